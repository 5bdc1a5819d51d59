// pip_physics.cuh -- per-cell and per-face physics of the PIP two-fluid step, device side.
//
// Every function keeps the operation order of the Fortran it restates (left-to-right
// evaluation, parentheses as written), so that a build without FMA contraction
// (-fmad=false) reproduces the FP64 CPU results bit for bit (up to exp()).  The functions
// are templated on the arithmetic type R (double for the drop-in path, float for the
// fluxes of the mixed-precision path).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cmath>

// Functions here compile for the device and, for host-side tests of the adjoint, for the
// host.
#if defined(__CUDACC__)
#define PIP_HD __host__ __device__ __forceinline__
#else
#define PIP_HD inline
#endif

namespace pip {

constexpr double kTiny = 1.0e-20;        // Globalvar.f90:101
constexpr double kHllcEpsi = 1.0e-10;    // HLL_rot.f90:12
constexpr double kHllcAcc = 1.03;        // HLL_rot.f90:12
constexpr double kHllgFactor = 1.001;    // HLL_rot.f90:702
constexpr double kMuP = 0.5;             // PIP_rot.f90:35
constexpr double kMuN = 1.0;             // PIP_rot.f90:36

template <typename R> PIP_HD R rmax(R a, R b) { return std::fmax(a, b); }
template <typename R> PIP_HD R rmin(R a, R b) { return std::fmin(a, b); }
template <> PIP_HD float rmax<float>(float a, float b) { return std::fmax(a, b); }
template <> PIP_HD float rmin<float>(float a, float b) { return std::fmin(a, b); }
PIP_HD double rsqrt_(double a) { return std::sqrt(a); }
PIP_HD float rsqrt_(float a) { return std::sqrt(a); }
// Reciprocal of the folded-division (rcp) forms below.  FP64 on the device: the hardware's
// approximate reciprocal (PTX rcp.approx.ftz.f64) refined by two Newton-Raphson steps,
// r <- r + r (1 - x r), each an error-compensated pair of FMAs, which take the seed's
// relative error e to about e^2 and then to the FP64 rounding level: within 1 ulp of the
// correctly rounded 1/x for normal x whose reciprocal is normal (tests/rcp_check.cu checks
// it against the IEEE division), inline and without branches.  Subnormal x or 1/x
// flush to zero and x = 0 gives NaN, outside the physical range of the denominators it
// serves (densities, wave-speed differences, the HLLD star denominators behind the HLLC-G
// guard).  FP32 and the host: the plain quotient.
PIP_HD double rcp_(double x) {
#if defined(__CUDA_ARCH__)
  double r, e;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
#else
  return 1.0 / x;
#endif
}
PIP_HD float rcp_(float x) { return 1.0f / x; }
PIP_HD double rabs(double a) { return std::fabs(a); }
PIP_HD float rabs(float a) { return std::fabs(a); }
PIP_HD double rsign1(double b) { return std::copysign(1.0, b); }
PIP_HD float rsign1(float b) { return std::copysign(1.0f, b); }

// ---------------------------------------------------------------- conversions

// u2v_mhd (HLL_rot.f90:1159-1186): conserved -> primitive with density/pressure floors.
template <typename R, int NVM>
PIP_HD void u2v_mhd(const R (&u)[NVM], R (&v)[NVM], R gm, R ro_lim, R pr_lim) {
  R ro = rmax(u[0], ro_lim);
  R roi = R(1) / ro;
  v[0] = ro;
  v[1] = u[1] * roi;
  v[2] = u[2] * roi;
  v[3] = u[3] * roi;
  R pr = (gm - R(1)) * (u[4] - R(0.5) * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * roi -
                        R(0.5) * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]));
  v[4] = pr < pr_lim ? pr_lim : pr;
  v[5] = u[5];
  v[6] = u[6];
  v[7] = u[7];
  if (NVM == 9) v[NVM - 1] = u[NVM - 1];
}

// u2v_hd (HLL_rot.f90:1136-1156).
template <typename R>
PIP_HD void u2v_hd(const R (&u)[5], R (&v)[5], R gm, R ro_lim, R pr_lim) {
  R ro = rmax(u[0], ro_lim);
  R roi = R(1) / ro;
  v[0] = ro;
  v[1] = u[1] * roi;
  v[2] = u[2] * roi;
  v[3] = u[3] * roi;
  R pr = (gm - R(1)) * (u[4] - R(0.5) * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * roi);
  v[4] = pr < pr_lim ? pr_lim : pr;
}

// Primitive set produced by cq2pv (density floored, velocity from the unfloored density).
template <typename R> struct Prim {
  R de, vx, vy, vz, pr;
};

// cq2pv_mhd (Scheme_rot.f90:153-179): floors and rewrites the conserved ion state through
// primitives, in place.  Returns the primitives.
template <typename R, int NVM>
PIP_HD Prim<R> cq2pv_mhd(R (&u)[NVM], R gm, R ro_lim, R pr_lim) {
  Prim<R> q;
  R de = u[0];
  R vx = u[1] / de, vy = u[2] / de, vz = u[3] / de;
  R bx = u[5], by = u[6], bz = u[7];
  R pr = (gm - R(1)) * (u[4] - R(0.5) * de * (vx * vx + vy * vy + vz * vz) -
                        R(0.5) * (bx * bx + by * by + bz * bz));
  pr = rmax(pr, pr_lim);
  de = rmax(de, ro_lim);
  u[0] = de;
  u[1] = vx * de;
  u[2] = vy * de;
  u[3] = vz * de;
  u[4] = pr / (gm - R(1)) + R(0.5) * de * (vx * vx + vy * vy + vz * vz) +
         R(0.5) * (bx * bx + by * by + bz * bz);
  q.de = de; q.vx = vx; q.vy = vy; q.vz = vz; q.pr = pr;
  return q;
}

// cq2pv_hd (Scheme_rot.f90:132-150).
template <typename R>
PIP_HD Prim<R> cq2pv_hd(R (&u)[5], R gm, R ro_lim, R pr_lim) {
  Prim<R> q;
  R de = u[0];
  R vx = u[1] / de, vy = u[2] / de, vz = u[3] / de;
  R pr = (gm - R(1)) * (u[4] - R(0.5) * de * (vx * vx + vy * vy + vz * vz));
  pr = rmax(pr, pr_lim);
  de = rmax(de, ro_lim);
  u[0] = de;
  u[1] = vx * de;
  u[2] = vy * de;
  u[3] = vz * de;
  u[4] = pr / (gm - R(1)) + R(0.5) * de * (vx * vx + vy * vy + vz * vz);
  q.de = de; q.vx = vx; q.vy = vy; q.vz = vz; q.pr = pr;
  return q;
}

// cq2pv with one division per species (reciprocal form, see below).
template <typename R, int NVM>
PIP_HD Prim<R> cq2pv_mhd_rcp(R (&u)[NVM], R gm, R igm1, R ro_lim, R pr_lim) {
  Prim<R> q;
  R de = u[0];
  const R inv = rcp_(de);
  R vx = u[1] * inv, vy = u[2] * inv, vz = u[3] * inv;
  const R kin = vx * vx + vy * vy + vz * vz;
  const R bb = u[5] * u[5] + u[6] * u[6] + u[7] * u[7];
  R pr = (gm - R(1)) * (u[4] - R(0.5) * de * kin - R(0.5) * bb);
  pr = rmax(pr, pr_lim);
  de = rmax(de, ro_lim);
  u[0] = de;
  u[1] = vx * de;
  u[2] = vy * de;
  u[3] = vz * de;
  u[4] = pr * igm1 + R(0.5) * de * kin + R(0.5) * bb;
  q.de = de; q.vx = vx; q.vy = vy; q.vz = vz; q.pr = pr;
  return q;
}
template <typename R>
PIP_HD Prim<R> cq2pv_hd_rcp(R (&u)[5], R gm, R igm1, R ro_lim, R pr_lim) {
  Prim<R> q;
  R de = u[0];
  const R inv = rcp_(de);
  R vx = u[1] * inv, vy = u[2] * inv, vz = u[3] * inv;
  const R kin = vx * vx + vy * vy + vz * vz;
  R pr = (gm - R(1)) * (u[4] - R(0.5) * de * kin);
  pr = rmax(pr, pr_lim);
  de = rmax(de, ro_lim);
  u[0] = de;
  u[1] = vx * de;
  u[2] = vy * de;
  u[3] = vz * de;
  u[4] = pr * igm1 + R(0.5) * de * kin;
  q.de = de; q.vx = vx; q.vy = vy; q.vz = vz; q.pr = pr;
  return q;
}

// CFL candidates of one interior cell (cfl_mhd Scheme_rot.f90:279-283, cfl_hd :229-233),
// from the primitives of the cq2pv rewrite.  sg = safety*gmin.
template <typename R>
PIP_HD R cfl_mhd_cell(const Prim<R>& q, R bx, R by, R bz, R gm, R sg) {
  R dm = rmax(q.de, R(kTiny));
  R cs2 = gm * q.pr / dm;
  R valf2 = (bx * bx + by * by + bz * bz) / dm;
  R vabs = rsqrt_(q.vx * q.vx + q.vy * q.vy + q.vz * q.vz);
  return sg / (vabs + rsqrt_(cs2 + valf2));
}
template <typename R>
PIP_HD R cfl_hd_cell(const Prim<R>& q, R gm, R sg) {
  R cs = rsqrt_(gm * q.pr / q.de);
  R vabs = rsqrt_(rmax(q.vx * q.vx + q.vy * q.vy + q.vz * q.vz, R(kTiny)));
  return sg / (vabs + cs);
}

// ---------------------------------------------------------------- reconstruction

// minmod_func (Util_rot.f90:59-76): slope at cell 1 of the triple (v0, v1, v2).
template <typename R>
PIP_HD R minmod(R v0, R v1, R v2) {
  R X = v2 - v1, Y = v1 - v0;
  R SX = rsign1(X);
  return SX * rmax(R(0), rmin(rabs(X), SX * Y));
}

// ---------------------------------------------------------------- Riemann solvers

// hllc_flux (HLL_rot.f90:615-687), primitive states (ro, vn, vt1, vt2, pr).
template <typename R>
PIP_HD void hllc_flux(const R (&v_l)[5], const R (&v_r)[5], R (&flx)[5], R gm) {
  const R gm1 = gm - R(1);
  R u_l[5], u_r[5], fl[5], fr[5], stl[5], str[5];
  u_l[0] = v_l[0]; u_l[1] = v_l[0] * v_l[1]; u_l[2] = v_l[0] * v_l[2]; u_l[3] = v_l[0] * v_l[3];
  u_l[4] = v_l[4] / gm1 + R(0.5) * v_l[0] * (v_l[1] * v_l[1] + v_l[2] * v_l[2] + v_l[3] * v_l[3]);
  u_r[0] = v_r[0]; u_r[1] = v_r[0] * v_r[1]; u_r[2] = v_r[0] * v_r[2]; u_r[3] = v_r[0] * v_r[3];
  u_r[4] = v_r[4] / gm1 + R(0.5) * v_r[0] * (v_r[1] * v_r[1] + v_r[2] * v_r[2] + v_r[3] * v_r[3]);
  const R pr_l = v_l[4], pr_r = v_r[4];
  fl[0] = u_l[1];
  fr[0] = u_r[1];
  fl[1] = pr_l + u_l[1] * u_l[1] / u_l[0];
  fr[1] = pr_r + u_r[1] * u_r[1] / u_r[0];
  fl[2] = u_l[1] * u_l[2] / u_l[0];
  fr[2] = u_r[1] * u_r[2] / u_r[0];
  fl[3] = u_l[1] * u_l[3] / u_l[0];
  fr[3] = u_r[1] * u_r[3] / u_r[0];
  fl[4] = u_l[1] * (u_l[4] + pr_l) / u_l[0];
  fr[4] = u_r[1] * (u_r[4] + pr_r) / u_r[0];
  const R cs_l = rsqrt_(gm * pr_l / u_l[0]);
  const R cs_r = rsqrt_(gm * pr_r / u_r[0]);
  const R vn_l = u_l[1] / u_l[0];
  const R vn_r = u_r[1] / u_r[0];
  const R sl = R(kHllcAcc) * rmin(vn_l - cs_l, vn_r - cs_r);
  const R sr = R(kHllcAcc) * rmax(vn_l + cs_l, vn_r + cs_r);
  const R sm = (u_r[1] * (sr - vn_r) - u_l[1] * (sl - vn_l) + pr_l - pr_r) /
               (u_r[0] * (sr - vn_r) - u_l[0] * (sl - vn_l));
  const R pr_m = sm * u_l[0] * (sl - vn_l) - u_l[1] * (sl - vn_l) + pr_l;
  stl[0] = u_l[0] * (sl - vn_l) / (sl - sm);
  str[0] = u_r[0] * (sr - vn_r) / (sr - sm);
  stl[1] = stl[0] * sm;
  str[1] = str[0] * sm;
  stl[2] = stl[0] * u_l[2] / u_l[0];
  str[2] = str[0] * u_r[2] / u_r[0];
  stl[3] = stl[0] * u_l[3] / u_l[0];
  str[3] = str[0] * u_r[3] / u_r[0];
  stl[4] = ((sl - vn_l) * u_l[4] - pr_l * vn_l + pr_m * sm) / (sl - sm);
  str[4] = ((sr - vn_r) * u_r[4] - pr_r * vn_r + pr_m * sm) / (sr - sm);
  const R thl = (rabs(sl) + sl) / rmax(R(2) * sl, R(kHllcEpsi));
  const R thm = (rabs(sm) + sm) / rmax(R(2) * sm, R(kHllcEpsi));
  const R thr = R(1) - (rabs(sr) + sr) / rmax(R(2) * sr, R(kHllcEpsi));
#pragma unroll
  for (int n = 0; n < 5; ++n)
    flx[n] = thr * fr[n] + thl * fl[n] +
             (R(1) - thl - thr) * (thm * (fl[n] + sl * (stl[n] - u_l[n])) +
                                   (R(1) - thm) * (fr[n] + sr * (str[n] - u_r[n])));
}

// hlld_flux (HLL_rot.f90:691-910): Miyoshi-Kusano HLLD with the HLLC-G fallback and the
// Dedner flux of (Bn, psi) when NVM == 9.  States are primitive
// (ro, vn, vt1, vt2, pr, Bn, Bt1, Bt2[, psi]).
template <typename R, int NVM>
PIP_HD void hlld_flux(const R (&v_l)[NVM], const R (&v_r)[NVM], R (&flx)[NVM],
                                          R gm, R cmax) {
  const R gm1 = gm - R(1);
  // v2u_1 energies (HLL_rot.f90:1201-1213)
  const R el = v_l[4] / gm1 + R(0.5) * v_l[0] * (v_l[1] * v_l[1] + v_l[2] * v_l[2] + v_l[3] * v_l[3]) +
               R(0.5) * (v_l[5] * v_l[5] + v_l[6] * v_l[6] + v_l[7] * v_l[7]);
  const R er = v_r[4] / gm1 + R(0.5) * v_r[0] * (v_r[1] * v_r[1] + v_r[2] * v_r[2] + v_r[3] * v_r[3]) +
               R(0.5) * (v_r[5] * v_r[5] + v_r[6] * v_r[6] + v_r[7] * v_r[7]);
  R u_l[8], u_r[8];
  u_l[0] = v_l[0]; u_l[1] = v_l[0] * v_l[1]; u_l[2] = v_l[0] * v_l[2]; u_l[3] = v_l[0] * v_l[3];
  u_l[4] = el; u_l[5] = v_l[5]; u_l[6] = v_l[6]; u_l[7] = v_l[7];
  u_r[0] = v_r[0]; u_r[1] = v_r[0] * v_r[1]; u_r[2] = v_r[0] * v_r[2]; u_r[3] = v_r[0] * v_r[3];
  u_r[4] = er; u_r[5] = v_r[5]; u_r[6] = v_r[6]; u_r[7] = v_r[7];

  const R b2_l = (v_l[5] * v_l[5] + v_l[6] * v_l[6] + v_l[7] * v_l[7]);
  const R pt_l = v_l[4] + R(0.5) * b2_l;
  const R vbL = v_l[1] * v_l[5] + v_l[2] * v_l[6] + v_l[3] * v_l[7];
  R fl[8], fr[8];
  fl[0] = v_l[0] * v_l[1];
  fl[1] = v_l[0] * (v_l[1] * v_l[1]) + v_l[4] + R(0.5) * b2_l - v_l[5] * v_l[5];
  fl[2] = v_l[0] * v_l[1] * v_l[2] - v_l[5] * v_l[6];
  fl[3] = v_l[0] * v_l[1] * v_l[3] - v_l[5] * v_l[7];
  fl[4] = (u_l[4] + pt_l) * v_l[1] - vbL * v_l[5];
  fl[5] = R(0);
  fl[6] = v_l[1] * v_l[6] - v_l[5] * v_l[2];
  fl[7] = v_l[1] * v_l[7] - v_l[5] * v_l[3];

  const R b2_r = (v_r[5] * v_r[5] + v_r[6] * v_r[6] + v_r[7] * v_r[7]);
  const R pt_r = v_r[4] + R(0.5) * b2_r;
  const R vbR = v_r[1] * v_r[5] + v_r[2] * v_r[6] + v_r[3] * v_r[7];
  fr[0] = v_r[0] * v_r[1];
  fr[1] = v_r[0] * (v_r[1] * v_r[1]) + v_r[4] + R(0.5) * b2_r - v_r[5] * v_r[5];
  fr[2] = v_r[0] * v_r[1] * v_r[2] - v_r[5] * v_r[6];
  fr[3] = v_r[0] * v_r[1] * v_r[3] - v_r[5] * v_r[7];
  fr[4] = (u_r[4] + pt_r) * v_r[1] - vbR * v_r[5];
  fr[5] = R(0);
  fr[6] = v_r[1] * v_r[6] - v_r[5] * v_r[2];
  fr[7] = v_r[1] * v_r[7] - v_r[5] * v_r[3];

  // fast mode speeds
  R f1 = gm * v_l[4];
  R f2 = R(4) * f1 * (v_l[5] * v_l[5]);
  const R vf_l = rsqrt_(((f1 + b2_l) + rsqrt_(rmax((f1 + b2_l) * (f1 + b2_l) - f2, R(0)))) / (R(2) * v_l[0]));
  f1 = gm * v_r[4];
  f2 = R(4) * f1 * (v_r[5] * v_r[5]);
  const R vf_r = rsqrt_(((f1 + b2_r) + rsqrt_(rmax((f1 + b2_r) * (f1 + b2_r) - f2, R(0)))) / (R(2) * v_r[0]));

  const R sl = rmin(v_l[1], v_r[1]) - rmax(vf_l, vf_r);
  const R sr = rmax(v_l[1], v_r[1]) + rmax(vf_l, vf_r);

  R out[8];
  if (sl >= R(0)) {
#pragma unroll
    for (int n = 0; n < 8; ++n) out[n] = fl[n];
  } else if (sr <= R(0)) {
#pragma unroll
    for (int n = 0; n < 8; ++n) out[n] = fr[n];
  } else {
    f1 = R(1) / (sr - sl);
    R uh[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) uh[n] = f1 * (sr * u_r[n] - sl * u_l[n] - fr[n] + fl[n]);
    const R sm = uh[1] / uh[0];
    const R pt = pt_l + v_l[0] * (sl - v_l[1]) * (sm - v_l[1]);
    const R ro_l1 = v_l[0] * (sl - v_l[1]) / (sl - sm);
    const R ro_r1 = v_r[0] * (sr - v_r[1]) / (sr - sm);
    const R sal = rabs(uh[5]) / rsqrt_(ro_l1);
    const R sar = rabs(uh[5]) / rsqrt_(ro_r1);

    if ((sl >= (sm - R(kHllgFactor) * sal)) || ((sm + R(kHllgFactor) * sar) >= sr)) {
      // revert to HLLC-G (HLL_rot.f90:776-807)
      const R vy_2 = uh[2] / uh[0];
      const R vz_2 = uh[3] / uh[0];
      if (sm >= R(0)) {
        const R e2 = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                      uh[5] * (vbL - sm * uh[5] - vy_2 * uh[6] - vz_2 * uh[7])) / (sl - sm);
        out[0] = sl * (ro_l1 - v_l[0]) + fl[0];
        out[1] = sl * (ro_l1 * sm - u_l[1]) + fl[1];
        out[2] = sl * (ro_l1 * vy_2 - u_l[2]) + fl[2];
        out[3] = sl * (ro_l1 * vz_2 - u_l[3]) + fl[3];
        out[4] = sl * (e2 - u_l[4]) + fl[4];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sl * (uh[n] - v_l[n]) + fl[n];
      } else {
        const R e2 = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                      uh[5] * (vbR - sm * uh[5] - vy_2 * uh[6] - vz_2 * uh[7])) / (sr - sm);
        out[0] = sr * (ro_r1 - v_r[0]) + fr[0];
        out[1] = sr * (ro_r1 * sm - u_r[1]) + fr[1];
        out[2] = sr * (ro_r1 * vy_2 - u_r[2]) + fr[2];
        out[3] = sr * (ro_r1 * vz_2 - u_r[3]) + fr[3];
        out[4] = sr * (e2 - u_r[4]) + fr[4];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sr * (uh[n] - v_r[n]) + fr[n];
      }
    } else {
      // intermediate states L*, R* (HLL_rot.f90:813-843)
      R ul1[8], ur1[8];
      f1 = R(1) / (v_l[0] * (sl - v_l[1]) * (sl - sm) - uh[5] * uh[5]);
      ul1[5] = uh[5];
      ul1[6] = v_l[6] * f1 * (v_l[0] * ((sl - v_l[1]) * (sl - v_l[1])) - uh[5] * uh[5]);
      ul1[7] = v_l[7] * f1 * (v_l[0] * ((sl - v_l[1]) * (sl - v_l[1])) - uh[5] * uh[5]);
      const R vy_l1 = v_l[2] - f1 * uh[5] * v_l[6] * (sm - v_l[1]);
      const R vz_l1 = v_l[3] - f1 * uh[5] * v_l[7] * (sm - v_l[1]);
      ul1[0] = ro_l1;
      ul1[4] = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                uh[5] * (vbL - sm * uh[5] - vy_l1 * ul1[6] - vz_l1 * ul1[7])) / (sl - sm);
      ul1[1] = ro_l1 * sm;
      ul1[2] = ro_l1 * vy_l1;
      ul1[3] = ro_l1 * vz_l1;

      f1 = R(1) / (v_r[0] * (sr - v_r[1]) * (sr - sm) - uh[5] * uh[5]);
      ur1[5] = uh[5];
      ur1[6] = v_r[6] * f1 * (v_r[0] * ((sr - v_r[1]) * (sr - v_r[1])) - uh[5] * uh[5]);
      ur1[7] = v_r[7] * f1 * (v_r[0] * ((sr - v_r[1]) * (sr - v_r[1])) - uh[5] * uh[5]);
      const R vy_r1 = v_r[2] - f1 * uh[5] * v_r[6] * (sm - v_r[1]);
      const R vz_r1 = v_r[3] - f1 * uh[5] * v_r[7] * (sm - v_r[1]);
      ur1[0] = ro_r1;
      ur1[4] = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                uh[5] * (vbR - sm * uh[5] - vy_r1 * ur1[6] - vz_r1 * ur1[7])) / (sr - sm);
      ur1[1] = ro_r1 * sm;
      ur1[2] = ro_r1 * vy_r1;
      ur1[3] = ro_r1 * vz_r1;

      const R sl1 = sm - sal;
      const R sr1 = sm + sar;
      if (sl1 >= R(0)) {
        out[0] = sl * (ul1[0] - v_l[0]) + fl[0];
#pragma unroll
        for (int n = 1; n < 5; ++n) out[n] = sl * (ul1[n] - u_l[n]) + fl[n];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sl * (ul1[n] - v_l[n]) + fl[n];
      } else if (sr1 <= R(0)) {
        out[0] = sr * (ur1[0] - v_r[0]) + fr[0];
#pragma unroll
        for (int n = 1; n < 5; ++n) out[n] = sr * (ur1[n] - u_r[n]) + fr[n];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sr * (ur1[n] - v_r[n]) + fr[n];
      } else {
        // central states L**, R** (HLL_rot.f90:861-898)
        const R ro_ls = rsqrt_(ro_l1);
        const R ro_rs = rsqrt_(ro_r1);
        f1 = R(1) / (ro_ls + ro_rs);
        f2 = rsign1(uh[5]);
        const R vy_2 = f1 * (ro_ls * vy_l1 + ro_rs * vy_r1 + (ur1[6] - ul1[6]) * f2);
        const R vz_2 = f1 * (ro_ls * vz_l1 + ro_rs * vz_r1 + (ur1[7] - ul1[7]) * f2);
        R u2[8];
        u2[5] = uh[5];
        u2[6] = f1 * (ro_ls * ur1[6] + ro_rs * ul1[6] + ro_ls * ro_rs * (vy_r1 - vy_l1) * f2);
        u2[7] = f1 * (ro_ls * ur1[7] + ro_rs * ul1[7] + ro_ls * ro_rs * (vz_r1 - vz_l1) * f2);
        if (sm >= R(0)) {
          u2[0] = ro_l1;
          u2[4] = ul1[4] - ro_ls * (vy_l1 * ul1[6] + vz_l1 * ul1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_l1 * sm;
          u2[2] = ro_l1 * vy_2;
          u2[3] = ro_l1 * vz_2;
          out[0] = sl1 * u2[0] - (sl1 - sl) * ul1[0] - sl * v_l[0] + fl[0];
#pragma unroll
          for (int n = 1; n < 5; ++n) out[n] = sl1 * u2[n] - (sl1 - sl) * ul1[n] - sl * u_l[n] + fl[n];
#pragma unroll
          for (int n = 5; n < 8; ++n) out[n] = sl1 * u2[n] - (sl1 - sl) * ul1[n] - sl * v_l[n] + fl[n];
        } else {
          u2[0] = ro_r1;
          u2[4] = ur1[4] + ro_rs * (vy_r1 * ur1[6] + vz_r1 * ur1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_r1 * sm;
          u2[2] = ro_r1 * vy_2;
          u2[3] = ro_r1 * vz_2;
          out[0] = sr1 * u2[0] - (sr1 - sr) * ur1[0] - sr * v_r[0] + fr[0];
#pragma unroll
          for (int n = 1; n < 5; ++n) out[n] = sr1 * u2[n] - (sr1 - sr) * ur1[n] - sr * u_r[n] + fr[n];
#pragma unroll
          for (int n = 5; n < 8; ++n) out[n] = sr1 * u2[n] - (sr1 - sr) * ur1[n] - sr * v_r[n] + fr[n];
        }
      }
    }
  }
#pragma unroll
  for (int n = 0; n < 8; ++n) flx[n] = out[n];
  if (NVM == 9) {
    // Dedner flux (HLL_rot.f90:904-908) with ch = cmax
    const R ch = cmax;
    flx[5] = R(0.5) * (v_l[NVM - 1] + v_r[NVM - 1] - ch * (v_r[5] - v_l[5]));
    flx[NVM - 1] = R(0.5) * (ch * ch * (v_l[5] + v_r[5]) - ch * (v_r[NVM - 1] - v_l[NVM - 1]));
  }
}

// ---------------------------------------------------------------- reciprocal forms
//
// The same Riemann solvers with the divisions folded: a shared denominator is inverted
// once, u/rho of a state built as rho*v is taken as v, and p/(gm-1) uses a precomputed
// 1/(gm-1).  Results differ from the literal forms above by a few ulps per face; they are
// used by the FMA build (held to 1e-10 relative L1 against the oracle over whole runs)
// and by the FP32-mixed form.

PIP_HD double rrsqrt(double a) {
#if defined(__CUDA_ARCH__)
  return rsqrt(a);
#else
  return 1.0 / std::sqrt(a);
#endif
}
PIP_HD float rrsqrt(float a) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(a);
#else
  return 1.0f / std::sqrt(a);
#endif
}

// A product the compiler may not fuse into an FMA.  At a mirror face (flag_bnd 2-7: the
// ghost state is the interior state with vn, and Bn or the tangential pairs, negated) the
// HLL averages sr*u_r - sl*u_l of the symmetric components cancel to exactly +0 only when
// both products are rounded alone; fused, the residue is one product's rounding error of
// either sign.  Its sign picks the L* or R* branch (sm) and sign(Bn), whose wall fluxes of
// vt, Bt and e are equal and opposite, so a fused average flips them from step to step.
PIP_HD double mul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
PIP_HD float mul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}

// HLLC smooth switch (|s|+s)/max(2s,eps) without a division: 1 for s >= eps/2, 0 for s<=0.
template <typename R>
PIP_HD R hllc_switch(R s) {
  return s >= R(0.5 * kHllcEpsi) ? R(1) : (s > R(0) ? R(2) * s * R(1.0 / kHllcEpsi) : R(0));
}

template <typename R>
PIP_HD void hllc_flux_rcp(const R (&v_l)[5], const R (&v_r)[5], R (&flx)[5], R gm,
                                              R igm1) {
  R u_l[5], u_r[5], fl[5], fr[5], stl[5], str[5];
  const R ke_l = v_l[1] * v_l[1] + v_l[2] * v_l[2] + v_l[3] * v_l[3];
  const R ke_r = v_r[1] * v_r[1] + v_r[2] * v_r[2] + v_r[3] * v_r[3];
  u_l[0] = v_l[0]; u_l[1] = v_l[0] * v_l[1]; u_l[2] = v_l[0] * v_l[2]; u_l[3] = v_l[0] * v_l[3];
  u_l[4] = v_l[4] * igm1 + R(0.5) * v_l[0] * ke_l;
  u_r[0] = v_r[0]; u_r[1] = v_r[0] * v_r[1]; u_r[2] = v_r[0] * v_r[2]; u_r[3] = v_r[0] * v_r[3];
  u_r[4] = v_r[4] * igm1 + R(0.5) * v_r[0] * ke_r;
  const R pr_l = v_l[4], pr_r = v_r[4];
  const R vn_l = v_l[1], vn_r = v_r[1];
  fl[0] = u_l[1];
  fr[0] = u_r[1];
  fl[1] = pr_l + u_l[1] * vn_l;
  fr[1] = pr_r + u_r[1] * vn_r;
  fl[2] = u_l[2] * vn_l;
  fr[2] = u_r[2] * vn_r;
  fl[3] = u_l[3] * vn_l;
  fr[3] = u_r[3] * vn_r;
  fl[4] = (u_l[4] + pr_l) * vn_l;
  fr[4] = (u_r[4] + pr_r) * vn_r;
  const R cs_l = rsqrt_(gm * pr_l / v_l[0]);
  const R cs_r = rsqrt_(gm * pr_r / v_r[0]);
  const R sl = R(kHllcAcc) * rmin(vn_l - cs_l, vn_r - cs_r);
  const R sr = R(kHllcAcc) * rmax(vn_l + cs_l, vn_r + cs_r);
  const R ql = u_l[0] * (sl - vn_l), qr = u_r[0] * (sr - vn_r);
  const R sm = (mul_rn(u_r[1], sr - vn_r) - mul_rn(u_l[1], sl - vn_l) + pr_l - pr_r) / (qr - ql);
  const R pr_m = sm * ql - u_l[1] * (sl - vn_l) + pr_l;
  const R il = rcp_(sl - sm), ir = rcp_(sr - sm);
  stl[0] = ql * il;
  str[0] = qr * ir;
  stl[1] = stl[0] * sm;
  str[1] = str[0] * sm;
  stl[2] = stl[0] * v_l[2];
  str[2] = str[0] * v_r[2];
  stl[3] = stl[0] * v_l[3];
  str[3] = str[0] * v_r[3];
  stl[4] = ((sl - vn_l) * u_l[4] - pr_l * vn_l + pr_m * sm) * il;
  str[4] = ((sr - vn_r) * u_r[4] - pr_r * vn_r + pr_m * sm) * ir;
  const R thl = hllc_switch(sl);
  const R thm = hllc_switch(sm);
  const R thr = R(1) - hllc_switch(sr);
#pragma unroll
  for (int n = 0; n < 5; ++n)
    flx[n] = thr * fr[n] + thl * fl[n] +
             (R(1) - thl - thr) * (thm * (fl[n] + sl * (stl[n] - u_l[n])) +
                                   (R(1) - thm) * (fr[n] + sr * (str[n] - u_r[n])));
}

template <typename R, int NVM>
PIP_HD void hlld_flux_rcp(const R (&v_l)[NVM], const R (&v_r)[NVM], R (&flx)[NVM],
                                              R gm, R igm1, R cmax) {
  const R b2_l = (v_l[5] * v_l[5] + v_l[6] * v_l[6] + v_l[7] * v_l[7]);
  const R b2_r = (v_r[5] * v_r[5] + v_r[6] * v_r[6] + v_r[7] * v_r[7]);
  const R el = v_l[4] * igm1 + R(0.5) * v_l[0] * (v_l[1] * v_l[1] + v_l[2] * v_l[2] + v_l[3] * v_l[3]) +
               R(0.5) * b2_l;
  const R er = v_r[4] * igm1 + R(0.5) * v_r[0] * (v_r[1] * v_r[1] + v_r[2] * v_r[2] + v_r[3] * v_r[3]) +
               R(0.5) * b2_r;
  R u_l[8], u_r[8];
  u_l[0] = v_l[0]; u_l[1] = v_l[0] * v_l[1]; u_l[2] = v_l[0] * v_l[2]; u_l[3] = v_l[0] * v_l[3];
  u_l[4] = el; u_l[5] = v_l[5]; u_l[6] = v_l[6]; u_l[7] = v_l[7];
  u_r[0] = v_r[0]; u_r[1] = v_r[0] * v_r[1]; u_r[2] = v_r[0] * v_r[2]; u_r[3] = v_r[0] * v_r[3];
  u_r[4] = er; u_r[5] = v_r[5]; u_r[6] = v_r[6]; u_r[7] = v_r[7];
  const R pt_l = v_l[4] + R(0.5) * b2_l;
  const R pt_r = v_r[4] + R(0.5) * b2_r;
  const R vbL = v_l[1] * v_l[5] + v_l[2] * v_l[6] + v_l[3] * v_l[7];
  const R vbR = v_r[1] * v_r[5] + v_r[2] * v_r[6] + v_r[3] * v_r[7];
  R fl[8], fr[8];
  fl[0] = u_l[1];
  fl[1] = u_l[1] * v_l[1] + pt_l - v_l[5] * v_l[5];
  fl[2] = u_l[1] * v_l[2] - v_l[5] * v_l[6];
  fl[3] = u_l[1] * v_l[3] - v_l[5] * v_l[7];
  fl[4] = (u_l[4] + pt_l) * v_l[1] - vbL * v_l[5];
  fl[5] = R(0);
  fl[6] = v_l[1] * v_l[6] - v_l[5] * v_l[2];
  fl[7] = v_l[1] * v_l[7] - v_l[5] * v_l[3];
  fr[0] = u_r[1];
  fr[1] = u_r[1] * v_r[1] + pt_r - v_r[5] * v_r[5];
  fr[2] = u_r[1] * v_r[2] - v_r[5] * v_r[6];
  fr[3] = u_r[1] * v_r[3] - v_r[5] * v_r[7];
  fr[4] = (u_r[4] + pt_r) * v_r[1] - vbR * v_r[5];
  fr[5] = R(0);
  fr[6] = v_r[1] * v_r[6] - v_r[5] * v_r[2];
  fr[7] = v_r[1] * v_r[7] - v_r[5] * v_r[3];

  R f1 = gm * v_l[4];
  const R vf_l = rsqrt_(((f1 + b2_l) + rsqrt_(rmax((f1 + b2_l) * (f1 + b2_l) - R(4) * f1 * (v_l[5] * v_l[5]), R(0)))) /
                        (R(2) * v_l[0]));
  f1 = gm * v_r[4];
  const R vf_r = rsqrt_(((f1 + b2_r) + rsqrt_(rmax((f1 + b2_r) * (f1 + b2_r) - R(4) * f1 * (v_r[5] * v_r[5]), R(0)))) /
                        (R(2) * v_r[0]));
  const R sl = rmin(v_l[1], v_r[1]) - rmax(vf_l, vf_r);
  const R sr = rmax(v_l[1], v_r[1]) + rmax(vf_l, vf_r);

  R out[8];
  if (sl >= R(0)) {
#pragma unroll
    for (int n = 0; n < 8; ++n) out[n] = fl[n];
  } else if (sr <= R(0)) {
#pragma unroll
    for (int n = 0; n < 8; ++n) out[n] = fr[n];
  } else {
    f1 = rcp_(sr - sl);
    R uh[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) uh[n] = f1 * (mul_rn(sr, u_r[n]) - mul_rn(sl, u_l[n]) - fr[n] + fl[n]);
    const R iuh0 = rcp_(uh[0]);
    const R sm = uh[1] * iuh0;
    const R pt = pt_l + v_l[0] * (sl - v_l[1]) * (sm - v_l[1]);
    const R ilm = rcp_(sl - sm), irm = rcp_(sr - sm);
    const R ro_l1 = v_l[0] * (sl - v_l[1]) * ilm;
    const R ro_r1 = v_r[0] * (sr - v_r[1]) * irm;
    const R rs_l = rrsqrt(ro_l1), rs_r = rrsqrt(ro_r1);
    const R bn = uh[5], bn2 = bn * bn;
    const R sal = rabs(bn) * rs_l;
    const R sar = rabs(bn) * rs_r;

    if ((sl >= (sm - R(kHllgFactor) * sal)) || ((sm + R(kHllgFactor) * sar) >= sr)) {
      const R vy_2 = uh[2] * iuh0;
      const R vz_2 = uh[3] * iuh0;
      if (sm >= R(0)) {
        const R e2 = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                      bn * (vbL - sm * bn - vy_2 * uh[6] - vz_2 * uh[7])) * ilm;
        out[0] = sl * (ro_l1 - v_l[0]) + fl[0];
        out[1] = sl * (ro_l1 * sm - u_l[1]) + fl[1];
        out[2] = sl * (ro_l1 * vy_2 - u_l[2]) + fl[2];
        out[3] = sl * (ro_l1 * vz_2 - u_l[3]) + fl[3];
        out[4] = sl * (e2 - u_l[4]) + fl[4];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sl * (uh[n] - v_l[n]) + fl[n];
      } else {
        const R e2 = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                      bn * (vbR - sm * bn - vy_2 * uh[6] - vz_2 * uh[7])) * irm;
        out[0] = sr * (ro_r1 - v_r[0]) + fr[0];
        out[1] = sr * (ro_r1 * sm - u_r[1]) + fr[1];
        out[2] = sr * (ro_r1 * vy_2 - u_r[2]) + fr[2];
        out[3] = sr * (ro_r1 * vz_2 - u_r[3]) + fr[3];
        out[4] = sr * (e2 - u_r[4]) + fr[4];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sr * (uh[n] - v_r[n]) + fr[n];
      }
    } else {
      R ul1[8], ur1[8];
      const R dl = v_l[0] * (sl - v_l[1]);
      f1 = rcp_(dl * (sl - sm) - bn2);
      const R gl = f1 * (dl * (sl - v_l[1]) - bn2);
      ul1[5] = bn;
      ul1[6] = v_l[6] * gl;
      ul1[7] = v_l[7] * gl;
      const R vy_l1 = v_l[2] - f1 * bn * v_l[6] * (sm - v_l[1]);
      const R vz_l1 = v_l[3] - f1 * bn * v_l[7] * (sm - v_l[1]);
      ul1[0] = ro_l1;
      ul1[4] = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                bn * (vbL - sm * bn - vy_l1 * ul1[6] - vz_l1 * ul1[7])) * ilm;
      ul1[1] = ro_l1 * sm;
      ul1[2] = ro_l1 * vy_l1;
      ul1[3] = ro_l1 * vz_l1;

      const R dr = v_r[0] * (sr - v_r[1]);
      f1 = rcp_(dr * (sr - sm) - bn2);
      const R gr = f1 * (dr * (sr - v_r[1]) - bn2);
      ur1[5] = bn;
      ur1[6] = v_r[6] * gr;
      ur1[7] = v_r[7] * gr;
      const R vy_r1 = v_r[2] - f1 * bn * v_r[6] * (sm - v_r[1]);
      const R vz_r1 = v_r[3] - f1 * bn * v_r[7] * (sm - v_r[1]);
      ur1[0] = ro_r1;
      ur1[4] = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                bn * (vbR - sm * bn - vy_r1 * ur1[6] - vz_r1 * ur1[7])) * irm;
      ur1[1] = ro_r1 * sm;
      ur1[2] = ro_r1 * vy_r1;
      ur1[3] = ro_r1 * vz_r1;

      const R sl1 = sm - sal;
      const R sr1 = sm + sar;
      if (sl1 >= R(0)) {
        out[0] = sl * (ul1[0] - v_l[0]) + fl[0];
#pragma unroll
        for (int n = 1; n < 5; ++n) out[n] = sl * (ul1[n] - u_l[n]) + fl[n];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sl * (ul1[n] - v_l[n]) + fl[n];
      } else if (sr1 <= R(0)) {
        out[0] = sr * (ur1[0] - v_r[0]) + fr[0];
#pragma unroll
        for (int n = 1; n < 5; ++n) out[n] = sr * (ur1[n] - u_r[n]) + fr[n];
#pragma unroll
        for (int n = 5; n < 8; ++n) out[n] = sr * (ur1[n] - v_r[n]) + fr[n];
      } else {
        const R ro_ls = ro_l1 * rs_l;   // sqrt(ro_l1)
        const R ro_rs = ro_r1 * rs_r;
        f1 = rcp_(ro_ls + ro_rs);
        const R f2 = rsign1(bn);
        const R vy_2 = f1 * (ro_ls * vy_l1 + ro_rs * vy_r1 + (ur1[6] - ul1[6]) * f2);
        const R vz_2 = f1 * (ro_ls * vz_l1 + ro_rs * vz_r1 + (ur1[7] - ul1[7]) * f2);
        R u2[8];
        u2[5] = bn;
        u2[6] = f1 * (ro_ls * ur1[6] + ro_rs * ul1[6] + ro_ls * ro_rs * (vy_r1 - vy_l1) * f2);
        u2[7] = f1 * (ro_ls * ur1[7] + ro_rs * ul1[7] + ro_ls * ro_rs * (vz_r1 - vz_l1) * f2);
        if (sm >= R(0)) {
          u2[0] = ro_l1;
          u2[4] = ul1[4] - ro_ls * (vy_l1 * ul1[6] + vz_l1 * ul1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_l1 * sm;
          u2[2] = ro_l1 * vy_2;
          u2[3] = ro_l1 * vz_2;
          out[0] = sl1 * u2[0] - (sl1 - sl) * ul1[0] - sl * v_l[0] + fl[0];
#pragma unroll
          for (int n = 1; n < 5; ++n) out[n] = sl1 * u2[n] - (sl1 - sl) * ul1[n] - sl * u_l[n] + fl[n];
#pragma unroll
          for (int n = 5; n < 8; ++n) out[n] = sl1 * u2[n] - (sl1 - sl) * ul1[n] - sl * v_l[n] + fl[n];
        } else {
          u2[0] = ro_r1;
          u2[4] = ur1[4] + ro_rs * (vy_r1 * ur1[6] + vz_r1 * ur1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_r1 * sm;
          u2[2] = ro_r1 * vy_2;
          u2[3] = ro_r1 * vz_2;
          out[0] = sr1 * u2[0] - (sr1 - sr) * ur1[0] - sr * v_r[0] + fr[0];
#pragma unroll
          for (int n = 1; n < 5; ++n) out[n] = sr1 * u2[n] - (sr1 - sr) * ur1[n] - sr * u_r[n] + fr[n];
#pragma unroll
          for (int n = 5; n < 8; ++n) out[n] = sr1 * u2[n] - (sr1 - sr) * ur1[n] - sr * v_r[n] + fr[n];
        }
      }
    }
  }
#pragma unroll
  for (int n = 0; n < 8; ++n) flx[n] = out[n];
  if (NVM == 9) {
    const R ch = cmax;
    flx[5] = R(0.5) * (v_l[NVM - 1] + v_r[NVM - 1] - ch * (v_r[5] - v_l[5]));
    flx[NVM - 1] = R(0.5) * (ch * ch * (v_l[5] + v_r[5]) - ch * (v_r[NVM - 1] - v_l[NVM - 1]));
  }
}

}  // namespace pip
