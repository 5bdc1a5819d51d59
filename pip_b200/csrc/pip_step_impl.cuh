// pip_step_impl.cuh -- FP64 kernels of the two-fluid step.  Included by pip_fp64_fast.cu
// (FMA contraction on) and pip_fp64_exact.cu (-fmad=false, bitwise comparable with the
// CPU restatement); PIP_FLAVOUR names the namespace and PIP_LAUNCHERS the table getter.
//
// Layout in HBM: one array of NV = nvm + 5 planes, each plane the Fortran
// (ix,jx) slab with ghosts (x fastest): ion planes 0..nvm-1 (ro, mx, my, mz, en, bx, by,
// bz[, psi]) then neutral planes nvm..nvm+4 (ro, mx, my, mz, en).  A step uses two such
// arrays: A holds U0 and receives U2 in place, B receives U1.
#pragma once

#include <cstring>

#include "pip_kernels.cuh"
#include "pip_physics.cuh"
#include "pip_tma.cuh"

namespace pip {
namespace PIP_FLAVOUR {

constexpr int kH = 2;  // stencil half-width of minmod MUSCL

template <int NDIM> struct Tile;
// 2D tile (compile-time tuning constants; 32x7 cells: 33x7 x faces + 32x8 y faces = 487
// faces = two rounds of 256 threads).
#ifndef PIP_FP64_TX
#define PIP_FP64_TX 32
#endif
#ifndef PIP_FP64_TY
#define PIP_FP64_TY 7
#endif
template <> struct Tile<2> {
  static constexpr int TX = PIP_FP64_TX, TY = PIP_FP64_TY, NT = (TX * TY + 255) / 256 * 256;
};
template <> struct Tile<1> {
  static constexpr int TX = 128, TY = 1, NT = 128;
};

// Conversions and Riemann solvers of this flavour: the literal reference expressions
// (FMA-free build) or the reciprocal forms (FMA build).
template <int NVM>
__device__ __forceinline__ Prim<double> rt_mhd(double (&u)[NVM], const KParams &p) {
#if PIP_RCP
  return cq2pv_mhd_rcp<double, NVM>(u, p.gm, p.igm1, p.ro_lim, p.pr_lim);
#else
  return cq2pv_mhd<double, NVM>(u, p.gm, p.ro_lim, p.pr_lim);
#endif
}
__device__ __forceinline__ Prim<double> rt_hd(double (&u)[5], const KParams &p) {
#if PIP_RCP
  return cq2pv_hd_rcp<double>(u, p.gm, p.igm1, p.ro_lim, p.pr_lim);
#else
  return cq2pv_hd<double>(u, p.gm, p.ro_lim, p.pr_lim);
#endif
}
template <int NVM>
__device__ __forceinline__ void riemann_mhd(const double (&vl)[NVM], const double (&vr)[NVM],
                                            double (&f)[NVM], const KParams &p, double cmax) {
#if PIP_RCP
  hlld_flux_rcp<double, NVM>(vl, vr, f, p.gm, p.igm1, cmax);
#else
  hlld_flux<double, NVM>(vl, vr, f, p.gm, cmax);
#endif
}
__device__ __forceinline__ void riemann_hd(const double (&vl)[5], const double (&vr)[5],
                                           double (&f)[5], const KParams &p) {
#if PIP_RCP
  hllc_flux_rcp<double>(vl, vr, f, p.gm, p.igm1);
#else
  hllc_flux<double>(vl, vr, f, p.gm);
#endif
}

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

// dt of the step from the reduced CFL terms (cfl, Scheme_rot.f90:183-213): the minimum
// CFL candidate (seeded with cfl_mhd's 10.0), cfl_pn_col and cfl_pip_ir.
__device__ __forceinline__ double finalize_dt(const KParams &p, const DevCtrl *c, int slot) {
  double dt = bitsd(c->red_dt[slot]);
  double rho = bitsd(c->red_rho[slot]);
  dt = fmin(dt, p.col_lim / rho);
  if (p.ir) dt = fmin(dt, p.ir_lim / fmax(bitsd(c->red_gr[slot]), 1.0e-5));
  if (p.irn) {
    // cfl_pip_ir's ion_pot term (flag_IR_type 0) and cfl_pip_ir_nexcite; the slots hold
    // the maxima already raised to 1e-5
    if (p.ir_type == 0) dt = fmin(dt, p.safety / bitsd(c->red_ip[slot]));
    dt = fmin(dt, p.nl_lim / bitsd(c->red_nx[slot]));
  }
  return dt;
}

// Ionisation/recombination rates of PIP_IR_POWERLAW from the ion state (get_Pr_MHD's
// pressure with floor, Scheme_rot.f90:112-121; get_Te_MHD's temperature, :104-110).
template <int NVM>
__device__ __forceinline__ void ir_rates(const double (&u)[NVM], const KParams &p, double &gr,
                                         double &gi) {
  const double gm = p.gm;
  double pr = (gm - 1.0) * (u[4] - 0.5 * ((u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
                                          u[5] * u[5] + u[6] * u[6] + u[7] * u[7]));
  pr = fmax(pr, p.pr_lim);
  const double te = 0.5 * gm * (pr / u[0]);
  const double rs = 1.0 / sqrt(te);
  gr = p.ir_rec * rs;
  gi = p.ir_ion * rs * exp(-p.ir_chi / te);
}

constexpr double kPiRef = 3.1415926535897932;  // pi of Parameters.f90:2

// Explicitly rounded operations: the alpha_c field is computed at several call sites (the
// stage kernels' cells, the exchanged ghost cells, the whole-grid pass), and FMA
// contraction would round each site differently in the contracted build.
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

// get_Te_MHD and get_Te_HD (Scheme_rot.f90:83-128) on one cell: the pressures with the
// floor (`if(minval(pr).le.pr_lim) pr=max(pr,pr_lim)` is the per-cell max), the energies
// um[4], uh[4] rewritten from them, and the temperatures Te_m = 0.5*gm*pr/ro, Te_h = gm*pr/ro.
// The FMA build multiplies by 1/ro and 1/(gm-1) (returned in rm, rh for the drift); the
// FMA-free build divides as the Fortran does.  Divisions by 2, 16 and 64 below are exact
// multiplications by their reciprocals.
template <int NVM>
__device__ __forceinline__ void get_te(double (&um)[NVM], double (&uh)[5], const KParams &p,
                                       double &te_m, double &te_h, double &rm, double &rh) {
  const double gm = p.gm, g1 = rsub(gm, 1.0);
  // (m.m)/ro + bx^2 + by^2 + bz^2, summed left to right
  const double mm = radd(radd(rmul(um[1], um[1]), rmul(um[2], um[2])), rmul(um[3], um[3]));
  const double mh = radd(radd(rmul(uh[1], uh[1]), rmul(uh[2], uh[2])), rmul(uh[3], uh[3]));
#if PIP_RCP
  rm = rdiv(1.0, um[0]);
  rh = rdiv(1.0, uh[0]);
  const double km = rmul(mm, rm), kh = rmul(mh, rh);
#else
  rm = rh = 0.0;
  const double km = rdiv(mm, um[0]), kh = rdiv(mh, uh[0]);
#endif
  const double em = radd(radd(radd(km, rmul(um[5], um[5])), rmul(um[6], um[6])),
                         rmul(um[7], um[7]));
  double pr = rmul(g1, rsub(um[4], rmul(0.5, em)));
  pr = fmax(pr, p.pr_lim);
#if PIP_RCP
  um[4] = radd(rmul(pr, p.igm1), rmul(0.5, em));
  te_m = rmul(rmul(0.5, gm), rmul(pr, rm));
  double ph = rmul(g1, rsub(uh[4], rmul(rmul(0.5, mh), rh)));
  ph = fmax(ph, p.pr_lim);
  uh[4] = radd(rmul(ph, p.igm1), rmul(0.5, kh));
  te_h = rmul(gm, rmul(ph, rh));
#else
  um[4] = radd(rdiv(pr, g1), rmul(0.5, em));
  te_m = rmul(rmul(0.5, gm), rdiv(pr, um[0]));
  double ph = rmul(g1, rsub(uh[4], rdiv(rmul(0.5, mh), uh[0])));   // 0.5*(m.m)/ro
  ph = fmax(ph, p.pr_lim);
  uh[4] = radd(rdiv(ph, g1), rmul(0.5, kh));                        // 0.5*((m.m)/ro)
  te_h = rmul(gm, rdiv(ph, uh[0]));
#endif
}

// set_collisional for col_type 1..6 (PIP_rot.f90:44-97) on one cell: rewrites the energies
// (get_te) and returns alpha_c from Te_h + Te_m and the drift of get_vel_diff
// (Scheme_rot.f90:988-999), in the Fortran operation order.
template <int NVM>
__device__ __forceinline__ double set_collisional_cell(double (&um)[NVM], double (&uh)[5],
                                                       const KParams &p) {
  double te_m, te_h, rm, rh;
  get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
  const double gm = p.gm, T = radd(te_h, te_m);
  double a = rmul(p.ac, __dsqrt_rn(rmul(T, 0.5)));
  const int type = p.col_type;
  if (type == 1) return rdiv(a, p.ac_sb);
  if (type == 2) return a;
#if PIP_RCP
  const double vdx = rsub(rmul(uh[1], rh), rmul(um[1], rm));
  const double vdy = rsub(rmul(uh[2], rh), rmul(um[2], rm));
  const double vdz = rsub(rmul(uh[3], rh), rmul(um[3], rm));
#else
  const double vdx = rsub(rdiv(uh[1], uh[0]), rdiv(um[1], um[0]));
  const double vdy = rsub(rdiv(uh[2], uh[0]), rdiv(um[2], um[0]));
  const double vdz = rsub(rdiv(uh[3], uh[0]), rdiv(um[3], um[0]));
#endif
  const double v2 = radd(radd(rmul(vdx, vdx), rmul(vdy, vdy)), rmul(vdz, vdz));
  // 9*pi/64*gm/2*v2/T, left to right
  const double k = rdiv(rmul(rmul(rmul(rmul(rmul(9.0, kPiRef), 0.015625), gm), 0.5), v2), T);
  a = rmul(a, __dsqrt_rn(radd(1.0, k)));
  if (type == 3) return rdiv(a, p.ac_sb);
  if (type == 4) return a;
  const double w = rmul(rmul(rmul(gm, kPiRef), 0.0625), v2);       // gm*pi/16*v2
  if (type == 5)
    return rmul(rdiv(a, p.ac_sb), pow(radd(rmul(rdiv(p.ac_b2g, T), 0.5), w), 0.125));
  return rdiv(a, pow(radd(rmul(T, 0.5), w), 0.125));
}

// set_IR types 1, 2 and 3 (PIP_rot.f90:134-228) for one cell from the ion density ro and the
// temperature te of get_Te_MHD, in the Fortran operation order (constants from the host).
__device__ __forceinline__ void ir_law_rates(const KParams &p, double ro, double te, double &gr,
                                              double &gi) {
  if (p.irf) {
    gr = rmul(rmul(rmul(pow(te, -0.5), rmul(ro, ro)), p.ir_recfac), p.ir_ionfac);
    gi = rmul(rmul(rmul(pow(te, 0.5), ro), pow(p.ir_factor, rdiv(1.0, te))), p.ir_ionfac);
  } else if (p.irs == 2) {
    const double a = rdiv(p.ir_c136, te);
    gr = rmul(rdiv(ro, __dsqrt_rn(te)), p.ir_recfac);
    gi = rmul(rdiv(rmul(rmul(rmul(rmul(p.ir_n6, ro), p.ir_c291), exp(-a)), pow(a, 0.39)),
                   radd(0.232, a)),
              p.ir_tir);
  } else {
    const double b = rmul(rdiv(p.ir_c136, te), p.ir_tfac);
    gr = rmul(rdiv(rmul(rdiv(ro, __dsqrt_rn(te)), p.ir_tir), p.ir_fp), p.ir_sqtfac);
    const double g = rmul(rmul(rmul(p.ir_c291n6, ro), exp(-b)), pow(b, 0.39));
    gi = rmul(rdiv(rdiv(rdiv(g, radd(0.232, b)), p.ir_recfac), p.ir_fp), p.ir_tir);
  }
}

// set_IR of types 1-3 on one cell: get_Te's energy rewrite, then the rates.
template <int NVM>
__device__ __forceinline__ void set_ir_cell(double (&um)[NVM], double (&uh)[5], const KParams &p,
                                            double &gr, double &gi) {
  double te_m, te_h, rm, rh;
  get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
  if (p.irn) {   // type 4: the rates come from nlev_rates_kernel (irg)
    gr = 0.0;
    gi = 0.0;
    return;
  }
  ir_law_rates(p, um[0], te_m, gr, gi);
}

// Collisional exchange dS of source_PIP (PIP_rot.f90:1333-1368) for one cell from the
// rewritten states um/uh, their primitives and the cell's alpha_c.
template <int NVM>
__device__ __forceinline__ void collision_ds(const double (&um)[NVM], const double (&uh)[5],
                                             const Prim<double> &qm, const Prim<double> &qh,
                                             const KParams &p, double ac, double dt_coll,
                                             double (&ds)[5]) {
  const double gm = p.gm;
  const double te = qm.pr / qm.de * gm * kMuP;
  const double nte = qh.pr / qh.de * gm * kMuN;
  ds[0] = 0.0;
  if (p.imp) {
    const double temp = dt_coll * (uh[0] + um[0]);
    const double e = (1.0 - exp(-ac * temp));
    ds[1] = (um[0] * uh[1] - uh[0] * um[1]) * e / temp;
    ds[2] = (um[0] * uh[2] - uh[0] * um[2]) * e / temp;
    ds[3] = (um[0] * uh[3] - uh[0] * um[3]) * e / temp;
    const double nde = qh.de, de = qm.de;
    const double lambda = ac * (nde + de);
    const double kap = 3.0 * (gm - 1.0) * ac * (kMuP * nde + kMuN * de);
    const double dvx = qh.vx - qm.vx, dvy = qh.vy - qm.vy, dvz = qh.vz - qm.vz;
    // the ion term multiplies (nvz-vz) by nvz, as PIP_rot.f90:1348 does
    const double B = -(1.0 / 3.0 * gm * kap / ((nde + de) * (kap - lambda)) *
                       (de * (dvx * qm.vx + dvy * qm.vy + dvz * qh.vz) +
                        nde * (dvx * qh.vx + dvy * qh.vy + dvz * qh.vz)));
    const double D = -(gm / 6.0 * kap * (de - nde) / ((de + nde) * (kap - 2.0 * lambda)) *
                       (dvx * dvx + dvy * dvy + dvz * dvz));
    ds[4] = -((3.0 / gm) * ac * de * nde / kap *
              (+(exp(-kap * dt_coll) - 1.0) * (nte - te) - (B + D) * exp(-kap * dt_coll) +
               B * exp(-lambda * dt_coll) + D * exp(-2.0 * lambda * dt_coll)) /
              dt_coll);
  } else {
    ds[1] = ac * (um[0] * uh[1] - uh[0] * um[1]);
    ds[2] = ac * (um[0] * uh[2] - uh[0] * um[2]);
    ds[3] = ac * (um[0] * uh[3] - uh[0] * um[3]);
    ds[4] = ac * qh.de * qm.de *
            (0.5 * ((qh.vx * qh.vx - qm.vx * qm.vx) + (qh.vy * qh.vy - qm.vy * qm.vy) +
                    (qh.vz * qh.vz - qm.vz * qm.vz)) +
             3.0 / gm / 2.0 * (nte - te));
  }
}

// IR exchange of source_PIP (PIP_rot.f90:1370-1411, flag_IR_type 0, 1 or 2; 0 has type 1's
// energy term, its ionisation potential is added by the caller).
__device__ __forceinline__ void ir_ds(const Prim<double> &qm, const Prim<double> &qh, double gr,
                                      double gi, const KParams &p, double (&ds)[5]) {
  const double gm = p.gm;
  ds[0] = gr * qm.de - gi * qh.de;
  ds[1] = gr * qm.de * qm.vx - gi * qh.de * qh.vx;
  ds[2] = gr * qm.de * qm.vy - gi * qh.de * qh.vy;
  ds[3] = gr * qm.de * qm.vz - gi * qh.de * qh.vz;
  const double kin = 0.5 * (gr * qm.de * (qm.vx * qm.vx + qm.vy * qm.vy + qm.vz * qm.vz) -
                            gi * qh.de * (qh.vx * qh.vx + qh.vy * qh.vy + qh.vz * qh.vz));
  if (p.ir_type != 2)
    ds[4] = kin - gi * qh.pr / (gm - 1.0) + 0.5 * gr * qm.pr / (gm - 1.0);
  else
    ds[4] = kin - gi * qh.pr / (gm - 1.0) + gr * qm.pr / (gm - 1.0);
}

// Splits a cell's NV planes into ion and neutral arrays.
template <int NVM>
__device__ __forceinline__ void load_cell(const double *__restrict__ U, long long q, long long nc,
                                          double (&um)[NVM], double (&uh)[5]) {
#pragma unroll
  for (int n = 0; n < NVM; ++n) um[n] = U[q + n * nc];
#pragma unroll
  for (int n = 0; n < 5; ++n) uh[n] = U[q + (NVM + n) * nc];
}

// Ghost images of one updated cell (PIPbnd after the stage: x faces first, then y faces,
// Boundary_rot.f90:54-125 order, so a corner ghost carries both sign flips).  Only cells
// within 2*margin of a boundary can be a ghost source; the values are re-read from the
// planes the same thread has just written.
template <int NDIM>
__device__ __forceinline__ bool near_boundary(const KParams &p, int gi, int gj) {
  return gi < 2 * p.m0 || gi >= p.ix - 2 * p.m0 ||
         (NDIM == 2 && (gj < 2 * p.m1 || gj >= p.jx - 2 * p.m1));
}

template <int NDIM>
__device__ __forceinline__ void write_ghosts(const KParams &p, int gi, int gj, double *U, int nplanes,
                                             bool unsigned_plane = false) {
  const long long nc = p.nc;
  const long long q = (long long)gj * p.ix + gi;
  int tx[2 * kMaxMargin], sx[2 * kMaxMargin], ntx = 0;
  int ty[2 * kMaxMargin], sy[2 * kMaxMargin], nty = 0;
  for (int s = 0; s < 2; ++s)
    for (int l = 0; l < p.m0; ++l)
      if (p.gx[s][l] == gi) {
        tx[ntx] = s == 0 ? l : p.ix - p.m0 + l;
        sx[ntx++] = s;
      }
  if (NDIM == 2)
    for (int s = 0; s < 2; ++s)
      for (int l = 0; l < p.m1; ++l)
        if (p.gy[s][l] == gj) {
          ty[nty] = s == 0 ? l : p.jx - p.m1 + l;
          sy[nty++] = s;
        }
#pragma unroll 1
  for (int n = 0; n < nplanes; ++n) {
    const double v = U[q + n * nc];
    for (int a = 0; a < ntx; ++a) {
      if (unsigned_plane) {
        U[(long long)gj * p.ix + tx[a] + n * nc] = v;
        for (int b = 0; b < nty; ++b) U[(long long)ty[b] * p.ix + tx[a] + n * nc] = v;
        continue;
      }
      const double g = (double)p.symx[sx[a]][n];
      U[(long long)gj * p.ix + tx[a] + n * nc] = g * v;
      for (int b = 0; b < nty; ++b)
        U[(long long)ty[b] * p.ix + tx[a] + n * nc] = (double)p.symy[sy[b]][n] * (g * v);
    }
    for (int b = 0; b < nty; ++b)
      U[(long long)ty[b] * p.ix + gi + n * nc] = unsigned_plane ? v : (double)p.symy[sy[b]][n] * v;
  }
}

// Writes a cell and its ghost images.
template <int NDIM, int NVM>
__device__ __forceinline__ void store_cell(double *U, const KParams &p, int gi, int gj,
                                           const double (&um)[NVM], const double (&uh)[5]) {
  const long long nc = p.nc;
  const long long q = (long long)gj * p.ix + gi;
#pragma unroll
  for (int n = 0; n < NVM; ++n) U[q + n * nc] = um[n];
#pragma unroll
  for (int n = 0; n < 5; ++n) U[q + (NVM + n) * nc] = uh[n];
  if (near_boundary<NDIM>(p, gi, gj)) write_ghosts<NDIM>(p, gi, gj, U, NVM + 5);
}

// Block-wide min/max into the reduction slots (one atomic per block).
template <int NT>
__device__ __forceinline__ void block_reduce_cfl(double dtc, double rho, double gr, DevCtrl *ctrl,
                                                 int slot) {
  __shared__ double s_red[3][NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
    rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
    gr = fmax(gr, __shfl_xor_sync(0xffffffffu, gr, o));
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) {
    s_red[0][w] = dtc;
    s_red[1][w] = rho;
    s_red[2][w] = gr;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < NT / 32; ++k) {
      dtc = fmin(dtc, s_red[0][k]);
      rho = fmax(rho, s_red[1][k]);
      gr = fmax(gr, s_red[2][k]);
    }
    // all values are positive (or +0), so the bit patterns order like the doubles
    atomicMin(&ctrl->red_dt[slot], dbits(dtc));
    atomicMax(&ctrl->red_rho[slot], dbits(rho));
    atomicMax(&ctrl->red_gr[slot], dbits(gr));
  }
}

// E = eta*curl B of one cell (get_rotation's s_order-2 branch, Util_rot.f90:148-236, and
// resistive_flux's ex, ey, ez, Solver_rot.f90:597-599) from the field planes bx, by, bz
// with row stride sy; gi, gj the cell's global indices (never on the outermost layer).
//
// With resi 2 the cell's eta is set_resistivity's (Res_rot.f90:37-60) from this curl B and
// the ion density ro[c]: resi_type 2 11 eta_0 where |curl B| >= j_cri, else eta_0;
// resi_type 3 eta_0 (vd/vd_cri - 1)**2 where vd = |curl B|/rho_i >= vd_cri, else 0.  The
// cell's eta is returned in eta.
template <int NDIM>
__device__ __forceinline__ void cell_e(const double *bx, const double *by, const double *bz,
                                       const double *ro, long long c, long long sy,
                                       const KParams &p, int gi, int gj, double &ex, double &ey,
                                       double &ez, double &eta) {
  double r1 = 0.0, r2, r3;
#if PIP_RCP
  // the FMA build multiplies by 1/(2 dx), 1/(2 dy)
  const double rx = 1.0 / (2.0 * p.dx[gi]);
  r2 = -((bz[c + 1] - bz[c - 1]) * rx);
  if (NDIM == 2) {
    const double ry = 1.0 / (2.0 * p.dy[gj]);
    r1 = (bz[c + sy] - bz[c - sy]) * ry;
    r3 = (by[c + 1] - by[c - 1]) * rx - (bx[c + sy] - bx[c - sy]) * ry;
  } else {
    r3 = (by[c + 1] - by[c - 1]) * rx;
  }
#else
  const double dx2 = 2.0 * p.dx[gi];
  r2 = -((bz[c + 1] - bz[c - 1]) / dx2);
  if (NDIM == 2) {
    const double dy2 = 2.0 * p.dy[gj];
    r1 = (bz[c + sy] - bz[c - sy]) / dy2;
    r3 = (by[c + 1] - by[c - 1]) / dx2 - (bx[c + sy] - bx[c - sy]) / dy2;
  } else {
    r3 = (by[c + 1] - by[c - 1]) / dx2;
  }
#endif
  if (p.resi == 2) {
    const double c2 = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    if (p.resi_type == 2) {
      eta = c2 >= p.j_cri ? p.eta0 * 11.0 : p.eta0;
    } else {
      const double vd = c2 / ro[c];
      const double a = vd / p.vd_cri - 1.0;
      eta = vd >= p.vd_cri ? p.eta0 * (a * a) : 0.0;
    }
  } else {
    eta = p.etaf[(long long)gj * p.ix + gi];
  }
  ex = r1 * eta;
  ey = r2 * eta;
  ez = r3 * eta;
}

// resistive_flux's face terms (Solver_rot.f90:601-636, flag_sch=0 branch) added to the MHD
// flux F (stride nf) of a face from E of its two cells (0: left/lower, 1: right/upper) and
// B there.
__device__ __forceinline__ void face_terms(double *F, long long nf, long long fo, bool ydir,
                                           double ex0, double ey0, double ez0, double ex1,
                                           double ey1, double ez1, double bx0, double bx1,
                                           double by0, double by1, double bz0, double bz1) {
  if (!ydir) {
    F[4 * nf + fo] = F[4 * nf + fo] + 0.25 * ((ey1 + ey0) * (bz0 + bz1) - (ez0 + ez1) * (by0 + by1));
    F[6 * nf + fo] = F[6 * nf + fo] - 0.5 * (ez0 + ez1);
    F[7 * nf + fo] = F[7 * nf + fo] + 0.5 * (ey0 + ey1);
  } else {
    F[4 * nf + fo] = F[4 * nf + fo] + 0.25 * ((ez1 + ez0) * (bx0 + bx1) - (ex0 + ex1) * (bz0 + bz1));
    F[5 * nf + fo] = F[5 * nf + fo] + 0.5 * (ez0 + ez1);
    F[7 * nf + fo] = F[7 * nf + fo] - 0.5 * (ex0 + ex1);
  }
}

// The face terms of the face between cells c0 and c1 = c0 + (x: 1, y: sy) of the field
// planes, E computed at both cells (the unit-level flux kernel; ro the ion density plane).
template <int NDIM>
__device__ __forceinline__ void add_resistive(double *F, long long nf, long long fo, bool ydir,
                                              const double *bx, const double *by, const double *bz,
                                              const double *ro, long long c0, long long sy,
                                              const KParams &p, int gi, int gj) {
  double ex0, ey0, ez0, ex1, ey1, ez1, e0, e1;
  const long long c1 = ydir ? c0 + sy : c0 + 1;
  cell_e<NDIM>(bx, by, bz, ro, c0, sy, p, gi, gj, ex0, ey0, ez0, e0);
  cell_e<NDIM>(bx, by, bz, ro, c1, sy, p, ydir ? gi : gi + 1, ydir ? gj + 1 : gj, ex1, ey1, ez1,
               e1);
  face_terms(F, nf, fo, ydir, ex0, ey0, ez0, ex1, ey1, ez1, bx[c0], bx[c1], by[c0], by[c1], bz[c0],
             bz[c1]);
}

// alpha_c of the ghost cells that the halo exchange filled (faces whose source is -1),
// from the stage-2 input state there, as set_collisional computes it on every cell after
// mpi_bnd.  The tiles along such a face take its ghost layers over their columns (rows in
// 1D), the edge tiles also the corner cells; the ranges of the tiles are disjoint.
template <int NDIM, int NVM, int TX, int TY, int NT>
__device__ void exchanged_ghost_ac(const KParams &p, const double *__restrict__ Us, int i0, int j0,
                                   int tid, int by, int nby) {
  const bool first_x = blockIdx.x == 0, last_x = blockIdx.x == gridDim.x - 1;
  const bool first_y = by == 0, last_y = by == nby - 1;
  const bool lo_x = first_x && p.gx[0][0] < 0, hi_x = last_x && p.gx[1][0] < 0;
  const bool lo_y = NDIM == 2 && first_y && p.gy[0][0] < 0;
  const bool hi_y = NDIM == 2 && last_y && p.gy[1][0] < 0;
  if (!(lo_x || hi_x || lo_y || hi_y)) return;
  const int ca = first_x ? 0 : i0;
  const int cb = last_x ? p.ix : i0 + TX;
  const int ra = NDIM == 2 ? (first_y ? 0 : j0) : 0;
  const int rb = NDIM == 2 ? (last_y ? p.jx : j0 + TY) : 1;
  const int w = cb - ca, n = w * (rb - ra);
  for (int t = tid; t < n; t += NT) {
    const int i = ca + t % w, j = ra + t / w;
    const bool ghost = (lo_x && i < p.m0) || (hi_x && i >= p.ix - p.m0) ||
                       (lo_y && j < p.m1) || (hi_y && j >= p.jx - p.m1);
    if (!ghost) continue;
    const long long q = (long long)j * p.ix + i;
    double um[NVM], uh[5];
    load_cell<NVM>(Us, q, p.nc, um, uh);
    p.acf[q] = set_collisional_cell<NVM>(um, uh, p);
  }
}

// One RK stage of run_solver (Solver_rot.f90:59-71) fused into one kernel per tile:
// u2v + get_Side minmod + HLLD/HLLC for every face of the tile (set_flux), the
// collisional/IR source (set_source), add_flux_rk + add_source + Dedner decay
// (time_integral) and the ghost fill (PIPbnd).  STAGE 2 optionally fuses the two cfl
// calls that follow run_solver and open the next step (main.f90:47 and :36): epi = 1
// applies one cq2pv rewrite; epi = 2 applies two and reduces the next dt; epi = -1 takes
// 1 or 2 from the control block's last-step flag.  X selects the extra physics of the
// instance: bit 0 set_coefficients at every stage (alpha_c per cell, col_type >= 1, and/or
// the Popescu IR rates), bit 1 resistivity; each combination is its own instance so that
// the others keep their register budget.
// Minimum of v over the block, taken into *dst (ordered bits of positive doubles) by one
// atomic per block.  Every thread of the block calls it.
template <int NT>
__device__ __forceinline__ void block_min_to(double v, unsigned long long *dst) {
  __shared__ double s_min[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (threadIdx.x % 32 == 0) s_min[threadIdx.x / 32] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < NT / 32; ++k) v = fmin(v, s_min[k]);
    atomicMin(dst, dbits(v));
  }
}

template <int NDIM, int NVM, int STAGE, int X>
__global__ void __launch_bounds__(Tile<NDIM>::NT, NDIM == 2 ? 2 : 4)
stage_kernel(const __grid_constant__ KParams p, const double *__restrict__ Us, const double *U0,
             double *Uo, DevCtrl *ctrl, int dt_mode, int epi,
             const __grid_constant__ CUtensorMap tmap, int use_tma, int rows) {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY, NT = Tile<NDIM>::NT;
  constexpr int NV = NVM + 5;
  constexpr int RX = TX + 2 * kH, RY = NDIM == 2 ? TY + 2 * kH : 1, RR = RX * RY;
  constexpr int NFX = (TX + 1) * TY, NFY = NDIM == 2 ? TX * (TY + 1) : 0;
  constexpr int EW = TX + 2, EH = NDIM == 2 ? TY + 2 : 1, EN = EW * EH;
  extern __shared__ __align__(128) double smem[];
  double *sV = smem;                 // first: the TMA destination (128-byte aligned)
  double *sFx = sV + NV * RR;
  double *sFy = sFx + NV * NFX;
  constexpr bool COL = (X & 1) != 0, RES = (X & 2) != 0;
  double *sE = sFy + NV * NFY;  // RES only: E of the tile's cells and one ring
  __shared__ double s_dt, s_cmax;
  __shared__ long long s_step;
  __shared__ int s_exit, s_epi;
  __shared__ __align__(8) unsigned long long s_bar;

  const int tid = threadIdx.x;
  // tile row of this CTA: every row (rows 0), the first and the last (1: the rows a halo
  // exchange sends, launched first), or the rows between them (2)
  const int nby = NDIM == 2 ? (p.ny + TY - 1) / TY : 1;
  const int by = NDIM == 1 || rows == 0 ? (int)blockIdx.y
                 : rows == 1 ? (blockIdx.y == 0 ? 0 : nby - 1) : (int)blockIdx.y + 1;
  const bool block0 = blockIdx.x == 0 && by == 0;
  if (tid == 0) {
    int ex = 0;
    if (STAGE == 1) {
      if (ctrl->done || ctrl->nan_flag) ex = 1;
    } else {
      if (ctrl->done) ex = 1;
    }
    double dt, cmax;
    if (STAGE == 1 && dt_mode == 1) {
      const long long st = ctrl->step;
      dt = finalize_dt(p, ctrl, (int)(st & 1));
      cmax = p.sg_all / dt;
    } else {
      dt = ctrl->dt;
      cmax = ctrl->cmax;
    }
    s_dt = dt;
    s_cmax = cmax;
    s_step = ctrl->step;
    s_exit = ex;
    s_epi = (STAGE == 2 && epi < 0) ? (ctrl->last ? 1 : 2) : epi;
  }
  __syncthreads();
  if (s_exit) {
    if (STAGE == 1 && block0 && tid == 0) {
      if (ctrl->nan_flag && ctrl->status == 0) ctrl->status = 3;  // PIP_ERR_NAN
      ctrl->done = 1;
    }
    return;
  }
  const double dt = s_dt, cmax = s_cmax;
  if (STAGE == 1 && dt_mode == 1 && block0 && tid == 0) {
    // loop bookkeeping of main.f90:31,58 for this step
    const long long st = ctrl->step;
    ctrl->dt = dt;
    ctrl->cmax = cmax;
    const double tn = ctrl->time + dt;
    ctrl->time_next = tn;
    ctrl->last = ((ctrl->t_end > 0.0 && tn >= ctrl->t_end) ||
                  (ctrl->nsteps > 0 && st + 1 >= ctrl->nsteps)) ? 1 : 0;
    const int ns = (int)((st + 1) & 1);
    ctrl->red_dt[ns] = dbits(fmin(10.0, p.resi_dt));  // cfl_mhd's start, cfl_resi's bound
    ctrl->red_rho[ns] = 0ull;
    ctrl->red_gr[ns] = 0ull;
    ctrl->red_ip[ns] = 0ull;
    ctrl->red_nx[ns] = 0ull;
  }

  if (STAGE == 1 && RES && p.resi == 2 && block0 && tid == 0) {
    // stage 2 takes the minimum of cfl_resi's bound into this word; no kernel reads it
    // between the stages
    *p.resi_bound = dbits(INFINITY);
  }

  const double gm = p.gm, ro_lim = p.ro_lim, pr_lim = p.pr_lim;
  const int i0 = p.m0 + blockIdx.x * TX;
  const int j0 = NDIM == 2 ? p.m1 + by * TY : 0;
  const long long nc = p.nc;

  // ---- 1. stage state of the tile and its halo -> primitives in shared memory
  if (NDIM == 2 && use_tma && (tma_smem_addr(sV) & 127u) == 0) {
    // all planes of the tile and its halo by one TMA load into sV (cells outside the array
    // read as zero), then the primitives in place, each thread on its own cells
    if (tid == 0) {
      tma_bar_init(&s_bar);
      tma_bar_expect(&s_bar, (uint32_t)(NV * RR * sizeof(double)));
      tma_load_tile(sV, &tmap, i0 - kH, j0 - kH, &s_bar);
    }
    __syncthreads();
    if (!tma_bar_wait(&s_bar, kTmaWaitLimit)) {
      // the tile did not arrive: flag the stage (the run stops with PIP_ERR_ITER; this
      // tile's results are void) and let the copy land (bounded) before going on, so that
      // no copy is in flight when the CTA's shared memory is released
      atomicCAS(&ctrl->status, 0, 5);
      ctrl->done = 1;
      tma_bar_wait(&s_bar, kTmaWaitLimit);
    }
    for (int idx = tid; idx < RR; idx += NT) {
      const int ri = idx % RX, rj = idx / RX;
      if (!RES && (ri < kH || ri >= TX + kH) && (rj < kH || rj >= TY + kH)) continue;
      const int gi = i0 - kH + ri, gj = j0 - kH + rj;
      if (gi >= p.ix || gj >= p.jx) continue;
      double um[NVM], uh[5], vm[NVM], vh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) um[n] = sV[n * RR + idx];
#pragma unroll
      for (int n = 0; n < 5; ++n) uh[n] = sV[(NVM + n) * RR + idx];
      if (COL) {
        double te_m, te_h, rm, rh;
        if (p.col_type) get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
        if (p.irs) get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
      }
      u2v_mhd<double, NVM>(um, vm, gm, ro_lim, pr_lim);
      u2v_hd<double>(uh, vh, gm, ro_lim, pr_lim);
#pragma unroll
      for (int n = 0; n < NVM; ++n) sV[n * RR + idx] = vm[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) sV[(NVM + n) * RR + idx] = vh[n];
    }
  } else
  for (int idx = tid; idx < RR; idx += NT) {
    const int ri = idx % RX, rj = idx / RX;
    // the corners only for the curl of B next to the tile's corner faces (resistivity)
    if (NDIM == 2 && !RES && (ri < kH || ri >= TX + kH) && (rj < kH || rj >= TY + kH))
      continue;
    const int gi = i0 - kH + ri, gj = NDIM == 2 ? j0 - kH + rj : 0;
    if (gi >= p.ix || gj >= p.jx) continue;
    double um[NVM], uh[5], vm[NVM], vh[5];
    load_cell<NVM>(Us, (long long)gj * p.ix + gi, nc, um, uh);
    if (COL) {
      // set_coefficients (Solver_rot.f90:62) rewrites the energies before set_flux: in
      // set_collisional and again in set_IR
      double te_m, te_h, rm, rh;
      if (p.col_type) get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
      if (p.irs) get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
    }
    u2v_mhd<double, NVM>(um, vm, gm, ro_lim, pr_lim);
    u2v_hd<double>(uh, vh, gm, ro_lim, pr_lim);
#pragma unroll
    for (int n = 0; n < NVM; ++n) sV[n * RR + idx] = vm[n];
#pragma unroll
    for (int n = 0; n < 5; ++n) sV[(NVM + n) * RR + idx] = vh[n];
  }
  __syncthreads();
  // resi 2, stage 2: cfl_resi's bound over this tile's interior cells with the eta of this
  // stage (the last set_resistivity before the next cfl)
  double rb = INFINITY;
  if (RES) {
    // E = eta*curl B once per cell of the tile and its first ring (each enters four faces)
    const int iend_ = p.m0 + p.nx, jend_ = NDIM == 2 ? p.m1 + p.ny : 1;
    for (int idx = tid; idx < EN; idx += NT) {
      const int er = idx % EW, ej = idx / EW;
      const int gi = i0 - 1 + er, gj = NDIM == 2 ? j0 - 1 + ej : 0;
      if (gi > p.ix - 2 || (NDIM == 2 && gj > p.jx - 2)) continue;
      const int c = (NDIM == 2 ? (ej + kH - 1) * RX : 0) + er + kH - 1;
      double ex, ey, ez, eta;
      cell_e<NDIM>(sV + 5 * RR, sV + 6 * RR, sV + 7 * RR, sV, c, RX, p, gi, gj, ex, ey, ez, eta);
      sE[idx] = ex;
      sE[EN + idx] = ey;
      sE[2 * EN + idx] = ez;
      if (STAGE == 2 && p.resi == 2 && er >= 1 && er <= TX && gi < iend_ &&
          (NDIM == 1 || (ej >= 1 && ej <= TY && gj < jend_))) {
        const double gmin = fmin(fmin(p.dx[gi], NDIM == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
        rb = fmin(rb, p.safety * (gmin * gmin) / fmax(eta, 1.0e-8));
      }
    }
    if (STAGE == 2 && p.resi == 2) block_min_to<NT>(rb, p.resi_bound);
    __syncthreads();
  }

  // ---- 2. face fluxes (set_flux): x faces then y faces of the tile
  const int iend = p.m0 + p.nx, jend = NDIM == 2 ? p.m1 + p.ny : 1;
  for (int f = tid; f < NFX + NFY; f += NT) {
    int a, s, perm_y;
    double *Fout;
    int fo, nf;
    if (f < NFX) {
      const int fi = f % (TX + 1), fj = f / (TX + 1);
      if (i0 + fi - 1 >= iend || (NDIM == 2 && j0 + fj >= jend)) continue;
      a = (NDIM == 2 ? (fj + kH) * RX : 0) + fi + kH - 1;  // left cell of the face
      s = 1;
      perm_y = 0;
      Fout = sFx;
      fo = f;
      nf = NFX;
    } else {
      const int g = f - NFX, fi = g % TX, fj = g / TX;
      if (i0 + fi >= iend || j0 + fj - 1 >= jend) continue;
      a = (fj + kH - 1) * RX + fi + kH;  // lower cell of the face
      s = RX;
      perm_y = 1;
      Fout = sFy;
      fo = g;
      nf = NFY;
    }
    {
      double vl[NVM], vr[NVM], fx[NVM];
#pragma unroll
      for (int n = 0; n < NVM; ++n) {
        // direction 2 swaps (vx,vy) and (bx,by) (set_HLLD_fluxes, HLL_rot.f90:365-383)
        const int src = perm_y ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        const double *v = sV + src * RR + a;
        const double v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
        vl[n] = v1 + 0.5 * minmod<double>(v0, v1, v2);
        vr[n] = v2 - 0.5 * minmod<double>(v1, v2, v3);
      }
      vl[0] = fmax(vl[0], ro_lim);
      vr[0] = fmax(vr[0], ro_lim);
      riemann_mhd<NVM>(vl, vr, fx, p, cmax);
#pragma unroll
      for (int n = 0; n < NVM; ++n) {
        const int dst = perm_y ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        Fout[dst * nf + fo] = fx[n];
      }
    }
    {
      double vl[5], vr[5], fx[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        const int src = perm_y ? (n == 1 ? 2 : n == 2 ? 1 : n) : n;
        const double *v = sV + (NVM + src) * RR + a;
        const double v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
        vl[n] = v1 + 0.5 * minmod<double>(v0, v1, v2);
        vr[n] = v2 - 0.5 * minmod<double>(v1, v2, v3);
      }
      vl[0] = fmax(vl[0], ro_lim);
      vr[0] = fmax(vr[0], ro_lim);
      riemann_hd(vl, vr, fx, p);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        const int dst = perm_y ? (n == 1 ? 2 : n == 2 ? 1 : n) : n;
        Fout[(NVM + dst) * nf + fo] = fx[n];
      }
    }
  }
  if (RES) {
    // resistive_flux's terms, added by the thread that wrote the face's flux (same faces
    // per thread as above), in a loop of their own to keep the Riemann solvers' registers
    for (int f = tid; f < NFX + NFY; f += NT) {
      int a, s, nf, fo, e0, e1;
      double *Fout;
      const bool ydir = f >= NFX;
      if (!ydir) {
        const int fi = f % (TX + 1), fj = f / (TX + 1);
        if (i0 + fi - 1 >= iend || (NDIM == 2 && j0 + fj >= jend)) continue;
        a = (NDIM == 2 ? (fj + kH) * RX : 0) + fi + kH - 1;
        s = 1;
        Fout = sFx;
        fo = f;
        nf = NFX;
        e0 = (NDIM == 2 ? (fj + 1) * EW : 0) + fi;
        e1 = e0 + 1;
      } else {
        const int g = f - NFX, fi = g % TX, fj = g / TX;
        if (i0 + fi >= iend || j0 + fj - 1 >= jend) continue;
        a = (fj + kH - 1) * RX + fi + kH;
        s = RX;
        Fout = sFy;
        fo = g;
        nf = NFY;
        e0 = fj * EW + fi + 1;
        e1 = e0 + EW;
      }
      const int a1 = a + s;
      const double *bx = sV + 5 * RR, *by = sV + 6 * RR, *bz = sV + 7 * RR;
      face_terms(Fout, nf, fo, ydir, sE[e0], sE[EN + e0], sE[2 * EN + e0], sE[e1], sE[EN + e1],
                 sE[2 * EN + e1], bx[a], bx[a1], by[a], by[a1], bz[a], bz[a1]);
    }
  }
  __syncthreads();

  // ---- 3. per-cell source, update, epilogue
  const int ti = tid % TX, tj = tid / TX;
  const int gi = i0 + ti, gj = j0 + tj;
  const bool valid = tj < TY && gi < iend && (NDIM == 1 || gj < jend);
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  if (valid) {
    const long long q = (long long)gj * p.ix + gi;
    const double dt_sub = STAGE == 1 ? dt / 2.0 : dt / 1.0;  // dt/(t_order-istep+1)
    const double dt_coll = dt * 0.5;                          // set_dt_coll, t_order=2
    double a_m[NVM], a_h[5];  // U0 of the cell
    load_cell<NVM>(U0, q, nc, a_m, a_h);
    double s_m[NVM], s_h[5];  // stage state of the cell
    if (STAGE == 1) {
#pragma unroll
      for (int n = 0; n < NVM; ++n) s_m[n] = a_m[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) s_h[n] = a_h[n];
    } else {
      load_cell<NVM>(Us, q, nc, s_m, s_h);
    }
    // alpha_c of the stage (set_coefficients at the stage start; U0 keeps its energies)
    double ac_s = p.ac;
    if (COL && p.col_type) ac_s = set_collisional_cell<NVM>(s_m, s_h, p);
    double gr = 0.0, gion = 0.0;
    if (COL && p.irs) {
      set_ir_cell<NVM>(s_m, s_h, p, gr, gion);  // set_IR of the stage
      if (p.irn) {                              // type 4: nlev_rates_kernel's rates
        gion = p.irg[q];
        gr = p.irg[nc + q];
      }
    } else if (COL && p.irf) {
      gion = p.irg[q];                          // the time loop's last set_IR
      gr = p.irg[nc + q];
    } else if (p.ir) {
      ir_rates<NVM>(a_m, p, gr, gion);
    }

    // exponential form: U0 carries the collision increments of the earlier stages
    if (p.imp && STAGE == 2) {
      double r_m[NVM], r_h[5], ds[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) r_m[n] = a_m[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) r_h[n] = a_h[n];
      double ac_r = p.ac;
      if (COL && p.col_type) ac_r = set_collisional_cell<NVM>(r_m, r_h, p);
      if (COL && p.irs) {
        double g1, g2;
        set_ir_cell<NVM>(r_m, r_h, p, g1, g2);
      }
      const Prim<double> qh = rt_hd(r_h, p);
      const Prim<double> qm = rt_mhd<NVM>(r_m, p);
      collision_ds<NVM>(r_m, r_h, qm, qh, p, ac_r, dt_coll, ds);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        a_h[n] = a_h[n] - dt_coll * ds[n];
        a_m[n] = a_m[n] + dt_coll * ds[n];
      }
    }
    // source_PIP on the stage state (rewrites it through primitives first)
    double S_m[5], S_h[5];
    {
      const Prim<double> qh = rt_hd(s_h, p);
      const Prim<double> qm = rt_mhd<NVM>(s_m, p);
      double ds[5];
      collision_ds<NVM>(s_m, s_h, qm, qh, p, ac_s, dt_coll, ds);
      if (p.imp) {
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          a_h[n] = a_h[n] - dt_coll * ds[n];
          a_m[n] = a_m[n] + dt_coll * ds[n];
          S_h[n] = 0.0;
          S_m[n] = 0.0;
        }
      } else {
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          S_h[n] = 0.0 - ds[n];
          S_m[n] = 0.0 + ds[n];
        }
      }
      if (p.ir) {
        ir_ds(qm, qh, gr, gion, p, ds);
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          S_h[n] = S_h[n] + ds[n];
          S_m[n] = S_m[n] - ds[n];
        }
        // flag_IR_type 0: S_m(5) - ion_pot + arb_heat (0), PIP_rot.f90:1397
        if (p.irn && p.ir_type == 0) S_m[4] = S_m[4] - p.nl_ip[q] + 0.0;
      }
    }
    // time_integral: add_flux_rk (x, then y) and add_source, per species
    const double cx = dt_sub / p.dx[gi];
    const double cy = NDIM == 2 ? dt_sub / p.dy[gj] : 0.0;
    const int fxl = tj * (TX + 1) + ti, fyl = tj * TX + ti;
    double n_m[NVM], n_h[5];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const double u0 = n < NVM ? a_m[n] : a_h[n - NVM];
      double u = u0 - cx * (sFx[n * NFX + fxl + 1] - sFx[n * NFX + fxl]);
      if (NDIM == 2) u = u - cy * (sFy[n * NFY + fyl + TX] - sFy[n * NFY + fyl]);
      if (n < NVM) {
        u = n < 5 ? u + S_m[n] * dt_sub : u + 0.0;
        n_m[n] = u;
      } else {
        n_h[n - NVM] = u + S_h[n - NVM] * dt_sub;
      }
    }
    if (NVM == 9) n_m[NVM - 1] = n_m[NVM - 1] * p.decay[STAGE - 1];

    // fused cfl rewrites (and the next step's CFL terms)
    const int ep = STAGE == 1 ? 0 : s_epi;  // stage 1 is never followed by a cfl
    if (ep >= 1) {
      if (COL && p.irl) {  // the time loop's set_IR before the cfl (main.f90:44-46)
        double g1, g2;
        set_ir_cell<NVM>(n_m, n_h, p, g1, g2);
      }
      const Prim<double> qm = rt_mhd<NVM>(n_m, p);
      const Prim<double> qh = rt_hd(n_h, p);
      (void)qm;
      (void)qh;
    }
    if (ep == 2) {
      if (COL && p.irl) {  // the next step's set_IR (main.f90:32-34): cfl_pip_ir's rates
        double g1, g2;
        set_ir_cell<NVM>(n_m, n_h, p, g1, g2);
        grc = fmax(g1, g2);
        if (p.irf) {       // type 1: the rates of the next step's stages
          p.irg[q] = g2;
          p.irg[nc + q] = g1;
        }
      }
      const Prim<double> qm = rt_mhd<NVM>(n_m, p);
      const Prim<double> qh = rt_hd(n_h, p);
      const double gmin = fmin(fmin(p.dx[gi], NDIM == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
      const double sg = p.safety * gmin;
      dtc = fmin(cfl_mhd_cell<double>(qm, n_m[5], n_m[6], n_m[7], gm, sg),
                 cfl_hd_cell<double>(qh, gm, sg));
      rhoc = fmax(n_m[0] * ac_s, n_h[0] * ac_s);
      if (p.ir && !p.irl) {
        double g1, g2;
        ir_rates<NVM>(n_m, p, g1, g2);
        grc = fmax(g1, g2);
      }
    }
    bool bad = false;
#pragma unroll
    for (int n = 0; n < NVM; ++n) bad |= !isfinite(n_m[n]);
#pragma unroll
    for (int n = 0; n < 5; ++n) bad |= !isfinite(n_h[n]);
    if (bad) atomicOr(&ctrl->nan_flag, 1);
    store_cell<NDIM, NVM>(Uo, p, gi, gj, n_m, n_h);
    if (STAGE == 2 && COL && p.col_type) {
      // the alpha_c field that the next cfl reads (cfl_pn_col, Scheme_rot.f90:305-313)
      p.acf[q] = ac_s;
      if (near_boundary<NDIM>(p, gi, gj)) write_ghosts<NDIM>(p, gi, gj, p.acf, 1, true);
    }
  }
  if (STAGE == 2 && COL && p.col_type) exchanged_ghost_ac<NDIM, NVM, TX, TY, NT>(p, Us, i0, j0, tid, by, nby);
  if (STAGE == 2 && s_epi == 2) {
    if (RES && p.resi == 2) dtc = fmin(dtc, rb);  // the next step's cfl_resi
    block_reduce_cfl<NT>(dtc, rhoc, grc, ctrl, (int)((s_step + 1) & 1));
  }
  if (STAGE == 2 && dt_mode == 1) {
    // end of step, done by the last block to finish (every block has read the control
    // block by then): time += dt and stop_sim's dt check (main.f90:58-66, IO_rot.f90:636)
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      const unsigned int nb = gridDim.x * nby;     // every tile of the stage's launches
      if (atomicAdd(&ctrl->blocks_done, 1u) == nb - 1) {
        __threadfence();
        ctrl->blocks_done = 0u;
        if (RES && p.resi == 2) {
          // the cfl after run_solver lowers the global dt that time advances by to
          // cfl_resi's bound of this stage's eta (main.f90:47,58; Scheme_rot.f90:298)
          const double tn = ctrl->time + fmin(dt, bitsd(atomicOr(p.resi_bound, 0ull)));
          ctrl->time = tn;
          ctrl->last = ((ctrl->t_end > 0.0 && tn >= ctrl->t_end) ||
                        (ctrl->nsteps > 0 && s_step + 1 >= ctrl->nsteps)) ? 1 : 0;
        } else {
          ctrl->time = ctrl->time_next;
        }
        ctrl->step = s_step + 1;
        if (ctrl->last) ctrl->done = 1;
        if (dt <= 1.0e-12) {
          ctrl->done = 1;
          if (ctrl->status == 0) ctrl->status = 4;  // PIP_ERR_DT
        }
      }
    }
  }
}

// cfl (Scheme_rot.f90:183-213) as a standalone pass over every cell: cq2pv rewrite of
// both species in place, CFL candidates of interior cells, rho*alpha_c and IR maxima of all
// cells into reduction slot `slot`.
template <int NVM>
__global__ void __launch_bounds__(256) cfl_kernel(const KParams p, double *U, DevCtrl *ctrl,
                                                  int slot) {
  const double gm = p.gm;
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  // cfl_resi with the eta of the last set_resistivity (resi 2; a fixed field's bound is
  // seeded into the slot by the host)
  if (p.resi == 2 && blockIdx.x == 0 && threadIdx.x == 0) dtc = bitsd(*p.resi_bound);
  const long long nc = p.nc;
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < nc; q += (long long)gridDim.x * 256) {
    double um[NVM], uh[5];
    load_cell<NVM>(U, q, nc, um, uh);
    double gp1 = 0.0, gp2 = 0.0;
    if (p.irl) {                                        // the time loop's set_IR before cfl
      set_ir_cell<NVM>(um, uh, p, gp1, gp2);
      if (p.irf) {
        p.irg[q] = gp2;
        p.irg[nc + q] = gp1;
      }
    }
    const Prim<double> qm = rt_mhd<NVM>(um, p);
    const Prim<double> qh = rt_hd(uh, p);
#pragma unroll
    for (int n = 0; n < 5; ++n) U[q + n * nc] = um[n];
#pragma unroll
    for (int n = 0; n < 5; ++n) U[q + (NVM + n) * nc] = uh[n];
    const int i = (int)(q % p.ix), j = (int)(q / p.ix);
    const bool interior = i >= p.m0 && i < p.ix - p.m0 && j >= p.m1 && j < p.jx - p.m1;
    if (interior) {
      const double gmin = fmin(fmin(p.dx[i], p.dy[j]), p.dz0);
      const double sg = p.safety * gmin;
      dtc = fmin(dtc, fmin(cfl_mhd_cell<double>(qm, um[5], um[6], um[7], gm, sg),
                           cfl_hd_cell<double>(qh, gm, sg)));
    }
    if (!p.col_type) {
      rhoc = fmax(rhoc, fmax(um[0] * p.ac, uh[0] * p.ac));
    } else {
      const double a = p.acf[q];
      rhoc = fmax(rhoc, fmax(um[0] * a, uh[0] * a));
    }
    if (p.irl) {
      grc = fmax(grc, fmax(gp1, gp2));
    } else if (p.ir) {
      double g1, g2;
      ir_rates<NVM>(um, p, g1, g2);
      grc = fmax(grc, fmax(g1, g2));
    }
  }
  block_reduce_cfl<256>(dtc, rhoc, grc, ctrl, slot);
}

// PIPbnd (Boundary_rot.f90:34-125): x ghost columns for every row, then (2D) y ghost rows
// for every column; boundary_control types 1 (periodic), 2 (mirror with sign table) and
// 10 (copy of the first interior layer).  Faces with a neighbouring rank (source -1) are
// left to the halo exchange, as MHDbnd/HDbnd skip faces whose neighbor is not -1.
__global__ void ghosts_x_kernel(const KParams p, double *U, int nplanes) {
  const long long nc = p.nc;
  const int ng = 2 * p.m0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)ng * p.jx;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(t % ng), j = (int)(t / ng);
    const int side = g / p.m0, l = g % p.m0;
    const int dst = side == 0 ? l : p.ix - p.m0 + l;
    const int src = p.gx[side][l];
    if (src < 0) continue;         // face filled by the halo exchange
    for (int n = 0; n < nplanes; ++n) {
      const double v = U[(long long)j * p.ix + src + n * nc];
      U[(long long)j * p.ix + dst + n * nc] = p.typex[side] == 10 ? v : (double)p.symx[side][n] * v;
    }
  }
}

__global__ void ghosts_y_kernel(const KParams p, double *U, int nplanes) {
  const long long nc = p.nc;
  const int ng = 2 * p.m1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)ng * p.ix;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % p.ix), g = (int)(t / p.ix);
    const int side = g / p.m1, l = g % p.m1;
    const int dst = side == 0 ? l : p.jx - p.m1 + l;
    const int src = p.gy[side][l];
    if (src < 0) continue;         // face filled by the halo exchange
    for (int n = 0; n < nplanes; ++n) {
      const double v = U[(long long)src * p.ix + i + n * nc];
      U[(long long)dst * p.ix + i + n * nc] = p.typey[side] == 10 ? v : (double)p.symy[side][n] * v;
    }
  }
}

// set_flux for one direction, faces adjacent to interior cells only; F has NV planes.
template <int NVM>
__global__ void flux_kernel(const KParams p, const double *__restrict__ U, double *F, int dir,
                            double cmax) {
  const double gm = p.gm, ro_lim = p.ro_lim, pr_lim = p.pr_lim;
  const long long nc = p.nc;
  const int ni = dir == 1 ? p.nx + 1 : p.nx;
  const int nj = dir == 1 ? (p.ndim == 2 ? p.ny : 1) : p.ny + 1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)ni * nj;
       t += (long long)gridDim.x * blockDim.x) {
    const int fi = (int)(t % ni), fj = (int)(t / ni);
    int i, j;
    long long s;
    if (dir == 1) {
      i = p.m0 - 1 + fi;
      j = p.ndim == 2 ? p.m1 + fj : 0;
      s = 1;
    } else {
      i = p.m0 + fi;
      j = p.m1 - 1 + fj;
      s = p.ix;
    }
    const long long qa = (long long)j * p.ix + i;
    double V[4][NVM + 5];
    for (int c = 0; c < 4; ++c) {
      double um[NVM], uh[5], vm[NVM], vh[5];
      load_cell<NVM>(U, qa + (c - 1) * s, nc, um, uh);
      u2v_mhd<double, NVM>(um, vm, gm, ro_lim, pr_lim);
      u2v_hd<double>(uh, vh, gm, ro_lim, pr_lim);
      for (int n = 0; n < NVM; ++n) V[c][n] = vm[n];
      for (int n = 0; n < 5; ++n) V[c][NVM + n] = vh[n];
    }
    const bool py = dir == 2;
    {
      double vl[NVM], vr[NVM], fx[NVM];
      for (int n = 0; n < NVM; ++n) {
        const int src = py ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        vl[n] = V[1][src] + 0.5 * minmod<double>(V[0][src], V[1][src], V[2][src]);
        vr[n] = V[2][src] - 0.5 * minmod<double>(V[1][src], V[2][src], V[3][src]);
      }
      vl[0] = fmax(vl[0], ro_lim);
      vr[0] = fmax(vr[0], ro_lim);
      riemann_mhd<NVM>(vl, vr, fx, p, cmax);
      for (int n = 0; n < NVM; ++n) {
        const int dst = py ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        F[qa + dst * nc] = fx[n];
      }
      if (p.resi) {
        if (p.ndim == 2)
          add_resistive<2>(F, nc, qa, py, U + 5 * nc, U + 6 * nc, U + 7 * nc, U, qa, p.ix, p, i, j);
        else
          add_resistive<1>(F, nc, qa, false, U + 5 * nc, U + 6 * nc, U + 7 * nc, U, qa, p.ix, p, i,
                           j);
      }
    }
    {
      double vl[5], vr[5], fx[5];
      for (int n = 0; n < 5; ++n) {
        const int src = NVM + (py ? (n == 1 ? 2 : n == 2 ? 1 : n) : n);
        vl[n] = V[1][src] + 0.5 * minmod<double>(V[0][src], V[1][src], V[2][src]);
        vr[n] = V[2][src] - 0.5 * minmod<double>(V[1][src], V[2][src], V[3][src]);
      }
      vl[0] = fmax(vl[0], ro_lim);
      vr[0] = fmax(vr[0], ro_lim);
      riemann_hd(vl, vr, fx, p);
      for (int n = 0; n < 5; ++n) {
        const int dst = py ? (n == 1 ? 2 : n == 2 ? 1 : n) : n;
        F[qa + (NVM + dst) * nc] = fx[n];
      }
    }
  }
}

// source_PIP over every cell (PIP_rot.f90:1309-1429): rewrites U and writes S (NV planes);
// with the exponential form S receives the U0 increments (-/+ dt_coll*dS).
template <int NVM>
__global__ void source_kernel(const KParams p, double *U, double *S, double dt_coll) {
  const long long nc = p.nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    double um[NVM], uh[5];
    load_cell<NVM>(U, q, nc, um, uh);
    double gr = 0.0, gion = 0.0;
    if (p.irs) {
      set_ir_cell<NVM>(um, uh, p, gr, gion);  // the rates of the state as given
      if (p.irn) {
        gion = p.irg[q];
        gr = p.irg[nc + q];
      }
    } else if (p.irf) {
      gion = p.irg[q];                        // the last set_IR's
      gr = p.irg[nc + q];
    } else if (p.ir) {
      ir_rates<NVM>(um, p, gr, gion);
    }
    const Prim<double> qh = rt_hd(uh, p);
    const Prim<double> qm = rt_mhd<NVM>(um, p);
    double ds[5], sm[5], sh[5];
    collision_ds<NVM>(um, uh, qm, qh, p, p.col_type ? p.acf[q] : p.ac, dt_coll, ds);
    for (int n = 0; n < 5; ++n) {
      if (p.imp) {
        sh[n] = 0.0 - dt_coll * ds[n];
        sm[n] = 0.0 + dt_coll * ds[n];
      } else {
        sh[n] = 0.0 - ds[n];
        sm[n] = 0.0 + ds[n];
      }
    }
    if (p.ir) {
      ir_ds(qm, qh, gr, gion, p, ds);
      for (int n = 0; n < 5; ++n) {
        sh[n] = sh[n] + ds[n];
        sm[n] = sm[n] - ds[n];
      }
      if (p.irn && p.ir_type == 0) sm[4] = sm[4] - p.nl_ip[q] + 0.0;
    }
    for (int n = 0; n < 5; ++n) {
      U[q + n * nc] = um[n];
      U[q + (NVM + n) * nc] = uh[n];
      S[q + n * nc] = sm[n];
      S[q + (NVM + n) * nc] = sh[n];
    }
    for (int n = 5; n < NVM; ++n) S[q + n * nc] = 0.0;
  }
}

// set_coefficients over every cell (Solver_rot.f90:95-122): set_collisional (col_type >= 1,
// alpha_c into p.acf) and set_IR (types 1-3; type 1's rates into p.irg), each rewriting
// both energies in place.
template <int NVM>
__global__ void coefficients_kernel(const KParams p, double *U) {
  const long long nc = p.nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    double um[NVM], uh[5];
    load_cell<NVM>(U, q, nc, um, uh);
    if (p.col_type) p.acf[q] = set_collisional_cell<NVM>(um, uh, p);
    if (p.irl) {
      double g1, g2;
      set_ir_cell<NVM>(um, uh, p, g1, g2);
      if (p.irf) {
        p.irg[q] = g2;
        p.irg[nc + q] = g1;
      }
    }
    U[q + 4 * nc] = um[4];
    U[q + (NVM + 4) * nc] = uh[4];
  }
}

// set_resistivity resi_type 2 or 3 over the state as it stands (the prologue's
// set_coefficients, Initial_rot.f90:140): cfl_resi's bound of that eta over the interior
// cells into *p.resi_bound (set to +inf before by resi_reset_kernel).
template <int NDIM>
__global__ void __launch_bounds__(256) resi_bound_kernel(const KParams p, const double *U) {
  const long long nc = p.nc, n = (long long)p.nx * p.ny;
  double rb = INFINITY;
  for (long long t = blockIdx.x * 256ll + threadIdx.x; t < n; t += (long long)gridDim.x * 256) {
    const int gi = p.m0 + (int)(t % p.nx), gj = p.m1 + (int)(t / p.nx);
    const long long q = (long long)gj * p.ix + gi;
    double ex, ey, ez, eta;
    cell_e<NDIM>(U + 5 * nc, U + 6 * nc, U + 7 * nc, U, q, p.ix, p, gi, gj, ex, ey, ez, eta);
    const double gmin = fmin(fmin(p.dx[gi], NDIM == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
    rb = fmin(rb, p.safety * (gmin * gmin) / fmax(eta, 1.0e-8));
  }
  block_min_to<256>(rb, p.resi_bound);
}
__global__ void resi_reset_kernel(unsigned long long *b) { *b = dbits(INFINITY); }

__global__ void nan_kernel(const double *__restrict__ U, long long n, int *flag) {
  int bad = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(U[t]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

#include "pip_nlevel_impl.cuh"

// ---------------------------------------------------------------- host launchers

template <int NDIM, int NVM, int X>
constexpr size_t stage_smem_bytes() {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY;
  constexpr int RR = (TX + 2 * kH) * (NDIM == 2 ? TY + 2 * kH : 1);
  constexpr int NFX = (TX + 1) * TY, NFY = NDIM == 2 ? TX * (TY + 1) : 0;
  constexpr int EN = (TX + 2) * (NDIM == 2 ? TY + 2 : 1);
  return sizeof(double) * ((NVM + 5) * (RR + NFX + NFY) + ((X & 2) ? 3 * EN : 0));
}

template <int NDIM, int NVM, int STAGE, int X>
static cudaError_t set_stage_attr_x() {
  return cudaFuncSetAttribute(stage_kernel<NDIM, NVM, STAGE, X>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)stage_smem_bytes<NDIM, NVM, X>());
}

template <int NDIM, int NVM, int STAGE>
static cudaError_t set_stage_attr() {
  cudaError_t e;
  if ((e = set_stage_attr_x<NDIM, NVM, STAGE, 0>()) != cudaSuccess) return e;
  if ((e = set_stage_attr_x<NDIM, NVM, STAGE, 1>()) != cudaSuccess) return e;
  if ((e = set_stage_attr_x<NDIM, NVM, STAGE, 2>()) != cudaSuccess) return e;
  return set_stage_attr_x<NDIM, NVM, STAGE, 3>();
}

// Raises the dynamic shared-memory limit of every stage-kernel instance on the current
// device; called once per context so that graph capture sees launches only.
static cudaError_t prepare() {
  cudaError_t e;
  if ((e = set_stage_attr<1, 8, 1>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<1, 8, 2>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<2, 8, 1>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<2, 8, 2>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<2, 9, 1>()) != cudaSuccess) return e;
  return set_stage_attr<2, 9, 2>();
}

template <int NDIM, int NVM, int STAGE>
static cudaError_t launch_stage_t(const KParams &p, const double *Us, const double *U0, double *Uo,
                                  DevCtrl *ctrl, int dt_mode, int epi, cudaStream_t s,
                                  const CUtensorMap *tm, int rows) {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY, NT = Tile<NDIM>::NT;
  const int nby = NDIM == 2 ? (p.ny + TY - 1) / TY : 1;
  if (NDIM == 1) rows = 0;
  const int gy = rows == 0 ? nby : rows == 1 ? (nby < 2 ? nby : 2) : nby - 2;
  if (gy <= 0) return cudaSuccess;   // no rows between the first and the last
  dim3 grid((p.nx + TX - 1) / TX, gy);
  CUtensorMap none;
  std::memset(&none, 0, sizeof none);
  const CUtensorMap &map = tm ? *tm : none;
  const int use = tm ? 1 : 0;
  switch ((p.col_type || p.irl ? 1 : 0) | (p.resi ? 2 : 0)) {
    case 0:
      stage_kernel<NDIM, NVM, STAGE, 0><<<grid, NT, stage_smem_bytes<NDIM, NVM, 0>(), s>>>(
          p, Us, U0, Uo, ctrl, dt_mode, epi, map, use, rows);
      break;
    case 1:
      stage_kernel<NDIM, NVM, STAGE, 1><<<grid, NT, stage_smem_bytes<NDIM, NVM, 1>(), s>>>(
          p, Us, U0, Uo, ctrl, dt_mode, epi, map, use, rows);
      break;
    case 2:
      stage_kernel<NDIM, NVM, STAGE, 2><<<grid, NT, stage_smem_bytes<NDIM, NVM, 2>(), s>>>(
          p, Us, U0, Uo, ctrl, dt_mode, epi, map, use, rows);
      break;
    default:
      stage_kernel<NDIM, NVM, STAGE, 3><<<grid, NT, stage_smem_bytes<NDIM, NVM, 3>(), s>>>(
          p, Us, U0, Uo, ctrl, dt_mode, epi, map, use, rows);
      break;
  }
  return cudaGetLastError();
}

static cudaError_t launch_stage(const KParams &p, int stage, const double *Us, const double *U0,
                                double *Uo, DevCtrl *ctrl, int dt_mode, int epi, cudaStream_t s,
                                const CUtensorMap *tm, int rows) {
  if (p.ndim == 1) {
    return stage == 1 ? launch_stage_t<1, 8, 1>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, nullptr, 0)
                      : launch_stage_t<1, 8, 2>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, nullptr, 0);
  }
  if (p.nvm == 9)
    return stage == 1 ? launch_stage_t<2, 9, 1>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, tm, rows)
                      : launch_stage_t<2, 9, 2>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, tm, rows);
  return stage == 1 ? launch_stage_t<2, 8, 1>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, tm, rows)
                    : launch_stage_t<2, 8, 2>(p, Us, U0, Uo, ctrl, dt_mode, epi, s, tm, rows);
}

static bool tile_map(const KParams &p, const double *U, CUtensorMap *map) {
  if (p.ndim != 2) return false;
  constexpr int TX = Tile<2>::TX, TY = Tile<2>::TY;
  if (!tma_tile_ok(U, p.ix, p.jx, p.nvm + 5, (int)sizeof(double), p.m0 - kH, TX, TX + 2 * kH,
                   TY + 2 * kH))
    return false;
  return tma_encode(map, U, p.ix, p.jx, p.nvm + 5, (int)sizeof(double), TX + 2 * kH, TY + 2 * kH);
}

static int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

static cudaError_t launch_cfl(const KParams &p, double *U, DevCtrl *ctrl, int slot,
                              cudaStream_t s) {
  const int g = grid_for(p.nc, 256);
  if (p.nvm == 9) cfl_kernel<9><<<g, 256, 0, s>>>(p, U, ctrl, slot);
  else cfl_kernel<8><<<g, 256, 0, s>>>(p, U, ctrl, slot);
  return cudaGetLastError();
}

static cudaError_t launch_ghosts(const KParams &p, double *U, cudaStream_t s) {
  const int np = p.nvm + 5;
  ghosts_x_kernel<<<grid_for(2ll * p.m0 * p.jx, 256), 256, 0, s>>>(p, U, np);
  if (p.ndim == 2) ghosts_y_kernel<<<grid_for(2ll * p.m1 * p.ix, 256), 256, 0, s>>>(p, U, np);
  return cudaGetLastError();
}

static cudaError_t launch_flux(const KParams &p, const double *U, double *F, int dir, double cmax,
                               cudaStream_t s) {
  const long long n = (long long)(p.nx + 1) * (p.ndim == 2 ? p.ny + 1 : 1);
  if (p.nvm == 9) flux_kernel<9><<<grid_for(n, 128), 128, 0, s>>>(p, U, F, dir, cmax);
  else flux_kernel<8><<<grid_for(n, 128), 128, 0, s>>>(p, U, F, dir, cmax);
  return cudaGetLastError();
}

static cudaError_t launch_source(const KParams &p, double *U, double *S, double dt_coll,
                                 cudaStream_t s) {
  if (p.nvm == 9) source_kernel<9><<<grid_for(p.nc, 128), 128, 0, s>>>(p, U, S, dt_coll);
  else source_kernel<8><<<grid_for(p.nc, 128), 128, 0, s>>>(p, U, S, dt_coll);
  return cudaGetLastError();
}

static cudaError_t launch_coefficients(const KParams &p, double *U, cudaStream_t s) {
  if (p.resi == 2) {  // set_resistivity comes first in set_coefficients; it reads B and rho
    resi_reset_kernel<<<1, 1, 0, s>>>(p.resi_bound);
    const long long n = (long long)p.nx * p.ny;
    if (p.ndim == 2) resi_bound_kernel<2><<<grid_for(n, 256), 256, 0, s>>>(p, U);
    else resi_bound_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(p, U);
  }
  if (!p.col_type && !p.irl) return cudaGetLastError();
  if (p.nvm == 9) coefficients_kernel<9><<<grid_for(p.nc, 256), 256, 0, s>>>(p, U);
  else coefficients_kernel<8><<<grid_for(p.nc, 256), 256, 0, s>>>(p, U);
  return cudaGetLastError();
}

static cudaError_t launch_nlev_ref(const KParams &p, double *out, cudaStream_t s) {
  nlev_ref_kernel<<<1, 32, 0, s>>>(p, out);
  return cudaGetLastError();
}

static cudaError_t launch_nlev_rates(const KParams &p, const double *U, int colrw, int ipmode,
                                     const double *crref, DevCtrl *ctrl, cudaStream_t s) {
  const int g = grid_for(p.nc, 128);
  if (p.nvm == 9) nlev_rates_kernel<9><<<g, 128, 0, s>>>(p, U, colrw, ipmode, crref, ctrl);
  else nlev_rates_kernel<8><<<g, 128, 0, s>>>(p, U, colrw, ipmode, crref, ctrl);
  return cudaGetLastError();
}

static cudaError_t launch_nlev_update(const KParams &p, const double *U, const DevCtrl *ctrl,
                                      int stage, cudaStream_t s) {
  const int g = grid_for((long long)p.nx * p.ny, 128);
  if (p.ndim == 1) nlev_update_kernel<1, 8><<<g, 128, 0, s>>>(p, U, ctrl, stage);
  else if (p.nvm == 9) nlev_update_kernel<2, 9><<<g, 128, 0, s>>>(p, U, ctrl, stage);
  else nlev_update_kernel<2, 8><<<g, 128, 0, s>>>(p, U, ctrl, stage);
  return cudaGetLastError();
}

static cudaError_t launch_nlev_cfl(const KParams &p, double *U, DevCtrl *ctrl, int slot,
                                   cudaStream_t s) {
  const int g = grid_for(p.nc, 256);
  if (p.ndim == 1) nlev_cfl_kernel<1, 8><<<g, 256, 0, s>>>(p, U, ctrl, slot);
  else if (p.nvm == 9) nlev_cfl_kernel<2, 9><<<g, 256, 0, s>>>(p, U, ctrl, slot);
  else nlev_cfl_kernel<2, 8><<<g, 256, 0, s>>>(p, U, ctrl, slot);
  return cudaGetLastError();
}

static cudaError_t launch_nan(const KParams &p, const double *U, int *flag, cudaStream_t s) {
  const long long n = p.nc * (p.nvm + 5);
  nan_kernel<<<grid_for(n, 256), 256, 0, s>>>(U, n, flag);
  return cudaGetLastError();
}

}  // namespace PIP_FLAVOUR

const Launchers &PIP_LAUNCHERS() {
  static const Launchers L = {PIP_FLAVOUR::prepare,       PIP_FLAVOUR::launch_stage,
                              PIP_FLAVOUR::launch_cfl,    PIP_FLAVOUR::launch_ghosts,
                              PIP_FLAVOUR::launch_flux,   PIP_FLAVOUR::launch_source,
                              PIP_FLAVOUR::launch_nan,    PIP_FLAVOUR::launch_coefficients,
                              PIP_FLAVOUR::tile_map,      PIP_FLAVOUR::launch_nlev_ref,
                              PIP_FLAVOUR::launch_nlev_rates, PIP_FLAVOUR::launch_nlev_update,
                              PIP_FLAVOUR::launch_nlev_cfl};
  return L;
}

}  // namespace pip
