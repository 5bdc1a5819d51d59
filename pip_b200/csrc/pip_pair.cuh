// pip_pair.cuh -- FP32 Riemann solvers of the mixed form with each face's left and right
// computations paired in the packed FP32x2 arithmetic of sm_100 (one FFMA2/FADD2/FMUL2 does
// the left state's and the right state's operation).  Lane x holds the left state, lane y the
// right state.  The operations and their order per lane are those of hllc_flux_rcp /
// hlld_flux_rcp (pip_physics.cuh); the packed forms round each product, sum or fused
// multiply-add once per lane as the scalar ones do, so results differ from the scalar
// solvers only where the compiler contracted a different pair of operations there.  The
// steps that mix the two states (wave speeds, HLL averages, the star-state speeds, the state
// selection) stay scalar.  Float; the host compilation (tests) restates the packed operations
// lane by lane.
#pragma once

#include <cuda_runtime.h>

#include "pip_physics.cuh"

namespace pip {
namespace pair {

PIP_HD float2 p2(float a, float b) { return make_float2(a, b); }
PIP_HD float2 s2(float a) { return make_float2(a, a); }
#if defined(__CUDA_ARCH__)
PIP_HD float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
PIP_HD float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
PIP_HD float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
#else
// host restatement (tests): the same per-lane roundings
PIP_HD float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
PIP_HD float2 mul2(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
PIP_HD float2 fma2(float2 a, float2 b, float2 c) {
  return make_float2(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y));
}
#endif
// a - b, rounded once (b * -1 is exact)
PIP_HD float2 sub2(float2 a, float2 b) { return fma2(b, s2(-1.0f), a); }

// hllc_flux_rcp<float> (HLL_rot.f90:615-687) with paired left/right work.
PIP_HD void hllc_flux(const float (&v_l)[5], const float (&v_r)[5],
                                          float (&flx)[5], float gm, float igm1) {
  float2 v[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) v[n] = p2(v_l[n], v_r[n]);
  const float2 ke = fma2(v[3], v[3], fma2(v[2], v[2], mul2(v[1], v[1])));
  float2 u[5], f[5];
  u[0] = v[0];
  u[1] = mul2(v[0], v[1]);
  u[2] = mul2(v[0], v[2]);
  u[3] = mul2(v[0], v[3]);
  u[4] = fma2(v[4], s2(igm1), mul2(mul2(s2(0.5f), v[0]), ke));
  const float2 pr = v[4], vn = v[1];
  f[0] = u[1];
  f[1] = fma2(u[1], vn, pr);
  f[2] = mul2(u[2], vn);
  f[3] = mul2(u[3], vn);
  f[4] = mul2(add2(u[4], pr), vn);
  const float2 gp = mul2(s2(gm), pr);
  const float cs_l = rsqrt_(gp.x / v[0].x), cs_r = rsqrt_(gp.y / v[0].y);
  const float2 cs = p2(cs_l, cs_r);
  const float2 lo = sub2(vn, cs), hi = add2(vn, cs);
  const float sl = float(kHllcAcc) * rmin(lo.x, lo.y);
  const float sr = float(kHllcAcc) * rmax(hi.x, hi.y);
  const float2 sp = p2(sl, sr);
  const float2 d = sub2(sp, vn);          // (sl - vn_l, sr - vn_r)
  const float2 q = mul2(u[0], d);         // (ql, qr)
  const float2 w = mul2(u[1], d);         // products rounded alone: +0 sums at a mirror face
  const float sm = (w.y - w.x + pr.x - pr.y) / (q.y - q.x);
  const float pr_m = sm * q.x - w.x + pr.x;
  const float2 den = sub2(sp, s2(sm));
  const float2 iv = p2(1.0f / den.x, 1.0f / den.y);
  float2 st[5];
  st[0] = mul2(q, iv);
  st[1] = mul2(st[0], s2(sm));
  st[2] = mul2(st[0], v[2]);
  st[3] = mul2(st[0], v[3]);
  st[4] = mul2(add2(sub2(mul2(d, u[4]), mul2(pr, vn)), s2(pr_m * sm)), iv);
  const float thl = hllc_switch(sl);
  const float thm = hllc_switch(sm);
  const float thr = 1.0f - hllc_switch(sr);
  const float2 tlr = p2(thl, thr), tm = p2(thm, 1.0f - thm);
  const float c = 1.0f - thl - thr;
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    const float2 g = fma2(sp, sub2(st[n], u[n]), f[n]);   // (fl + sl (stl - ul), fr + sr (str - ur))
    const float2 a = mul2(tlr, f[n]);
    const float2 b = mul2(tm, g);
    flx[n] = a.y + a.x + c * (b.x + b.y);
  }
}


// hlld_flux_rcp<float, 8> (HLL_rot.f90:691-910 without the Dedner flux, which the mixed
// form takes in FP64) with paired left/right work: the conversions, the one-sided fluxes,
// the fast speeds, the star states L* and R* and their fluxes.  The HLL average, the contact
// and Alfven speeds, the HLLC-G fallback, the central states L** and R** and the choice of
// the state stay scalar.
PIP_HD void hlld_flux(const float (&v_l)[8], const float (&v_r)[8],
                                          float (&flx)[8], float gm, float igm1) {
  float2 v[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) v[n] = p2(v_l[n], v_r[n]);
  const float2 half = s2(0.5f);
  const float2 b2 = fma2(v[7], v[7], fma2(v[6], v[6], mul2(v[5], v[5])));
  const float2 ke = fma2(v[3], v[3], fma2(v[2], v[2], mul2(v[1], v[1])));
  float2 u[8], f[8];
  u[0] = v[0];
  u[1] = mul2(v[0], v[1]);
  u[2] = mul2(v[0], v[2]);
  u[3] = mul2(v[0], v[3]);
  u[4] = fma2(v[4], s2(igm1), fma2(mul2(half, v[0]), ke, mul2(half, b2)));
  u[5] = v[5];
  u[6] = v[6];
  u[7] = v[7];
  const float2 pt = fma2(half, b2, v[4]);
  const float2 vb = fma2(v[3], v[7], fma2(v[2], v[6], mul2(v[1], v[5])));
  f[0] = u[1];
  f[1] = sub2(fma2(u[1], v[1], pt), mul2(v[5], v[5]));
  f[2] = sub2(mul2(u[1], v[2]), mul2(v[5], v[6]));
  f[3] = sub2(mul2(u[1], v[3]), mul2(v[5], v[7]));
  f[4] = sub2(mul2(add2(u[4], pt), v[1]), mul2(vb, v[5]));
  f[5] = s2(0.0f);
  f[6] = sub2(mul2(v[1], v[6]), mul2(v[5], v[2]));
  f[7] = sub2(mul2(v[1], v[7]), mul2(v[5], v[3]));

  // fast magnetosonic speeds
  const float2 gp = mul2(s2(gm), v[4]);
  const float2 a = add2(gp, b2);
  const float2 disc = sub2(mul2(a, a), mul2(mul2(s2(4.0f), gp), mul2(v[5], v[5])));
  const float2 num = add2(a, p2(rsqrt_(rmax(disc.x, 0.0f)), rsqrt_(rmax(disc.y, 0.0f))));
  const float2 den2 = mul2(s2(2.0f), v[0]);
  const float vf = rmax(rsqrt_(num.x / den2.x), rsqrt_(num.y / den2.y));
  const float sl = rmin(v[1].x, v[1].y) - vf;
  const float sr = rmax(v[1].x, v[1].y) + vf;

  if (sl >= 0.0f) {
#pragma unroll
    for (int n = 0; n < 8; ++n) flx[n] = f[n].x;
    return;
  }
  if (sr <= 0.0f) {
#pragma unroll
    for (int n = 0; n < 8; ++n) flx[n] = f[n].y;
    return;
  }
  const float2 sp = p2(sl, sr);
  const float ihll = 1.0f / (sr - sl);
  float uh[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const float2 w = mul2(sp, u[n]);      // products rounded alone (mirror faces: +0)
    uh[n] = ihll * (w.y - w.x - f[n].y + f[n].x);
  }
  const float iuh0 = 1.0f / uh[0];
  const float sm = uh[1] * iuh0;
  const float2 d = sub2(sp, v[1]);                     // (sl - vn_l, sr - vn_r)
  const float pts = pt.x + v[0].x * d.x * (sm - v[1].x);
  const float2 dsm = sub2(sp, s2(sm));                 // (sl - sm, sr - sm)
  const float2 ilr = p2(1.0f / dsm.x, 1.0f / dsm.y);
  const float2 dlr = mul2(v[0], d);
  const float2 ro1 = mul2(dlr, ilr);                   // (ro_l1, ro_r1)
  const float2 rs = p2(rrsqrt(ro1.x), rrsqrt(ro1.y));
  const float bn = uh[5], bn2 = bn * bn;
  const float2 sa = mul2(s2(rabs(bn)), rs);            // (sal, sar)

  if ((sl >= (sm - float(kHllgFactor) * sa.x)) || ((sm + float(kHllgFactor) * sa.y) >= sr)) {
    // HLLC-G (HLL_rot.f90:776-807)
    const float vy_2 = uh[2] * iuh0;
    const float vz_2 = uh[3] * iuh0;
    const bool left = sm >= 0.0f;
    const float s = left ? sl : sr, dd = left ? d.x : d.y, ro = left ? ro1.x : ro1.y;
    const float e2 = (dd * (left ? u[4].x : u[4].y) - (left ? pt.x : pt.y) * (left ? v[1].x : v[1].y) +
                      pts * sm + bn * ((left ? vb.x : vb.y) - sm * bn - vy_2 * uh[6] - vz_2 * uh[7])) *
                     (left ? ilr.x : ilr.y);
    const float st[8] = {ro, ro * sm, ro * vy_2, ro * vz_2, e2, uh[5], uh[6], uh[7]};
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const float un = left ? u[n].x : u[n].y, fn = left ? f[n].x : f[n].y;
      flx[n] = s * (st[n] - un) + fn;
    }
    return;
  }

  // L* and R* (HLL_rot.f90:813-843)
  const float2 tden = sub2(mul2(dlr, dsm), s2(bn2));
  const float2 fi = p2(1.0f / tden.x, 1.0f / tden.y);
  const float2 glr = mul2(fi, sub2(mul2(dlr, d), s2(bn2)));
  float2 us[8];
  us[5] = s2(bn);
  us[6] = mul2(v[6], glr);
  us[7] = mul2(v[7], glr);
  const float2 smv = sub2(s2(sm), v[1]);               // (sm - vn_l, sm - vn_r)
  const float2 fb = mul2(fi, s2(bn));
  const float2 vy1 = sub2(v[2], mul2(mul2(fb, v[6]), smv));
  const float2 vz1 = sub2(v[3], mul2(mul2(fb, v[7]), smv));
  us[0] = ro1;
  {
    const float2 inner = sub2(sub2(sub2(vb, s2(sm * bn)), mul2(vy1, us[6])), mul2(vz1, us[7]));
    const float2 t = add2(add2(sub2(mul2(d, u[4]), mul2(pt, v[1])), s2(pts * sm)),
                          mul2(s2(bn), inner));
    us[4] = mul2(t, ilr);
  }
  us[1] = mul2(ro1, s2(sm));
  us[2] = mul2(ro1, vy1);
  us[3] = mul2(ro1, vz1);

  const float sl1 = sm - sa.x;
  const float sr1 = sm + sa.y;
  if (sl1 >= 0.0f || sr1 <= 0.0f) {
    const bool left = sl1 >= 0.0f;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const float2 o = fma2(sp, sub2(us[n], u[n]), f[n]);   // s (U* - U) + F, both sides
      flx[n] = left ? o.x : o.y;
    }
    return;
  }
  // L** and R** (HLL_rot.f90:861-898)
  const float2 ros = mul2(ro1, rs);                    // sqrt(ro_l1), sqrt(ro_r1)
  const float fq = 1.0f / (ros.x + ros.y);
  const float sg = rsign1(bn);
  const float vy_2 = fq * (ros.x * vy1.x + ros.y * vy1.y + (us[6].y - us[6].x) * sg);
  const float vz_2 = fq * (ros.x * vz1.x + ros.y * vz1.y + (us[7].y - us[7].x) * sg);
  float u2[8];
  u2[5] = bn;
  u2[6] = fq * (ros.x * us[6].y + ros.y * us[6].x + ros.x * ros.y * (vy1.y - vy1.x) * sg);
  u2[7] = fq * (ros.x * us[7].y + ros.y * us[7].x + ros.x * ros.y * (vz1.y - vz1.x) * sg);
  const bool left = sm >= 0.0f;
  const float ro = left ? ro1.x : ro1.y;
  const float s = left ? sl : sr, s1 = left ? sl1 : sr1;
  const float rsd = left ? ros.x : ros.y;
  const float vy = left ? vy1.x : vy1.y, vz = left ? vz1.x : vz1.y;
  const float b6 = left ? us[6].x : us[6].y, b7 = left ? us[7].x : us[7].y;
  const float e1 = left ? us[4].x : us[4].y;
  const float de = rsd * (vy * b6 + vz * b7 - vy_2 * u2[6] - vz_2 * u2[7]) * sg;
  u2[0] = ro;
  u2[4] = left ? e1 - de : e1 + de;
  u2[1] = ro * sm;
  u2[2] = ro * vy_2;
  u2[3] = ro * vz_2;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const float usn = left ? us[n].x : us[n].y;
    const float un = left ? u[n].x : u[n].y, fn = left ? f[n].x : f[n].y;
    flx[n] = s1 * u2[n] - (s1 - s) * usn - s * un + fn;
  }
}

}  // namespace pair
}  // namespace pip
