// pip_adjoint_physics.cuh -- hand-written reverse-mode derivatives (vector-Jacobian
// products) of the per-cell and per-face physics of the FP64 two-fluid step.
//
// Each *_vjp function recomputes the forward quantities it needs from the same inputs as
// the forward function in pip_physics.cuh (the reciprocal forms used by the FMA build) and
// then runs the reverse sweep by hand: every branch (min/max, minmod slope choice, HLLD
// fan region, HLLC-G fallback, floors) is differentiated on the side the forward takes.
// Cotangents are ACCUMULATED into the a_* outputs (callers zero them).  The functions
// compile for the host too, so that they can be checked against central finite
// differences without a GPU.
#pragma once

#include "pip_physics.cuh"

namespace pip {
namespace adj {

// derivative of |x| (0 at x == 0)
PIP_HD double dabs(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// ---------------------------------------------------------------- conversions

// u2v_mhd (HLL_rot.f90:1159-1186), NVM = 8.
PIP_HD void u2v_mhd_vjp(const double (&u)[8], const double (&a_v)[8], double gm, double ro_lim,
                        double pr_lim, double (&a_u)[8]) {
  const double ro = rmax(u[0], ro_lim);
  const double roi = 1.0 / ro;
  const double m2 = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  const double pr = (gm - 1.0) * (u[4] - 0.5 * m2 * roi - 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]));
  const double a_pr = pr < pr_lim ? 0.0 : a_v[4];
  double a_roi = -(gm - 1.0) * 0.5 * m2 * a_pr;
  a_u[4] += (gm - 1.0) * a_pr;
  for (int k = 1; k <= 3; ++k) {
    a_u[k] += -(gm - 1.0) * u[k] * roi * a_pr + roi * a_v[k];
    a_roi += u[k] * a_v[k];
  }
  for (int k = 5; k <= 7; ++k) a_u[k] += -(gm - 1.0) * u[k] * a_pr + a_v[k];
  const double a_ro = a_v[0] - roi * roi * a_roi;
  if (u[0] >= ro_lim) a_u[0] += a_ro;
}

// u2v_hd (HLL_rot.f90:1136-1156).
PIP_HD void u2v_hd_vjp(const double (&u)[5], const double (&a_v)[5], double gm, double ro_lim,
                       double pr_lim, double (&a_u)[5]) {
  const double ro = rmax(u[0], ro_lim);
  const double roi = 1.0 / ro;
  const double m2 = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  const double pr = (gm - 1.0) * (u[4] - 0.5 * m2 * roi);
  const double a_pr = pr < pr_lim ? 0.0 : a_v[4];
  double a_roi = -(gm - 1.0) * 0.5 * m2 * a_pr;
  a_u[4] += (gm - 1.0) * a_pr;
  for (int k = 1; k <= 3; ++k) {
    a_u[k] += -(gm - 1.0) * u[k] * roi * a_pr + roi * a_v[k];
    a_roi += u[k] * a_v[k];
  }
  const double a_ro = a_v[0] - roi * roi * a_roi;
  if (u[0] >= ro_lim) a_u[0] += a_ro;
}

// Reverse of cq2pv_*_rcp (Scheme_rot.f90:132-179) for a consumer of both the rewritten
// conserved state (a_w, planes 0..4) and the primitives (a_q: de, vx, vy, vz, pr).  NB is
// the number of magnetic components (3 for ions, 0 for neutrals) read from u[5..7].
template <int N, int NB>
PIP_HD void cq2pv_vjp(const double (&u)[N], const double (&a_w)[5], const double (&a_q)[5],
                      double gm, double igm1, double ro_lim, double pr_lim, double (&a_u)[N]) {
  const double de = u[0];
  const double inv = 1.0 / de;
  double v[3] = {u[1] * inv, u[2] * inv, u[3] * inv};
  const double kin = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  double bb = 0.0;
  for (int k = 0; k < NB; ++k) bb += u[5 + k] * u[5 + k];
  const double pr_raw = (gm - 1.0) * (u[4] - 0.5 * de * kin - 0.5 * bb);
  const double de_f = rmax(de, ro_lim);
  const double pr_f = rmax(pr_raw, pr_lim);
  (void)pr_f;
  // outputs: w0 = de_f, w_k = v_k de_f, w4 = pr_f igm1 + 0.5 de_f kin + 0.5 bb;
  //          q = (de_f, v, pr_f)
  double a_def = a_w[0] + a_q[0] + 0.5 * kin * a_w[4];
  double a_v[3], a_kin = 0.5 * de_f * a_w[4], a_bb = 0.5 * a_w[4];
  for (int k = 0; k < 3; ++k) {
    a_def += v[k] * a_w[1 + k];
    a_v[k] = de_f * a_w[1 + k] + a_q[1 + k];
  }
  const double a_prf = igm1 * a_w[4] + a_q[4];
  const double a_prraw = pr_raw >= pr_lim ? a_prf : 0.0;
  double a_de = de >= ro_lim ? a_def : 0.0;
  a_u[4] += (gm - 1.0) * a_prraw;
  a_de += -(gm - 1.0) * 0.5 * kin * a_prraw;
  a_kin += -(gm - 1.0) * 0.5 * de * a_prraw;
  a_bb += -(gm - 1.0) * 0.5 * a_prraw;
  double a_inv = 0.0;
  for (int k = 0; k < 3; ++k) {
    a_v[k] += 2.0 * v[k] * a_kin;
    a_u[1 + k] += inv * a_v[k];
    a_inv += u[1 + k] * a_v[k];
  }
  for (int k = 0; k < NB; ++k) a_u[5 + k] += 2.0 * u[5 + k] * a_bb;
  a_de += -inv * inv * a_inv;
  a_u[0] += a_de;
}

// ---------------------------------------------------------------- reconstruction

// Which branch minmod(v0, v1, v2) (Util_rot.f90:59-76) takes: 0 -> slope 0, 1 -> slope
// v2 - v1, 2 -> slope v1 - v0.
PIP_HD int minmod_mode(double v0, double v1, double v2) {
  const double X = v2 - v1, Y = v1 - v0;
  const double SX = rsign1(X);
  const double m = rmin(rabs(X), SX * Y);
  if (!(m > 0.0)) return 0;
  return rabs(X) <= SX * Y ? 1 : 2;
}

// Cotangents of (v0, v1, v2) from cotangent g of the minmod slope.
PIP_HD void minmod_vjp(int mode, double g, double &a0, double &a1, double &a2) {
  if (mode == 1) {
    a2 += g;
    a1 -= g;
  } else if (mode == 2) {
    a1 += g;
    a0 -= g;
  }
}

// ---------------------------------------------------------------- HLLC (reciprocal form)

PIP_HD double hllc_switch_d(double s) {
  return (s >= 0.5 * kHllcEpsi) ? 0.0 : (s > 0.0 ? 2.0 * (1.0 / kHllcEpsi) : 0.0);
}

// Reverse of hllc_flux_rcp (HLL_rot.f90:615-687); optionally returns the flux.
PIP_HD void hllc_vjp(const double (&vl)[5], const double (&vr)[5], const double (&a_f)[5],
                     double gm, double igm1, double (&a_vl)[5], double (&a_vr)[5],
                     double *flx_out = nullptr) {
  // ---- forward
  const double kel = vl[1] * vl[1] + vl[2] * vl[2] + vl[3] * vl[3];
  const double ker = vr[1] * vr[1] + vr[2] * vr[2] + vr[3] * vr[3];
  double ul[5], ur[5], fl[5], fr[5], stl[5], str[5];
  ul[0] = vl[0]; ul[1] = vl[0] * vl[1]; ul[2] = vl[0] * vl[2]; ul[3] = vl[0] * vl[3];
  ul[4] = vl[4] * igm1 + 0.5 * vl[0] * kel;
  ur[0] = vr[0]; ur[1] = vr[0] * vr[1]; ur[2] = vr[0] * vr[2]; ur[3] = vr[0] * vr[3];
  ur[4] = vr[4] * igm1 + 0.5 * vr[0] * ker;
  const double prl = vl[4], prr = vr[4], vnl = vl[1], vnr = vr[1];
  fl[0] = ul[1]; fr[0] = ur[1];
  fl[1] = prl + ul[1] * vnl; fr[1] = prr + ur[1] * vnr;
  fl[2] = ul[2] * vnl; fr[2] = ur[2] * vnr;
  fl[3] = ul[3] * vnl; fr[3] = ur[3] * vnr;
  fl[4] = (ul[4] + prl) * vnl; fr[4] = (ur[4] + prr) * vnr;
  const double Xl = gm * prl / vl[0], Xr = gm * prr / vr[0];
  const double csl = rsqrt_(Xl), csr = rsqrt_(Xr);
  const bool sl_left = (vnl - csl) <= (vnr - csr);
  const bool sr_left = (vnl + csl) >= (vnr + csr);
  const double sl = kHllcAcc * (sl_left ? vnl - csl : vnr - csr);
  const double sr = kHllcAcc * (sr_left ? vnl + csl : vnr + csr);
  const double ql = ul[0] * (sl - vnl), qr = ur[0] * (sr - vnr);
  const double Nn = mul_rn(ur[1], sr - vnr) - mul_rn(ul[1], sl - vnl) + prl - prr;
  const double Dd = qr - ql;
  const double sm = Nn / Dd;
  const double prm = sm * ql - ul[1] * (sl - vnl) + prl;
  const double il = 1.0 / (sl - sm), ir = 1.0 / (sr - sm);
  stl[0] = ql * il; str[0] = qr * ir;
  stl[1] = stl[0] * sm; str[1] = str[0] * sm;
  stl[2] = stl[0] * vl[2]; str[2] = str[0] * vr[2];
  stl[3] = stl[0] * vl[3]; str[3] = str[0] * vr[3];
  const double Tl = (sl - vnl) * ul[4] - prl * vnl + prm * sm;
  const double Tr = (sr - vnr) * ur[4] - prr * vnr + prm * sm;
  stl[4] = Tl * il; str[4] = Tr * ir;
  const double thl = hllc_switch(sl), thm = hllc_switch(sm), thr = 1.0 - hllc_switch(sr);
  double Ml[5], Mr[5], C[5];
  for (int n = 0; n < 5; ++n) {
    Ml[n] = fl[n] + sl * (stl[n] - ul[n]);
    Mr[n] = fr[n] + sr * (str[n] - ur[n]);
    C[n] = thm * Ml[n] + (1.0 - thm) * Mr[n];
    if (flx_out) flx_out[n] = thr * fr[n] + thl * fl[n] + (1.0 - thl - thr) * C[n];
  }
  // ---- reverse
  double a_ul[5] = {0, 0, 0, 0, 0}, a_ur[5] = {0, 0, 0, 0, 0};
  double a_fl[5], a_fr[5], a_stl[5], a_str[5];
  double a_thl = 0, a_thm = 0, a_thr = 0, a_sl = 0, a_sr = 0, a_sm = 0;
  for (int n = 0; n < 5; ++n) {
    const double a = a_f[n];
    a_thr += a * (fr[n] - C[n]);
    a_thl += a * (fl[n] - C[n]);
    const double aC = (1.0 - thl - thr) * a;
    a_thm += aC * (Ml[n] - Mr[n]);
    const double aMl = thm * aC, aMr = (1.0 - thm) * aC;
    a_fl[n] = thl * a + aMl;
    a_fr[n] = thr * a + aMr;
    a_sl += aMl * (stl[n] - ul[n]);
    a_sr += aMr * (str[n] - ur[n]);
    a_stl[n] = sl * aMl;
    a_str[n] = sr * aMr;
    a_ul[n] -= sl * aMl;
    a_ur[n] -= sr * aMr;
  }
  a_sr -= hllc_switch_d(sr) * a_thr;
  a_sl += hllc_switch_d(sl) * a_thl;
  a_sm += hllc_switch_d(sm) * a_thm;
  double a_il = 0, a_ir = 0, a_prm = 0, a_vnl = 0, a_vnr = 0, a_prl = 0, a_prr = 0;
  {
    const double aT = il * a_stl[4];
    a_il += Tl * a_stl[4];
    a_sl += ul[4] * aT;
    a_vnl -= (ul[4] + prl) * aT;
    a_ul[4] += (sl - vnl) * aT;
    a_prl -= vnl * aT;
    a_prm += sm * aT;
    a_sm += prm * aT;
  }
  {
    const double aT = ir * a_str[4];
    a_ir += Tr * a_str[4];
    a_sr += ur[4] * aT;
    a_vnr -= (ur[4] + prr) * aT;
    a_ur[4] += (sr - vnr) * aT;
    a_prr -= vnr * aT;
    a_prm += sm * aT;
    a_sm += prm * aT;
  }
  double a_stl0 = a_stl[0] + vl[2] * a_stl[2] + vl[3] * a_stl[3] + sm * a_stl[1];
  double a_str0 = a_str[0] + vr[2] * a_str[2] + vr[3] * a_str[3] + sm * a_str[1];
  a_vl[2] += stl[0] * a_stl[2];
  a_vl[3] += stl[0] * a_stl[3];
  a_vr[2] += str[0] * a_str[2];
  a_vr[3] += str[0] * a_str[3];
  a_sm += stl[0] * a_stl[1] + str[0] * a_str[1];
  double a_ql = il * a_stl0, a_qr = ir * a_str0;
  a_il += ql * a_stl0;
  a_ir += qr * a_str0;
  a_sl -= il * il * a_il;
  a_sm += il * il * a_il;
  a_sr -= ir * ir * a_ir;
  a_sm += ir * ir * a_ir;
  // prm = sm*ql - ul1*(sl - vnl) + prl
  a_sm += ql * a_prm;
  a_ql += sm * a_prm;
  a_ul[1] -= (sl - vnl) * a_prm;
  a_sl -= ul[1] * a_prm;
  a_vnl += ul[1] * a_prm;
  a_prl += a_prm;
  // sm = Nn / Dd
  const double a_N = a_sm / Dd;
  const double a_D = -sm / Dd * a_sm;
  a_qr += a_D;
  a_ql -= a_D;
  a_ur[1] += (sr - vnr) * a_N;
  a_sr += ur[1] * a_N;
  a_vnr -= ur[1] * a_N;
  a_ul[1] -= (sl - vnl) * a_N;
  a_sl -= ul[1] * a_N;
  a_vnl += ul[1] * a_N;
  a_prl += a_N;
  a_prr -= a_N;
  // ql = ul0*(sl - vnl), qr = ur0*(sr - vnr)
  a_ul[0] += (sl - vnl) * a_ql;
  a_sl += ul[0] * a_ql;
  a_vnl -= ul[0] * a_ql;
  a_ur[0] += (sr - vnr) * a_qr;
  a_sr += ur[0] * a_qr;
  a_vnr -= ur[0] * a_qr;
  // wave speeds
  double a_csl = 0, a_csr = 0;
  if (sl_left) { a_vnl += kHllcAcc * a_sl; a_csl -= kHllcAcc * a_sl; }
  else { a_vnr += kHllcAcc * a_sl; a_csr -= kHllcAcc * a_sl; }
  if (sr_left) { a_vnl += kHllcAcc * a_sr; a_csl += kHllcAcc * a_sr; }
  else { a_vnr += kHllcAcc * a_sr; a_csr += kHllcAcc * a_sr; }
  if (csl > 0.0) {
    const double aX = a_csl / (2.0 * csl);
    a_prl += gm / vl[0] * aX;
    a_vl[0] -= Xl / vl[0] * aX;
  }
  if (csr > 0.0) {
    const double aX = a_csr / (2.0 * csr);
    a_prr += gm / vr[0] * aX;
    a_vr[0] -= Xr / vr[0] * aX;
  }
  // physical fluxes
  a_ul[1] += a_fl[0] + vnl * a_fl[1];
  a_prl += a_fl[1] + vnl * a_fl[4];
  a_vnl += ul[1] * a_fl[1] + ul[2] * a_fl[2] + ul[3] * a_fl[3] + (ul[4] + prl) * a_fl[4];
  a_ul[2] += vnl * a_fl[2];
  a_ul[3] += vnl * a_fl[3];
  a_ul[4] += vnl * a_fl[4];
  a_ur[1] += a_fr[0] + vnr * a_fr[1];
  a_prr += a_fr[1] + vnr * a_fr[4];
  a_vnr += ur[1] * a_fr[1] + ur[2] * a_fr[2] + ur[3] * a_fr[3] + (ur[4] + prr) * a_fr[4];
  a_ur[2] += vnr * a_fr[2];
  a_ur[3] += vnr * a_fr[3];
  a_ur[4] += vnr * a_fr[4];
  // conserved from primitive
  a_vl[1] += a_vnl;
  a_vl[4] += a_prl + igm1 * a_ul[4];
  a_vl[0] += a_ul[0] + 0.5 * kel * a_ul[4];
  a_vr[1] += a_vnr;
  a_vr[4] += a_prr + igm1 * a_ur[4];
  a_vr[0] += a_ur[0] + 0.5 * ker * a_ur[4];
  for (int k = 1; k <= 3; ++k) {
    a_vl[0] += vl[k] * a_ul[k];
    a_vl[k] += vl[0] * a_ul[k] + vl[0] * vl[k] * a_ul[4];
    a_vr[0] += vr[k] * a_ur[k];
    a_vr[k] += vr[0] * a_ur[k] + vr[0] * vr[k] * a_ur[4];
  }
}

// ---------------------------------------------------------------- HLLD (reciprocal form)

// Intermediate (single-star) state of one side, HLL_rot.f90:813-843, with everything the
// reverse sweep needs.  s = +1 for the left side (uses sl), -1 for the right.
struct StarSide {
  double d, den, f1, num, g;      // d = ro*(S - vn), f1 = 1/den, g = f1*num
  double vy1, vz1, u1[8], E, iS;  // iS = 1/(S - sm)
};

PIP_HD void star_forward(const double (&v)[8], const double (&u)[8], double S, double iS, double sm,
                         double bn, double bn2, double pt, double pts, double vb, double ro1,
                         StarSide &st) {
  st.iS = iS;
  st.d = v[0] * (S - v[1]);
  st.den = st.d * (S - sm) - bn2;
  st.f1 = 1.0 / st.den;
  st.num = st.d * (S - v[1]) - bn2;
  st.g = st.f1 * st.num;
  st.u1[5] = bn;
  st.u1[6] = v[6] * st.g;
  st.u1[7] = v[7] * st.g;
  st.vy1 = v[2] - st.f1 * bn * v[6] * (sm - v[1]);
  st.vz1 = v[3] - st.f1 * bn * v[7] * (sm - v[1]);
  st.u1[0] = ro1;
  st.E = (S - v[1]) * u[4] - pts * v[1] + pt * sm +
         bn * (vb - sm * bn - st.vy1 * st.u1[6] - st.vz1 * st.u1[7]);
  st.u1[4] = st.E * iS;
  st.u1[1] = ro1 * sm;
  st.u1[2] = ro1 * st.vy1;
  st.u1[3] = ro1 * st.vz1;
}

// Reverse of star_forward: a_u1[8], a_vy1, a_vz1 in; accumulates into the shared adjoints.
PIP_HD void star_reverse(const double (&v)[8], const double (&u)[8], double S, double sm, double bn,
                         double pt, double pts, double vb, double ro1, const StarSide &st,
                         double (&a_u1)[8], double a_vy1, double a_vz1, double (&a_v)[8],
                         double (&a_u)[8], double &a_S, double &a_sm, double &a_bn,
                         double &a_bn2, double &a_pt, double &a_pts, double &a_vb,
                         double &a_ro1, double &a_iS) {
  // u1[1..3]
  a_ro1 += sm * a_u1[1] + st.vy1 * a_u1[2] + st.vz1 * a_u1[3] + a_u1[0];
  a_sm += ro1 * a_u1[1];
  a_vy1 += ro1 * a_u1[2];
  a_vz1 += ro1 * a_u1[3];
  a_bn += a_u1[5];
  // u1[4] = E*iS
  const double aE = st.iS * a_u1[4];
  a_iS += st.E * a_u1[4];
  const double Q = vb - sm * bn - st.vy1 * st.u1[6] - st.vz1 * st.u1[7];
  a_S += u[4] * aE;
  a_v[1] -= (u[4] + pts) * aE;
  a_u[4] += (S - v[1]) * aE;
  a_pts -= v[1] * aE;
  a_pt += sm * aE;
  a_sm += pt * aE;
  a_bn += (Q - bn * sm) * aE;
  a_vb += bn * aE;
  a_sm -= bn * bn * aE;
  a_vy1 -= bn * st.u1[6] * aE;
  double a_u16 = a_u1[6] - bn * st.vy1 * aE;
  a_vz1 -= bn * st.u1[7] * aE;
  double a_u17 = a_u1[7] - bn * st.vz1 * aE;
  // vy1 = v2 - f1*bn*v6*(sm - v1), vz1 likewise
  double a_f1 = 0.0;
  a_v[2] += a_vy1;
  a_f1 -= bn * v[6] * (sm - v[1]) * a_vy1;
  a_bn -= st.f1 * v[6] * (sm - v[1]) * a_vy1;
  a_v[6] -= st.f1 * bn * (sm - v[1]) * a_vy1;
  a_sm -= st.f1 * bn * v[6] * a_vy1;
  a_v[1] += st.f1 * bn * v[6] * a_vy1;
  a_v[3] += a_vz1;
  a_f1 -= bn * v[7] * (sm - v[1]) * a_vz1;
  a_bn -= st.f1 * v[7] * (sm - v[1]) * a_vz1;
  a_v[7] -= st.f1 * bn * (sm - v[1]) * a_vz1;
  a_sm -= st.f1 * bn * v[7] * a_vz1;
  a_v[1] += st.f1 * bn * v[7] * a_vz1;
  // u1[6] = v6*g, u1[7] = v7*g
  a_v[6] += st.g * a_u16;
  a_v[7] += st.g * a_u17;
  const double a_g = v[6] * a_u16 + v[7] * a_u17;
  a_f1 += st.num * a_g;
  const double a_num = st.f1 * a_g;
  double a_d = (S - v[1]) * a_num;
  a_S += st.d * a_num;
  a_v[1] -= st.d * a_num;
  a_bn2 -= a_num;
  const double a_den = -st.f1 * st.f1 * a_f1;
  a_d += (S - sm) * a_den;
  a_S += st.d * a_den;
  a_sm -= st.d * a_den;
  a_bn2 -= a_den;
  a_v[0] += (S - v[1]) * a_d;
  a_S += v[0] * a_d;
  a_v[1] -= v[0] * a_d;
}

// Reverse of hlld_flux_rcp<double, 8> (HLL_rot.f90:691-910 without the Dedner flux).
// Returns the region taken (0: F_L, 1: F_R, 2/3: HLLC-G left/right, 4/5: L*/R*,
// 6/7: L**/R**); optionally the flux.
PIP_HD int hlld_vjp(const double (&vl)[8], const double (&vr)[8], const double (&a_f)[8],
                    double gm, double igm1, double (&a_vl)[8], double (&a_vr)[8],
                    double *flx_out = nullptr) {
  // ---- forward prefix
  const double b2l = vl[5] * vl[5] + vl[6] * vl[6] + vl[7] * vl[7];
  const double b2r = vr[5] * vr[5] + vr[6] * vr[6] + vr[7] * vr[7];
  const double kel = vl[1] * vl[1] + vl[2] * vl[2] + vl[3] * vl[3];
  const double ker = vr[1] * vr[1] + vr[2] * vr[2] + vr[3] * vr[3];
  double ul[8], ur[8];
  ul[0] = vl[0]; ul[1] = vl[0] * vl[1]; ul[2] = vl[0] * vl[2]; ul[3] = vl[0] * vl[3];
  ul[4] = vl[4] * igm1 + 0.5 * vl[0] * kel + 0.5 * b2l; ul[5] = vl[5]; ul[6] = vl[6]; ul[7] = vl[7];
  ur[0] = vr[0]; ur[1] = vr[0] * vr[1]; ur[2] = vr[0] * vr[2]; ur[3] = vr[0] * vr[3];
  ur[4] = vr[4] * igm1 + 0.5 * vr[0] * ker + 0.5 * b2r; ur[5] = vr[5]; ur[6] = vr[6]; ur[7] = vr[7];
  const double ptl = vl[4] + 0.5 * b2l, ptr = vr[4] + 0.5 * b2r;
  const double vbL = vl[1] * vl[5] + vl[2] * vl[6] + vl[3] * vl[7];
  const double vbR = vr[1] * vr[5] + vr[2] * vr[6] + vr[3] * vr[7];
  double fl[8], fr[8];
  fl[0] = ul[1];
  fl[1] = ul[1] * vl[1] + ptl - vl[5] * vl[5];
  fl[2] = ul[1] * vl[2] - vl[5] * vl[6];
  fl[3] = ul[1] * vl[3] - vl[5] * vl[7];
  fl[4] = (ul[4] + ptl) * vl[1] - vbL * vl[5];
  fl[5] = 0.0;
  fl[6] = vl[1] * vl[6] - vl[5] * vl[2];
  fl[7] = vl[1] * vl[7] - vl[5] * vl[3];
  fr[0] = ur[1];
  fr[1] = ur[1] * vr[1] + ptr - vr[5] * vr[5];
  fr[2] = ur[1] * vr[2] - vr[5] * vr[6];
  fr[3] = ur[1] * vr[3] - vr[5] * vr[7];
  fr[4] = (ur[4] + ptr) * vr[1] - vbR * vr[5];
  fr[5] = 0.0;
  fr[6] = vr[1] * vr[6] - vr[5] * vr[2];
  fr[7] = vr[1] * vr[7] - vr[5] * vr[3];
  const double f1l = gm * vl[4], Al = f1l + b2l;
  const double discl = Al * Al - 4.0 * f1l * (vl[5] * vl[5]);
  const double ddl = rsqrt_(rmax(discl, 0.0));
  const double Ql = (Al + ddl) / (2.0 * vl[0]);
  const double vfl = rsqrt_(Ql);
  const double f1r = gm * vr[4], Ar = f1r + b2r;
  const double discr = Ar * Ar - 4.0 * f1r * (vr[5] * vr[5]);
  const double ddr = rsqrt_(rmax(discr, 0.0));
  const double Qr = (Ar + ddr) / (2.0 * vr[0]);
  const double vfr = rsqrt_(Qr);
  const bool vmin_left = vl[1] <= vr[1];
  const bool vmax_left = vl[1] >= vr[1];
  const bool vf_left = vfl >= vfr;
  const double vfm = vf_left ? vfl : vfr;
  const double sl = (vmin_left ? vl[1] : vr[1]) - vfm;
  const double sr = (vmax_left ? vl[1] : vr[1]) + vfm;

  double a_ul[8] = {0, 0, 0, 0, 0, 0, 0, 0}, a_ur[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double a_fl[8] = {0, 0, 0, 0, 0, 0, 0, 0}, a_fr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double a_sl = 0, a_sr = 0, a_ptl = 0, a_ptr = 0, a_vbL = 0, a_vbR = 0;
  int region;
  if (sl >= 0.0) {
    region = 0;
    for (int n = 0; n < 8; ++n) {
      a_fl[n] += a_f[n];
      if (flx_out) flx_out[n] = fl[n];
    }
  } else if (sr <= 0.0) {
    region = 1;
    for (int n = 0; n < 8; ++n) {
      a_fr[n] += a_f[n];
      if (flx_out) flx_out[n] = fr[n];
    }
  } else {
    const double f1 = 1.0 / (sr - sl);
    double uh[8], w[8];
    for (int n = 0; n < 8; ++n) {
      w[n] = mul_rn(sr, ur[n]) - mul_rn(sl, ul[n]) - fr[n] + fl[n];
      uh[n] = f1 * w[n];
    }
    const double iuh0 = 1.0 / uh[0];
    const double sm = uh[1] * iuh0;
    const double pt = ptl + vl[0] * (sl - vl[1]) * (sm - vl[1]);
    const double ilm = 1.0 / (sl - sm), irm = 1.0 / (sr - sm);
    const double rol1 = vl[0] * (sl - vl[1]) * ilm;
    const double ror1 = vr[0] * (sr - vr[1]) * irm;
    const double rsl = rrsqrt(rol1), rsr = rrsqrt(ror1);
    const double bn = uh[5], bn2 = bn * bn;
    const double sal = rabs(bn) * rsl, sar = rabs(bn) * rsr;

    double a_uh[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double a_sm = 0, a_pt = 0, a_ilm = 0, a_irm = 0, a_rol1 = 0, a_ror1 = 0, a_rsl = 0,
           a_rsr = 0, a_bn = 0, a_bn2 = 0, a_sal = 0, a_sar = 0, a_iuh0 = 0;
    double out[8];
    if ((sl >= (sm - kHllgFactor * sal)) || ((sm + kHllgFactor * sar) >= sr)) {
      // HLLC-G (HLL_rot.f90:776-807).  The side is selected element by element (no pointer
      // to one side's arrays), so that every array stays in registers.
      const double vy2 = uh[2] * iuh0, vz2 = uh[3] * iuh0;
      const bool left = sm >= 0.0;
      double us[8], st[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) us[n] = left ? ul[n] : ur[n];
      const double v1 = left ? vl[1] : vr[1];
      const double S = left ? sl : sr;
      const double ro1 = left ? rol1 : ror1;
      const double iS = left ? ilm : irm;
      const double pts = left ? ptl : ptr;
      const double vb = left ? vbL : vbR;
      const double Q = vb - sm * bn - vy2 * uh[6] - vz2 * uh[7];
      const double E = (S - v1) * us[4] - pts * v1 + pt * sm + bn * Q;
      const double e2 = E * iS;
      st[0] = ro1; st[1] = ro1 * sm; st[2] = ro1 * vy2; st[3] = ro1 * vz2; st[4] = e2;
      st[5] = uh[5]; st[6] = uh[6]; st[7] = uh[7];
#pragma unroll
      for (int n = 0; n < 8; ++n) out[n] = S * (st[n] - us[n]) + (left ? fl[n] : fr[n]);
      region = left ? 2 : 3;
      // reverse
      double a_S = 0, a_st[8], a_us[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        a_S += a_f[n] * (st[n] - us[n]);
        a_st[n] = S * a_f[n];
        a_us[n] = -S * a_f[n];
      }
      double a_ro1 = a_st[0] + sm * a_st[1] + vy2 * a_st[2] + vz2 * a_st[3];
      a_sm += ro1 * a_st[1];
      double a_vy2 = ro1 * a_st[2], a_vz2 = ro1 * a_st[3];
      a_uh[5] += a_st[5];
      a_uh[6] += a_st[6];
      a_uh[7] += a_st[7];
      const double aE = iS * a_st[4];
      const double a_iS = E * a_st[4];
      a_S += us[4] * aE;
      const double a_v1 = -(us[4] + pts) * aE;
      a_us[4] += (S - v1) * aE;
      const double a_pts = -v1 * aE;
      a_pt += sm * aE;
      a_sm += pt * aE;
      a_bn += (Q - bn * sm) * aE;
      const double a_vb = bn * aE;
      a_sm -= bn * bn * aE;
      a_vy2 -= bn * uh[6] * aE;
      a_uh[6] -= bn * vy2 * aE;
      a_vz2 -= bn * uh[7] * aE;
      a_uh[7] -= bn * vz2 * aE;
      a_uh[2] += iuh0 * a_vy2;
      a_uh[3] += iuh0 * a_vz2;
      a_iuh0 += uh[2] * a_vy2 + uh[3] * a_vz2;
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        a_fl[n] += left ? a_f[n] : 0.0;
        a_fr[n] += left ? 0.0 : a_f[n];
        a_ul[n] += left ? a_us[n] : 0.0;
        a_ur[n] += left ? 0.0 : a_us[n];
      }
      a_vl[1] += left ? a_v1 : 0.0;
      a_vr[1] += left ? 0.0 : a_v1;
      a_sl += left ? a_S : 0.0;
      a_sr += left ? 0.0 : a_S;
      a_rol1 += left ? a_ro1 : 0.0;
      a_ror1 += left ? 0.0 : a_ro1;
      a_ilm += left ? a_iS : 0.0;
      a_irm += left ? 0.0 : a_iS;
      a_ptl += left ? a_pts : 0.0;
      a_ptr += left ? 0.0 : a_pts;
      a_vbL += left ? a_vb : 0.0;
      a_vbR += left ? 0.0 : a_vb;
    } else {
      StarSide L, Rt;
      star_forward(vl, ul, sl, ilm, sm, bn, bn2, pt, ptl, vbL, rol1, L);
      star_forward(vr, ur, sr, irm, sm, bn, bn2, pt, ptr, vbR, ror1, Rt);
      const double sl1 = sm - sal, sr1 = sm + sar;
      double a_L[8] = {0, 0, 0, 0, 0, 0, 0, 0}, a_R[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      double a_vyl1 = 0, a_vzl1 = 0, a_vyr1 = 0, a_vzr1 = 0;
      if (sl1 >= 0.0) {
        region = 4;
        for (int n = 0; n < 8; ++n) {
          out[n] = sl * (L.u1[n] - ul[n]) + fl[n];
          a_fl[n] += a_f[n];
          a_sl += a_f[n] * (L.u1[n] - ul[n]);
          a_L[n] += sl * a_f[n];
          a_ul[n] -= sl * a_f[n];
        }
      } else if (sr1 <= 0.0) {
        region = 5;
        for (int n = 0; n < 8; ++n) {
          out[n] = sr * (Rt.u1[n] - ur[n]) + fr[n];
          a_fr[n] += a_f[n];
          a_sr += a_f[n] * (Rt.u1[n] - ur[n]);
          a_R[n] += sr * a_f[n];
          a_ur[n] -= sr * a_f[n];
        }
      } else {
        // central states (HLL_rot.f90:861-898)
        const double rols = rol1 * rsl, rors = ror1 * rsr;
        const double s = rols + rors;
        const double f1c = 1.0 / s;
        const double f2 = rsign1(bn);
        const double Y = rols * L.vy1 + rors * Rt.vy1 + (Rt.u1[6] - L.u1[6]) * f2;
        const double Z = rols * L.vz1 + rors * Rt.vz1 + (Rt.u1[7] - L.u1[7]) * f2;
        const double vy2 = f1c * Y, vz2 = f1c * Z;
        const double B6 = rols * Rt.u1[6] + rors * L.u1[6] + rols * rors * (Rt.vy1 - L.vy1) * f2;
        const double B7 = rols * Rt.u1[7] + rors * L.u1[7] + rols * rors * (Rt.vz1 - L.vz1) * f2;
        double u2[8];
        u2[5] = bn;
        u2[6] = f1c * B6;
        u2[7] = f1c * B7;
        const bool left = sm >= 0.0;
        region = left ? 6 : 7;
        double Pu1[8], us[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          Pu1[n] = left ? L.u1[n] : Rt.u1[n];
          us[n] = left ? ul[n] : ur[n];
        }
        const double Pvy1 = left ? L.vy1 : Rt.vy1, Pvz1 = left ? L.vz1 : Rt.vz1;
        const double ro1 = left ? rol1 : ror1;
        const double ros = left ? rols : rors;
        const double S1 = left ? sl1 : sr1;
        const double S = left ? sl : sr;
        const double sg = left ? -1.0 : 1.0;   // u2[4] = P.u1[4] + sg*ros*W*f2
        const double W = Pvy1 * Pu1[6] + Pvz1 * Pu1[7] - vy2 * u2[6] - vz2 * u2[7];
        u2[0] = ro1;
        u2[4] = Pu1[4] + sg * ros * W * f2;
        u2[1] = ro1 * sm;
        u2[2] = ro1 * vy2;
        u2[3] = ro1 * vz2;
        double a_S1 = 0, a_S = 0, a_u2[8], a_P[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          out[n] = S1 * u2[n] - (S1 - S) * Pu1[n] - S * us[n] + (left ? fl[n] : fr[n]);
          a_S1 += a_f[n] * (u2[n] - Pu1[n]);
          a_S += a_f[n] * (Pu1[n] - us[n]);
          a_u2[n] = S1 * a_f[n];
          a_P[n] = -(S1 - S) * a_f[n];
          a_fl[n] += left ? a_f[n] : 0.0;
          a_fr[n] += left ? 0.0 : a_f[n];
          a_ul[n] -= left ? S * a_f[n] : 0.0;
          a_ur[n] -= left ? 0.0 : S * a_f[n];
        }
        // u2[4]
        a_P[4] += a_u2[4];
        double a_ros = sg * W * f2 * a_u2[4];
        const double a_W = sg * ros * f2 * a_u2[4];
        const double a_Pvy1 = Pu1[6] * a_W, a_Pvz1 = Pu1[7] * a_W;
        a_P[6] += Pvy1 * a_W;
        a_P[7] += Pvz1 * a_W;
        double a_vy2 = -u2[6] * a_W, a_vz2 = -u2[7] * a_W;
        a_u2[6] -= vy2 * a_W;
        a_u2[7] -= vz2 * a_W;
        // u2[0..3]
        const double a_ro1 = a_u2[0] + sm * a_u2[1] + vy2 * a_u2[2] + vz2 * a_u2[3];
        a_sm += ro1 * a_u2[1];
        a_vy2 += ro1 * a_u2[2];
        a_vz2 += ro1 * a_u2[3];
        a_bn += a_u2[5];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          a_L[n] += left ? a_P[n] : 0.0;
          a_R[n] += left ? 0.0 : a_P[n];
        }
        a_rol1 += left ? a_ro1 : 0.0;
        a_ror1 += left ? 0.0 : a_ro1;
        a_vyl1 += left ? a_Pvy1 : 0.0;
        a_vyr1 += left ? 0.0 : a_Pvy1;
        a_vzl1 += left ? a_Pvz1 : 0.0;
        a_vzr1 += left ? 0.0 : a_Pvz1;
        double a_rols = left ? a_ros : 0.0, a_rors = left ? 0.0 : a_ros;
        // u2[6] = f1c*B6, u2[7] = f1c*B7
        double a_f1c = B6 * a_u2[6] + B7 * a_u2[7];
        const double aB6 = f1c * a_u2[6], aB7 = f1c * a_u2[7];
        a_rols += Rt.u1[6] * aB6 + rors * (Rt.vy1 - L.vy1) * f2 * aB6 +
                  Rt.u1[7] * aB7 + rors * (Rt.vz1 - L.vz1) * f2 * aB7;
        a_rors += L.u1[6] * aB6 + rols * (Rt.vy1 - L.vy1) * f2 * aB6 +
                  L.u1[7] * aB7 + rols * (Rt.vz1 - L.vz1) * f2 * aB7;
        a_R[6] += rols * aB6;
        a_L[6] += rors * aB6;
        a_R[7] += rols * aB7;
        a_L[7] += rors * aB7;
        a_vyr1 += rols * rors * f2 * aB6;
        a_vyl1 -= rols * rors * f2 * aB6;
        a_vzr1 += rols * rors * f2 * aB7;
        a_vzl1 -= rols * rors * f2 * aB7;
        // vy2 = f1c*Y, vz2 = f1c*Z
        a_f1c += Y * a_vy2 + Z * a_vz2;
        const double aY = f1c * a_vy2, aZ = f1c * a_vz2;
        a_rols += L.vy1 * aY + L.vz1 * aZ;
        a_rors += Rt.vy1 * aY + Rt.vz1 * aZ;
        a_vyl1 += rols * aY;
        a_vyr1 += rors * aY;
        a_vzl1 += rols * aZ;
        a_vzr1 += rors * aZ;
        a_R[6] += f2 * aY;
        a_L[6] -= f2 * aY;
        a_R[7] += f2 * aZ;
        a_L[7] -= f2 * aZ;
        // f1c = 1/s
        const double a_s = -f1c * f1c * a_f1c;
        a_rols += a_s;
        a_rors += a_s;
        a_rol1 += rsl * a_rols;
        a_rsl += rol1 * a_rols;
        a_ror1 += rsr * a_rors;
        a_rsr += ror1 * a_rors;
        // S1: sl1 = sm - sal, sr1 = sm + sar
        a_sm += a_S1;
        if (left) {
          a_sal -= a_S1;
          a_sl += a_S;
        } else {
          a_sar += a_S1;
          a_sr += a_S;
        }
      }
      // single-star states
      star_reverse(vl, ul, sl, sm, bn, pt, ptl, vbL, rol1, L, a_L, a_vyl1, a_vzl1, a_vl, a_ul,
                   a_sl, a_sm, a_bn, a_bn2, a_pt, a_ptl, a_vbL, a_rol1, a_ilm);
      star_reverse(vr, ur, sr, sm, bn, pt, ptr, vbR, ror1, Rt, a_R, a_vyr1, a_vzr1, a_vr, a_ur,
                   a_sr, a_sm, a_bn, a_bn2, a_pt, a_ptr, a_vbR, a_ror1, a_irm);
    }
    if (flx_out)
      for (int n = 0; n < 8; ++n) flx_out[n] = out[n];
    // ---- reverse of the shared fan quantities
    a_bn += 2.0 * bn * a_bn2;
    a_bn += dabs(bn) * (rsl * a_sal + rsr * a_sar);
    a_rsl += rabs(bn) * a_sal;
    a_rsr += rabs(bn) * a_sar;
    a_uh[5] += a_bn;
    a_rol1 += -0.5 * rsl * rsl * rsl * a_rsl;
    a_ror1 += -0.5 * rsr * rsr * rsr * a_rsr;
    // rol1 = vl0*(sl - vl1)*ilm, ror1 likewise
    a_vl[0] += (sl - vl[1]) * ilm * a_rol1;
    a_sl += vl[0] * ilm * a_rol1;
    a_vl[1] -= vl[0] * ilm * a_rol1;
    a_ilm += vl[0] * (sl - vl[1]) * a_rol1;
    a_vr[0] += (sr - vr[1]) * irm * a_ror1;
    a_sr += vr[0] * irm * a_ror1;
    a_vr[1] -= vr[0] * irm * a_ror1;
    a_irm += vr[0] * (sr - vr[1]) * a_ror1;
    // ilm = 1/(sl - sm), irm = 1/(sr - sm)
    a_sl -= ilm * ilm * a_ilm;
    a_sm += ilm * ilm * a_ilm;
    a_sr -= irm * irm * a_irm;
    a_sm += irm * irm * a_irm;
    // pt = ptl + vl0*(sl - vl1)*(sm - vl1)
    a_ptl += a_pt;
    a_vl[0] += (sl - vl[1]) * (sm - vl[1]) * a_pt;
    a_sl += vl[0] * (sm - vl[1]) * a_pt;
    a_sm += vl[0] * (sl - vl[1]) * a_pt;
    a_vl[1] -= vl[0] * ((sm - vl[1]) + (sl - vl[1])) * a_pt;
    // sm = uh1*iuh0, iuh0 = 1/uh0
    a_uh[1] += iuh0 * a_sm;
    a_iuh0 += uh[1] * a_sm;
    a_uh[0] -= iuh0 * iuh0 * a_iuh0;
    // uh = f1*(sr*ur - sl*ul - fr + fl)
    double a_f1 = 0.0;
    for (int n = 0; n < 8; ++n) {
      a_f1 += w[n] * a_uh[n];
      a_sr += f1 * ur[n] * a_uh[n];
      a_ur[n] += f1 * sr * a_uh[n];
      a_sl -= f1 * ul[n] * a_uh[n];
      a_ul[n] -= f1 * sl * a_uh[n];
      a_fr[n] -= f1 * a_uh[n];
      a_fl[n] += f1 * a_uh[n];
    }
    a_sr -= f1 * f1 * a_f1;
    a_sl += f1 * f1 * a_f1;
  }
  // ---- reverse of the wave speeds
  {
    double a_vfm = a_sr - a_sl;
    if (vmin_left) a_vl[1] += a_sl; else a_vr[1] += a_sl;
    if (vmax_left) a_vl[1] += a_sr; else a_vr[1] += a_sr;
    const double a_vfl = vf_left ? a_vfm : 0.0, a_vfr = vf_left ? 0.0 : a_vfm;
    double a_b2l = 0.0, a_b2r = 0.0;
    if (vfl > 0.0 && a_vfl != 0.0) {
      const double aQ = a_vfl / (2.0 * vfl);
      double a_A = aQ / (2.0 * vl[0]);
      const double a_dd = aQ / (2.0 * vl[0]);
      a_vl[0] -= Ql / vl[0] * aQ;
      if (discl > 0.0) {
        const double a_disc = a_dd / (2.0 * ddl);
        a_A += 2.0 * Al * a_disc;
        const double a_f1 = -4.0 * (vl[5] * vl[5]) * a_disc;
        a_vl[5] += -8.0 * f1l * vl[5] * a_disc;
        a_vl[4] += gm * (a_f1 + a_A);
      } else {
        a_vl[4] += gm * a_A;
      }
      a_b2l += a_A;
    }
    if (vfr > 0.0 && a_vfr != 0.0) {
      const double aQ = a_vfr / (2.0 * vfr);
      double a_A = aQ / (2.0 * vr[0]);
      const double a_dd = aQ / (2.0 * vr[0]);
      a_vr[0] -= Qr / vr[0] * aQ;
      if (discr > 0.0) {
        const double a_disc = a_dd / (2.0 * ddr);
        a_A += 2.0 * Ar * a_disc;
        const double a_f1 = -4.0 * (vr[5] * vr[5]) * a_disc;
        a_vr[5] += -8.0 * f1r * vr[5] * a_disc;
        a_vr[4] += gm * (a_f1 + a_A);
      } else {
        a_vr[4] += gm * a_A;
      }
      a_b2r += a_A;
    }
    // physical fluxes
    a_ul[1] += a_fl[0] + vl[1] * a_fl[1] + vl[2] * a_fl[2] + vl[3] * a_fl[3];
    a_vl[1] += ul[1] * a_fl[1] + (ul[4] + ptl) * a_fl[4] + vl[6] * a_fl[6] + vl[7] * a_fl[7];
    a_ptl += a_fl[1] + vl[1] * a_fl[4];
    a_vl[5] += -2.0 * vl[5] * a_fl[1] - vl[6] * a_fl[2] - vl[7] * a_fl[3] - vbL * a_fl[4] -
               vl[2] * a_fl[6] - vl[3] * a_fl[7];
    a_vl[2] += ul[1] * a_fl[2] - vl[5] * a_fl[6];
    a_vl[3] += ul[1] * a_fl[3] - vl[5] * a_fl[7];
    a_vl[6] += -vl[5] * a_fl[2] + vl[1] * a_fl[6];
    a_vl[7] += -vl[5] * a_fl[3] + vl[1] * a_fl[7];
    a_ul[4] += vl[1] * a_fl[4];
    a_vbL -= vl[5] * a_fl[4];
    a_ur[1] += a_fr[0] + vr[1] * a_fr[1] + vr[2] * a_fr[2] + vr[3] * a_fr[3];
    a_vr[1] += ur[1] * a_fr[1] + (ur[4] + ptr) * a_fr[4] + vr[6] * a_fr[6] + vr[7] * a_fr[7];
    a_ptr += a_fr[1] + vr[1] * a_fr[4];
    a_vr[5] += -2.0 * vr[5] * a_fr[1] - vr[6] * a_fr[2] - vr[7] * a_fr[3] - vbR * a_fr[4] -
               vr[2] * a_fr[6] - vr[3] * a_fr[7];
    a_vr[2] += ur[1] * a_fr[2] - vr[5] * a_fr[6];
    a_vr[3] += ur[1] * a_fr[3] - vr[5] * a_fr[7];
    a_vr[6] += -vr[5] * a_fr[2] + vr[1] * a_fr[6];
    a_vr[7] += -vr[5] * a_fr[3] + vr[1] * a_fr[7];
    a_ur[4] += vr[1] * a_fr[4];
    a_vbR -= vr[5] * a_fr[4];
    // vb, pt
    a_vl[1] += vl[5] * a_vbL; a_vl[5] += vl[1] * a_vbL;
    a_vl[2] += vl[6] * a_vbL; a_vl[6] += vl[2] * a_vbL;
    a_vl[3] += vl[7] * a_vbL; a_vl[7] += vl[3] * a_vbL;
    a_vr[1] += vr[5] * a_vbR; a_vr[5] += vr[1] * a_vbR;
    a_vr[2] += vr[6] * a_vbR; a_vr[6] += vr[2] * a_vbR;
    a_vr[3] += vr[7] * a_vbR; a_vr[7] += vr[3] * a_vbR;
    a_vl[4] += a_ptl;
    a_b2l += 0.5 * a_ptl;
    a_vr[4] += a_ptr;
    a_b2r += 0.5 * a_ptr;
    // conserved vectors
    a_vl[0] += a_ul[0] + 0.5 * kel * a_ul[4];
    a_vr[0] += a_ur[0] + 0.5 * ker * a_ur[4];
    a_vl[4] += igm1 * a_ul[4];
    a_vr[4] += igm1 * a_ur[4];
    a_b2l += 0.5 * a_ul[4];
    a_b2r += 0.5 * a_ur[4];
    for (int k = 1; k <= 3; ++k) {
      a_vl[0] += vl[k] * a_ul[k];
      a_vl[k] += vl[0] * a_ul[k] + vl[0] * vl[k] * a_ul[4];
      a_vr[0] += vr[k] * a_ur[k];
      a_vr[k] += vr[0] * a_ur[k] + vr[0] * vr[k] * a_ur[4];
    }
    for (int k = 5; k <= 7; ++k) {
      a_vl[k] += a_ul[k] + 2.0 * vl[k] * a_b2l;
      a_vr[k] += a_ur[k] + 2.0 * vr[k] * a_b2r;
    }
  }
  return region;
}

// ---------------------------------------------------------------- collision source

// Reverse of the explicit collision exchange of source_PIP (PIP_rot.f90:1333-1368,
// flag_pip_imp = 0) taken on the cq2pv rewrite of the stage state of one cell.  a_ds[k]
// (k = 1..4) is the cotangent of dS_k; the ion state gains +dS and the neutral state -dS.
// Returns d(dS)/d(alpha_c) . a_ds.
PIP_HD double collision_vjp(const double (&um)[8], const double (&uh)[5], const double (&a_ds)[5],
                            double gm, double igm1, double ac, double ro_lim, double pr_lim,
                            double (&a_um)[8], double (&a_uh)[5]) {
  // forward: rewrite through primitives (in copies)
  double wm[8], wh[5];
  for (int n = 0; n < 8; ++n) wm[n] = um[n];
  for (int n = 0; n < 5; ++n) wh[n] = uh[n];
  const Prim<double> qm = cq2pv_mhd_rcp<double, 8>(wm, gm, igm1, ro_lim, pr_lim);
  const Prim<double> qh = cq2pv_hd_rcp<double>(wh, gm, igm1, ro_lim, pr_lim);
  const double te = qm.pr / qm.de * gm * kMuP;
  const double nte = qh.pr / qh.de * gm * kMuN;
  const double c32g = 3.0 / gm / 2.0;
  const double Qb = 0.5 * ((qh.vx * qh.vx - qm.vx * qm.vx) + (qh.vy * qh.vy - qm.vy * qm.vy) +
                           (qh.vz * qh.vz - qm.vz * qm.vz)) +
                    c32g * (nte - te);
  double dac = 0.0;
  double a_wm[5] = {0, 0, 0, 0, 0}, a_wh[5] = {0, 0, 0, 0, 0};
  double a_qm[5] = {0, 0, 0, 0, 0}, a_qh[5] = {0, 0, 0, 0, 0};
  for (int k = 1; k <= 3; ++k) {
    const double a = a_ds[k];
    dac += a * (wm[0] * wh[k] - wh[0] * wm[k]);
    a_wm[0] += ac * wh[k] * a;
    a_wh[k] += ac * wm[0] * a;
    a_wh[0] -= ac * wm[k] * a;
    a_wm[k] -= ac * wh[0] * a;
  }
  {
    const double a = a_ds[4];
    dac += a * qh.de * qm.de * Qb;
    a_qh[0] += ac * qm.de * Qb * a;
    a_qm[0] += ac * qh.de * Qb * a;
    const double aQ = ac * qh.de * qm.de * a;
    a_qh[1] += qh.vx * aQ; a_qh[2] += qh.vy * aQ; a_qh[3] += qh.vz * aQ;
    a_qm[1] -= qm.vx * aQ; a_qm[2] -= qm.vy * aQ; a_qm[3] -= qm.vz * aQ;
    const double a_nte = c32g * aQ, a_te = -c32g * aQ;
    a_qm[4] += gm * kMuP / qm.de * a_te;
    a_qm[0] -= te / qm.de * a_te;
    a_qh[4] += gm * kMuN / qh.de * a_nte;
    a_qh[0] -= nte / qh.de * a_nte;
  }
  cq2pv_vjp<8, 3>(um, a_wm, a_qm, gm, igm1, ro_lim, pr_lim, a_um);
  cq2pv_vjp<5, 0>(uh, a_wh, a_qh, gm, igm1, ro_lim, pr_lim, a_uh);
  return dac;
}

// ---------------------------------------------------------------- CFL candidates

// Gradient of cfl_mhd_cell (Scheme_rot.f90:279-283) with respect to the conserved ion
// state of the cell (primitives by cq2pv).  Returns the candidate.
PIP_HD double cfl_mhd_grad(const double (&u)[8], double gm, double ro_lim, double pr_lim, double sg,
                           double (&g)[8]) {
  const double inv = 1.0 / u[0];
  const double v[3] = {u[1] * inv, u[2] * inv, u[3] * inv};
  const double kin = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double bb = u[5] * u[5] + u[6] * u[6] + u[7] * u[7];
  const double pr_raw = (gm - 1.0) * (u[4] - 0.5 * u[0] * kin - 0.5 * bb);
  const double pr = rmax(pr_raw, pr_lim);
  const double de = rmax(u[0], ro_lim);
  const double dm = rmax(de, kTiny);
  const double cs2 = gm * pr / dm, valf2 = bb / dm;
  const double vabs = rsqrt_(kin);
  const double c = rsqrt_(cs2 + valf2);
  const double Dn = vabs + c;
  const double cand = sg / Dn;
  for (int n = 0; n < 8; ++n) g[n] = 0.0;
  const double a_Dn = -sg / (Dn * Dn);
  const double a_w = c > 0.0 ? a_Dn / (2.0 * c) : 0.0;
  double a_pr = gm / dm * a_w;
  const double a_dm = -(cs2 + valf2) / dm * a_w;
  double a_bb = a_w / dm;
  double a_de = de >= kTiny ? a_dm : 0.0;
  double a_v[3] = {0, 0, 0};
  if (vabs > 0.0)
    for (int k = 0; k < 3; ++k) a_v[k] = v[k] / vabs * a_Dn;
  const double a_prraw = pr_raw >= pr_lim ? a_pr : 0.0;
  double a_u0 = u[0] >= ro_lim ? a_de : 0.0;
  g[4] += (gm - 1.0) * a_prraw;
  a_u0 += -(gm - 1.0) * 0.5 * kin * a_prraw;
  a_bb += -(gm - 1.0) * 0.5 * a_prraw;
  for (int k = 0; k < 3; ++k) {
    a_v[k] += -(gm - 1.0) * u[0] * v[k] * a_prraw;
    g[1 + k] += inv * a_v[k];
    a_u0 -= v[k] * inv * a_v[k];
  }
  for (int k = 5; k <= 7; ++k) g[k] += 2.0 * u[k] * a_bb;
  g[0] += a_u0;
  (void)a_pr;
  return cand;
}

// Gradient of cfl_hd_cell (Scheme_rot.f90:229-233).  Returns the candidate.
PIP_HD double cfl_hd_grad(const double (&u)[5], double gm, double ro_lim, double pr_lim, double sg,
                          double (&g)[5]) {
  const double inv = 1.0 / u[0];
  const double v[3] = {u[1] * inv, u[2] * inv, u[3] * inv};
  const double kin = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double pr_raw = (gm - 1.0) * (u[4] - 0.5 * u[0] * kin);
  const double pr = rmax(pr_raw, pr_lim);
  const double de = rmax(u[0], ro_lim);
  const double X = gm * pr / de;
  const double cs = rsqrt_(X);
  const double kc = rmax(kin, kTiny);
  const double vabs = rsqrt_(kc);
  const double Dn = vabs + cs;
  const double cand = sg / Dn;
  for (int n = 0; n < 5; ++n) g[n] = 0.0;
  const double a_Dn = -sg / (Dn * Dn);
  const double a_X = cs > 0.0 ? a_Dn / (2.0 * cs) : 0.0;
  const double a_pr = gm / de * a_X;
  const double a_de = -X / de * a_X;
  double a_v[3] = {0, 0, 0};
  if (kin >= kTiny)
    for (int k = 0; k < 3; ++k) a_v[k] = v[k] / vabs * a_Dn;
  const double a_prraw = pr_raw >= pr_lim ? a_pr : 0.0;
  double a_u0 = u[0] >= ro_lim ? a_de : 0.0;
  g[4] += (gm - 1.0) * a_prraw;
  a_u0 += -(gm - 1.0) * 0.5 * kin * a_prraw;
  for (int k = 0; k < 3; ++k) {
    a_v[k] += -(gm - 1.0) * u[0] * v[k] * a_prraw;
    g[1 + k] += inv * a_v[k];
    a_u0 -= v[k] * inv * a_v[k];
  }
  g[0] += a_u0;
  return cand;
}

}  // namespace adj
}  // namespace pip
