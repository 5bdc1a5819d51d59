// Host check of the hand-written vector-Jacobian products in pip_adjoint_physics.cuh
// against central finite differences of the forward functions of pip_physics.cuh.
//
// For random states in every branch region, random cotangents a and random directions d:
//   <VJP(a), d>  vs  (phi(x + h d) - phi(x - h d)) / 2h,   phi(x) = <a, f(x)>.
// Cases whose branch (minmod slope, HLLD region, floor) differs between x - h d and
// x + h d are skipped (the derivative is taken on the branch the forward takes).
// Prints one line per function and exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <functional>

#include "pip_adjoint_physics.cuh"

using namespace pip;

static std::mt19937_64 rng(20260311);
static double unif(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }
static double gaus() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

static const double GM = 5.0 / 3.0, IGM1 = 1.0 / (GM - 1.0), RO_LIM = 1e-6, PR_LIM = 1e-6;

struct Stat {
  const char *name;
  int checked = 0, skipped = 0, failed = 0;
  double worst = 0.0;
  void add(double vjp, double fd, double scale, double tol) {
    // relative to |fd|, floored at 1e-4 of the summed term magnitudes: the central
    // difference itself carries ~eps*|phi|/h of rounding error
    const double err = std::fabs(vjp - fd) / (std::fabs(fd) + scale * 1e-4 + 1e-300);
    ++checked;
    if (err > worst) worst = err;
    if (err > tol) {
      ++failed;
      if (failed <= 3) std::printf("  %s: vjp %.15e fd %.15e rel %.3e\n", name, vjp, fd, err);
    }
  }
  bool report() const {
    std::printf("%-14s checked %5d skipped %4d failed %3d worst_rel %.3e\n", name, checked, skipped,
                failed, worst);
    return failed == 0 && checked > 0;
  }
};

// central difference of phi along d with step h (relative to the inputs' scale)
template <int N>
static double fd(const std::function<double(const double *)> &phi, const double *x, const double *d,
                 double h) {
  double xp[N], xm[N];
  for (int i = 0; i < N; ++i) {
    xp[i] = x[i] + h * d[i];
    xm[i] = x[i] - h * d[i];
  }
  return (phi(xp) - phi(xm)) / (2.0 * h);
}

// a primitive MHD state (ro, vn, vt1, vt2, pr, bn, bt1, bt2)
static void mhd_state(double (&v)[8], double vn, double bn, double bt) {
  v[0] = unif(0.5, 2.0);
  v[1] = vn + 0.2 * gaus();
  v[2] = 0.3 * gaus();
  v[3] = 0.3 * gaus();
  v[4] = unif(0.2, 1.5);
  v[5] = bn + 0.1 * gaus();
  v[6] = bt * gaus();
  v[7] = bt * gaus();
}

static bool check_hlld() {
  Stat st{"hlld"};
  int region_hits[8] = {0};
  struct Case { double vn, bn, bt, pr_scale, ro_scale; };
  const Case cases[] = {
      {10.0, 0.5, 0.5, 1.0, 1.0},   // supersonic right: F_L
      {-10.0, 0.5, 0.5, 1.0, 1.0},  // supersonic left: F_R
      {0.0, 1.0, 0.5, 1.0, 1.0},    // central states
      {0.0, 0.05, 0.8, 1.0, 1.0},   // weak normal field: star states / central
      {1.2, 0.05, 0.8, 1.0, 1.0},   // flow with weak normal field: L*
      {-1.2, 0.05, 0.8, 1.0, 1.0},  // R*
      {0.0, 2.5, 0.0, 0.05, 1.0},   // field-aligned, Alfven > sound: HLLC-G
      {0.3, 2.5, 0.01, 0.05, 1.0},
      {-0.3, 2.5, 0.01, 0.05, 1.0},
  };
  for (const Case &c : cases) {
    for (int trial = 0; trial < 400; ++trial) {
      double vl[8], vr[8], a[8], d[16], x[16];
      mhd_state(vl, c.vn, c.bn, c.bt);
      mhd_state(vr, c.vn, c.bn, c.bt);
      vl[4] *= c.pr_scale;
      vr[4] *= c.pr_scale;
      vr[5] = vl[5];  // continuous normal field, as the scheme sees it most of the time
      if (trial % 3 == 0) vr[5] = vl[5] + 0.05 * gaus();
      for (int n = 0; n < 8; ++n) a[n] = gaus();
      for (int n = 0; n < 16; ++n) d[n] = gaus();
      for (int n = 0; n < 8; ++n) { x[n] = vl[n]; x[8 + n] = vr[n]; }
      double a_vl[8] = {0}, a_vr[8] = {0}, flx[8], ref[8];
      const int region = adj::hlld_vjp(vl, vr, a, GM, IGM1, a_vl, a_vr, flx);
      hlld_flux_rcp<double, 8>(vl, vr, ref, GM, IGM1, 0.0);
      for (int n = 0; n < 8; ++n)
        if (std::fabs(flx[n] - ref[n]) > 1e-13 * (1.0 + std::fabs(ref[n]))) {
          std::printf("  hlld flux mismatch region %d n %d: %.17g vs %.17g\n", region, n, flx[n], ref[n]);
          st.failed++;
        }
      const double h = 1e-6;
      // branch at the two ends
      double xp[16], xm[16], dum[8], za[8] = {0};
      for (int i = 0; i < 16; ++i) { xp[i] = x[i] + h * d[i]; xm[i] = x[i] - h * d[i]; }
      double lp[8], rp[8], lm[8], rm[8];
      for (int n = 0; n < 8; ++n) { lp[n] = xp[n]; rp[n] = xp[8 + n]; lm[n] = xm[n]; rm[n] = xm[8 + n]; }
      double t1[8] = {0}, t2[8] = {0}, t3[8] = {0}, t4[8] = {0};
      const int rpn = adj::hlld_vjp(lp, rp, za, GM, IGM1, t1, t2, dum);
      const int rmn = adj::hlld_vjp(lm, rm, za, GM, IGM1, t3, t4, dum);
      if (rpn != region || rmn != region) { st.skipped++; continue; }
      auto phi = [&](const double *y) {
        double l[8], r[8], f[8];
        for (int n = 0; n < 8; ++n) { l[n] = y[n]; r[n] = y[8 + n]; }
        hlld_flux_rcp<double, 8>(l, r, f, GM, IGM1, 0.0);
        double s = 0.0;
        for (int n = 0; n < 8; ++n) s += a[n] * f[n];
        return s;
      };
      const double g = fd<16>(phi, x, d, h);
      double v = 0.0, scale = 0.0;
      for (int n = 0; n < 8; ++n) {
        v += a_vl[n] * d[n] + a_vr[n] * d[8 + n];
        scale += std::fabs(a_vl[n] * d[n]) + std::fabs(a_vr[n] * d[8 + n]);
      }
      st.add(v, g, scale, 2e-6);
      region_hits[region]++;
    }
  }
  std::printf("  hlld regions checked:");
  for (int r = 0; r < 8; ++r) std::printf(" %d:%d", r, region_hits[r]);
  std::printf("\n");
  bool all = true;
  for (int r = 0; r < 8; ++r) all &= region_hits[r] > 0;
  if (!all) std::printf("  hlld: some region never checked\n");
  return st.report() && all;
}

static bool check_hllc() {
  Stat st{"hllc"};
  const double vns[] = {0.0, 0.5, -0.5, 3.0, -3.0};
  for (double vn : vns)
    for (int trial = 0; trial < 400; ++trial) {
      double vl[5], vr[5], a[5], d[10], x[10];
      for (int s = 0; s < 2; ++s) {
        double *v = s ? vr : vl;
        v[0] = unif(0.5, 2.0);
        v[1] = vn + 0.3 * gaus();
        v[2] = 0.3 * gaus();
        v[3] = 0.3 * gaus();
        v[4] = unif(0.2, 1.5);
      }
      for (int n = 0; n < 5; ++n) { a[n] = gaus(); x[n] = vl[n]; x[5 + n] = vr[n]; }
      for (int n = 0; n < 10; ++n) d[n] = gaus();
      double a_vl[5] = {0}, a_vr[5] = {0}, flx[5], ref[5];
      adj::hllc_vjp(vl, vr, a, GM, IGM1, a_vl, a_vr, flx);
      hllc_flux_rcp<double>(vl, vr, ref, GM, IGM1);
      for (int n = 0; n < 5; ++n)
        if (std::fabs(flx[n] - ref[n]) > 1e-13 * (1.0 + std::fabs(ref[n]))) {
          std::printf("  hllc flux mismatch n %d\n", n);
          st.failed++;
        }
      auto phi = [&](const double *y) {
        double l[5], r[5], f[5];
        for (int n = 0; n < 5; ++n) { l[n] = y[n]; r[n] = y[5 + n]; }
        hllc_flux_rcp<double>(l, r, f, GM, IGM1);
        double s = 0.0;
        for (int n = 0; n < 5; ++n) s += a[n] * f[n];
        return s;
      };
      const double h = 1e-6;
      const double g = fd<10>(phi, x, d, h);
      double v = 0.0, scale = 0.0;
      for (int n = 0; n < 5; ++n) {
        v += a_vl[n] * d[n] + a_vr[n] * d[5 + n];
        scale += std::fabs(a_vl[n] * d[n]) + std::fabs(a_vr[n] * d[5 + n]);
      }
      st.add(v, g, scale, 2e-6);
    }
  return st.report();
}

static bool check_u2v() {
  Stat sm{"u2v_mhd"}, sh{"u2v_hd"};
  for (int trial = 0; trial < 2000; ++trial) {
    double u[8], a[8], d[8];
    u[0] = unif(0.3, 2.0);
    for (int k = 1; k <= 3; ++k) u[k] = u[0] * 0.5 * gaus();
    for (int k = 5; k <= 7; ++k) u[k] = 0.7 * gaus();
    const double pr = unif(0.1, 1.0);
    u[4] = pr / (GM - 1.0) + 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
           0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
    for (int n = 0; n < 8; ++n) { a[n] = gaus(); d[n] = gaus(); }
    double g[8] = {0};
    adj::u2v_mhd_vjp(u, a, GM, RO_LIM, PR_LIM, g);
    auto phi = [&](const double *y) {
      double uu[8], v[8];
      for (int n = 0; n < 8; ++n) uu[n] = y[n];
      u2v_mhd<double, 8>(uu, v, GM, RO_LIM, PR_LIM);
      double s = 0.0;
      for (int n = 0; n < 8; ++n) s += a[n] * v[n];
      return s;
    };
    double v = 0.0, sc = 0.0;
    for (int n = 0; n < 8; ++n) { v += g[n] * d[n]; sc += std::fabs(g[n] * d[n]); }
    sm.add(v, fd<8>(phi, u, d, 1e-6), sc, 1e-6);

    double uh[5] = {u[0], u[1], u[2], u[3], pr / (GM - 1.0) + 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]};
    double gh[5] = {0};
    adj::u2v_hd_vjp(uh, *reinterpret_cast<double(*)[5]>(a), GM, RO_LIM, PR_LIM, gh);
    auto phih = [&](const double *y) {
      double uu[5], vv[5];
      for (int n = 0; n < 5; ++n) uu[n] = y[n];
      u2v_hd<double>(uu, vv, GM, RO_LIM, PR_LIM);
      double s = 0.0;
      for (int n = 0; n < 5; ++n) s += a[n] * vv[n];
      return s;
    };
    v = 0.0; sc = 0.0;
    for (int n = 0; n < 5; ++n) { v += gh[n] * d[n]; sc += std::fabs(gh[n] * d[n]); }
    sh.add(v, fd<5>(phih, uh, d, 1e-6), sc, 1e-6);
  }
  // floored density: the primitives no longer depend on u0
  {
    double u[8] = {1e-9, 0.3e-9, 0.0, 0.0, 1.0, 0.2, 0.0, 0.0}, a[8] = {1, 1, 1, 1, 1, 1, 1, 1};
    double g[8] = {0};
    adj::u2v_mhd_vjp(u, a, GM, RO_LIM, PR_LIM, g);
    if (g[0] != 0.0) {
      std::printf("  u2v_mhd: floored density has d/du0 = %g\n", g[0]);
      sm.failed++;
    }
  }
  return sm.report() & sh.report();
}

static bool check_minmod() {
  Stat st{"muscl"};
  for (int trial = 0; trial < 4000; ++trial) {
    double v[4], d[4];
    for (int i = 0; i < 4; ++i) { v[i] = gaus(); d[i] = gaus(); }
    const double aL = gaus(), aR = gaus();
    // face states of cells 1, 2 of the 4-cell stencil
    auto phi = [&](const double *y) {
      const double vl = y[1] + 0.5 * minmod<double>(y[0], y[1], y[2]);
      const double vr = y[2] - 0.5 * minmod<double>(y[1], y[2], y[3]);
      return aL * vl + aR * vr;
    };
    const double h = 1e-6;
    double xp[4], xm[4];
    for (int i = 0; i < 4; ++i) { xp[i] = v[i] + h * d[i]; xm[i] = v[i] - h * d[i]; }
    const int mL = adj::minmod_mode(v[0], v[1], v[2]), mR = adj::minmod_mode(v[1], v[2], v[3]);
    if (adj::minmod_mode(xp[0], xp[1], xp[2]) != mL || adj::minmod_mode(xm[0], xm[1], xm[2]) != mL ||
        adj::minmod_mode(xp[1], xp[2], xp[3]) != mR || adj::minmod_mode(xm[1], xm[2], xm[3]) != mR) {
      st.skipped++;
      continue;
    }
    double g[4] = {0, 0, 0, 0};
    g[1] += aL;
    g[2] += aR;
    adj::minmod_vjp(mL, 0.5 * aL, g[0], g[1], g[2]);
    adj::minmod_vjp(mR, -0.5 * aR, g[1], g[2], g[3]);
    double v1 = 0.0, sc = 0.0;
    for (int i = 0; i < 4; ++i) { v1 += g[i] * d[i]; sc += std::fabs(g[i] * d[i]); }
    st.add(v1, fd<4>(phi, v, d, h), sc, 1e-6);
  }
  return st.report();
}

static bool check_collision() {
  Stat st{"collision"}, sa{"collision_ac"};
  for (int trial = 0; trial < 2000; ++trial) {
    double um[8], uh[5], a[5], d[13];
    um[0] = unif(0.3, 2.0);
    uh[0] = unif(0.3, 2.0);
    for (int k = 1; k <= 3; ++k) { um[k] = um[0] * 0.5 * gaus(); uh[k] = uh[0] * 0.5 * gaus(); }
    for (int k = 5; k <= 7; ++k) um[k] = 0.7 * gaus();
    um[4] = unif(0.1, 1.0) / (GM - 1.0) + 0.5 * (um[1] * um[1] + um[2] * um[2] + um[3] * um[3]) / um[0] +
            0.5 * (um[5] * um[5] + um[6] * um[6] + um[7] * um[7]);
    uh[4] = unif(0.1, 1.0) / (GM - 1.0) + 0.5 * (uh[1] * uh[1] + uh[2] * uh[2] + uh[3] * uh[3]) / uh[0];
    a[0] = 0.0;
    for (int k = 1; k < 5; ++k) a[k] = gaus();
    for (int n = 0; n < 13; ++n) d[n] = gaus();
    const double ac = unif(0.5, 50.0);
    double gm_[8] = {0}, gh_[5] = {0};
    const double dac = adj::collision_vjp(um, uh, a, GM, IGM1, ac, RO_LIM, PR_LIM, gm_, gh_);
    auto ds_of = [&](const double *y, double acx) {
      double m[8], hh[5];
      for (int n = 0; n < 8; ++n) m[n] = y[n];
      for (int n = 0; n < 5; ++n) hh[n] = y[8 + n];
      const Prim<double> qh = cq2pv_hd_rcp<double>(hh, GM, IGM1, RO_LIM, PR_LIM);
      const Prim<double> qm = cq2pv_mhd_rcp<double, 8>(m, GM, IGM1, RO_LIM, PR_LIM);
      const double te = qm.pr / qm.de * GM * kMuP, nte = qh.pr / qh.de * GM * kMuN;
      double s = 0.0;
      for (int k = 1; k <= 3; ++k) s += a[k] * acx * (m[0] * hh[k] - hh[0] * m[k]);
      s += a[4] * acx * qh.de * qm.de *
           (0.5 * ((qh.vx * qh.vx - qm.vx * qm.vx) + (qh.vy * qh.vy - qm.vy * qm.vy) +
                   (qh.vz * qh.vz - qm.vz * qm.vz)) +
            3.0 / GM / 2.0 * (nte - te));
      return s;
    };
    double x[13];
    for (int n = 0; n < 8; ++n) x[n] = um[n];
    for (int n = 0; n < 5; ++n) x[8 + n] = uh[n];
    auto phi = [&](const double *y) { return ds_of(y, ac); };
    double v = 0.0, sc = 0.0;
    for (int n = 0; n < 8; ++n) { v += gm_[n] * d[n]; sc += std::fabs(gm_[n] * d[n]); }
    for (int n = 0; n < 5; ++n) { v += gh_[n] * d[8 + n]; sc += std::fabs(gh_[n] * d[8 + n]); }
    st.add(v, fd<13>(phi, x, d, 1e-6), sc, 1e-6);
    const double h = 1e-6 * ac;
    const double fda = (ds_of(x, ac + h) - ds_of(x, ac - h)) / (2.0 * h);
    sa.add(dac, fda, std::fabs(dac), 1e-6);
  }
  return st.report() & sa.report();
}

static bool check_cfl() {
  Stat sm{"cfl_mhd"}, sh{"cfl_hd"};
  for (int trial = 0; trial < 2000; ++trial) {
    double u[8], d[8];
    u[0] = unif(0.3, 2.0);
    for (int k = 1; k <= 3; ++k) u[k] = u[0] * 0.5 * gaus();
    for (int k = 5; k <= 7; ++k) u[k] = 0.7 * gaus();
    u[4] = unif(0.1, 1.0) / (GM - 1.0) + 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
           0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
    for (int n = 0; n < 8; ++n) d[n] = gaus();
    const double sg = 0.3 * 0.01;
    double g[8];
    adj::cfl_mhd_grad(u, GM, RO_LIM, PR_LIM, sg, g);
    auto phi = [&](const double *y) {
      double w[8];
      for (int n = 0; n < 8; ++n) w[n] = y[n];
      const Prim<double> q = cq2pv_mhd_rcp<double, 8>(w, GM, IGM1, RO_LIM, PR_LIM);
      return cfl_mhd_cell<double>(q, w[5], w[6], w[7], GM, sg);
    };
    double v = 0.0, sc = 0.0;
    for (int n = 0; n < 8; ++n) { v += g[n] * d[n]; sc += std::fabs(g[n] * d[n]); }
    sm.add(v, fd<8>(phi, u, d, 1e-6), sc, 1e-6);
    double uh[5] = {u[0], u[1], u[2], u[3], unif(0.1, 1.0) / (GM - 1.0) + 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]};
    double gh[5];
    adj::cfl_hd_grad(uh, GM, RO_LIM, PR_LIM, sg, gh);
    auto phih = [&](const double *y) {
      double w[5];
      for (int n = 0; n < 5; ++n) w[n] = y[n];
      const Prim<double> q = cq2pv_hd_rcp<double>(w, GM, IGM1, RO_LIM, PR_LIM);
      return cfl_hd_cell<double>(q, GM, sg);
    };
    v = 0.0; sc = 0.0;
    for (int n = 0; n < 5; ++n) { v += gh[n] * d[n]; sc += std::fabs(gh[n] * d[n]); }
    sh.add(v, fd<5>(phih, uh, d, 1e-6), sc, 1e-6);
  }
  return sm.report() & sh.report();
}

int main() {
  bool ok = true;
  ok &= check_u2v();
  ok &= check_minmod();
  ok &= check_hllc();
  ok &= check_hlld();
  ok &= check_collision();
  ok &= check_cfl();
  std::printf(ok ? "ALL OK\n" : "FAILURES\n");
  return ok ? 0 : 1;
}
