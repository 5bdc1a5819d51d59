// pip_nlevel.cu -- host side of set_IR type 4 (the 6-level hydrogen model): the
// cell-independent coefficients of get_col_ion_coeff and the exponential-integral table that
// expintread loads (PIP_rot.f90:315-357) from expintcalc/colexp.dat, regenerated here by the
// algorithm of that file's generator (expintcalc/colexpintcalc.f90).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "../../include/pip_gpu.h"
#include "pip_kernels.cuh"

namespace pip {

// get_col_ion_coeff's constants (PIP_rot.f90:378-439) and, per level pair ii < jj,
// xrat, Enn, rnn, the Gaunt factor, fnn, Ann, Bnn (:411-434) and the ionisation
// coefficients An0, Bn0 (:507-524), in the Fortran operation order.  2.18e-18 is a
// default-real literal there (rounded to float); Eev of IRgetionpot likewise (:1170).
void nlev_constants(NlevConst *k) {
  static const double ev[6] = {13.6, 3.4, 1.51, 0.85, 0.54, 0.0};
  static const double gw[6] = {2.0, 8.0, 18.0, 32.0, 50.0, 1.0};
  static const float eevf[6] = {13.6f, 3.4f, 1.51f, 0.85f, 0.54f, 0.0f};
  const double ej = (double)2.18e-18f, pi = 3.1415926535897932;
  *k = NlevConst{};
  for (int m = 0; m < 6; ++m) {
    const double n = (double)(m + 1);
    k->gw[m] = gw[m];
    k->eion[m] = ev[m] / 13.6 * ej;
    k->rn[m] = m == 0 ? 0.45 : 1.94 * std::pow(n, -1.57);
    k->eev[m] = (double)eevf[m];
  }
  double bn[6];
  for (int m = 0; m < 6; ++m) {
    const double n = (double)(m + 1);
    bn[m] = m == 0 ? -0.603 : (1.0 / n) * (4.0 - 18.63 / n + 36.24 / (n * n) - 28.09 / (n * n * n));
  }
  for (int a = 0; a < 5; ++a) {
    const double ri = (double)(a + 1);
    for (int b = a + 1; b < 5; ++b) {
      const double rj = (double)(b + 1), r = ri / rj;
      const double x = 1.0 - r * r;
      double g;
      if (a == 0) {
        g = 1.1330 - 0.4059 / x + 0.07014 / (x * x);
      } else if (a == 1) {
        g = 1.0785 - 0.2319 / x + 0.02947 / (x * x);
      } else {
        g = 0.9935 + 0.2328 / ri - 0.1296 / (ri * ri) -
            (1.0 / x) * (1.0 / ri) * (0.6282 - 0.5598 / ri + 0.5299 / (ri * ri)) +
            (1.0 / x) * (1.0 / x) * (1.0 / (ri * ri)) * (0.3887 - 1.181 / ri + 1.470 / (ri * ri));
      }
      const double fnn = 32.0 / 3.0 / std::sqrt(3.0) / pi * ri / (rj * rj * rj) / (x * x * x) * g;
      k->xrat[a][b] = x;
      k->enn[a][b] = k->eion[a] - k->eion[b];
      k->rnn[a][b] = k->rn[a] * x;
      k->ann[a][b] = 2.0 * (ri * ri) / x * fnn;
      k->bnn[a][b] = 4.0 * ((ri * ri) * (ri * ri)) / (rj * rj * rj) / (x * x) *
                     (1.0 + 4.0 / 3.0 / x + bn[a] / (x * x));
      k->lgt[a][b] = std::log(2.0 * (ri * ri) / x);
    }
    double g1, g2, g3;
    if (a == 0) {
      g1 = 1.1330; g2 = -0.4059; g3 = 0.07014;
    } else if (a == 1) {
      g1 = 1.0785; g2 = -0.2319; g3 = 0.02947;
    } else {
      g1 = 0.9935 + 0.2328 / ri - 0.1296 / (ri * ri);
      g2 = (-1.0 / ri) * (0.6282 - 0.5598 / ri + 0.5299 / (ri * ri));
      g3 = (1.0 / ri) * (1.0 / ri) * (0.3887 - 1.181 / ri + 1.470 / (ri * ri));
    }
    for (int b = a + 1; b < 5; ++b) {
      k->ixrat[a][b] = 1.0 / k->xrat[a][b];
      k->gwq[a][b] = k->gw[a] / k->gw[b];
    }
    k->gwh[a] = k->gw[a] / k->gw[5] / 2.0;
    k->an0[a] = 32.0 / 3.0 / std::sqrt(3.0) / pi * ri + g1 / 3.0 + g2 / 4.0 + g3 / 5.0;
    k->bn0[a] = 2.0 / 3.0 * (ri * ri) * (5.0 + bn[a]);
    k->lgi[a] = std::log(2.0 * (ri * ri));
  }
}

namespace {

// ionexpfittest of the generator: trapezoid sum of exp(-z*t)*t**(-istar) from t = 1 in steps
// of 0.001 until a step adds no more than 1e-4 of the first one.
double expint_trap(double zhat, double istar) {
  const double stepsize = 0.001, tol = 0.0001;
  double a = 1.0, b = a + stepsize;
  double fa = std::exp(-zhat * a) * std::pow(a, -istar);
  double fb = std::exp(-zhat * b) * std::pow(b, -istar);
  const double sol0 = 0.5 * (b - a) * (fa + fb);
  double sol = sol0, dif = 1.0;
  while (dif > tol) {
    a = b;
    b = a + stepsize;
    fa = std::exp(-zhat * a) * std::pow(a, -istar);
    fb = std::exp(-zhat * b) * std::pow(b, -istar);
    const double solt = 0.5 * (b - a) * (fa + fb);
    sol = sol + solt;
    dif = solt / sol0;
  }
  return sol;
}

}  // namespace
}  // namespace pip

extern "C" int pip_colexp_table(int64_t nsamps, double *out) {
  if (!out) return PIP_ERR_NULL;
  if (nsamps < 2) return PIP_ERR_PARAM;
  // ymin: 0.54 eV at 1e5 K (the generator's bound), ymax 108 (E_n ~ 1e-50 beyond)
  const double kb = (double)1.38064852e-23f;
  const double ymin = 0.54 / 13.6 * (double)2.18e-18f / kb / 100000.0, ymax = 108.0;
  const double dy = (ymax - ymin) / (double)nsamps;
  // rows are independent; small yn take the longest sums, so threads take rows in chunks
  std::atomic<int64_t> next{0};
  const int64_t chunk = 256;
  auto work = [&]() {
    for (;;) {
      const int64_t t0 = next.fetch_add(chunk);
      if (t0 > nsamps) return;
      const int64_t t1 = std::min<int64_t>(t0 + chunk, nsamps + 1);
      for (int64_t t = t0; t < t1; ++t) {
        const double yn = ymin + (double)t * dy;
        out[4 * t] = yn;
        out[4 * t + 1] = pip::expint_trap(yn, 0.0);
        out[4 * t + 2] = pip::expint_trap(yn, 1.0);
        out[4 * t + 3] = pip::expint_trap(yn, 2.0);
      }
    }
  };
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 64) nt = 64;
  std::vector<std::thread> pool;
  for (unsigned i = 1; i < nt; ++i) pool.emplace_back(work);
  work();
  for (auto &th : pool) th.join();
  return PIP_OK;
}
