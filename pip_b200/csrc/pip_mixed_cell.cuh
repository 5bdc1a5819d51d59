// pip_mixed_cell.cuh -- FP64 per-cell parts of the FP32-mixed form (primitives, floors,
// collisional and ionisation/recombination source), shared by the 1D/2D mixed stage
// kernels and the batched ensemble so that both compute identical cell updates.
#pragma once

#include "pip_kernels.cuh"
#include "pip_physics.cuh"

namespace pip {
namespace mixed {

// FP64 primitives of a conserved cell (cq2pv's expressions, without the rewrite).
template <int NVM>
__device__ __forceinline__ Prim<double> prim_mhd(const double (&u)[NVM], const KParams &p) {
  Prim<double> q;
  const double de = u[0];
  const double inv = 1.0 / de;
  q.vx = u[1] * inv;
  q.vy = u[2] * inv;
  q.vz = u[3] * inv;
  q.pr = fmax((p.gm - 1.0) * (u[4] - 0.5 * de * (q.vx * q.vx + q.vy * q.vy + q.vz * q.vz) -
                              0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7])), p.pr_lim);
  q.de = fmax(de, p.ro_lim);
  return q;
}
__device__ __forceinline__ Prim<double> prim_hd(const double (&u)[5], const KParams &p) {
  Prim<double> q;
  const double de = u[0];
  const double inv = 1.0 / de;
  q.vx = u[1] * inv;
  q.vy = u[2] * inv;
  q.vz = u[3] * inv;
  q.pr = fmax((p.gm - 1.0) * (u[4] - 0.5 * de * (q.vx * q.vx + q.vy * q.vy + q.vz * q.vz)), p.pr_lim);
  q.de = fmax(de, p.ro_lim);
  return q;
}

// Density/pressure floors of cq2pv (Scheme_rot.f90:171-178), applied only when they fire;
// an FP32 estimate skips the FP64 test far from the floors.
template <int NVM>
__device__ __forceinline__ void floors_mhd(double (&u)[NVM], const KParams &p) {
  {
    const float d = (float)u[0];
    const float pf = (float)(p.gm - 1.0) *
                     ((float)u[4] - 0.5f * ((float)u[1] * (float)u[1] + (float)u[2] * (float)u[2] +
                                            (float)u[3] * (float)u[3]) / d -
                      0.5f * ((float)u[5] * (float)u[5] + (float)u[6] * (float)u[6] +
                              (float)u[7] * (float)u[7]));
    if (d > 2.0f * (float)p.ro_lim && pf > 2.0f * (float)p.pr_lim + 1e-3f * (float)u[4]) return;
  }
  const double de = u[0];
  const double k = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / de;
  const double b = 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
  const double pr = (p.gm - 1.0) * (u[4] - k - b);
  if (pr <= p.pr_lim || de <= p.ro_lim) cq2pv_mhd<double, NVM>(u, p.gm, p.ro_lim, p.pr_lim);
}
__device__ __forceinline__ void floors_hd(double (&u)[5], const KParams &p) {
  {
    const float d = (float)u[0];
    const float pf = (float)(p.gm - 1.0) *
                     ((float)u[4] - 0.5f * ((float)u[1] * (float)u[1] + (float)u[2] * (float)u[2] +
                                            (float)u[3] * (float)u[3]) / d);
    if (d > 2.0f * (float)p.ro_lim && pf > 2.0f * (float)p.pr_lim + 1e-3f * (float)u[4]) return;
  }
  const double de = u[0];
  const double pr = (p.gm - 1.0) * (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / de);
  if (pr <= p.pr_lim || de <= p.ro_lim) cq2pv_hd<double>(u, p.gm, p.ro_lim, p.pr_lim);
}

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

// FP64 collisional dS (PIP_rot.f90:1333-1368) from FP64 primitives.
template <int NVM>
__device__ __forceinline__ void collision_ds(const double (&um)[NVM], const double (&uh)[5],
                                             const Prim<double> &qm, const Prim<double> &qh,
                                             const KParams &p, double dt_coll, double (&ds)[5]) {
  const double gm = p.gm, ac = p.ac;
  ds[0] = 0.0;
  if (p.imp) {
    const double te = qm.pr / qm.de * gm * kMuP;
    const double nte = qh.pr / qh.de * gm * kMuN;
    const double temp = dt_coll * (uh[0] + um[0]);
    const double e = (1.0 - exp(-ac * temp));
    ds[1] = (um[0] * uh[1] - uh[0] * um[1]) * e / temp;
    ds[2] = (um[0] * uh[2] - uh[0] * um[2]) * e / temp;
    ds[3] = (um[0] * uh[3] - uh[0] * um[3]) * e / temp;
    const double nde = qh.de, de = qm.de;
    const double lambda = ac * (nde + de);
    const double kap = 3.0 * (gm - 1.0) * ac * (kMuP * nde + kMuN * de);
    const double dvx = qh.vx - qm.vx, dvy = qh.vy - qm.vy, dvz = qh.vz - qm.vz;
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
    // 3/gm/2 (nte - te) with te = 0.5 gm pr/de, nte = gm npr/nde: the gm cancels
    const double dte = 1.5 * (qh.pr / qh.de - 0.5 * (qm.pr / qm.de));
    ds[4] = ac * qh.de * qm.de *
            (0.5 * ((qh.vx * qh.vx - qm.vx * qm.vx) + (qh.vy * qh.vy - qm.vy * qm.vy) +
                    (qh.vz * qh.vz - qm.vz * qm.vz)) +
             dte);
  }
}

__device__ __forceinline__ void ir_ds(const Prim<double> &qm, const Prim<double> &qh, double gr,
                                      double gi, const KParams &p, double (&ds)[5]) {
  const double gm = p.gm;
  ds[0] = gr * qm.de - gi * qh.de;
  ds[1] = gr * qm.de * qm.vx - gi * qh.de * qh.vx;
  ds[2] = gr * qm.de * qm.vy - gi * qh.de * qh.vy;
  ds[3] = gr * qm.de * qm.vz - gi * qh.de * qh.vz;
  const double kin = 0.5 * (gr * qm.de * (qm.vx * qm.vx + qm.vy * qm.vy + qm.vz * qm.vz) -
                            gi * qh.de * (qh.vx * qh.vx + qh.vy * qh.vy + qh.vz * qh.vz));
  if (p.ir_type == 1)
    ds[4] = kin - gi * qh.pr / (gm - 1.0) + 0.5 * gr * qm.pr / (gm - 1.0);
  else
    ds[4] = kin - gi * qh.pr / (gm - 1.0) + gr * qm.pr / (gm - 1.0);
}

// Ghost images of one updated cell (PIPbnd after the stage, x faces then y faces, so a
// corner ghost carries both sign flips).  Only cells within 2*margin of a boundary can be
// a ghost source; the caller tests that first.  The values are re-read from the planes the
// same thread has just written.
template <int NDIM>
__device__ __forceinline__ bool near_boundary(const KParams &p, int gi, int gj) {
  return gi < 2 * p.m0 || gi >= p.ix - 2 * p.m0 ||
         (NDIM == 2 && (gj < 2 * p.m1 || gj >= p.jx - 2 * p.m1));
}

template <int NDIM>
__device__ __noinline__ void write_ghosts(const KParams &p, int gi, int gj, float *hi, float *lo,
                                          int nplanes) {
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
    const float h = hi[q + n * nc];
    const float w = lo ? lo[q + n * nc] : 0.0f;
    for (int a = 0; a < ntx; ++a) {
      const float g = (float)p.symx[sx[a]][n];
      const long long t = (long long)gj * p.ix + tx[a];
      hi[t + n * nc] = g * h;
      if (lo) lo[t + n * nc] = g * w;
      for (int b = 0; b < nty; ++b) {
        const float g2 = (float)p.symy[sy[b]][n];
        const long long c = (long long)ty[b] * p.ix + tx[a];
        hi[c + n * nc] = g2 * (g * h);
        if (lo) lo[c + n * nc] = g2 * (g * w);
      }
    }
    for (int b = 0; b < nty; ++b) {
      const float g2 = (float)p.symy[sy[b]][n];
      const long long t = (long long)ty[b] * p.ix + gi;
      hi[t + n * nc] = g2 * h;
      if (lo) lo[t + n * nc] = g2 * w;
    }
  }
}

}  // namespace mixed
}  // namespace pip
