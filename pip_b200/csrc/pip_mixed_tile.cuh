// pip_mixed_tile.cuh -- one RK stage of the FP32-mixed form on one tile, shared by the
// stage kernels (pip_mixed.cu, one tile per CTA) and the batched ensemble (pip_ensemble.cu,
// a CTA walking a 2D member's tiles).  Compiled in both with the same flags
// (-ftz=true -prec-div=false -prec-sqrt=false).
#pragma once

#include "pip_kernels.cuh"
#include "pip_mixed_cell.cuh"
#include "pip_pair.cuh"
#include "pip_physics.cuh"

namespace pip {
namespace mixed {

// One RK stage on the TX x TY cells from (i0, j0) (the arithmetic is that of run_solver's
// stage, see the FP64 stage_kernel): FP32 primitives of the tile and its kH-cell halo, FP32
// face fluxes (HLLD on the ion planes 0-7, HLLC on the neutral ones, each face's left and
// right work paired in packed FP32x2 arithmetic, pip_pair.cuh; with NVM == 9 the
// normal-field and psi fluxes in FP64), then per cell the FP64 source and the compensated
// update into Ohi (and Olo in stage 2) with the ghost images.  Stage 1: Us = U0hi = A.hi;
// stage 2: Us = U1, U0 = A.hi + A.lo.  staged: sV already holds the raw planes of the tile
// (a TMA load), else they are read from Us.  ep (stage 2): 1 the cfl rewrite's floors, 2
// also the next step's CFL terms, folded into dtc (min), rhoc and grc (max).  bad is set
// for a non-finite updated cell.  Every thread of the CTA calls it; it synchronises the CTA
// between its phases, but not after the update.
template <int NDIM, int NVM, int STAGE, int TX, int TY, int NT, int kH>
__device__ __forceinline__ void tile_stage(const KParams &p, const float *__restrict__ Us,
                                           const float *U0hi, const float *U0lo, float *Ohi,
                                           float *Olo, int i0, int j0, double dt, double cmax,
                                           int ep, bool staged, float *sV, double *sD6,
                                           double *sD9, float *sFx, float *sFy, double &dtc,
                                           double &rhoc, double &grc, bool &bad) {
  constexpr int NV = NVM + 5;
  constexpr int RX = TX + 2 * kH, RY = NDIM == 2 ? TY + 2 * kH : 1, RR = RX * RY;
  constexpr int NFX = (TX + 1) * TY, NFY = NDIM == 2 ? TX * (TY + 1) : 0;
  const int tid = threadIdx.x;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  const float igm1f = (float)p.igm1;
  const long long nc = p.nc;
  if (STAGE == 1) ep = 0;   // stage 1 is never followed by a cfl

  // ---- 1. FP32 primitives of the tile and its halo
  if (staged) {
    for (int idx = tid; idx < RR; idx += NT) {
      const int ri = idx % RX, rj = idx / RX;
      if ((ri < kH || ri >= TX + kH) && (rj < kH || rj >= TY + kH)) continue;
      const int gi = i0 - kH + ri, gj = j0 - kH + rj;
      if (gi >= p.ix || gj >= p.jx) continue;
      float um[NVM], uh[5], vm[NVM], vh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) um[n] = sV[n * RR + idx];
#pragma unroll
      for (int n = 0; n < 5; ++n) uh[n] = sV[(NVM + n) * RR + idx];
      u2v_mhd<float, NVM>(um, vm, gmf, rolf, prlf);
      u2v_hd<float>(uh, vh, gmf, rolf, prlf);
#pragma unroll
      for (int n = 0; n < NVM; ++n) sV[n * RR + idx] = vm[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) sV[(NVM + n) * RR + idx] = vh[n];
    }
  } else
  for (int idx = tid; idx < RR; idx += NT) {
    const int ri = idx % RX, rj = idx / RX;
    if (NDIM == 2 && (ri < kH || ri >= TX + kH) && (rj < kH || rj >= TY + kH)) continue;
    const int gi = i0 - kH + ri, gj = NDIM == 2 ? j0 - kH + rj : 0;
    if (gi >= p.ix || gj >= p.jx) continue;
    const long long q = (long long)gj * p.ix + gi;
    float um[NVM], uh[5], vm[NVM], vh[5];
#pragma unroll
    for (int n = 0; n < NVM; ++n) um[n] = Us[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n) uh[n] = Us[q + (NVM + n) * nc];
    u2v_mhd<float, NVM>(um, vm, gmf, rolf, prlf);
    u2v_hd<float>(uh, vh, gmf, rolf, prlf);
#pragma unroll
    for (int n = 0; n < NVM; ++n) sV[n * RR + idx] = vm[n];
#pragma unroll
    for (int n = 0; n < 5; ++n) sV[(NVM + n) * RR + idx] = vh[n];
  }
  __syncthreads();

  // ---- 2. FP32 face fluxes
  const int iend = p.m0 + p.nx, jend = NDIM == 2 ? p.m1 + p.ny : 1;
  for (int f = tid; f < NFX + NFY; f += NT) {
    // x faces first, then y faces, each in row order (constant divisors in each branch)
    int a, s, py, fo, nf;
    float *Fout;
    if (f < NFX) {
      const int fi = f % (TX + 1), fj = f / (TX + 1);
      if (i0 + fi - 1 >= iend || (NDIM == 2 && j0 + fj >= jend)) continue;
      a = (NDIM == 2 ? (fj + kH) * RX : 0) + fi + kH - 1;
      s = 1;
      py = 0;
      Fout = sFx;
      fo = f;
      nf = NFX;
    } else {
      const int g = f - NFX, fi = g % TX, fj = g / TX;
      if (i0 + fi >= iend || j0 + fj - 1 >= jend) continue;
      a = (fj + kH - 1) * RX + fi + kH;
      s = RX;
      py = 1;
      Fout = sFy;
      fo = g;
      nf = NFY;
    }
    {
      // the HLLD of planes 0-7; with Dedner cleaning the normal-field and psi fluxes are the
      // FP64 ones below, so the FP32 solver neither reconstructs psi nor stores those two
      float vl[8], vr[8], fx[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        const int src = py ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        const float *v = sV + src * RR + a;
        const float v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
        vl[n] = v1 + 0.5f * minmod<float>(v0, v1, v2);
        vr[n] = v2 - 0.5f * minmod<float>(v1, v2, v3);
      }
      vl[0] = fmaxf(vl[0], rolf);
      vr[0] = fmaxf(vr[0], rolf);
      pair::hlld_flux(vl, vr, fx, gmf, igm1f);
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        if (NVM == 9 && n == 5) continue;
        const int dst = py ? (n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n) : n;
        Fout[dst * nf + fo] = fx[n];
      }
      if (NVM == 9) {
        // reconstruct Bn and psi in FP64 from the FP32 cell values
        const float *vb = sV + (py ? 6 : 5) * RR + a;
        const float *vp = sV + (NVM - 1) * RR + a;
        const double b0 = vb[-s], b1 = vb[0], b2 = vb[s], b3 = vb[2 * s];
        const double p0 = vp[-s], p1 = vp[0], p2 = vp[s], p3 = vp[2 * s];
        const double bl = b1 + 0.5 * minmod<double>(b0, b1, b2);
        const double br = b2 - 0.5 * minmod<double>(b1, b2, b3);
        const double pl = p1 + 0.5 * minmod<double>(p0, p1, p2);
        const double pr = p2 - 0.5 * minmod<double>(p1, p2, p3);
        const double ch = cmax;
        sD6[f] = 0.5 * (pl + pr - ch * (br - bl));
        sD9[f] = 0.5 * (ch * ch * (bl + br) - ch * (pr - pl));
      }
    }
    {
      float vl[5], vr[5], fx[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        const int src = py ? (n == 1 ? 2 : n == 2 ? 1 : n) : n;
        const float *v = sV + (NVM + src) * RR + a;
        const float v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
        vl[n] = v1 + 0.5f * minmod<float>(v0, v1, v2);
        vr[n] = v2 - 0.5f * minmod<float>(v1, v2, v3);
      }
      vl[0] = fmaxf(vl[0], rolf);
      vr[0] = fmaxf(vr[0], rolf);
      pair::hllc_flux(vl, vr, fx, gmf, igm1f);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        const int dst = py ? (n == 1 ? 2 : n == 2 ? 1 : n) : n;
        Fout[(NVM + dst) * nf + fo] = fx[n];
      }
    }
  }
  __syncthreads();

  // ---- 3. FP64 source and compensated update
  const int ti = tid % TX, tj = tid / TX;
  const int gi = i0 + ti, gj = j0 + tj;
  const bool valid = tj < TY && gi < iend && (NDIM == 1 || gj < jend);
  if (valid) {
    const long long q = (long long)gj * p.ix + gi;
    const double dt_sub = STAGE == 1 ? dt / 2.0 : dt;
    const double dt_coll = dt * 0.5;
    double a_m[NVM], a_h[5], s_m[NVM], s_h[5];
#pragma unroll
    for (int n = 0; n < NVM; ++n) {
      a_m[n] = (double)U0hi[q + n * nc];
      if (STAGE == 2) a_m[n] += (double)U0lo[q + n * nc];
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      a_h[n] = (double)U0hi[q + (NVM + n) * nc];
      if (STAGE == 2) a_h[n] += (double)U0lo[q + (NVM + n) * nc];
    }
    if (STAGE == 1) {
#pragma unroll
      for (int n = 0; n < NVM; ++n) s_m[n] = a_m[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) s_h[n] = a_h[n];
    } else {
#pragma unroll
      for (int n = 0; n < NVM; ++n) s_m[n] = (double)Us[q + n * nc];
#pragma unroll
      for (int n = 0; n < 5; ++n) s_h[n] = (double)Us[q + (NVM + n) * nc];
    }
    double gr = 0.0, gion = 0.0;
    if (p.ir) ir_rates<NVM>(a_m, p, gr, gion);
    if (p.imp && STAGE == 2) {
      double ds[5];
      const Prim<double> qh = prim_hd(a_h, p);
      const Prim<double> qm = prim_mhd<NVM>(a_m, p);
      collision_ds<NVM>(a_m, a_h, qm, qh, p, dt_coll, ds);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        a_h[n] = a_h[n] - dt_coll * ds[n];
        a_m[n] = a_m[n] + dt_coll * ds[n];
      }
    }
    double S_m[5], S_h[5];
    {
      const Prim<double> qh = prim_hd(s_h, p);
      const Prim<double> qm = prim_mhd<NVM>(s_m, p);
      double ds[5];
      collision_ds<NVM>(s_m, s_h, qm, qh, p, dt_coll, ds);
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
          S_h[n] = -ds[n];
          S_m[n] = ds[n];
        }
      }
      if (p.ir) {
        ir_ds(qm, qh, gr, gion, p, ds);
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          S_h[n] += ds[n];
          S_m[n] -= ds[n];
        }
      }
    }
    const double cx = dt_sub * p.rdx[gi];
    const double cy = NDIM == 2 ? dt_sub * p.rdy[gj] : 0.0;
    const int fxl = tj * (TX + 1) + ti, fyl = tj * TX + ti;
    double n_m[NVM], n_h[5];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double u = n < NVM ? a_m[n] : a_h[n - NVM];
      // x faces: Bx (plane 5) and psi take the FP64 Dedner fluxes; y faces: By (6) and psi
      const bool dx64 = NVM == 9 && (n == 5 || n == NVM - 1);
      const bool dy64 = NVM == 9 && (n == 6 || n == NVM - 1);
      const double *Dx = n == NVM - 1 ? sD9 : sD6;
      if (dx64) u -= cx * (Dx[fxl + 1] - Dx[fxl]);
      else u -= cx * (double)(sFx[n * NFX + fxl + 1] - sFx[n * NFX + fxl]);
      if (NDIM == 2) {
        if (dy64) u -= cy * (Dx[NFX + fyl + TX] - Dx[NFX + fyl]);
        else u -= cy * (double)(sFy[n * NFY + fyl + TX] - sFy[n * NFY + fyl]);
      }
      if (n < NVM) {
        if (n < 5) u += S_m[n] * dt_sub;
        n_m[n] = u;
      } else {
        n_h[n - NVM] = u + S_h[n - NVM] * dt_sub;
      }
    }
    if (NVM == 9) n_m[NVM - 1] *= p.decay[STAGE - 1];
    if (ep >= 1) {
      floors_mhd<NVM>(n_m, p);
      floors_hd(n_h, p);
    }
    if (ep == 2) {
      // CFL terms of the next step in FP32 from the new state
      float um[NVM], uh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) um[n] = (float)n_m[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) uh[n] = (float)n_h[n];
      const Prim<float> qm = cq2pv_mhd<float, NVM>(um, gmf, rolf, prlf);
      const Prim<float> qh = cq2pv_hd<float>(uh, gmf, rolf, prlf);
      const double gmin = fmin(fmin(p.dx[gi], NDIM == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
      const float sg = (float)(p.safety * gmin);
      dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, um[5], um[6], um[7], gmf, sg),
                                    cfl_hd_cell<float>(qh, gmf, sg)));
      rhoc = fmax(rhoc, fmax(n_m[0] * p.ac, n_h[0] * p.ac));
      if (p.ir) {
        double g1, g2;
        ir_rates<NVM>(n_m, p, g1, g2);
        grc = fmax(grc, fmax(g1, g2));
      }
    }
#pragma unroll
    for (int n = 0; n < NVM; ++n) bad |= !isfinite(n_m[n]);
#pragma unroll
    for (int n = 0; n < 5; ++n) bad |= !isfinite(n_h[n]);
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const double u = n < NVM ? n_m[n] : n_h[n - NVM];
      const float hi = (float)u;
      Ohi[q + n * nc] = hi;
      if (STAGE == 2) Olo[q + n * nc] = (float)(u - (double)hi);
    }
    if (near_boundary<NDIM>(p, gi, gj)) write_ghosts<NDIM>(p, gi, gj, Ohi, STAGE == 2 ? Olo : nullptr, NV);
  }
}

}  // namespace mixed
}  // namespace pip
