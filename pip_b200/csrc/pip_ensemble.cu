// pip_ensemble.cu -- batched ensemble of independent 1D two-fluid runs in one persistent
// launch (FP32-mixed form).
//
// Each CTA takes a run from a work queue (runs ordered longest first), owns the whole
// run and advances it to its end time with its own dt: per step stage 1, stage 2 and the
// fused cfl, with block-wide reductions and no grid synchronisation.  Within a stage the
// CTA walks the run in chunks of NT-1 cells: primitives of the chunk and its halo into
// shared memory, the NT faces of the chunk (one per thread), then the per-cell update.
// The per-cell arithmetic is the mixed stage kernel's (pip_mixed_cell.cuh and the same
// Riemann solvers), so a member evolves exactly as a single-run mixed context does.
//
// Packed storage: member r's planes start at off[r] floats in three arrays (hi, lo, U1),
// NV = 13 planes of ix_r floats each.  A run's KParams (with its dx tables) sits in a
// device array.  The launch (queue reset + persistent kernel) is captured in a CUDA graph.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/pip_ensemble.h"
#include "../../include/pip_gpu.h"
#include "pip_kernels.cuh"
#include "pip_mixed_cell.cuh"
#include "pip_mixed_tile.cuh"
#include "pip_physics.cuh"

namespace pip {
namespace ens {

constexpr int NVM = 8, NV = 13, kH = 2;
// 2D members: the mixed stage kernels' 16x14 tiles, walked by one CTA
constexpr int TX2 = 16, TY2 = 14;

struct Member {
  long long off;      // first float of the member's planes in hi/lo/U1
  int kp;             // index of its KParams
};

struct RunState {
  double time, dt;
  long long steps;
  int status;         // 0, PIP_ERR_NAN (3) or PIP_ERR_DT (4)
  int blocks;         // thread blocks that stepped it in the last launch that advanced it
  unsigned long long t_start, t_end;  // device global timer (ns) when the last launch that
                                      // advanced the run took it from the queue and left it
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double finalize_dt(const KParams &p, double red_dt, double red_rho,
                                              double red_gr) {
  double dt = fmin(red_dt, p.col_lim / red_rho);
  if (p.ir) dt = fmin(dt, p.ir_lim / fmax(red_gr, 1.0e-5));
  return dt;
}

template <int NT>
__device__ __forceinline__ void block_minmax(double &dtc, double &rho, double &gr, double *s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
    rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
    gr = fmax(gr, __shfl_xor_sync(0xffffffffu, gr, o));
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) {
    s_red[w] = dtc;
    s_red[NT / 32 + w] = rho;
    s_red[2 * (NT / 32) + w] = gr;
  }
  __syncthreads();
  dtc = s_red[0];
  rho = s_red[NT / 32];
  gr = s_red[2 * (NT / 32)];
  for (int k = 1; k < NT / 32; ++k) {
    dtc = fmin(dtc, s_red[k]);
    rho = fmax(rho, s_red[NT / 32 + k]);
    gr = fmax(gr, s_red[2 * (NT / 32) + k]);
  }
}

// Barrier of the CTAs that share a member: the cluster barrier (arrive.release /
// wait.acquire at cluster scope, so the global writes of one CTA's cells and ghosts before
// it are seen by the others after it), or the block barrier when one CTA owns the member.
template <int CL>
__device__ __forceinline__ void member_sync() {
  if constexpr (CL > 1) cooperative_groups::this_cluster().sync();
  else __syncthreads();
}

// The CFL terms and the NaN flag of a member shared by the CL CTAs of a cluster: each CTA's
// block result goes to its slot in its own shared memory, and after the cluster barrier
// every CTA reads all CL slots through distributed shared memory and reduces them in rank
// order (min and max are exact, so every CTA, and a one-CTA run, gets the same dt).  A slot
// is written again only after the next member_sync, when every CTA has read it.
template <int CL>
__device__ __forceinline__ void cluster_minmax(double &dtc, double &rho, double &gr, int &bad,
                                               double *s_slot, double *s_res) {
  if constexpr (CL > 1) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x == 0) {
      s_slot[0] = dtc;
      s_slot[1] = rho;
      s_slot[2] = gr;
      s_slot[3] = bad ? 1.0 : 0.0;
    }
    cl.sync();
    if (threadIdx.x < 32) {
      const int k = threadIdx.x;
      double d = 10.0, r = 0.0, g = 0.0, b = 0.0;
      if (k < CL) {
        const double *q = cl.map_shared_rank(s_slot, k);
        d = q[0];
        r = q[1];
        g = q[2];
        b = q[3];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        d = fmin(d, __shfl_xor_sync(0xffffffffu, d, o));
        r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
        g = fmax(g, __shfl_xor_sync(0xffffffffu, g, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
      }
      if (k == 0) {
        s_res[0] = d;
        s_res[1] = r;
        s_res[2] = g;
        s_res[3] = b;
      }
    }
    __syncthreads();
    dtc = s_res[0];
    rho = s_res[1];
    gr = s_res[2];
    bad = s_res[3] != 0.0;
    __syncthreads();   // s_res is rewritten by the next reduction
  }
}

// One RK stage of a member (the 1D mixed stage kernel's arithmetic, chunk by chunk).
// Returns, for stage 2 with ep == 2, this thread's CFL terms of the next step.
// Cells [cbeg, cend) of the interior: all of it for a member one CTA owns, this CTA's part
// of it for a member a cluster shares.
template <int NT, int STAGE>
__device__ void run_stage(const KParams &p, const float *Us, float *Ahi, float *Alo, float *Bf,
                          double dt, int ep, float *sV, float *sF, double &dtc, double &rhoc,
                          double &grc, int &bad, int cbeg, int iend) {
  constexpr int CN = NT - 1;          // cells per chunk
  constexpr int RX = CN + 2 * kH;     // region cells
  const int tid = threadIdx.x;
  const long long nc = p.nc;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  const float igm1f = (float)p.igm1;
  float *Ohi = STAGE == 1 ? Bf : Ahi;
  for (int c0 = cbeg; c0 < iend; c0 += CN) {
    const int cn = min(CN, iend - c0);
    // primitives of the chunk and its halo
    for (int idx = tid; idx < cn + 2 * kH; idx += NT) {
      const int gi = c0 - kH + idx;
      float um[NVM], uh[5], vm[NVM], vh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) um[n] = Us[gi + n * nc];
#pragma unroll
      for (int n = 0; n < 5; ++n) uh[n] = Us[gi + (NVM + n) * nc];
      u2v_mhd<float, NVM>(um, vm, gmf, rolf, prlf);
      u2v_hd<float>(uh, vh, gmf, rolf, prlf);
#pragma unroll
      for (int n = 0; n < NVM; ++n) sV[n * RX + idx] = vm[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) sV[(NVM + n) * RX + idx] = vh[n];
    }
    __syncthreads();
    // faces: face t lies between cells c0-1+t and c0+t
    if (tid <= cn) {
      const int a = tid + kH - 1;
      {
        float vl[NVM], vr[NVM], fx[NVM];
#pragma unroll
        for (int n = 0; n < NVM; ++n) {
          const float *v = sV + n * RX + a;
          const float v0 = v[-1], v1 = v[0], v2 = v[1], v3 = v[2];
          vl[n] = v1 + 0.5f * minmod<float>(v0, v1, v2);
          vr[n] = v2 - 0.5f * minmod<float>(v1, v2, v3);
        }
        vl[0] = fmaxf(vl[0], rolf);
        vr[0] = fmaxf(vr[0], rolf);
        hlld_flux_rcp<float, NVM>(vl, vr, fx, gmf, igm1f, 0.0f);
#pragma unroll
        for (int n = 0; n < NVM; ++n) sF[n * NT + tid] = fx[n];
      }
      {
        float vl[5], vr[5], fx[5];
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          const float *v = sV + (NVM + n) * RX + a;
          const float v0 = v[-1], v1 = v[0], v2 = v[1], v3 = v[2];
          vl[n] = v1 + 0.5f * minmod<float>(v0, v1, v2);
          vr[n] = v2 - 0.5f * minmod<float>(v1, v2, v3);
        }
        vl[0] = fmaxf(vl[0], rolf);
        vr[0] = fmaxf(vr[0], rolf);
        hllc_flux_rcp<float>(vl, vr, fx, gmf, igm1f);
#pragma unroll
        for (int n = 0; n < 5; ++n) sF[(NVM + n) * NT + tid] = fx[n];
      }
    }
    __syncthreads();
    // per-cell source and update
    if (tid < cn) {
      const int gi = c0 + tid;
      const double dt_sub = STAGE == 1 ? dt / 2.0 : dt;
      const double dt_coll = dt * 0.5;
      double a_m[NVM], a_h[5], s_m[NVM], s_h[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) {
        a_m[n] = (double)Ahi[gi + n * nc];
        if (STAGE == 2) a_m[n] += (double)Alo[gi + n * nc];
      }
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        a_h[n] = (double)Ahi[gi + (NVM + n) * nc];
        if (STAGE == 2) a_h[n] += (double)Alo[gi + (NVM + n) * nc];
      }
      if (STAGE == 1) {
#pragma unroll
        for (int n = 0; n < NVM; ++n) s_m[n] = a_m[n];
#pragma unroll
        for (int n = 0; n < 5; ++n) s_h[n] = a_h[n];
      } else {
#pragma unroll
        for (int n = 0; n < NVM; ++n) s_m[n] = (double)Us[gi + n * nc];
#pragma unroll
        for (int n = 0; n < 5; ++n) s_h[n] = (double)Us[gi + (NVM + n) * nc];
      }
      double gr = 0.0, gion = 0.0;
      if (p.ir) mixed::ir_rates<NVM>(a_m, p, gr, gion);
      if (p.imp && STAGE == 2) {
        double ds[5];
        const Prim<double> qh = mixed::prim_hd(a_h, p);
        const Prim<double> qm = mixed::prim_mhd<NVM>(a_m, p);
        mixed::collision_ds<NVM>(a_m, a_h, qm, qh, p, dt_coll, ds);
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          a_h[n] = a_h[n] - dt_coll * ds[n];
          a_m[n] = a_m[n] + dt_coll * ds[n];
        }
      }
      double S_m[5], S_h[5];
      {
        const Prim<double> qh = mixed::prim_hd(s_h, p);
        const Prim<double> qm = mixed::prim_mhd<NVM>(s_m, p);
        double ds[5];
        mixed::collision_ds<NVM>(s_m, s_h, qm, qh, p, dt_coll, ds);
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
          mixed::ir_ds(qm, qh, gr, gion, p, ds);
#pragma unroll
          for (int n = 0; n < 5; ++n) {
            S_h[n] += ds[n];
            S_m[n] -= ds[n];
          }
        }
      }
      const double cx = dt_sub * p.rdx[gi];
      double n_m[NVM], n_h[5];
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        double u = n < NVM ? a_m[n] : a_h[n - NVM];
        u -= cx * (double)(sF[n * NT + tid + 1] - sF[n * NT + tid]);
        if (n < NVM) {
          if (n < 5) u += S_m[n] * dt_sub;
          n_m[n] = u;
        } else {
          n_h[n - NVM] = u + S_h[n - NVM] * dt_sub;
        }
      }
      if (ep >= 1) {
        mixed::floors_mhd<NVM>(n_m, p);
        mixed::floors_hd(n_h, p);
      }
      if (ep == 2) {
        float um[NVM], uh[5];
#pragma unroll
        for (int n = 0; n < NVM; ++n) um[n] = (float)n_m[n];
#pragma unroll
        for (int n = 0; n < 5; ++n) uh[n] = (float)n_h[n];
        const Prim<float> qm = cq2pv_mhd<float, NVM>(um, gmf, rolf, prlf);
        const Prim<float> qh = cq2pv_hd<float>(uh, gmf, rolf, prlf);
        const double gmin = fmin(fmin(p.dx[gi], p.dy[0]), p.dz0);
        const float sg = (float)(p.safety * gmin);
        dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, um[5], um[6], um[7], gmf, sg),
                                      cfl_hd_cell<float>(qh, gmf, sg)));
        rhoc = fmax(rhoc, fmax(n_m[0] * p.ac, n_h[0] * p.ac));
        if (p.ir) {
          double g1, g2;
          mixed::ir_rates<NVM>(n_m, p, g1, g2);
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
        Ohi[gi + n * nc] = hi;
        if (STAGE == 2) Alo[gi + n * nc] = (float)(u - (double)hi);
      }
      if (mixed::near_boundary<1>(p, gi, 0))
        mixed::write_ghosts<1>(p, gi, 0, Ohi, STAGE == 2 ? Alo : nullptr, NV);
    }
    __syncthreads();
  }
}

// Shared memory of a 2D member's tile step (the mixed stage kernel's layout).
template <int NVM2>
constexpr size_t smem_2d() {
  constexpr int RR = (TX2 + 2 * kH) * (TY2 + 2 * kH);
  constexpr int NFX = (TX2 + 1) * TY2, NFY = TX2 * (TY2 + 1);
  return sizeof(float) * (NVM2 + 5) * (RR + NFX + NFY) +
         (NVM2 == 9 ? 2 * sizeof(double) * (NFX + NFY) : 0);
}

// A 2D member (ion planes NVM2 = 8, or 9 with Dedner cleaning) advanced by one CTA to the
// end time: its cfl, then per step stage 1 over every tile and stage 2 over every tile
// (mixed::tile_stage, the single-run mixed kernels' arithmetic), the CTA synchronised
// between tiles and stages.
template <int NT, int NVM2>
__device__ void run_member_2d(const KParams &p, float *Ahi, float *Alo, float *B, RunState &rs,
                              double t_end, long long max_steps, float *smem, double *s_red) {
  constexpr int NV2 = NVM2 + 5;
  constexpr int RR = (TX2 + 2 * kH) * (TY2 + 2 * kH);
  constexpr int NFX = (TX2 + 1) * TY2, NFY = TX2 * (TY2 + 1);
  float *sV = smem;
  double *sD6 = reinterpret_cast<double *>(sV + NV2 * RR);
  double *sD9 = sD6 + (NVM2 == 9 ? NFX + NFY : 0);
  float *sFx = reinterpret_cast<float *>(sD9 + (NVM2 == 9 ? NFX + NFY : 0));
  float *sFy = sFx + NV2 * NFX;
  const int tid = threadIdx.x;
  const long long nc = p.nc;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  // cfl of the first step: floors of every cell and the CFL terms (the mixed cfl kernel's
  // arithmetic)
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  for (long long q = tid; q < nc; q += NT) {
    double um[NVM2], uh[5];
#pragma unroll
    for (int n = 0; n < NVM2; ++n) um[n] = (double)Ahi[q + n * nc] + (double)Alo[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n)
      uh[n] = (double)Ahi[q + (NVM2 + n) * nc] + (double)Alo[q + (NVM2 + n) * nc];
    mixed::floors_mhd<NVM2>(um, p);
    mixed::floors_hd(uh, p);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      float h = (float)um[n];
      Ahi[q + n * nc] = h;
      Alo[q + n * nc] = (float)(um[n] - (double)h);
      h = (float)uh[n];
      Ahi[q + (NVM2 + n) * nc] = h;
      Alo[q + (NVM2 + n) * nc] = (float)(uh[n] - (double)h);
    }
    const int i = (int)(q % p.ix), j = (int)(q / p.ix);
    if (i >= p.m0 && i < p.ix - p.m0 && j >= p.m1 && j < p.jx - p.m1) {
      float fm[NVM2], fh[5];
#pragma unroll
      for (int n = 0; n < NVM2; ++n) fm[n] = (float)um[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) fh[n] = (float)uh[n];
      const Prim<float> qm = cq2pv_mhd<float, NVM2>(fm, gmf, rolf, prlf);
      const Prim<float> qh = cq2pv_hd<float>(fh, gmf, rolf, prlf);
      const float sg = (float)(p.safety * fmin(fmin(p.dx[i], p.dy[j]), p.dz0));
      dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, fm[5], fm[6], fm[7], gmf, sg),
                                    cfl_hd_cell<float>(qh, gmf, sg)));
    }
    rhoc = fmax(rhoc, fmax(um[0] * p.ac, uh[0] * p.ac));
    if (p.ir) {
      double g1, g2;
      mixed::ir_rates<NVM2>(um, p, g1, g2);
      grc = fmax(grc, fmax(g1, g2));
    }
  }
  block_minmax<NT>(dtc, rhoc, grc, s_red);
  double dt = finalize_dt(p, dtc, rhoc, grc);
  // the prologue's PIPbnd after its cfl (Initial_rot.f90:152-159): ghost images of the
  // rewritten interior, as the single run's pip_fill_ghosts (a no-op on ghosts that already
  // hold them)
  __syncthreads();
  for (long long t = tid; t < (long long)p.nx * p.ny; t += NT) {
    const int gi = p.m0 + (int)(t % p.nx), gj = p.m1 + (int)(t / p.nx);
    if (mixed::near_boundary<2>(p, gi, gj)) mixed::write_ghosts<2>(p, gi, gj, Ahi, Alo, NV2);
  }
  __syncthreads();
  const int ntx = (p.nx + TX2 - 1) / TX2, nty = (p.ny + TY2 - 1) / TY2, ntiles = ntx * nty;
  bool bad = false;
  for (;;) {
    const double tn = rs.time + dt;
    const bool last = (t_end > 0.0 && tn >= t_end) || (max_steps > 0 && rs.steps + 1 >= max_steps);
    const double cmax = p.sg_all / dt;
    double d1 = 10.0, r1 = 0.0, g1 = 0.0;
    for (int t = 0; t < ntiles; ++t) {
      const int i0 = p.m0 + (t % ntx) * TX2, j0 = p.m1 + (t / ntx) * TY2;
      mixed::tile_stage<2, NVM2, 1, TX2, TY2, NT, kH>(p, Ahi, Ahi, Alo, B, nullptr, i0, j0, dt, cmax,
                                                     0, false, sV, sD6, sD9, sFx, sFy, d1, r1, g1,
                                                     bad);
      __syncthreads();   // the next tile reuses the shared memory
    }
    double d2 = 10.0, r2 = 0.0, g2 = 0.0;
    for (int t = 0; t < ntiles; ++t) {
      const int i0 = p.m0 + (t % ntx) * TX2, j0 = p.m1 + (t / ntx) * TY2;
      mixed::tile_stage<2, NVM2, 2, TX2, TY2, NT, kH>(p, B, Ahi, Alo, Ahi, Alo, i0, j0, dt, cmax,
                                                     last ? 1 : 2, false, sV, sD6, sD9, sFx, sFy,
                                                     d2, r2, g2, bad);
      __syncthreads();
    }
    rs.time = tn;
    rs.steps += 1;
    rs.dt = dt;
    if (__syncthreads_or(bad)) {
      rs.status = 3;  // PIP_ERR_NAN
      break;
    }
    if (dt <= 1.0e-12) {
      rs.status = 4;  // PIP_ERR_DT
      break;
    }
    if (last) break;
    block_minmax<NT>(d2, r2, g2, s_red);
    dt = finalize_dt(p, d2, r2, g2);
  }
}

// A 1D member advanced to the end time by CL CTAs (CL = 1: one CTA owns it; CL > 1: the
// CTAs of a thread-block cluster, rank `rank`, each stepping a contiguous 1/CL of the
// interior and meeting at the cluster barrier after each stage).  The cells' arithmetic
// and the reductions are the same for every CL, so a shared member takes the steps a
// member one CTA owns takes, its state equal up to the FMA contraction of each instance.
// Not inlined: the cluster kernels call the same one-CTA runner as the plain kernels, so
// their unshared runs keep its register allocation (inlined next to the shared runner they
// ran 10% slower per step).
template <int NT, int CL>
__device__ __noinline__ void run_member_1d(const KParams &p, float *Ahi, float *Alo, float *B,
                                           RunState &rs, double t_end, long long max_steps,
                                           float *sV, float *sF, double *s_red, double *s_slot,
                                           double *s_res, int rank) {
  const int tid = threadIdx.x;
  const long long nc = p.nc;
  // cfl of the first step: floors of every cell (cq2pv, Scheme_rot.f90:132-179) and the
  // CFL terms (the mixed cfl kernel's arithmetic)
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  for (int i = rank * NT + tid; i < p.ix; i += NT * CL) {
    double um[NVM], uh[5];
#pragma unroll
    for (int n = 0; n < NVM; ++n) um[n] = (double)Ahi[i + n * nc] + (double)Alo[i + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n) uh[n] = (double)Ahi[i + (NVM + n) * nc] + (double)Alo[i + (NVM + n) * nc];
    mixed::floors_mhd<NVM>(um, p);
    mixed::floors_hd(uh, p);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      float h = (float)um[n];
      Ahi[i + n * nc] = h;
      Alo[i + n * nc] = (float)(um[n] - (double)h);
      h = (float)uh[n];
      Ahi[i + (NVM + n) * nc] = h;
      Alo[i + (NVM + n) * nc] = (float)(uh[n] - (double)h);
    }
    if (i >= p.m0 && i < p.ix - p.m0) {
      float fm[NVM], fh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) fm[n] = (float)um[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) fh[n] = (float)uh[n];
      const Prim<float> qm = cq2pv_mhd<float, NVM>(fm, gmf, rolf, prlf);
      const Prim<float> qh = cq2pv_hd<float>(fh, gmf, rolf, prlf);
      const float sg = (float)(p.safety * fmin(fmin(p.dx[i], p.dy[0]), p.dz0));
      dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, fm[5], fm[6], fm[7], gmf, sg),
                                    cfl_hd_cell<float>(qh, gmf, sg)));
    }
    rhoc = fmax(rhoc, fmax(um[0] * p.ac, uh[0] * p.ac));
    if (p.ir) {
      double g1, g2;
      mixed::ir_rates<NVM>(um, p, g1, g2);
      grc = fmax(grc, fmax(g1, g2));
    }
  }
  block_minmax<NT>(dtc, rhoc, grc, s_red);
  int bad = 0;
  cluster_minmax<CL>(dtc, rhoc, grc, bad, s_slot, s_res);
  double dt = finalize_dt(p, dtc, rhoc, grc);
  // the prologue's PIPbnd after its cfl (Initial_rot.f90:152-159)
  __syncthreads();
  for (int i = p.m0 + rank * NT + tid; i < p.ix - p.m0; i += NT * CL)
    if (mixed::near_boundary<1>(p, i, 0)) mixed::write_ghosts<1>(p, i, 0, Ahi, Alo, NVM + 5);
  member_sync<CL>();
  const int per = (p.nx + CL - 1) / CL;
  const int cb = p.m0 + min(p.nx, rank * per), ce = p.m0 + min(p.nx, (rank + 1) * per);
  // the time loop (main.f90:31-68) of this run
  for (;;) {
    const double tn = rs.time + dt;
    const bool last = (t_end > 0.0 && tn >= t_end) || (max_steps > 0 && rs.steps + 1 >= max_steps);
    double d1 = 10.0, r1 = 0.0, g1 = 0.0;
    run_stage<NT, 1>(p, Ahi, Ahi, Alo, B, dt, 0, sV, sF, d1, r1, g1, bad, cb, ce);
    if constexpr (CL > 1) member_sync<CL>();   // stage 2 reads the others' stage-1 cells
    double d2 = 10.0, r2 = 0.0, g2 = 0.0;
    run_stage<NT, 2>(p, B, Ahi, Alo, B, dt, last ? 1 : 2, sV, sF, d2, r2, g2, bad, cb, ce);
    rs.time = tn;
    rs.steps += 1;
    rs.dt = dt;
    int anybad = __syncthreads_or(bad);
    if constexpr (CL > 1) {
      // one exchange per step carries the next dt and the NaN flag; its barrier also
      // orders this step's stage-2 writes before the next step's stage 1
      block_minmax<NT>(d2, r2, g2, s_red);
      cluster_minmax<CL>(d2, r2, g2, anybad, s_slot, s_res);
    }
    if (anybad) {
      rs.status = 3;  // PIP_ERR_NAN
      break;
    }
    if (dt <= 1.0e-12) {
      rs.status = 4;  // PIP_ERR_DT
      break;
    }
    if (last) break;
    if constexpr (CL == 1) block_minmax<NT>(d2, r2, g2, s_red);
    dt = finalize_dt(p, d2, r2, g2);
  }
}

// Persistent ensemble kernel: CTAs take runs from the queue until it is empty.  HAS2D: the
// instance that can also step 2D members (its larger register footprint stays out of
// ensembles of 1D members only).  The 1D instance of 256 threads is held to 128 registers,
// two CTAs per SM, the configuration the tuner most often picks.
//
// CL > 1 (1D members only): the grid is made of clusters of CL CTAs.  The first nbig entries
// of the queue order (the runs estimated longest) are taken a cluster at a time, rank 0
// drawing from queue[1] and the cluster sharing the run; once they are gone every CTA
// takes the remaining runs alone from queue[0], as with CL = 1.
template <int NT, bool HAS2D, int CL>
__global__ void __launch_bounds__(NT, (NT == 256 && !HAS2D) ? 2 : 1)
    ensemble_kernel(const Member *mem, const KParams *kps, const int *order, int nmem, int nbig,
                    float *hi, float *lo, float *U1, RunState *st, unsigned *queue,
                    double t_end, long long max_steps) {
  constexpr int CN = NT - 1, RX = CN + 2 * kH;
  extern __shared__ float smem[];
  float *sV = smem;
  float *sF = sV + NV * RX;
  __shared__ double s_red[3 * (NT / 32)];
  __shared__ double s_slot[4], s_res[4];
  __shared__ KParams sp;
  __shared__ int s_r;
  const int tid = threadIdx.x;
  if constexpr (CL > 1) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    for (;;) {
      if (rank == 0 && tid == 0) s_r = (int)atomicAdd(queue + 1, 1u);
      cl.sync();
      const int rq = *cl.map_shared_rank(&s_r, 0);
      cl.sync();   // read by all before rank 0 draws again or leaves
      if (rq >= nbig) break;
      const int r = order[rq];
      if (tid == 0) sp = kps[mem[r].kp];
      __syncthreads();
      const KParams &p = sp;
      RunState rs = st[r];
      if (rs.status == 0 && !(t_end > 0.0 && rs.time >= t_end)) {
        rs.t_start = global_ns();
        rs.blocks = CL;
        run_member_1d<NT, CL>(p, hi + mem[r].off, lo + mem[r].off, U1 + mem[r].off, rs, t_end,
                              max_steps, sV, sF, s_red, s_slot, s_res, rank);
        rs.t_end = global_ns();
        if (rank == 0 && tid == 0) st[r] = rs;
      }
      __syncthreads();
    }
  }
  for (;;) {
    if (tid == 0) s_r = nbig + (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int rq = s_r;
    if (rq >= nmem) return;
    const int r = order[rq];
    if (tid == 0) sp = kps[mem[r].kp];
    __syncthreads();
    const KParams &p = sp;
    float *Ahi = hi + mem[r].off, *Alo = lo + mem[r].off, *B = U1 + mem[r].off;
    RunState rs = st[r];
    if (rs.status != 0 || (t_end > 0.0 && rs.time >= t_end)) {
      __syncthreads();
      continue;
    }
    rs.t_start = global_ns();
    rs.blocks = 1;
    if (HAS2D && p.ndim == 2) {
      // (the host allows 2D members only with NT >= TX2 * TY2 threads)
      if (NT >= TX2 * TY2) {
        if (p.nvm == 9) run_member_2d<NT, 9>(p, Ahi, Alo, B, rs, t_end, max_steps, smem, s_red);
        else run_member_2d<NT, 8>(p, Ahi, Alo, B, rs, t_end, max_steps, smem, s_red);
      }
    } else {
      run_member_1d<NT, 1>(p, Ahi, Alo, B, rs, t_end, max_steps, sV, sF, s_red, s_slot, s_res, 0);
    }
    rs.t_end = global_ns();
    if (tid == 0) st[r] = rs;
    __syncthreads();
  }
}

// dynamic shared memory of a launch: the 1D chunk layout, and the 2D tile layout when the
// ensemble holds 2D members
constexpr size_t smem_1d(int nt) { return sizeof(float) * NV * ((nt - 1 + 2 * kH) + nt); }
constexpr size_t smem_bytes(int nt, bool has2d) {
  return has2d && smem_2d<9>() > smem_1d(nt) ? smem_2d<9>() : smem_1d(nt);
}

// Initial dt of each run from its current state (the prologue's cfl terms without its
// floors' writes), one CTA per run: the work estimate (interior cells x remaining steps)
// that orders the queue and picks the runs a cluster shares.
template <int NT>
__global__ void __launch_bounds__(NT) dt0_kernel(const Member *mem, const KParams *kps,
                                                 const float *hi, const float *lo, double *dt0) {
  __shared__ double s_red[3 * (NT / 32)];
  const KParams &p = kps[mem[blockIdx.x].kp];
  const float *Ahi = hi + mem[blockIdx.x].off, *Alo = lo + mem[blockIdx.x].off;
  const long long nc = p.nc;
  const int nvm = p.nvm;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  for (long long q = threadIdx.x; q < nc; q += NT) {
    double um[NVM], uh[5];
#pragma unroll
    for (int n = 0; n < NVM; ++n) um[n] = (double)Ahi[q + n * nc] + (double)Alo[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n) uh[n] = (double)Ahi[q + (nvm + n) * nc] + (double)Alo[q + (nvm + n) * nc];
    mixed::floors_mhd<NVM>(um, p);
    mixed::floors_hd(uh, p);
    const int i = (int)(q % p.ix), j = (int)(q / p.ix);
    const bool inner = i >= p.m0 && i < p.ix - p.m0 &&
                       (p.ndim == 1 || (j >= p.m1 && j < p.jx - p.m1));
    if (inner) {
      float fm[NVM], fh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) fm[n] = (float)um[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) fh[n] = (float)uh[n];
      const Prim<float> qm = cq2pv_mhd<float, NVM>(fm, gmf, rolf, prlf);
      const Prim<float> qh = cq2pv_hd<float>(fh, gmf, rolf, prlf);
      const float sg = (float)(p.safety * fmin(fmin(p.dx[i], p.dy[p.ndim == 2 ? j : 0]), p.dz0));
      dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, fm[5], fm[6], fm[7], gmf, sg),
                                    cfl_hd_cell<float>(qh, gmf, sg)));
    }
    rhoc = fmax(rhoc, fmax(um[0] * p.ac, uh[0] * p.ac));
    if (p.ir) {
      double g1, g2;
      mixed::ir_rates<NVM>(um, p, g1, g2);
      grc = fmax(grc, fmax(g1, g2));
    }
  }
  block_minmax<NT>(dtc, rhoc, grc, s_red);
  if (threadIdx.x == 0) dt0[blockIdx.x] = finalize_dt(p, dtc, rhoc, grc);
}

cudaError_t launch_dt0(int n, cudaStream_t s, const Member *mem, const KParams *kps,
                       const float *hi, const float *lo, double *dt0) {
  dt0_kernel<256><<<n, 256, 0, s>>>(mem, kps, hi, lo, dt0);
  return cudaGetLastError();
}

// Launch configuration of a cluster instance (CL CTAs per cluster along x).
template <int NT, int CL>
cudaLaunchConfig_t cluster_config(int grid, cudaStream_t s, cudaLaunchAttribute *at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem_bytes(NT, false);
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

template <int NT, int CL>
cudaError_t launch_cluster(int grid, cudaStream_t s, const Member *mem, const KParams *kps,
                           const int *order, int nmem, int nbig, float *hi, float *lo, float *U1,
                           RunState *st, unsigned *queue, double t_end, long long max_steps) {
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cluster_config<NT, CL>(grid, s, at);
  return cudaLaunchKernelEx(&cfg, ensemble_kernel<NT, false, CL>, mem, kps, order, nmem, nbig,
                            hi, lo, U1, st, queue, t_end, max_steps);
}

cudaError_t launch(int nt, bool has2d, int cl, int grid, cudaStream_t s, const Member *mem,
                   const KParams *kps, const int *order, int nmem, int nbig, float *hi, float *lo,
                   float *U1, RunState *st, unsigned *queue, double t_end, long long max_steps) {
  if (cl > 1) {
    if (has2d) return cudaErrorInvalidValue;
    if (nt == 256 && cl == 4)
      return launch_cluster<256, 4>(grid, s, mem, kps, order, nmem, nbig, hi, lo, U1, st, queue, t_end, max_steps);
    if (nt == 256 && cl == 8)
      return launch_cluster<256, 8>(grid, s, mem, kps, order, nmem, nbig, hi, lo, U1, st, queue, t_end, max_steps);
    if (nt == 512 && cl == 4)
      return launch_cluster<512, 4>(grid, s, mem, kps, order, nmem, nbig, hi, lo, U1, st, queue, t_end, max_steps);
    if (nt == 512 && cl == 8)
      return launch_cluster<512, 8>(grid, s, mem, kps, order, nmem, nbig, hi, lo, U1, st, queue, t_end, max_steps);
    return cudaErrorInvalidValue;
  }
#define PIP_ENS_CASE(NTV)                                                                      \
  case NTV:                                                                                    \
    if (has2d)                                                                                 \
      ensemble_kernel<NTV, true, 1><<<grid, NTV, smem_bytes(NTV, true), s>>>(                  \
          mem, kps, order, nmem, 0, hi, lo, U1, st, queue, t_end, max_steps);                  \
    else                                                                                       \
      ensemble_kernel<NTV, false, 1><<<grid, NTV, smem_bytes(NTV, false), s>>>(                \
          mem, kps, order, nmem, 0, hi, lo, U1, st, queue, t_end, max_steps);                  \
    break;
  switch (nt) {
    PIP_ENS_CASE(128)
    PIP_ENS_CASE(256)
    PIP_ENS_CASE(512)
    PIP_ENS_CASE(1024)
    default: return cudaErrorInvalidValue;
  }
#undef PIP_ENS_CASE
  return cudaGetLastError();
}

template <int NT, bool HAS2D, int CL = 1>
cudaError_t set_smem() {
  return cudaFuncSetAttribute(ensemble_kernel<NT, HAS2D, CL>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes(NT, HAS2D));
}

cudaError_t prepare() {
  cudaError_t e;
  if ((e = set_smem<128, false>()) != cudaSuccess || (e = set_smem<256, false>()) != cudaSuccess ||
      (e = set_smem<512, false>()) != cudaSuccess || (e = set_smem<1024, false>()) != cudaSuccess ||
      (e = set_smem<256, true>()) != cudaSuccess || (e = set_smem<512, true>()) != cudaSuccess ||
      (e = set_smem<1024, true>()) != cudaSuccess || (e = set_smem<256, false, 4>()) != cudaSuccess ||
      (e = set_smem<256, false, 8>()) != cudaSuccess || (e = set_smem<512, false, 4>()) != cudaSuccess ||
      (e = set_smem<512, false, 8>()) != cudaSuccess)
    return e;
  return cudaSuccess;
}

template <int NT, bool HAS2D>
int occupancy() {
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &n, ensemble_kernel<NT, HAS2D, 1>, NT, smem_bytes(NT, HAS2D));
  return e == cudaSuccess ? n : 0;
}

int max_ctas_per_sm(int nt, bool has2d) {
  switch (nt) {
    case 128: return has2d ? 0 : occupancy<128, false>();
    case 256: return has2d ? occupancy<256, true>() : occupancy<256, false>();
    case 512: return has2d ? occupancy<512, true>() : occupancy<512, false>();
    case 1024: return has2d ? occupancy<1024, true>() : occupancy<1024, false>();
    default: return 0;
  }
}

template <int NT, int CL>
int cluster_count() {
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cluster_config<NT, CL>(CL, nullptr, at);
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveClusters(&n, ensemble_kernel<NT, false, CL>, &cfg);
  return e == cudaSuccess ? n : 0;
}

// Clusters of CL CTAs of nt threads the device keeps resident at once (0: no such instance).
int max_clusters(int nt, int cl) {
  if (nt == 256 && cl == 4) return cluster_count<256, 4>();
  if (nt == 256 && cl == 8) return cluster_count<256, 8>();
  if (nt == 512 && cl == 4) return cluster_count<512, 4>();
  if (nt == 512 && cl == 8) return cluster_count<512, 8>();
  return 0;
}

}  // namespace ens
}  // namespace pip

// ------------------------------------------------------------------------------ C ABI

using pip::ens::Member;
using pip::ens::RunState;

struct pip_ensemble {
  int n = 0;
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<pip::KParams> kp;
  std::vector<Member> mem;
  std::vector<long long> cost;
  long long total_floats = 0;
  Member *d_mem = nullptr;
  pip::KParams *d_kp = nullptr;
  int *d_order = nullptr;
  float *hi = nullptr, *lo = nullptr, *U1 = nullptr;
  float *save_hi = nullptr, *save_lo = nullptr;  // state snapshot for the autotuner
  double *d_dx = nullptr;                         // dx, 1/dx, dy tables of all members
  double *stage64 = nullptr;                      // FP64 staging of one member
  RunState *d_st = nullptr;
  unsigned *d_queue = nullptr;
  int threads = 256, ctas_per_sm = 2;
  int cluster = 0;                                // 0: chosen per launch, 1: off, 4 or 8
  double share = 0.25;                            // shared: work above share x an even share
  bool has2d = false;                             // some member is 2D
  double *d_dt0 = nullptr;                        // each run's initial dt (work estimate)
  std::vector<int> order;                         // queue order of the last launch
  int cl = 1, nbig = 0, grid = 0;                 // cluster size, shared runs, CTAs launched
  cudaGraphExec_t graph = nullptr;
  double graph_t_end = -1.0;
  long long graph_steps = -1;
  int graph_threads = 0, graph_ctas = 0, graph_cl = 0, graph_nbig = -1, graph_grid = 0;
};

#define EK(call)                        \
  do {                                  \
    cudaError_t e__ = (call);           \
    if (e__ != cudaSuccess) {           \
      pip::record_cuda_error((int)e__);      \
      return PIP_ERR_CUDA;              \
    }                                   \
  } while (0)

extern "C" {

int pip_ensemble_create(const pip_params *members, int n, pip_ensemble **out) {
  if (!members || !out) return PIP_ERR_NULL;
  *out = nullptr;
  if (n <= 0) return PIP_ERR_PARAM;
  pip_ensemble *e = new (std::nothrow) pip_ensemble();
  if (!e) return PIP_ERR_NOMEM;
  e->n = n;
  e->kp.resize(n);
  e->mem.resize(n);
  e->cost.resize(n);
  long long off = 0, dxoff = 0;
  std::vector<double> dxtab;
  for (int r = 0; r < n; ++r) {
    const pip_params &p = members[r];
    if ((p.ndim != 1 && p.ndim != 2) || p.precision != PIP_MIXED) {
      delete e;
      return PIP_ERR_PARAM;
    }
    int st = pip::kparams_from_params(&p, &e->kp[r]);
    if (st != PIP_OK) {
      delete e;
      return st;
    }
    e->mem[r].off = off;
    e->mem[r].kp = r;
    const long long nc = (long long)p.ix * p.jx;
    off += (long long)(p.nvar_m + 5) * nc;
    // dx, 1/dx, dy (and in 2D 1/dy) of this member, pointed at after the upload of the table
    const int ny = p.ndim == 2 ? p.jx : 1;
    for (int i = 0; i < p.ix; ++i) dxtab.push_back(p.dx[i]);
    for (int i = 0; i < p.ix; ++i) dxtab.push_back(1.0 / p.dx[i]);
    for (int j = 0; j < ny; ++j) dxtab.push_back(p.dy[j]);
    if (p.ndim == 2)
      for (int j = 0; j < ny; ++j) dxtab.push_back(1.0 / p.dy[j]);
    e->kp[r].dx = reinterpret_cast<const double *>(dxoff);
    e->kp[r].rdx = reinterpret_cast<const double *>(dxoff + p.ix);
    e->kp[r].dy = reinterpret_cast<const double *>(dxoff + 2 * p.ix);
    e->kp[r].rdy = p.ndim == 2 ? reinterpret_cast<const double *>(dxoff + 2 * p.ix + ny) : nullptr;
    dxoff += 2 * p.ix + (p.ndim == 2 ? 2 * ny : 1);
    // cells x steps: the steps go as the finest width
    e->cost[r] = nc * std::max(p.ix, p.ndim == 2 ? p.jx : 0);
    if (p.ndim == 2) e->has2d = true;
  }
  if (e->has2d) e->threads = std::max(e->threads, 256);
  e->total_floats = off;
  auto fail = [&](cudaError_t c) {
    pip::record_cuda_error((int)c);
    pip_ensemble_destroy(e);
    return c == cudaErrorMemoryAllocation ? PIP_ERR_NOMEM : PIP_ERR_CUDA;
  };
  cudaError_t c;
  if ((c = cudaGetDevice(&e->device)) != cudaSuccess) return fail(c);
  cudaDeviceProp prop;
  if ((c = cudaGetDeviceProperties(&prop, e->device)) != cudaSuccess) return fail(c);
  e->sms = prop.multiProcessorCount;
  if ((c = pip::ens::prepare()) != cudaSuccess) return fail(c);
  if ((c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(c);
  const size_t fb = sizeof(float) * (size_t)off;
  if ((c = cudaMalloc(&e->hi, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMalloc(&e->lo, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMalloc(&e->U1, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMemset(e->hi, 0, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMemset(e->lo, 0, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMemset(e->U1, 0, fb)) != cudaSuccess) return fail(c);
  if ((c = cudaMalloc(&e->d_dx, sizeof(double) * dxtab.size())) != cudaSuccess) return fail(c);
  if ((c = cudaMemcpy(e->d_dx, dxtab.data(), sizeof(double) * dxtab.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(c);
  for (int r = 0; r < n; ++r) {
    e->kp[r].dx = e->d_dx + reinterpret_cast<long long>(e->kp[r].dx);
    e->kp[r].rdx = e->d_dx + reinterpret_cast<long long>(e->kp[r].rdx);
    e->kp[r].dy = e->d_dx + reinterpret_cast<long long>(e->kp[r].dy);
    if (e->kp[r].rdy) e->kp[r].rdy = e->d_dx + reinterpret_cast<long long>(e->kp[r].rdy);
  }
  if ((c = cudaMalloc(&e->d_kp, sizeof(pip::KParams) * n)) != cudaSuccess) return fail(c);
  if ((c = cudaMemcpy(e->d_kp, e->kp.data(), sizeof(pip::KParams) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(c);
  if ((c = cudaMalloc(&e->d_mem, sizeof(Member) * n)) != cudaSuccess) return fail(c);
  if ((c = cudaMemcpy(e->d_mem, e->mem.data(), sizeof(Member) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(c);
  // longest runs first (cost ~ cells x steps ~ ix^2)
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->cost[a] > e->cost[b]; });
  if ((c = cudaMalloc(&e->d_order, sizeof(int) * n)) != cudaSuccess) return fail(c);
  if ((c = cudaMemcpy(e->d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(c);
  e->order = order;
  if ((c = cudaMalloc(&e->d_st, sizeof(RunState) * n)) != cudaSuccess) return fail(c);
  if ((c = cudaMemset(e->d_st, 0, sizeof(RunState) * n)) != cudaSuccess) return fail(c);
  if ((c = cudaMalloc(&e->d_queue, 2 * sizeof(unsigned))) != cudaSuccess) return fail(c);
  if ((c = cudaMalloc(&e->d_dt0, sizeof(double) * n)) != cudaSuccess) return fail(c);
  long long maxst = 0;
  for (int r = 0; r < n; ++r)
    maxst = std::max(maxst, (long long)(members[r].nvar_m + 5) * members[r].ix * members[r].jx);
  if ((c = cudaMalloc(&e->stage64, sizeof(double) * maxst)) != cudaSuccess) return fail(c);
  *out = e;
  return PIP_OK;
}

void pip_ensemble_destroy(pip_ensemble *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  cudaFree(e->hi);
  cudaFree(e->lo);
  cudaFree(e->U1);
  cudaFree(e->save_hi);
  cudaFree(e->save_lo);
  cudaFree(e->d_dx);
  cudaFree(e->d_kp);
  cudaFree(e->d_mem);
  cudaFree(e->d_order);
  cudaFree(e->d_st);
  cudaFree(e->d_queue);
  cudaFree(e->d_dt0);
  cudaFree(e->stage64);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

int pip_ensemble_upload(pip_ensemble *e, int member, const double *U_h, const double *U_m) {
  if (!e || !U_h || !U_m) return PIP_ERR_NULL;
  if (member < 0 || member >= e->n) return PIP_ERR_PARAM;
  EK(cudaSetDevice(e->device));
  const pip::KParams &k = e->kp[member];
  const size_t pb = sizeof(double) * (size_t)k.nc;
  EK(cudaMemcpyAsync(e->stage64, U_m, pb * k.nvm, cudaMemcpyHostToDevice, e->stream));
  EK(cudaMemcpyAsync(e->stage64 + k.nvm * k.nc, U_h, pb * 5, cudaMemcpyHostToDevice, e->stream));
  EK(pip::mixed_split(e->stage64, e->hi + e->mem[member].off, e->lo + e->mem[member].off,
                      (k.nvm + 5) * k.nc, e->stream));
  RunState z;
  std::memset(&z, 0, sizeof z);
  EK(cudaMemcpyAsync(e->d_st + member, &z, sizeof z, cudaMemcpyHostToDevice, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  return PIP_OK;
}

int pip_ensemble_member(pip_ensemble *e, int member, double *U_h, double *U_m, double *time,
                        int64_t *steps, int *status) {
  if (!e) return PIP_ERR_NULL;
  if (member < 0 || member >= e->n) return PIP_ERR_PARAM;
  EK(cudaSetDevice(e->device));
  const pip::KParams &k = e->kp[member];
  const size_t pb = sizeof(double) * (size_t)k.nc;
  RunState rs;
  EK(cudaMemcpyAsync(&rs, e->d_st + member, sizeof rs, cudaMemcpyDeviceToHost, e->stream));
  if (U_h && U_m) {
    EK(pip::mixed_join(e->hi + e->mem[member].off, e->lo + e->mem[member].off, e->stage64,
                       (k.nvm + 5) * k.nc, e->stream));
    EK(cudaMemcpyAsync(U_m, e->stage64, pb * k.nvm, cudaMemcpyDeviceToHost, e->stream));
    EK(cudaMemcpyAsync(U_h, e->stage64 + k.nvm * k.nc, pb * 5, cudaMemcpyDeviceToHost, e->stream));
  }
  EK(cudaStreamSynchronize(e->stream));
  if (time) *time = rs.time;
  if (steps) *steps = rs.steps;
  if (status) *status = rs.status;
  return PIP_OK;
}

int pip_ensemble_timings(pip_ensemble *e, double *start_us, double *end_us) {
  if (!e || !start_us || !end_us) return PIP_ERR_NULL;
  EK(cudaSetDevice(e->device));
  std::vector<RunState> all((size_t)e->n);
  EK(cudaMemcpyAsync(all.data(), e->d_st, sizeof(RunState) * e->n, cudaMemcpyDeviceToHost, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  unsigned long long t0 = ~0ull;
  for (const RunState &r : all)
    if (r.t_end != 0 && r.t_start < t0) t0 = r.t_start;
  for (int m = 0; m < e->n; ++m) {
    const RunState &r = all[(size_t)m];
    start_us[m] = r.t_end == 0 ? -1.0 : 1.0e-3 * (double)(r.t_start - t0);
    end_us[m] = r.t_end == 0 ? -1.0 : 1.0e-3 * (double)(r.t_end - t0);
  }
  return PIP_OK;
}

int pip_ensemble_blocks(pip_ensemble *e, int *blocks) {
  if (!e || !blocks) return PIP_ERR_NULL;
  EK(cudaSetDevice(e->device));
  std::vector<RunState> all((size_t)e->n);
  EK(cudaMemcpyAsync(all.data(), e->d_st, sizeof(RunState) * e->n, cudaMemcpyDeviceToHost, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  for (int m = 0; m < e->n; ++m) blocks[m] = all[(size_t)m].t_end == 0 ? 0 : all[(size_t)m].blocks;
  return PIP_OK;
}

int pip_ensemble_slots(pip_ensemble *e, int *slots) {
  if (!e || !slots) return PIP_ERR_NULL;
  *slots = e->grid > 0 ? e->grid : e->sms * e->ctas_per_sm;
  return PIP_OK;
}

int pip_ensemble_set_cluster(pip_ensemble *e, int cluster, double share) {
  if (!e) return PIP_ERR_NULL;
  if (cluster != 0 && cluster != 1 && cluster != 4 && cluster != 8) return PIP_ERR_PARAM;
  if (cluster > 1 && (e->has2d || (e->threads != 256 && e->threads != 512))) return PIP_ERR_PARAM;
  if (!(share > 0.0)) return PIP_ERR_PARAM;
  e->cluster = cluster;
  e->share = share;
  return PIP_OK;
}

int pip_ensemble_plan(pip_ensemble *e, int *cluster, int *shared_runs, int *grid) {
  if (!e) return PIP_ERR_NULL;
  if (cluster) *cluster = e->cl;
  if (shared_runs) *shared_runs = e->nbig;
  if (grid) *grid = e->grid;
  return PIP_OK;
}

int pip_ensemble_set_config(pip_ensemble *e, int threads, int ctas_per_sm) {
  if (!e) return PIP_ERR_NULL;
  if (threads != 128 && threads != 256 && threads != 512 && threads != 1024) return PIP_ERR_PARAM;
  if (e->has2d && threads < 256) return PIP_ERR_PARAM;   // a 2D tile needs 224 threads
  const int mx = pip::ens::max_ctas_per_sm(threads, e->has2d);
  if (ctas_per_sm < 1 || ctas_per_sm > mx) return PIP_ERR_PARAM;
  e->threads = threads;
  e->ctas_per_sm = ctas_per_sm;
  return PIP_OK;
}

static int ens_enqueue(pip_ensemble *e, double t_end, long long max_steps) {
  EK(cudaMemsetAsync(e->d_queue, 0, 2 * sizeof(unsigned), e->stream));
  EK(pip::ens::launch(e->threads, e->has2d, e->cl, e->grid, e->stream, e->d_mem, e->d_kp,
                      e->d_order, e->n, e->nbig, e->hi, e->lo, e->U1, e->d_st, e->d_queue, t_end,
                      max_steps));
  return PIP_OK;
}

// Work estimate and queue order of a launch: each run's interior cells x the steps its
// initial dt gives to the end (a step limit caps it), runs in decreasing order.  With
// clusters (1D ensembles of 256 or 512 threads) the runs above `share` (default 0.25) of an
// even share of the total work are shared by a cluster each: 4 CTAs, or 8 when the longest
// run exceeds 4 even shares.  cluster = 1 keeps every run on one CTA.
static int ens_plan(pip_ensemble *e, double t_end, long long max_steps) {
  const int n = e->n;
  EK(pip::ens::launch_dt0(n, e->stream, e->d_mem, e->d_kp, e->hi, e->lo, e->d_dt0));
  std::vector<double> dt0((size_t)n);
  std::vector<RunState> st((size_t)n);
  EK(cudaMemcpyAsync(dt0.data(), e->d_dt0, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream));
  EK(cudaMemcpyAsync(st.data(), e->d_st, sizeof(RunState) * n, cudaMemcpyDeviceToHost, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  std::vector<double> work((size_t)n);
  double total = 0.0, longest = 0.0;
  for (int r = 0; r < n; ++r) {
    const pip::KParams &k = e->kp[r];
    double steps = 1.0;
    if (st[r].status == 0) {
      const double left = t_end > 0.0 ? t_end - st[r].time : 0.0;
      steps = t_end > 0.0 && dt0[r] > 0.0 && std::isfinite(dt0[r]) ? std::max(left / dt0[r], 0.0) + 1.0
                                                                 : (double)max_steps;
      if (max_steps > 0) steps = std::min(steps, (double)max_steps);
    }
    work[r] = (double)k.nx * (k.ndim == 2 ? (double)k.ny : 1.0) * steps;
    total += work[r];
    longest = std::max(longest, work[r]);
  }
  std::vector<int> order((size_t)n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  const bool can = !e->has2d && (e->threads == 256 || e->threads == 512) && e->cluster != 1;
  int cl = 1, nbig = 0, grid = e->sms * e->ctas_per_sm;
  if (can) {
    const int c4 = pip::ens::max_clusters(e->threads, 4), c8 = pip::ens::max_clusters(e->threads, 8);
    const double even4 = c4 > 0 ? total / (4.0 * c4) : 0.0;
    int want = e->cluster;
    if (want == 0 && c4 > 0 && longest > 0.75 * even4) want = longest > 4.0 * 4.0 * even4 && c8 > 0 ? 8 : 4;
    const int cc = want == 4 ? c4 : want == 8 ? c8 : 0;
    if (cc > 0) {
      cl = want;
      grid = cc * cl;
      const double even = total / (double)grid;
      while (nbig < n && work[(size_t)order[(size_t)nbig]] > e->share * even) ++nbig;
    }
  }
  if (order != e->order) {
    EK(cudaMemcpyAsync(e->d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->stream));
    EK(cudaStreamSynchronize(e->stream));
    e->order = order;
  }
  e->cl = cl;
  e->nbig = nbig;
  e->grid = grid;
  return PIP_OK;
}

int pip_ensemble_run(pip_ensemble *e, double t_end, int64_t max_steps, float *device_ms) {
  if (!e) return PIP_ERR_NULL;
  if (!(t_end > 0.0) && max_steps <= 0) return PIP_ERR_PARAM;
  EK(cudaSetDevice(e->device));
  const int pl = ens_plan(e, t_end, max_steps);
  if (pl != PIP_OK) return pl;
  // one graph per (end time, step limit, configuration): queue reset + persistent kernel
  if (!e->graph || e->graph_t_end != t_end || e->graph_steps != max_steps ||
      e->graph_threads != e->threads || e->graph_ctas != e->ctas_per_sm ||
      e->graph_cl != e->cl || e->graph_nbig != e->nbig || e->graph_grid != e->grid) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    cudaGraph_t g = nullptr;
    EK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    const int st = ens_enqueue(e, t_end, max_steps);
    cudaError_t c = cudaStreamEndCapture(e->stream, &g);
    if (st != PIP_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    EK(c);
    c = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    EK(c);
    e->graph_t_end = t_end;
    e->graph_steps = max_steps;
    e->graph_threads = e->threads;
    e->graph_ctas = e->ctas_per_sm;
    e->graph_cl = e->cl;
    e->graph_nbig = e->nbig;
    e->graph_grid = e->grid;
  }
  cudaEvent_t a = nullptr, b = nullptr;
  if (device_ms) {
    EK(cudaEventCreate(&a));
    EK(cudaEventCreate(&b));
    EK(cudaEventRecord(a, e->stream));
  }
  EK(cudaGraphLaunch(e->graph, e->stream));
  if (device_ms) EK(cudaEventRecord(b, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  if (device_ms) {
    EK(cudaEventElapsedTime(device_ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  return PIP_OK;
}

// Autotuner: times every (threads, CTAs per SM) the device can hold on a short run from
// the current state (restored after each trial) and keeps the fastest.
int pip_ensemble_tune(pip_ensemble *e, double t_probe, int *threads, int *ctas_per_sm, float *best_ms) {
  if (!e) return PIP_ERR_NULL;
  if (!(t_probe > 0.0)) return PIP_ERR_PARAM;
  EK(cudaSetDevice(e->device));
  const size_t fb = sizeof(float) * (size_t)e->total_floats;
  if (!e->save_hi) EK(cudaMalloc(&e->save_hi, fb));
  if (!e->save_lo) EK(cudaMalloc(&e->save_lo, fb));
  std::vector<RunState> st0(e->n);
  EK(cudaMemcpyAsync(e->save_hi, e->hi, fb, cudaMemcpyDeviceToDevice, e->stream));
  EK(cudaMemcpyAsync(e->save_lo, e->lo, fb, cudaMemcpyDeviceToDevice, e->stream));
  EK(cudaMemcpyAsync(st0.data(), e->d_st, sizeof(RunState) * e->n, cudaMemcpyDeviceToHost, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  float best = 1e30f;
  int bt = e->threads, bc = e->ctas_per_sm;
  const int cand_t[4] = {128, 256, 512, 1024};
  for (int ti = 0; ti < 4; ++ti) {
    if (e->has2d && cand_t[ti] < 256) continue;
    const int mx = std::min(pip::ens::max_ctas_per_sm(cand_t[ti], e->has2d), 8);
    for (int cps = 1; cps <= mx; ++cps) {
      e->threads = cand_t[ti];
      e->ctas_per_sm = cps;
      // probe run: every member advances to t_probe from the saved state
      EK(cudaMemcpyAsync(e->hi, e->save_hi, fb, cudaMemcpyDeviceToDevice, e->stream));
      EK(cudaMemcpyAsync(e->lo, e->save_lo, fb, cudaMemcpyDeviceToDevice, e->stream));
      EK(cudaMemcpyAsync(e->d_st, st0.data(), sizeof(RunState) * e->n, cudaMemcpyHostToDevice, e->stream));
      float ms = 0.f;
      const int st = pip_ensemble_run(e, t_probe, 0, &ms);
      if (st != PIP_OK) return st;
      if (ms < best) {
        best = ms;
        bt = cand_t[ti];
        bc = cps;
      }
    }
  }
  EK(cudaMemcpyAsync(e->hi, e->save_hi, fb, cudaMemcpyDeviceToDevice, e->stream));
  EK(cudaMemcpyAsync(e->lo, e->save_lo, fb, cudaMemcpyDeviceToDevice, e->stream));
  EK(cudaMemcpyAsync(e->d_st, st0.data(), sizeof(RunState) * e->n, cudaMemcpyHostToDevice, e->stream));
  EK(cudaStreamSynchronize(e->stream));
  e->threads = bt;
  e->ctas_per_sm = bc;
  if (threads) *threads = bt;
  if (ctas_per_sm) *ctas_per_sm = bc;
  if (best_ms) *best_ms = best;
  return PIP_OK;
}

}  // extern "C"
