// pip_mixed.cu -- FP32-mixed form of the two-fluid step.
//
// Storage: the stage state and the fluxes are FP32.  U0 (array A) is kept as an FP32
// pair (hi, lo) with hi + lo = the FP64 value, so that the conservative update
// U2 = U0 - dt*div(F) + dt*S is accumulated in FP64 across the RK stages (compensated
// accumulation) and the stored state keeps ~48 significant bits.  The collisional and
// ionisation/recombination source (the stiff part) is evaluated in FP64.  The cq2pv
// rewrites of the FP64 path change a state only below the pair's precision except where
// a density or pressure floor fires; this form applies the floors (in FP64) and skips the
// round trip otherwise.
//
// Bytes per cell and step (14 planes): stage 1 reads hi and writes U1 (8 B/plane), stage 2
// reads U1, hi, lo and writes hi, lo (20 B/plane): 392 B.
//
// Compiled with -ftz=true -prec-div=false -prec-sqrt=false: FP32 division and square root
// are the approximate hardware forms; FP64 arithmetic is unaffected.
#include <cstring>

#include "pip_kernels.cuh"
#include "pip_mixed_cell.cuh"
#include "pip_physics.cuh"
#include "pip_mixed_tile.cuh"
#include "pip_tma.cuh"

namespace pip {
namespace mixed {

// 2D tile height and CTAs per SM of the stage kernels (compile-time tuning constants).
#ifndef PIP_MIXED_TX
#define PIP_MIXED_TX 16
#endif
#ifndef PIP_MIXED_TY
#define PIP_MIXED_TY 14
#endif
#ifndef PIP_MIXED_MINB
#define PIP_MIXED_MINB 3
#endif

constexpr int kH = 2;
template <int NDIM> struct Tile;
template <> struct Tile<2> {
  // 16x14 cells: 17x14 x faces + 16x15 y faces = 478 faces, two rounds of 256 threads;
  // primitives for 20x18 - 16 = 344 cells (1.54 per updated cell; 1.70 with 32x7)
  static constexpr int TX = PIP_MIXED_TX, TY = PIP_MIXED_TY, NT = (TX * TY + 255) / 256 * 256;
};
template <> struct Tile<1> {
  static constexpr int TX = 128, TY = 1, NT = 128;
};

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

__device__ __forceinline__ double finalize_dt(const KParams &p, const DevCtrl *c, int slot) {
  double dt = bitsd(c->red_dt[slot]);
  double rho = bitsd(c->red_rho[slot]);
  dt = fmin(dt, p.col_lim / rho);
  if (p.ir) dt = fmin(dt, p.ir_lim / fmax(bitsd(c->red_gr[slot]), 1.0e-5));
  return dt;
}

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
    atomicMin(&ctrl->red_dt[slot], dbits(dtc));
    atomicMax(&ctrl->red_rho[slot], dbits(rho));
    atomicMax(&ctrl->red_gr[slot], dbits(gr));
  }
}

// One RK stage (see the FP64 stage_kernel for the structure).  Stage 1: Us = A.hi,
// U0 = A.hi, output B (FP32).  Stage 2: Us = B, U0 = A.hi + A.lo, output A (hi, lo).
// The parameter block is __grid_constant__: the out-of-line ghost writer takes its address,
// which would otherwise copy the whole block to every thread's stack.  With use_tma (2D),
// the tile and its halo of all planes of Us arrive by one TMA load (tmap describes Us).
template <int NDIM, int NVM, int STAGE>
__global__ void __launch_bounds__(Tile<NDIM>::NT, NDIM == 2 ? PIP_MIXED_MINB : 4)
stage_kernel(const __grid_constant__ KParams p, const float *__restrict__ Us, const float *U0hi, const float *U0lo,
             float *Ohi, float *Olo, DevCtrl *ctrl, int dt_mode, int epi,
             const __grid_constant__ CUtensorMap tmap, int use_tma, int rows) {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY, NT = Tile<NDIM>::NT;
  constexpr int NV = NVM + 5;
  constexpr int RX = TX + 2 * kH, RY = NDIM == 2 ? TY + 2 * kH : 1, RR = RX * RY;
  constexpr int NFX = (TX + 1) * TY, NFY = NDIM == 2 ? TX * (TY + 1) : 0;
  extern __shared__ __align__(128) double smd[];
  // the tile's primitives first (128-byte aligned: the TMA destination), then the FP64
  // Dedner fluxes (Bn and psi components, HLL_rot.f90:904-908) of every face -- the psi
  // flux carries ch^2 (BnL+BnR), whose face-to-face difference cancels in FP32 -- then the
  // FP32 fluxes
  float *sV = reinterpret_cast<float *>(smd);
  double *sD6 = reinterpret_cast<double *>(sV + NV * RR);
  double *sD9 = sD6 + (NVM == 9 ? NFX + NFY : 0);
  float *sFx = reinterpret_cast<float *>(sD9 + (NVM == 9 ? NFX + NFY : 0));
  float *sFy = sFx + NV * NFX;
  static_assert((NV * RR * sizeof(float)) % sizeof(double) == 0, "Dedner planes alignment");
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ double s_dt, s_cmax;
  __shared__ long long s_step;
  __shared__ int s_exit, s_epi;

  const int tid = threadIdx.x;
  // tile row: every row (rows 0), the first and the last (1), the rows between them (2)
  const int nby = NDIM == 2 ? (p.ny + TY - 1) / TY : 1;
  const int by = NDIM == 1 || rows == 0 ? (int)blockIdx.y
                 : rows == 1 ? (blockIdx.y == 0 ? 0 : nby - 1) : (int)blockIdx.y + 1;
  const bool block0 = blockIdx.x == 0 && by == 0;
  if (tid == 0) {
    int ex = STAGE == 1 ? (ctrl->done || ctrl->nan_flag) : ctrl->done;
    double dt, cmax;
    if (STAGE == 1 && dt_mode == 1) {
      dt = finalize_dt(p, ctrl, (int)(ctrl->step & 1));
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
      if (ctrl->nan_flag && ctrl->status == 0) ctrl->status = 3;
      ctrl->done = 1;
    }
    return;
  }
  const double dt = s_dt;
  if (STAGE == 1 && dt_mode == 1 && block0 && tid == 0) {
    const long long st = ctrl->step;
    ctrl->dt = dt;
    ctrl->cmax = s_cmax;
    const double tn = ctrl->time + dt;
    ctrl->time_next = tn;
    ctrl->last = ((ctrl->t_end > 0.0 && tn >= ctrl->t_end) ||
                  (ctrl->nsteps > 0 && st + 1 >= ctrl->nsteps)) ? 1 : 0;
    const int ns = (int)((st + 1) & 1);
    ctrl->red_dt[ns] = dbits(10.0);
    ctrl->red_rho[ns] = 0ull;
    ctrl->red_gr[ns] = 0ull;
  }
  const int i0 = p.m0 + blockIdx.x * TX;
  const int j0 = NDIM == 2 ? p.m1 + by * TY : 0;

  // ---- 1.-3. the tile (primitives, face fluxes, source and update)
  // (the TMA writes shared memory only at 128-byte aligned destinations)
  bool staged = false;
  if (NDIM == 2 && use_tma && (tma_smem_addr(sV) & 127u) == 0) {
    // the raw planes by one TMA load into sV (cells outside the array read as zero); the
    // tile step forms the primitives in place
    if (tid == 0) {
      tma_bar_init(&s_bar);
      tma_bar_expect(&s_bar, (uint32_t)(NV * RR * sizeof(float)));
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
    staged = true;
  }
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  bool bad = false;
  tile_stage<NDIM, NVM, STAGE, TX, TY, NT, kH>(p, Us, U0hi, U0lo, Ohi, Olo, i0, j0, dt, s_cmax,
                                              s_epi, staged, sV, sD6, sD9, sFx, sFy, dtc, rhoc,
                                              grc, bad);
  if (bad) atomicOr(&ctrl->nan_flag, 1);
  if (STAGE == 2 && s_epi == 2) block_reduce_cfl<NT>(dtc, rhoc, grc, ctrl, (int)((s_step + 1) & 1));
  if (STAGE == 2 && dt_mode == 1) {
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      const unsigned int nb = gridDim.x * nby;     // every tile of the stage's launches
      if (atomicAdd(&ctrl->blocks_done, 1u) == nb - 1) {
        __threadfence();
        ctrl->blocks_done = 0u;
        ctrl->time = ctrl->time_next;
        ctrl->step = s_step + 1;
        if (ctrl->last) ctrl->done = 1;
        if (dt <= 1.0e-12) {
          ctrl->done = 1;
          if (ctrl->status == 0) ctrl->status = 4;
        }
      }
    }
  }
}

// cfl over every cell for the mixed state: floors (in FP64 on hi+lo) and FP32 CFL terms.
template <int NVM>
__global__ void __launch_bounds__(256) cfl_kernel(const KParams p, float *Uhi, float *Ulo,
                                                  DevCtrl *ctrl, int slot) {
  double dtc = 10.0, rhoc = 0.0, grc = 0.0;
  const long long nc = p.nc;
  const float gmf = (float)p.gm, rolf = (float)p.ro_lim, prlf = (float)p.pr_lim;
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < nc; q += (long long)gridDim.x * 256) {
    double um[NVM], uh[5];
#pragma unroll
    for (int n = 0; n < NVM; ++n) um[n] = (double)Uhi[q + n * nc] + (double)Ulo[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n)
      uh[n] = (double)Uhi[q + (NVM + n) * nc] + (double)Ulo[q + (NVM + n) * nc];
    floors_mhd<NVM>(um, p);
    floors_hd(uh, p);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      float h = (float)um[n];
      Uhi[q + n * nc] = h;
      Ulo[q + n * nc] = (float)(um[n] - (double)h);
      h = (float)uh[n];
      Uhi[q + (NVM + n) * nc] = h;
      Ulo[q + (NVM + n) * nc] = (float)(uh[n] - (double)h);
    }
    const int i = (int)(q % p.ix), j = (int)(q / p.ix);
    const bool interior = i >= p.m0 && i < p.ix - p.m0 && j >= p.m1 && j < p.jx - p.m1;
    if (interior) {
      float fm[NVM], fh[5];
#pragma unroll
      for (int n = 0; n < NVM; ++n) fm[n] = (float)um[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) fh[n] = (float)uh[n];
      const Prim<float> qm = cq2pv_mhd<float, NVM>(fm, gmf, rolf, prlf);
      const Prim<float> qh = cq2pv_hd<float>(fh, gmf, rolf, prlf);
      const float sg = (float)(p.safety * fmin(fmin(p.dx[i], p.dy[j]), p.dz0));
      dtc = fmin(dtc, (double)fminf(cfl_mhd_cell<float>(qm, fm[5], fm[6], fm[7], gmf, sg),
                                    cfl_hd_cell<float>(qh, gmf, sg)));
    }
    rhoc = fmax(rhoc, fmax(um[0] * p.ac, uh[0] * p.ac));
    if (p.ir) {
      double g1, g2;
      ir_rates<NVM>(um, p, g1, g2);
      grc = fmax(grc, fmax(g1, g2));
    }
  }
  block_reduce_cfl<256>(dtc, rhoc, grc, ctrl, slot);
}

// FP64 <-> (hi, lo) conversions of whole state arrays.
__global__ void split_kernel(const double *__restrict__ U, float *hi, float *lo, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double u = U[t];
    const float h = (float)u;
    hi[t] = h;
    lo[t] = (float)(u - (double)h);
  }
}
__global__ void join_kernel(const float *__restrict__ hi, const float *__restrict__ lo, double *U,
                            long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    U[t] = (double)hi[t] + (double)lo[t];
}

template <int NDIM, int NVM>
constexpr size_t smem_bytes() {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY;
  constexpr int RR = (TX + 2 * kH) * (NDIM == 2 ? TY + 2 * kH : 1);
  constexpr int NFX = (TX + 1) * TY, NFY = NDIM == 2 ? TX * (TY + 1) : 0;
  return sizeof(float) * (NVM + 5) * (RR + NFX + NFY) +
         (NVM == 9 ? 2 * sizeof(double) * (NFX + NFY) : 0);
}

template <int NDIM, int NVM, int STAGE>
static cudaError_t set_attr() {
  return cudaFuncSetAttribute(stage_kernel<NDIM, NVM, STAGE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes<NDIM, NVM>());
}

template <int NDIM, int NVM, int STAGE>
static cudaError_t launch_t(const KParams &p, const float *Us, const float *U0hi, const float *U0lo,
                            float *Ohi, float *Olo, DevCtrl *ctrl, int dt_mode, int epi,
                            cudaStream_t s, const CUtensorMap *tm, int rows) {
  constexpr int TX = Tile<NDIM>::TX, TY = Tile<NDIM>::TY, NT = Tile<NDIM>::NT;
  const int nby = NDIM == 2 ? (p.ny + TY - 1) / TY : 1;
  if (NDIM == 1) rows = 0;
  const int gy = rows == 0 ? nby : rows == 1 ? (nby < 2 ? nby : 2) : nby - 2;
  if (gy <= 0) return cudaSuccess;   // no rows between the first and the last
  dim3 grid((p.nx + TX - 1) / TX, gy);
  CUtensorMap none;
  std::memset(&none, 0, sizeof none);
  stage_kernel<NDIM, NVM, STAGE><<<grid, NT, smem_bytes<NDIM, NVM>(), s>>>(
      p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, tm ? *tm : none, tm ? 1 : 0, rows);
  return cudaGetLastError();
}

static int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace mixed

cudaError_t mixed_prepare() {
  cudaError_t e;
  if ((e = mixed::set_attr<1, 8, 1>()) != cudaSuccess) return e;
  if ((e = mixed::set_attr<1, 8, 2>()) != cudaSuccess) return e;
  if ((e = mixed::set_attr<2, 8, 1>()) != cudaSuccess) return e;
  if ((e = mixed::set_attr<2, 8, 2>()) != cudaSuccess) return e;
  if ((e = mixed::set_attr<2, 9, 1>()) != cudaSuccess) return e;
  return mixed::set_attr<2, 9, 2>();
}

cudaError_t mixed_stage(const KParams &p, int stage, const float *Us, const float *U0hi,
                        const float *U0lo, float *Ohi, float *Olo, DevCtrl *ctrl, int dt_mode,
                        int epi, cudaStream_t s, const CUtensorMap *tm, int rows) {
  using namespace mixed;
  if (p.ndim == 1)
    return stage == 1 ? launch_t<1, 8, 1>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, nullptr, 0)
                      : launch_t<1, 8, 2>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, nullptr, 0);
  if (p.nvm == 9)
    return stage == 1 ? launch_t<2, 9, 1>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, tm, rows)
                      : launch_t<2, 9, 2>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, tm, rows);
  return stage == 1 ? launch_t<2, 8, 1>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, tm, rows)
                    : launch_t<2, 8, 2>(p, Us, U0hi, U0lo, Ohi, Olo, ctrl, dt_mode, epi, s, tm, rows);
}

bool mixed_tile_map(const KParams &p, const float *Us, CUtensorMap *map) {
  using namespace mixed;
  if (p.ndim != 2) return false;
  constexpr int TX = Tile<2>::TX, TY = Tile<2>::TY;
  if (!tma_tile_ok(Us, p.ix, p.jx, p.nvm + 5, (int)sizeof(float), p.m0 - kH, TX, TX + 2 * kH,
                   TY + 2 * kH))
    return false;
  return tma_encode(map, Us, p.ix, p.jx, p.nvm + 5, (int)sizeof(float), TX + 2 * kH, TY + 2 * kH);
}

cudaError_t mixed_cfl(const KParams &p, float *hi, float *lo, DevCtrl *ctrl, int slot,
                      cudaStream_t s) {
  const int g = mixed::grid_for(p.nc, 256);
  if (p.nvm == 9) mixed::cfl_kernel<9><<<g, 256, 0, s>>>(p, hi, lo, ctrl, slot);
  else mixed::cfl_kernel<8><<<g, 256, 0, s>>>(p, hi, lo, ctrl, slot);
  return cudaGetLastError();
}

cudaError_t mixed_split(const double *U, float *hi, float *lo, long long n, cudaStream_t s) {
  mixed::split_kernel<<<mixed::grid_for(n, 256), 256, 0, s>>>(U, hi, lo, n);
  return cudaGetLastError();
}

cudaError_t mixed_join(const float *hi, const float *lo, double *U, long long n, cudaStream_t s) {
  mixed::join_kernel<<<mixed::grid_for(n, 256), 256, 0, s>>>(hi, lo, U, n);
  return cudaGetLastError();
}

}  // namespace pip
