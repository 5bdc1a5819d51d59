// pip_conduction.cu -- implicit anisotropic conduction of the ion species (HC(U_m,nvar_m,1),
// HC_rot.f90:67-140) on the device: cq2pv rewrite and temperature, the 9-point matrix of
// set_matrix_source_MHD2D9 (HC_rot.f90:643-739) with set_matrix_boundary's folding
// (:468-529), BiCGstab (:187-299, hc_split = 2) and the conversion back (pv2cq_mhd,
// Scheme_rot.f90:43-79).
//
// The matrix is held as face factors rather than nine planes: eta = kapper dt (gm-1) gm / ro
// per cell, te^2.5 nx nx and te^2.5 nx ny per x-face, te^2.5 ny ny and te^2.5 ny nx per
// y-face (nx, ny the components of the unit field vector at the face), and per column /
// row the grid factors 1/(dxc dx), 1/dxc, ...; each kernel rebuilds the nine entries of its
// row (the reference's combinations and boundary folds) in registers.  That is 5 planes
// read per matrix application instead of 9; the entries differ from the reference's
// left-to-right products (eta*te25*n*n/dxc/dx) by rounding only.
//
// BiCGstab keeps the reference's structure (the residual is recomputed from the iterate
// every iteration, so the stopping test sees the true residual).  One iteration is three
// kernels over the interior cells:
//   k1  p' = r + beta (p - omega Ap)  (p' = p in the first iteration); Ap' = A p';
//                                                    sums (r,r0), (r0,Ap')  -> alpha
//   k2  t  = r - alpha Ap';  At = A t;               sums (t,At), (At,At)   -> omega
//   k3  x' = x + alpha p' + omega t;  r = b - A x';  sums (r0,r), (r,r)     -> beta,
//       relative residual, stop flag
// A block owns 128 columns and a range of rows; the inputs of each row are staged into
// shared memory by bulk async copies rows ahead (two stages of two rows), and each thread
// keeps the 3x3 neighbourhood of the vector the matrix is applied to (p', t or x', formed
// from its inputs once per point) in registers as it walks down its column.  p, Ap and x are
// double-buffered (iteration i reads buffer i&1 and writes (i+1)&1), so no kernel reads
// what it writes.  Scalars are reduced by the last block of each kernel to finish (fixed
// order: deterministic) into a device block; every kernel returns at once when the stop
// flag is set, so the host launches iterations in groups and reads the flag between
// groups.  Vectors and matrix are templated: FP64 for the plain path; FP32 (FP32 products
// and sums, FP64 dot products) for the inner solve of the mixed path, whose FP64 outer
// loop (iterative refinement) recomputes the residual in FP64 and corrects x in FP64 until
// the FP64 relative residual reaches the target.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <initializer_list>
#include <new>

#include "pip_kernels.cuh"
#include "pip_physics.cuh"

namespace pip {
namespace hc {

constexpr int NT = 256;             // one-thread-per-cell kernels
constexpr int SX = 128;             // BiCGstab kernels: interior columns (threads) per block
// Pipeline of the BiCGstab kernels: NS stages of RS rows each, per precision (compile-time
// tuning, measured on KH 2048x1024: FP64 4 stages of 1 row, 122 us per iteration against
// 125 with 2 of 2; FP32 2 stages of 2 rows, 120 us against 123 with 4 of 1).
#ifndef PIP_HC_STAGES
#define PIP_HC_STAGES 4
#endif
#ifndef PIP_HC_ROWS
#define PIP_HC_ROWS 1
#endif
#ifndef PIP_HC_STAGES32
#define PIP_HC_STAGES32 2
#endif
#ifndef PIP_HC_ROWS32
#define PIP_HC_ROWS32 2
#endif
template <typename T>
__host__ __device__ constexpr int stages() {
  return sizeof(T) == 4 ? PIP_HC_STAGES32 : PIP_HC_STAGES;
}
// rows per stage: one wait per group
template <typename T>
__host__ __device__ constexpr int rows() {
  return sizeof(T) == 4 ? PIP_HC_ROWS32 : PIP_HC_ROWS;
}
constexpr int SLOT = 136;           // elements per staged row segment (SX + 2 + alignment)
constexpr int kWaitLimit = 1 << 22; // polls of an mbarrier before a block gives up
constexpr double kEpsi = 1.0e-5;    // HC_rot.f90:17

struct Scal {
  double rr, bb;                  // sum r^2, sum b^2
  double alphau, alphad, alpha;
  double omegau, omegad, omega;
  double betau, beta;
  double relres, tol;
  int count, hc_max, done, fault;
  unsigned int blocks_done;
  int wait_limit;                 // polls of a staging mbarrier before a block gives up
  unsigned int body;              // k3 launches of the solve's device-side loop
};

__device__ __forceinline__ bool interior_cell(const KParams &p, long long t, int &i, int &j) {
  const long long n = (long long)p.nx * p.ny;
  if (t >= n) return false;
  i = p.m0 + (int)(t % p.nx);
  j = p.m1 + (int)(t / p.nx);
  return true;
}

// Face-factor planes of the matrix.
constexpr int NPL = 5;   // 0 eta (cell), 1 fxx, 2 fxy (x-face i-1/2), 3 fyy, 4 fyx (y-face j-1/2)

// The face factors of one row: eta of the cell, (fxx, fxy) of its left (l) and right (r)
// x-faces, (fyy, fyx) of its lower (d) and upper (u) y-faces, and the grid factors
// 1/(dx_i dx_{i-1}), 1/(dx_i dx_i), 1/dx_i of its column and the same in y of its row.
template <typename T>
struct RowFactors {
  T eta, fxxl, fxxr, fxyl, fxyr, fyyd, fyyu, fyxd, fyxu;
  T cxl, cxr, idx, cyd, cyu, idy;
};

// The nine entries of row (i,j), in the reference's neighbour order 0 (i,j), 1 (i-1,j),
// 2 (i+1,j), 3 (i,j-1), 4 (i,j+1), 5 (i-1,j-1), 6 (i+1,j-1), 7 (i-1,j+1), 8 (i+1,j+1),
// with set_matrix_boundary's folds (HC_rot.f90:468-529) on the sides without a neighbouring
// rank (boundary type 0 marks an exchanged face: pip_set_neighbors).  One rank per
// direction: every side folds (MPI_rot.f90:123).
template <typename T>
__device__ __forceinline__ void entries(const KParams &p, const RowFactors<T> &f, int i, int j,
                                        T (&c)[9]) {
  const T eta = f.eta;
  const T exy = eta * (T(0.25) * f.idx * f.idy);
  const T bxxl = -(eta * f.fxxl * f.cxl);
  const T bxxr = -(eta * f.fxxr * f.cxr);
  const T byyd = -(eta * f.fyyd * f.cyd);
  const T byyu = -(eta * f.fyyu * f.cyu);
  const T bxyl = -(exy * f.fxyl);
  const T bxyr = -(exy * f.fxyr);
  const T byxd = -(exy * f.fyxd);
  const T byxu = -(exy * f.fyxu);
  c[1] = bxxl - (byxu - byxd);
  c[2] = bxxr + (byxu - byxd);
  c[3] = byyd - (bxyr - bxyl);
  c[4] = byyu + (bxyr - bxyl);
  c[5] = bxyl + byxd;
  c[6] = -(bxyr + byxd);
  c[7] = -(bxyl + byxu);
  c[8] = bxyr + byxu;
  c[0] = T(1) - (c[1] + c[2] + c[3] + c[4]);
  if (i == p.m0 && p.typex[0] != 0) {                 // x-minus
    c[0] = c[1] + c[0]; c[1] = T(0);
    c[3] = c[3] + c[5]; c[5] = T(0);
    c[4] = c[4] + c[7]; c[7] = T(0);
  }
  if (i == p.m0 + p.nx - 1 && p.typex[1] != 0) {      // x-plus
    c[0] = c[2] + c[0]; c[2] = T(0);
    c[3] = c[3] + c[6]; c[6] = T(0);
    c[4] = c[4] + c[8]; c[8] = T(0);
  }
  if (j == p.m1 && p.typey[0] != 0) {                 // y-minus
    c[0] = c[3] + c[0]; c[3] = T(0);
    c[1] = c[5] + c[1]; c[5] = T(0);
    c[2] = c[6] + c[2]; c[6] = T(0);
  }
  if (j == p.m1 + p.ny - 1 && p.typey[1] != 0) {      // y-plus
    c[0] = c[4] + c[0]; c[4] = T(0);
    c[1] = c[1] + c[7]; c[7] = T(0);
    c[2] = c[2] + c[8]; c[8] = T(0);
  }
}

// w is the 3x3 neighbourhood [dj+1][di+1] of a vector; sum_n c_n * w_n, n = 0..8 left to
// right, in T.
template <typename T>
__device__ __forceinline__ T stencil(const T (&c)[9], const T (&w)[3][3]) {
  T s = c[0] * w[1][1];
  s = s + c[1] * w[1][0];
  s = s + c[2] * w[1][2];
  s = s + c[3] * w[0][1];
  s = s + c[4] * w[2][1];
  s = s + c[5] * w[0][0];
  s = s + c[6] * w[0][2];
  s = s + c[7] * w[2][0];
  s = s + c[8] * w[2][2];
  return s;
}

// Block sums of 2 values into part[k*nb + block]; returns true in thread 0 of the last
// block to finish, which then holds the totals (summed in block order) in tot[].  NTB
// threads per block; the last block's sum over the blocks runs on its first NR threads
// (strided slices, then a tree), so the order of the additions depends on NR only.
template <int NTB, int NR = NTB>
__device__ bool reduce2(double a, double b, double *part, unsigned int *counter, double (&tot)[2]) {
  __shared__ double s[2][NTB / 32];
  __shared__ bool s_last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x / 32;
  if (threadIdx.x % 32 == 0) {
    s[0][w] = a;
    s[1][w] = b;
  }
  __syncthreads();
  const unsigned int nb = gridDim.x;
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int k = 0; k < NTB / 32; ++k) {
      x += s[0][k];
      y += s[1][k];
    }
    part[blockIdx.x] = x;
    part[nb + blockIdx.x] = y;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  // the last block: totals in block order (each thread a strided slice, then a tree)
  __threadfence();
  double x = 0.0, y = 0.0;
  if (threadIdx.x < NR)
    for (unsigned int k = threadIdx.x; k < nb; k += NR) {
      x += part[k];
      y += part[nb + k];
    }
  __shared__ double s2[2][NR];
  if (threadIdx.x < NR) {
    s2[0][threadIdx.x] = x;
    s2[1][threadIdx.x] = y;
  }
  __syncthreads();
  for (int h = NR / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      s2[0][threadIdx.x] += s2[0][threadIdx.x + h];
      s2[1][threadIdx.x] += s2[1][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return false;
  *counter = 0u;
  tot[0] = s2[0][0];
  tot[1] = s2[1][0];
  return true;
}

// cq2pv_mhd on every cell (rewrites the ion planes in place), te = gm*(pr/ro), and the
// kinetic and magnetic energy terms of pv2cq_mhd for the conversion back.
__global__ void setup_kernel(const KParams p, double *U, double *te, double *b, double *kin,
                             double *mag) {
  const long long nc = p.nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    double u[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) u[n] = U[q + n * nc];
    const Prim<double> s = cq2pv_mhd<double, 8>(u, p.gm, p.ro_lim, p.pr_lim);
#pragma unroll
    for (int n = 0; n < 5; ++n) U[q + n * nc] = u[n];
    const double t = p.gm * (s.pr / s.de);
    te[q] = t;
    b[q] = t;
    kin[q] = 0.5 * s.de * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz);
    mag[q] = 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
  }
}

// The face factors of set_matrix_source_MHD2D9 (HC_rot.f90:643-739, dxc = dx, dyc = dy):
// thread (i,j) over i = m0..m0+nx, j = m1..m1+ny writes the x-face i-1/2 of row j (j
// interior), the y-face j-1/2 of column i (i interior) and eta of cell (i,j) (interior).
// The face quantities of the reference (bxl, al, nxl, te_xm, ...) are symmetric in the two
// cells of the face, so each face is computed once.  Writes the FP64 planes and, when m32
// is given, their FP32 copy.
__global__ void matrix_kernel(const KParams p, const double *__restrict__ U, const double *__restrict__ te,
                              const double *dtp, double *m64, float *m32) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long w = p.nx + 1;
  if (t >= w * (p.ny + 1)) return;
  const int i = p.m0 + (int)(t % w), j = p.m1 + (int)(t / w);
  const bool row_in = j < p.m1 + p.ny, col_in = i < p.m0 + p.nx;
  const long long nc = p.nc, ix = p.ix;
  const long long q = (long long)j * ix + i;
  const double *bx = U + 5 * nc, *by = U + 6 * nc, *bz = U + 7 * nc;
  double f[NPL] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int have = 0;
  auto face = [&](long long o, double &fnn, double &fnt, bool x_face) {
    const double b1 = (bx[o] + bx[q]) / 2.0, b2 = (by[o] + by[q]) / 2.0, b3 = (bz[o] + bz[q]) / 2.0;
    const double a = fmax(sqrt(b1 * b1 + b2 * b2 + b3 * b3), kEpsi);
    const double n1 = b1 / a, n2 = b2 / a;
    const double tm = 0.5 * (te[q] + te[o]);
    const double t25 = tm * tm * sqrt(tm);
    if (x_face) {
      fnn = t25 * n1 * n1;
      fnt = n1 * n2 * t25;
    } else {
      fnn = t25 * n2 * n2;
      fnt = n2 * n1 * t25;
    }
  };
  if (row_in) {
    face(q - 1, f[1], f[2], true);
    have |= 6;
  }
  if (col_in) {
    face(q - ix, f[3], f[4], false);
    have |= 24;
  }
  if (row_in && col_in) {
    const double gm = p.gm, dt = *dtp;
    f[0] = p.hc_kapper * dt * (gm - 1.0) / U[q] * gm;
    have |= 1;
  }
#pragma unroll
  for (int n = 0; n < NPL; ++n) {
    if (!(have >> n & 1)) continue;
    m64[q + n * nc] = f[n];
    if (m32) m32[q + n * nc] = (float)f[n];
  }
}

// Grid factors per column (1/(dx_i dx_{i-1}), 1/(dx_i dx_i), 1/dx_i: three arrays of ix)
// and per row (the same in y: three arrays of jx, after the column ones).
__global__ void geometry_kernel(const KParams p, double *g64, float *g32) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool col = t < p.ix;
  if (!col && t >= p.ix + p.jx) return;
  const int k = col ? t : t - p.ix;
  const int n = col ? p.ix : p.jx;
  const double *d = col ? p.dx : p.dy;
  const long long base = col ? 0 : 3LL * p.ix;
  double v[3] = {0.0, 0.0, 0.0};
  if (k >= 1) {
    v[0] = 1.0 / (d[k] * d[k - 1]);
    v[1] = 1.0 / (d[k] * d[k]);
    v[2] = 1.0 / d[k];
  }
  for (int c = 0; c < 3; ++c) {
    g64[base + (long long)c * n + k] = v[c];
    if (g32) g32[base + (long long)c * n + k] = (float)v[c];
  }
}

// ---- shared-memory staging by bulk async copies (the TMA engine) on mbarriers ----

__device__ __forceinline__ uint32_t smem_addr(const void *ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Bounded wait on phase `parity` of bar; false when `limit` polls ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int k = 0; k < limit; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// The four BiCGstab kernels share one body.  A block owns SX interior columns starting at
// i0 and a contiguous range of rows [ja, jb); the rows of a column block are divided evenly
// among its blocks (one wave over the SMs).  Rows are staged in groups of RS, NS groups
// ahead, as row segments copied into shared memory (one bulk copy per segment, a full and
// an empty mbarrier per stage, see the block layout below).  For row j:
//   window vectors (row j+1, columns i0-1 .. i0+SX)   -- the vector A is applied to is
//                                                        formed from these at each point
//   own vectors    (row j, columns i0 .. i0+SX-1)
//   eta (row j), fxx and fxy (row j, columns i0 .. i0+SX: both x-faces of every cell),
//   fyy and fyx (rows j and j+1: both y-faces).
// Window rows ja-1 and ja come from plain loads before the pipeline starts.  A segment is
// copied from its start rounded down to 16 bytes, its length rounded up to 16 bytes and cut
// at the end of its allocation (conduction runs with at least two ghost rows, so the cut
// never reaches a value that is used).
enum Kind { KINIT = 0, K1 = 1, K2 = 2, K3 = 3 };
template <int KIND> struct KindShape;
template <> struct KindShape<KINIT> { static constexpr int nw = 1, no = 1; };  // x | b
template <> struct KindShape<K1> { static constexpr int nw = 3, no = 2; };     // p, Ap, r | r, r0
template <> struct KindShape<K2> { static constexpr int nw = 2, no = 0; };     // r, Ap' |
template <> struct KindShape<K3> { static constexpr int nw = 3, no = 2; };     // x, p', t | b, r0
constexpr int kMatCopies = 7;

template <int KIND>
__host__ __device__ constexpr int n_copies() {
  return KindShape<KIND>::nw + KindShape<KIND>::no + kMatCopies;
}

template <typename T, int KIND>
__host__ __device__ constexpr size_t stage_smem() {
  return (size_t)stages<T>() * rows<T>() * n_copies<KIND>() * SLOT * sizeof(T) +
         2 * stages<T>() * sizeof(unsigned long long);
}

template <typename T>
struct BicgArgs {
  const T *m, *g;            // face-factor planes (NPL*nc) and grid factors
  const T *w[3];             // window vectors
  const T *o[2];             // own vectors
  T *out[3];                 // INIT: r, r0, p;  K1: p', Ap';  K2: t;  K3: x', r
  double *part;
  Scal *sc;
  int ncb, nrb;              // column blocks, row ranges per column block
  cudaGraphConditionalHandle loop;  // k3 in the device-side loop: its while condition
  int in_loop;
};

// Copy c of a row: its source plane, row offset, first column offset (from i0), number of
// elements and the end of the allocation it lies in.
template <typename T, int KIND>
__device__ __forceinline__ void copy_desc(const BicgArgs<T> &a, long long nc, int c, const T *&base,
                                          int &dj, int &di, int &n, const T *&lim) {
  constexpr int NW = KindShape<KIND>::nw, NO = KindShape<KIND>::no;
  if (c < NW) {
    base = a.w[c]; dj = 1; di = -1; n = SX + 2; lim = a.w[c] + nc;
  } else if (c < NW + NO) {
    base = a.o[c - NW]; dj = 0; di = 0; n = SX; lim = a.o[c - NW] + nc;
  } else {
    const int k = c - NW - NO;     // eta, fxx, fxy, fyy(j), fyy(j+1), fyx(j), fyx(j+1)
    const int plane = k == 0 ? 0 : (k <= 2 ? k : (k <= 4 ? 3 : 4));
    base = a.m + plane * nc;
    dj = (k == 4 || k == 6) ? 1 : 0;
    di = 0;
    n = (k == 1 || k == 2) ? SX + 1 : SX;
    lim = a.m + NPL * nc;
  }
}

// Block layout: SX consumer threads (one interior column each) and one producer warp
// (threads SX .. SX+31) that stages the row groups.  Stage st has a `full` barrier (the
// producer's expect_tx arrival plus the bytes of its copies) and an `empty` barrier (one
// arrival per consumer warp when it has read the group), so neither side waits at a block
// barrier inside the row loop: a consumer warp waits only for its group's bytes, the
// producer only for the stage it refills.  Every wait is bounded; a wait that runs out
// sets the shared fault flag, the others stop at their next wait, and the producer lets
// the copies it issued land before the block leaves.
constexpr int kConsumerWarps = SX / 32;
constexpr int kBlock = SX + 32;

template <typename T, int KIND>
__global__ void __launch_bounds__(kBlock) bicg_kernel(const __grid_constant__ KParams p,
                                                     const __grid_constant__ BicgArgs<T> a) {
  constexpr int NW = KindShape<KIND>::nw, NO = KindShape<KIND>::no;
  constexpr int NCP = n_copies<KIND>();
  constexpr int NS = stages<T>(), RS = rows<T>();
  extern __shared__ __align__(128) unsigned char smem[];
  T *buf = reinterpret_cast<T *>(smem);
  unsigned long long *full =
      reinterpret_cast<unsigned long long *>(smem + (size_t)NS * RS * NCP * SLOT * sizeof(T));
  unsigned long long *empty = full + NS;
  static_assert(RS * NCP <= 32, "one lane of the producer warp per staged copy");
  __shared__ int off[NS][RS][NCP];
  __shared__ volatile int s_fault;

  const int t = threadIdx.x;
  const bool producer = t >= SX;
  const int cb = blockIdx.x % a.ncb, rb = blockIdx.x / a.ncb;
  const int i0 = p.m0 + cb * SX, i = i0 + t;
  const bool active = !producer && i < p.m0 + p.nx;
  const int ja = p.m1 + (int)((long long)p.ny * rb / a.nrb);
  const int jb = p.m1 + (int)((long long)p.ny * (rb + 1) / a.nrb);
  const int nrows = jb - ja;
  const int ngroups = (nrows + RS - 1) / RS;
  const long long ix = p.ix, nc = p.nc;

  if (t == 0) {
    for (int st = 0; st < NS; ++st) {
      mbar_init(smem_addr(&full[st]), 1u);
      mbar_init(smem_addr(&empty[st]), (uint32_t)kConsumerWarps);
    }
    s_fault = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  // Launched as a programmatic dependent of the solve's previous kernel: everything above
  // reads only the arguments; the vectors and scalars that kernel wrote are read after it
  // has completed.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  Scal *sc = a.sc;
  if (KIND == K3 && a.in_loop && blockIdx.x == 0 && t == 0) {
    // the loop ends once the solve has stopped (converged, out of iterations or faulted);
    // the count of k3 launches bounds it whatever the scalars say
    const unsigned int b = ++sc->body;
    if (sc->done || sc->fault || b > (unsigned int)sc->hc_max + 8u) cudaGraphSetConditional(a.loop, 0u);
  }
  if (sc->done || sc->fault) return;
  const int wait_limit = sc->wait_limit;
  __syncthreads();

  double acc0 = 0.0, acc1 = 0.0;
  if (producer) {
    // lane rr*NCP + c owns copy c of row rr of a group: its source address at row ja + rr,
    // the length and the allocation end; the first element of that copy inside its staged
    // segment goes to off[stage][rr][c] for the consumers
    const int lane = t - SX;
    const int lrow = lane / NCP, lcopy = lane % NCP;
    uintptr_t c_addr = 0, c_cap = 0;
    uint32_t c_len = 0;
    if (lane < RS * NCP) {
      const T *base, *lim;
      int dj, di, n;
      copy_desc<T, KIND>(a, nc, lcopy, base, dj, di, n, lim);
      c_addr = (uintptr_t)(base + ((long long)(ja + lrow + dj) * ix + i0 + di));
      c_len = (uint32_t)(n * sizeof(T));
      c_cap = (uintptr_t)lim & ~(uintptr_t)15;
    }
    const uintptr_t row_bytes = (uintptr_t)ix * sizeof(T);
    int issued = 0;
    for (int g = 0; g < ngroups; ++g) {
      const int st = g % NS;
      if (g >= NS) {
        // the consumers' reads of group g - NS free the stage
        const bool ok = mbar_wait(smem_addr(&empty[st]), (uint32_t)((g / NS - 1) & 1), wait_limit);
        if (!ok || s_fault) {
          if (!ok) s_fault = 1;
          break;
        }
      }
      uintptr_t a0 = 0;
      uint32_t bytes = 0;
      if (lane < RS * NCP && g * RS + lrow < nrows) {
        const uintptr_t ad = c_addr + (uintptr_t)(g * RS) * row_bytes;
        a0 = ad & ~(uintptr_t)15;
        uintptr_t end = (ad + c_len + 15) & ~(uintptr_t)15;
        if (end > c_cap) end = c_cap;
        bytes = (uint32_t)(end - a0);
        off[st][lrow][lcopy] = (int)((ad - a0) / sizeof(T));
      }
      uint32_t total = bytes;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      const uint32_t fb = smem_addr(&full[st]);
      __syncwarp();                               // every lane's off[st] before the arrival
      if (lane == 0) mbar_expect_tx(fb, total);   // releases off[st] to the consumers
      __syncwarp();
      if (bytes)
        bulk_load(smem_addr(buf + ((size_t)(st * RS + lrow) * NCP + lcopy) * SLOT),
                  (const void *)a0, bytes, fb);
      issued = g + 1;
    }
    // let every copy in flight land before the block can leave (the consumers have waited
    // for all of them on the normal path; after a fault some were never waited for)
    if (lane == 0)
      for (int g = issued - NS > 0 ? issued - NS : 0; g < issued; ++g)
        mbar_wait(smem_addr(&full[g % NS]), (uint32_t)((g / NS) & 1), kWaitLimit);
    __syncwarp();
  } else {
    // scalars of the update formed at each point
    T s1 = T(0), s2 = T(0);
    bool first = false;
    if (KIND == K1) {
      first = sc->count == 0;
      s1 = (T)sc->beta;
      s2 = (T)sc->omega;
    } else if (KIND == K2) {
      s1 = (T)sc->alpha;
    } else if (KIND == K3) {
      s1 = (T)sc->alpha;
      s2 = (T)sc->omega;
    }
    auto form = [&](const T (&v)[3]) -> T {
      if (KIND == KINIT) return v[0];
      if (KIND == K1) return first ? v[0] : v[2] + s1 * (v[0] - s2 * v[1]);
      if (KIND == K2) return v[0] - s1 * v[1];
      return v[0] + s1 * v[1] + s2 * v[2];
    };

    T w[3][3];
    RowFactors<T> f;
    if (active && nrows > 0) {
#pragma unroll
      for (int dr = 0; dr < 2; ++dr)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const long long k = (long long)(ja - 1 + dr) * ix + i - 1 + d;
          T v[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) v[c] = c < NW ? a.w[c][k] : T(0);
          w[dr][d] = form(v);
        }
      f.cxl = a.g[i];
      f.cxr = a.g[ix + i];
      f.idx = a.g[2 * ix + i];
    }
    const T *gy = a.g + 3 * ix;
    const int lane = t & 31;
    for (int g = 0; g < ngroups; ++g) {
      const int st = g % NS;
      bool ok = false;
      for (int k = 0; k < wait_limit && !ok; ++k) {
        ok = mbar_try_wait(smem_addr(&full[st]), (uint32_t)((g / NS) & 1));
        if (!ok && s_fault) break;
      }
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) s_fault = 1;
        break;
      }
#pragma unroll
      for (int rr = 0; rr < RS; ++rr) {
        const int r = g * RS + rr, j = ja + r;
        if (r >= nrows) break;
        const T *sb = buf + (size_t)(st * RS + rr) * NCP * SLOT;
        const int *of = off[st][rr];
        if (active) {
          const long long q = (long long)j * ix + i;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            T v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = c < NW ? sb[c * SLOT + of[c] + t + d] : T(0);
            w[2][d] = form(v);
          }
          T own[2];
#pragma unroll
          for (int c = 0; c < 2; ++c)
            own[c] = c < NO ? sb[(NW + c) * SLOT + of[NW + c] + t] : T(0);
          constexpr int mc = NW + NO;
          f.eta = sb[mc * SLOT + of[mc] + t];
          f.fxxl = sb[(mc + 1) * SLOT + of[mc + 1] + t];
          f.fxxr = sb[(mc + 1) * SLOT + of[mc + 1] + t + 1];
          f.fxyl = sb[(mc + 2) * SLOT + of[mc + 2] + t];
          f.fxyr = sb[(mc + 2) * SLOT + of[mc + 2] + t + 1];
          f.fyyd = sb[(mc + 3) * SLOT + of[mc + 3] + t];
          f.fyyu = sb[(mc + 4) * SLOT + of[mc + 4] + t];
          f.fyxd = sb[(mc + 5) * SLOT + of[mc + 5] + t];
          f.fyxu = sb[(mc + 6) * SLOT + of[mc + 6] + t];
          f.cyd = gy[j];
          f.cyu = gy[p.jx + j];
          f.idy = gy[2 * p.jx + j];
          T c[9];
          entries(p, f, i, j, c);
          if (KIND == KINIT) {
            // r = b - A x term by term, as the reference's initial residual
            const T bq = own[0];
            T v = bq;
            v = v - c[0] * w[1][1];
            v = v - c[1] * w[1][0];
            v = v - c[2] * w[1][2];
            v = v - c[3] * w[0][1];
            v = v - c[4] * w[2][1];
            v = v - c[5] * w[0][0];
            v = v - c[6] * w[0][2];
            v = v - c[7] * w[2][0];
            v = v - c[8] * w[2][2];
            a.out[0][q] = v;
            a.out[1][q] = v;
            a.out[2][q] = v;
            acc0 += (double)v * (double)v;
            acc1 += (double)bq * (double)bq;
          } else if (KIND == K1) {
            a.out[0][q] = w[1][1];
            const T av = stencil(c, w);
            a.out[1][q] = av;
            const double r0q = (double)own[1];
            acc0 += (double)own[0] * r0q;
            acc1 += r0q * (double)av;
          } else if (KIND == K2) {
            a.out[0][q] = w[1][1];
            const T at = stencil(c, w);
            acc0 += (double)w[1][1] * (double)at;
            acc1 += (double)at * (double)at;
          } else {
            a.out[0][q] = w[1][1];
            const T v = own[0] - stencil(c, w);
            a.out[1][q] = v;
            acc0 += (double)own[1] * (double)v;
            acc1 += (double)v * (double)v;
          }
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            w[0][d] = w[1][d];
            w[1][d] = w[2][d];
          }
        }
      }
      __syncwarp();                // the warp's reads of stage st are done
      if (lane == 0) mbar_arrive(smem_addr(&empty[st]));
    }
  }
  // the next kernel of the solve may start its launch (it waits for this one to complete
  // before it reads anything this one writes)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  __syncthreads();
  if (s_fault) {
    // a staged group never arrived (or its stage was never freed): flag it and leave the
    // scalars alone (the host reads the flag and stops; later kernels return at once)
    if (t == 0) atomicExch(&sc->fault, 1);
    return;
  }
  double tot[2];
  if (reduce2<kBlock, SX>(acc0, acc1, a.part, &sc->blocks_done, tot)) {
    if (KIND == KINIT) {
      sc->rr = tot[0];
      sc->bb = tot[1];
      sc->count = 0;
      sc->relres = tot[1] > 0.0 ? sqrt(tot[0] / tot[1]) : 0.0;
      sc->done = !(sc->relres > sc->tol && sc->count <= sc->hc_max);
    } else if (KIND == K1) {
      sc->alphau = tot[0];
      sc->alphad = tot[1];
      sc->alpha = tot[0] / tot[1];
    } else if (KIND == K2) {
      sc->omegau = tot[0];
      sc->omegad = tot[1];
      sc->omega = tot[0] / tot[1];
    } else {
      sc->betau = tot[0];
      sc->rr = tot[1];
      sc->beta = tot[0] / sc->alphau * sc->alpha / sc->omega;
      sc->count = sc->count + 1;
      sc->relres = sqrt(tot[1] / sc->bb);
      sc->done = !(sc->relres > sc->tol && sc->count <= sc->hc_max);
      if (a.in_loop && sc->done) cudaGraphSetConditional(a.loop, 0u);
    }
  }
}

// pr = (te*ro)/gm and the ion energy of pv2cq_mhd on the interior cells (the ghost cells
// are filled afterwards).
__global__ void writeback_kernel(const KParams p, double *U, const double *__restrict__ te,
                                 const double *__restrict__ kin, const double *__restrict__ mag) {
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long q = (long long)j * p.ix + i;
  const double ro = U[q];
  const double pr = (te[q] * ro) / p.gm;
  U[q + 4 * p.nc] = pr / (p.gm - 1.0) + kin[q] + mag[q];
}

__global__ void cast_kernel(const KParams p, const double *__restrict__ a, float *b) {
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long q = (long long)j * p.ix + i;
  b[q] = (float)a[q];
}

__global__ void correct_kernel(const KParams p, double *x, const float *__restrict__ d) {
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long q = (long long)j * p.ix + i;
  x[q] = x[q] + (double)d[q];
}

__global__ void set_scal_kernel(Scal *sc, double tol, int hc_max, int wait_limit) {
  sc->tol = tol;
  sc->hc_max = hc_max;
  sc->wait_limit = wait_limit;
  sc->done = 0;
  sc->fault = 0;
  sc->count = 0;
  sc->blocks_done = 0u;
  sc->body = 0u;
}

// One wave of BiCGstab blocks: ncb column blocks x nrb row ranges.
struct Grid {
  int ncb = 1, nrb = 1, nb = 1;
};

template <typename T, int KIND>
cudaError_t kind_blocks(int *bps) {
  const size_t smem = stage_smem<T, KIND>();
  cudaError_t err = cudaFuncSetAttribute(bicg_kernel<T, KIND>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int n = 0;
  if (err == cudaSuccess)
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bicg_kernel<T, KIND>, kBlock, smem);
  if (err == cudaSuccess) *bps = std::min(*bps, std::max(n, 1));
  return err;
}

// The grid of the four kernels of precision T: as many row ranges per column block as fill
// every SM at the occupancy of the most demanding kernel.
template <typename T>
cudaError_t make_grid(const KParams &k, int sms, Grid *g) {
  int bps = 1 << 20;
  cudaError_t err = kind_blocks<T, KINIT>(&bps);
  if (err == cudaSuccess) err = kind_blocks<T, K1>(&bps);
  if (err == cudaSuccess) err = kind_blocks<T, K2>(&bps);
  if (err == cudaSuccess) err = kind_blocks<T, K3>(&bps);
  if (err != cudaSuccess) return err;
  g->ncb = (k.nx + SX - 1) / SX;
  g->nrb = std::max(1, std::min(k.ny, sms * bps / g->ncb));
  g->nb = g->ncb * g->nrb;
  return cudaSuccess;
}

template <typename T, int KIND>
void launch(const Grid &g, const KParams &k, BicgArgs<T> a, cudaStream_t s) {
  a.ncb = g.ncb;
  a.nrb = g.nrb;
  // programmatic dependent launch: the kernel's set-up overlaps the previous kernel's tail
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)g.nb, 1, 1);
  cfg.blockDim = dim3(kBlock, 1, 1);
  cfg.dynamicSmemBytes = stage_smem<T, KIND>();
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, bicg_kernel<T, KIND>, k, a);
}

template <typename T>
BicgArgs<T> make_args(const T *m, const T *g, std::initializer_list<const T *> w,
                      std::initializer_list<const T *> o, std::initializer_list<T *> out,
                      double *part, Scal *sc) {
  BicgArgs<T> a{};
  a.m = m;
  a.g = g;
  int n = 0;
  for (const T *v : w) a.w[n++] = v;
  n = 0;
  for (const T *v : o) a.o[n++] = v;
  n = 0;
  for (T *v : out) a.out[n++] = v;
  a.part = part;
  a.sc = sc;
  return a;
}

}  // namespace hc

struct HcEngine {
  long long nc = 0;
  hc::Grid grid64, grid32;          // BiCGstab grids of the FP64 and FP32 kernels
  bool mixed = false;
  double *m64 = nullptr, *g64 = nullptr, *b = nullptr, *kin = nullptr, *mag = nullptr;
  double *x[2] = {nullptr, nullptr}, *p[2] = {nullptr, nullptr}, *ap[2] = {nullptr, nullptr};
  double *r = nullptr, *r0 = nullptr, *t = nullptr;
  float *m32 = nullptr, *g32 = nullptr, *b32 = nullptr, *r32 = nullptr, *r032 = nullptr,
        *t32 = nullptr;
  float *x32[2] = {nullptr, nullptr}, *p32[2] = {nullptr, nullptr}, *ap32[2] = {nullptr, nullptr};
  double *part = nullptr;
  hc::Scal *sc = nullptr, *sc32 = nullptr;
  hc::Scal *h_sc = nullptr;         // pinned
  int wait_limit = hc::kWaitLimit;  // polls of a staging mbarrier (hc_set_wait_limit)
  // distributed solve (hcd_*): per-block partial sums on the device and their pinned copy
  double *dpart = nullptr, *h_dpart = nullptr;
  int dnb = 0;
  // the BiCGstab iterations as a device-side loop (a conditional while node over two
  // iterations, k3 ending it), FP64 [0] and FP32 [1]; built at the first solve; a device
  // that cannot build it runs the host-checked groups instead
  cudaGraphExec_t loop[2] = {nullptr, nullptr};
  bool no_loop[2] = {false, false};
  bool host_groups = false;         // hc_set_loop(e, 0): the host-checked groups regardless
};

void hc_set_wait_limit(HcEngine *e, int polls) {
  if (e) e->wait_limit = polls < 0 ? hc::kWaitLimit : polls;
}

void hc_set_loop(HcEngine *e, int device_loop) {
  if (e) e->host_groups = device_loop == 0;
}

void hc_destroy(HcEngine *e) {
  if (!e) return;
  void *bufs[] = {e->m64, e->g64, e->b, e->kin, e->mag, e->x[0], e->x[1], e->p[0], e->p[1],
                  e->ap[0], e->ap[1], e->r, e->r0, e->t, e->m32, e->g32, e->b32, e->r32,
                  e->r032, e->t32, e->x32[0], e->x32[1], e->p32[0], e->p32[1], e->ap32[0],
                  e->ap32[1], e->part, e->sc, e->sc32};
  for (void *b : bufs)
    if (b) cudaFree(b);
  for (cudaGraphExec_t g : e->loop)
    if (g) cudaGraphExecDestroy(g);
  if (e->dpart) cudaFree(e->dpart);
  if (e->h_dpart) cudaFreeHost(e->h_dpart);
  if (e->h_sc) cudaFreeHost(e->h_sc);
  delete e;
}

cudaError_t hc_create(const KParams &k, bool mixed, HcEngine **out) {
  *out = nullptr;
  // the staged row segments reach up to two ghost rows past the interior
  if (k.m0 < 2 || k.m1 < 2) return cudaErrorInvalidValue;
  HcEngine *e = new (std::nothrow) HcEngine();
  if (!e) return cudaErrorMemoryAllocation;
  e->nc = k.nc;
  e->mixed = mixed;
  int dev = 0, sms = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err == cudaSuccess) err = hc::make_grid<double>(k, sms, &e->grid64);
  if (err == cudaSuccess && mixed) err = hc::make_grid<float>(k, sms, &e->grid32);
  if (err != cudaSuccess) {
    delete e;
    return err;
  }
  const size_t dv = sizeof(double) * (size_t)k.nc, fv = sizeof(float) * (size_t)k.nc;
  const size_t ng = 3 * ((size_t)k.ix + (size_t)k.jx);
  auto md = [&](double **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes);
    if (err == cudaSuccess) err = cudaMemset(*p, 0, bytes);
  };
  auto mf = [&](float **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes);
    if (err == cudaSuccess) err = cudaMemset(*p, 0, bytes);
  };
  md(&e->m64, hc::NPL * dv);
  md(&e->g64, sizeof(double) * ng);
  md(&e->b, dv); md(&e->kin, dv); md(&e->mag, dv);
  for (int h = 0; h < 2; ++h) {
    md(&e->x[h], dv); md(&e->p[h], dv); md(&e->ap[h], dv);
  }
  md(&e->r, dv); md(&e->r0, dv); md(&e->t, dv);
  if (mixed) {
    mf(&e->m32, hc::NPL * fv);
    mf(&e->g32, sizeof(float) * ng);
    mf(&e->b32, fv); mf(&e->r32, fv); mf(&e->r032, fv); mf(&e->t32, fv);
    for (int h = 0; h < 2; ++h) {
      mf(&e->x32[h], fv); mf(&e->p32[h], fv); mf(&e->ap32[h], fv);
    }
  }
  md(&e->part, sizeof(double) * 2 * (size_t)std::max(e->grid64.nb, e->grid32.nb));
  if (err == cudaSuccess) err = cudaMalloc(&e->sc, sizeof(hc::Scal));
  if (err == cudaSuccess) err = cudaMemset(e->sc, 0, sizeof(hc::Scal));
  if (err == cudaSuccess) err = cudaMalloc(&e->sc32, sizeof(hc::Scal));
  if (err == cudaSuccess) err = cudaMemset(e->sc32, 0, sizeof(hc::Scal));
  if (err == cudaSuccess) err = cudaMallocHost(&e->h_sc, sizeof(hc::Scal));
  if (err != cudaSuccess) {
    hc_destroy(e);
    return err;
  }
  *out = e;
  return cudaSuccess;
}

namespace {

// Two BiCGstab iterations (the double-buffered vectors' two parities) into the body of a
// conditional while node; k3 of the loop ends it (sets the condition to 0) once the solve has
// stopped.  The arguments (the engine's buffers and scalars) are fixed, so the loop graph is
// built once per precision.
template <typename T>
cudaError_t build_loop(const hc::Grid &gr, const KParams &k, const T *m, const T *g,
                       T *const (&x)[2], const T *b, T *r, T *r0, T *const (&pv)[2],
                       T *const (&ap)[2], T *tv, double *part, hc::Scal *sc, cudaStream_t s,
                       cudaGraphExec_t *out) {
  using namespace hc;
  cudaGraph_t graph = nullptr;
  cudaError_t err = cudaGraphCreate(&graph, 0);
  if (err != cudaSuccess) return err;
  cudaGraphConditionalHandle cond;
  err = cudaGraphConditionalHandleCreate(&cond, graph, 1u, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (err == cudaSuccess) err = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
  if (err == cudaSuccess)
    err = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) {
    cudaGraphDestroy(graph);
    return err;
  }
  for (int a = 0; a < 2; ++a) {
    const int z = a ^ 1;
    launch<T, K1>(gr, k, make_args<T>(m, g, {pv[a], ap[a], r}, {r, r0}, {pv[z], ap[z]}, part, sc), s);
    launch<T, K2>(gr, k, make_args<T>(m, g, {r, ap[z]}, {}, {tv}, part, sc), s);
    BicgArgs<T> a3 = make_args<T>(m, g, {x[a], pv[z], tv}, {b, r0}, {x[z], r}, part, sc);
    a3.loop = cond;
    a3.in_loop = 1;
    launch<T, K3>(gr, k, a3, s);
  }
  cudaGraph_t captured = nullptr;
  err = cudaStreamEndCapture(s, &captured);
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  return err;
}

// BiCGstab on the interior cells from x[0] until the stop flag of sc is set: the iterations
// run as the device-side loop (one host wait per solve), or, where that loop cannot be built,
// in groups after which the host reads the flag.  On return h holds the scalars; the iterate
// is in x[h->count & 1].
template <typename T>
cudaError_t bicgstab(HcEngine *e, const hc::Grid &gr, const KParams &k, const T *m, const T *g,
                     T *const (&x)[2], const T *b, T *r, T *r0, T *const (&pv)[2],
                     T *const (&ap)[2], T *tv, hc::Scal *sc, double tol, int hc_max,
                     cudaStream_t s, hc::Scal *h) {
  using namespace hc;
  set_scal_kernel<<<1, 1, 0, s>>>(sc, tol, hc_max, e->wait_limit);
  launch<T, KINIT>(gr, k, make_args<T>(m, g, {x[0]}, {b}, {r, r0, pv[0]}, e->part, sc), s);
  const int li = sizeof(T) == 8 ? 0 : 1;
  if (!e->host_groups && !e->loop[li] && !e->no_loop[li]) {
    if (build_loop<T>(gr, k, m, g, x, b, r, r0, pv, ap, tv, e->part, sc, s, &e->loop[li]) !=
        cudaSuccess) {
      cudaGetLastError();           // (a failed build leaves no error behind)
      e->loop[li] = nullptr;
      e->no_loop[li] = true;
    }
  }
  if (!e->host_groups && e->loop[li]) {
    cudaError_t err = cudaGraphLaunch(e->loop[li], s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(h, sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return err;
    if (h->fault) return cudaErrorLaunchTimeout;
    return cudaSuccess;
  }
  const int group = 4;
  for (int it = 0; it <= hc_max; it += group) {
    for (int u = 0; u < group; ++u) {
      const int a = (it + u) & 1, z = a ^ 1;
      launch<T, K1>(gr, k, make_args<T>(m, g, {pv[a], ap[a], r}, {r, r0}, {pv[z], ap[z]}, e->part, sc), s);
      launch<T, K2>(gr, k, make_args<T>(m, g, {r, ap[z]}, {}, {tv}, e->part, sc), s);
      launch<T, K3>(gr, k, make_args<T>(m, g, {x[a], pv[z], tv}, {b, r0}, {x[z], r}, e->part, sc), s);
    }
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    err = cudaMemcpyAsync(h, sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return err;
    if (h->fault) return cudaErrorLaunchTimeout;
    if (h->done) break;
  }
  return cudaSuccess;
}

// The FP64 residual r = b - A x[0] (r0 = p = r as well) and its scalars into h.
cudaError_t residual64(HcEngine *e, const KParams &k, double tol, cudaStream_t s, hc::Scal *h) {
  using namespace hc;
  set_scal_kernel<<<1, 1, 0, s>>>(e->sc, tol, 0, e->wait_limit);
  launch<double, KINIT>(e->grid64, k,
                        make_args<double>(e->m64, e->g64, {e->x[0]}, {e->b}, {e->r, e->r0, e->p[0]},
                                          e->part, e->sc),
                        s);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaMemcpyAsync(h, e->sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err == cudaSuccess && h->fault) err = cudaErrorLaunchTimeout;
  return err;
}

}  // namespace

cudaError_t hc_run(HcEngine *e, const KParams &k, double *U, const double *dtp, double tol,
                   int hc_max, cudaStream_t s, int *iters, double *relres, int *status) {
  using namespace hc;
  const long long nc = k.nc;
  const int gu = (int)std::min<long long>((nc + 255) / 256, 148 * 8);
  const int gi = (int)(((long long)k.nx * k.ny + NT - 1) / NT);
  const int gf = (int)(((long long)(k.nx + 1) * (k.ny + 1) + NT - 1) / NT);
  setup_kernel<<<gu, 256, 0, s>>>(k, U, e->x[0], e->b, e->kin, e->mag);
  matrix_kernel<<<gf, NT, 0, s>>>(k, U, e->x[0], dtp, e->m64, e->mixed ? e->m32 : nullptr);
  geometry_kernel<<<(k.ix + k.jx + NT - 1) / NT, NT, 0, s>>>(k, e->g64, e->mixed ? e->g32 : nullptr);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  int total = 0;
  Scal *h = e->h_sc;
  const double *xf = e->x[0];
  if (!e->mixed) {
    err = bicgstab<double>(e, e->grid64, k, e->m64, e->g64, e->x, e->b, e->r, e->r0, e->p, e->ap,
                           e->t, e->sc, tol, hc_max, s, h);
    if (err != cudaSuccess) return err;
    total = h->count;
    xf = e->x[h->count & 1];
  } else {
    // iterative refinement: FP64 residual of the FP64 matrix, FP32 BiCGstab on the
    // correction, FP64 update of x[0]; at most hc_max inner iterations in total.  A loose
    // inner tolerance: each refinement restarts BiCGstab where it converges fastest, while
    // a tight FP32 solve stagnates near FP32 precision (KH 2048x1024, kapper 0.01, first 60
    // steps: 21.6 inner iterations per step at 3e-3, 23.4 at 1e-3, 35.5 at 1e-4, 29 at
    // 1e-6, 23 at 1e-2; over 1000 steps 18.4 at 3e-3 against 19.3 at 1e-4).
#ifndef PIP_HC_INNER_TOL
#define PIP_HC_INNER_TOL 3.0e-3
#endif
    const double inner_tol = PIP_HC_INNER_TOL;
    bool fp64_scalars = false;      // h holds the FP64 residual of the current x[0]
    for (int outer = 0; outer < 32; ++outer) {
      err = residual64(e, k, tol, s, h);
      if (err != cudaSuccess) return err;
      fp64_scalars = true;
      if (!(h->relres > tol) || total > hc_max) break;
      cast_kernel<<<gi, NT, 0, s>>>(k, e->r, e->b32);
      err = cudaMemsetAsync(e->x32[0], 0, sizeof(float) * (size_t)nc, s);
      if (err != cudaSuccess) return err;
      err = bicgstab<float>(e, e->grid32, k, e->m32, e->g32, e->x32, e->b32, e->r32, e->r032,
                            e->p32, e->ap32, e->t32, e->sc32, inner_tol,
                            std::max(1, hc_max - total), s, h);
      if (err != cudaSuccess) return err;
      fp64_scalars = false;
      total += h->count;
      correct_kernel<<<gi, NT, 0, s>>>(k, e->x[0], e->x32[h->count & 1]);
    }
    if (!fp64_scalars) {
      // the FP64 residual of the final iterate
      err = residual64(e, k, tol, s, h);
      if (err != cudaSuccess) return err;
    }
  }
  writeback_kernel<<<gi, NT, 0, s>>>(k, U, xf, e->kin, e->mag);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  if (iters) *iters = total;
  if (relres) *relres = h->relres;
  if (status) *status = h->relres <= tol ? 0 : 5;  // PIP_ERR_ITER
  return cudaSuccess;
}


// ---------------------------------------------------------------- distributed BiCGstab
//
// BiCGstabMPI (HC_rot.f90:303-466, hc_split = 2) for a block whose y faces may border other
// ranks, as phases between which the caller reduces two scalars over the ranks (SUM) and
// exchanges one halo row of a vector.  The matrix is the single-rank one (face factors and
// entries(), folded only on faces without a neighbour), so the ranks together hold the rows
// of the undecomposed matrix bit for bit.  Per iteration:
//   phase 1  Ap = A p                 sums (r, r0), (r0, Ap)   -> alpha; exchange Ap
//   phase 2  t = r - alpha Ap; At     sums (t, At), (At, At)   -> omega
//   phase 3  x = x + alpha p + omega t
//   phase 4  r = b - A x              sums (r0, r), (r, r)     -> beta, residual; exchange r
//   phase 5  p = r + beta (p - omega Ap)
// t, x and p are formed on every cell, so their halo rows follow from the exchanged r and Ap
// rows (and from x's and p's own consistent halo rows): only Ap and r cross between ranks,
// one row each way, as the reference's mpiBND of apk and residual (its mpiBND of te is
// implied here).  The reference takes omega from the rank's own sums (HC_rot.f90:425-427),
// which makes its iterates depend on the decomposition; here every scalar is the global one,
// so the ranks iterate as the single domain does (the sums group differently: rounding).
// Sums: per-block partials in a fixed cell order, added on the host in block order.
namespace hcd {

using namespace pip::hc;
constexpr int NT = 256;

__device__ __forceinline__ RowFactors<double> factors(const KParams &p, const double *__restrict__ m,
                                                      const double *__restrict__ g, int i, int j) {
  const long long nc = p.nc, ix = p.ix, q = (long long)j * ix + i;
  RowFactors<double> f;
  f.eta = m[q];
  f.fxxl = m[nc + q];
  f.fxxr = m[nc + q + 1];
  f.fxyl = m[2 * nc + q];
  f.fxyr = m[2 * nc + q + 1];
  f.fyyd = m[3 * nc + q];
  f.fyyu = m[3 * nc + q + ix];
  f.fyxd = m[4 * nc + q];
  f.fyxu = m[4 * nc + q + ix];
  f.cxl = g[i];
  f.cxr = g[ix + i];
  f.idx = g[2 * ix + i];
  const double *gy = g + 3 * ix;
  f.cyd = gy[j];
  f.cyu = gy[p.jx + j];
  f.idy = gy[2 * p.jx + j];
  return f;
}

__device__ __forceinline__ void window(const KParams &p, const double *__restrict__ v, long long q,
                                       double (&w)[3][3]) {
#pragma unroll
  for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
    for (int di = -1; di <= 1; ++di) w[dj + 1][di + 1] = v[q + dj * (long long)p.ix + di];
}

// Block sums of two values into part[2*block + k] (tree order fixed by the block size).
__device__ __forceinline__ void block_sums(double a0, double a1, double *part) {
  __shared__ double s2[2][NT];
  s2[0][threadIdx.x] = a0;
  s2[1][threadIdx.x] = a1;
  __syncthreads();
  for (int h = NT / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      s2[0][threadIdx.x] += s2[0][threadIdx.x + h];
      s2[1][threadIdx.x] += s2[1][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s2[0][0];
    part[2 * blockIdx.x + 1] = s2[1][0];
  }
}

// Interior-cell kernels: 0 r = b - A x term by term, r0 = p = r, sums (r,r), (b,b);
// 1 Ap = A p, sums (r,r0), (r0,Ap); 2 At = A t, sums (t,At), (At,At); 4 r = b - A x, sums
// (r0,r), (r,r).
template <int KIND>
__global__ void __launch_bounds__(NT) spmv_kernel(const KParams p, const double *__restrict__ m,
                                                  const double *__restrict__ g, const double *__restrict__ v,
                                                  const double *__restrict__ b, double *r,
                                                  double *r0, double *out, double *part) {
  int i, j;
  const long long t = blockIdx.x * (long long)NT + threadIdx.x;
  double a0 = 0.0, a1 = 0.0;
  if (interior_cell(p, t, i, j)) {
    const long long q = (long long)j * p.ix + i;
    double w[3][3], c[9];
    window(p, v, q, w);
    entries(p, factors(p, m, g, i, j), i, j, c);
    if (KIND == 0) {
      const double bq = b[q];
      double x = bq;
      x = x - c[0] * w[1][1];
      x = x - c[1] * w[1][0];
      x = x - c[2] * w[1][2];
      x = x - c[3] * w[0][1];
      x = x - c[4] * w[2][1];
      x = x - c[5] * w[0][0];
      x = x - c[6] * w[0][2];
      x = x - c[7] * w[2][0];
      x = x - c[8] * w[2][2];
      r[q] = x;
      r0[q] = x;
      out[q] = x;
      a0 = x * x;
      a1 = bq * bq;
    } else if (KIND == 1) {
      const double av = stencil(c, w);
      out[q] = av;
      a0 = r[q] * r0[q];
      a1 = r0[q] * av;
    } else if (KIND == 2) {
      const double at = stencil(c, w);
      a0 = w[1][1] * at;
      a1 = at * at;
    } else {
      const double x = b[q] - stencil(c, w);
      r[q] = x;
      a0 = r0[q] * x;
      a1 = x * x;
    }
  }
  block_sums(a0, a1, part);
}

// Every-cell updates: 0 p = r; 2 t = r - c0 Ap; 3 x = x + c0 p + c1 t; 5 p = r + c0 (p - c1 Ap).
template <int KIND>
__global__ void __launch_bounds__(NT) axpy_kernel(long long nc, double c0, double c1, const double *r,
                                                  const double *ap, double *t, double *x, double *pv) {
  for (long long q = blockIdx.x * (long long)NT + threadIdx.x; q < nc; q += (long long)gridDim.x * NT) {
    if (KIND == 0) pv[q] = r[q];
    else if (KIND == 2) t[q] = r[q] - c0 * ap[q];
    else if (KIND == 3) x[q] = x[q] + c0 * pv[q] + c1 * t[q];
    else pv[q] = r[q] + c0 * (pv[q] - c1 * ap[q]);
  }
}

}  // namespace hcd

namespace {

// Per-block partials of the last spmv_kernel, summed in block order on the host.
cudaError_t hcd_sums(HcEngine *e, cudaStream_t s, double sums[2]) {
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->h_dpart, e->dpart, sizeof(double) * 2 * e->dnb, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return err;
  double a0 = 0.0, a1 = 0.0;
  for (int k = 0; k < e->dnb; ++k) {
    a0 += e->h_dpart[2 * k];
    a1 += e->h_dpart[2 * k + 1];
  }
  sums[0] = a0;
  sums[1] = a1;
  return cudaSuccess;
}

}  // namespace

cudaError_t hcd_begin(HcEngine *e, const KParams &k, double *U, const double *dtp, cudaStream_t s,
                      double sums[2]) {
  using namespace hc;
  const long long nc = k.nc;
  const int nb = (int)(((long long)k.nx * k.ny + hcd::NT - 1) / hcd::NT);
  if (nb > e->dnb) {
    if (e->dpart) cudaFree(e->dpart);
    if (e->h_dpart) cudaFreeHost(e->h_dpart);
    e->dpart = nullptr;
    e->h_dpart = nullptr;
    e->dnb = 0;
    cudaError_t err = cudaMalloc(&e->dpart, sizeof(double) * 2 * nb);
    if (err == cudaSuccess) err = cudaMallocHost(&e->h_dpart, sizeof(double) * 2 * nb);
    if (err != cudaSuccess) return err;
    e->dnb = nb;
  }
  e->dnb = nb;
  const int gu = (int)std::min<long long>((nc + 255) / 256, 148 * 8);
  const int gf = (int)(((long long)(k.nx + 1) * (k.ny + 1) + NT - 1) / NT);
  // every cell, ghost rows included: the halo rows hold the neighbours' state after the
  // stage's exchange, so te, b and the face factors next to an exchanged face are the
  // undecomposed ones
  setup_kernel<<<gu, 256, 0, s>>>(k, U, e->x[0], e->b, e->kin, e->mag);
  matrix_kernel<<<gf, NT, 0, s>>>(k, U, e->x[0], dtp, e->m64, nullptr);
  geometry_kernel<<<(k.ix + k.jx + NT - 1) / NT, NT, 0, s>>>(k, e->g64, nullptr);
  cudaError_t err = cudaMemsetAsync(e->ap[0], 0, sizeof(double) * (size_t)nc, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->t, 0, sizeof(double) * (size_t)nc, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->r, 0, sizeof(double) * (size_t)nc, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->p[0], 0, sizeof(double) * (size_t)nc, s);
  if (err != cudaSuccess) return err;
  hcd::spmv_kernel<0><<<nb, hcd::NT, 0, s>>>(k, e->m64, e->g64, e->x[0], e->b, e->r, e->r0, e->p[0],
                                             e->dpart);
  return hcd_sums(e, s, sums);
}

cudaError_t hcd_phase(HcEngine *e, const KParams &k, int phase, const double coef[2], cudaStream_t s,
                      double sums[2]) {
  const long long nc = k.nc;
  const int nb = e->dnb;
  const int ga = (int)std::min<long long>((nc + hcd::NT - 1) / hcd::NT, 148 * 8);
  const double c0 = coef ? coef[0] : 0.0, c1 = coef ? coef[1] : 0.0;
  switch (phase) {
    case 0:
      hcd::axpy_kernel<0><<<ga, hcd::NT, 0, s>>>(nc, 0.0, 0.0, e->r, nullptr, nullptr, nullptr, e->p[0]);
      return cudaGetLastError();
    case 1:
      hcd::spmv_kernel<1><<<nb, hcd::NT, 0, s>>>(k, e->m64, e->g64, e->p[0], nullptr, e->r, e->r0,
                                                 e->ap[0], e->dpart);
      return hcd_sums(e, s, sums);
    case 2:
      hcd::axpy_kernel<2><<<ga, hcd::NT, 0, s>>>(nc, c0, 0.0, e->r, e->ap[0], e->t, nullptr, nullptr);
      hcd::spmv_kernel<2><<<nb, hcd::NT, 0, s>>>(k, e->m64, e->g64, e->t, nullptr, nullptr, nullptr,
                                                 nullptr, e->dpart);
      return hcd_sums(e, s, sums);
    case 3:
      hcd::axpy_kernel<3><<<ga, hcd::NT, 0, s>>>(nc, c0, c1, nullptr, nullptr, e->t, e->x[0], e->p[0]);
      return cudaGetLastError();
    case 4:
      hcd::spmv_kernel<4><<<nb, hcd::NT, 0, s>>>(k, e->m64, e->g64, e->x[0], e->b, e->r, e->r0,
                                                 nullptr, e->dpart);
      return hcd_sums(e, s, sums);
    case 5:
      hcd::axpy_kernel<5><<<ga, hcd::NT, 0, s>>>(nc, c0, c1, e->r, e->ap[0], nullptr, nullptr, e->p[0]);
      return cudaGetLastError();
    default:
      return cudaErrorInvalidValue;
  }
}

double *hcd_vector(HcEngine *e, int vec) {
  return vec == 0 ? e->x[0] : vec == 1 ? e->r : vec == 2 ? e->ap[0] : nullptr;
}

cudaError_t hcd_end(HcEngine *e, const KParams &k, double *U, cudaStream_t s) {
  const int gi = (int)(((long long)k.nx * k.ny + hc::NT - 1) / hc::NT);
  hc::writeback_kernel<<<gi, hc::NT, 0, s>>>(k, U, e->x[0], e->kin, e->mag);
  return cudaGetLastError();
}

}  // namespace pip
