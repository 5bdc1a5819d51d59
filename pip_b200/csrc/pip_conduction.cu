// pip_conduction.cu -- implicit anisotropic conduction of the ion species (HC(U_m,nvar_m,1),
// HC_rot.f90:67-140) on the device: cq2pv rewrite and temperature, the 9-point matrix of
// set_matrix_source_MHD2D9 (HC_rot.f90:643-739) with set_matrix_boundary's folding
// (:468-529), BiCGstab (:187-299, hc_split = 2) and the conversion back (pv2cq_mhd,
// Scheme_rot.f90:43-79).
//
// BiCGstab keeps the reference's structure (the residual is recomputed from the iterate
// every iteration, so the stopping test sees the true residual).  One iteration is five
// kernels over the interior cells:
//   k0  p  = r + beta (p - omega Ap)                      (from the second iteration)
//   k1  Ap = A p;             sums (r,r0), (r0,Ap)   -> alpha
//   k2  t  = r - alpha Ap;    At = A t (t at the neighbours formed on the fly);
//                             sums (t,At), (At,At)   -> omega
//   k3  x  = x + alpha p + omega t
//   k4  r  = b - A x;         sums (r0,r), (r,r)     -> beta, relative residual, stop flag
// Scalars are reduced by the last block of each kernel to finish (fixed order:
// deterministic) into a device block; every kernel returns at once when the stop flag is
// set, so the host launches iterations in groups and reads the flag between groups.
// Vectors and matrix are templated: FP64 for the plain path; FP32 for the inner solve of
// the mixed path, whose FP64 outer loop (iterative refinement) recomputes the residual in
// FP64 and corrects x in FP64 until the FP64 relative residual reaches the target.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "pip_kernels.cuh"
#include "pip_physics.cuh"

namespace pip {
namespace hc {

constexpr int NT = 256;
constexpr double kEpsi = 1.0e-5;   // HC_rot.f90:17

struct Scal {
  double rr, bb;                  // sum r^2, sum b^2
  double alphau, alphad, alpha;
  double omegau, omegad, omega;
  double betau, beta;
  double relres, tol;
  int count, hc_max, done, pad;
  unsigned int blocks_done;
};

__device__ __forceinline__ bool interior_cell(const KParams &p, long long t, int &i, int &j) {
  const long long n = (long long)p.nx * p.ny;
  if (t >= n) return false;
  i = p.m0 + (int)(t % p.nx);
  j = p.m1 + (int)(t / p.nx);
  return true;
}

// matrix(i,j,:) . v over the stencil (0: (i,j), 1: i-1, 2: i+1, 3: j-1, 4: j+1, 5: (i-1,j-1),
// 6: (i+1,j-1), 7: (i-1,j+1), 8: (i+1,j+1)), summed left to right.
template <typename T>
__device__ __forceinline__ double apply9(const T *__restrict__ m, const T *__restrict__ v,
                                         long long q, long long nc, long long ix) {
  return (double)m[q] * (double)v[q] + (double)m[q + nc] * (double)v[q - 1] +
         (double)m[q + 2 * nc] * (double)v[q + 1] + (double)m[q + 3 * nc] * (double)v[q - ix] +
         (double)m[q + 4 * nc] * (double)v[q + ix] + (double)m[q + 5 * nc] * (double)v[q - 1 - ix] +
         (double)m[q + 6 * nc] * (double)v[q + 1 - ix] + (double)m[q + 7 * nc] * (double)v[q - 1 + ix] +
         (double)m[q + 8 * nc] * (double)v[q + 1 + ix];
}

// Block sums of up to 2 values into part[k*nb + block]; returns true in thread 0 of the last
// block to finish, which then holds the totals (summed in block order) in tot[].
__device__ bool reduce2(double a, double b, double *part, unsigned int *counter, double (&tot)[2]) {
  __shared__ double s[2][NT / 32];
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
    for (int k = 0; k < NT / 32; ++k) {
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
  // the last block: totals in block order (each thread a strided slice, then warp order)
  __threadfence();
  double x = 0.0, y = 0.0;
  for (unsigned int k = threadIdx.x; k < nb; k += NT) {
    x += part[k];
    y += part[nb + k];
  }
  __shared__ double s2[2][NT];
  s2[0][threadIdx.x] = x;
  s2[1][threadIdx.x] = y;
  __syncthreads();
  for (int h = NT / 2; h > 0; h >>= 1) {
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

// set_matrix_source_MHD2D9 for the interior cells (dxc = dx, dyc = dy) and
// set_matrix_boundary on all four sides (one rank per direction: every neighbour is -1,
// MPI_rot.f90:123), folded per cell in the order x-, x+, y-, y+.  Writes the FP64 matrix
// and, when m32 is given, its FP32 copy.
__global__ void matrix_kernel(const KParams p, const double *__restrict__ U, const double *__restrict__ te,
                              const double *dtp, double *m64, float *m32) {
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long nc = p.nc, ix = p.ix;
  const long long q = (long long)j * ix + i;
  const double *ro = U, *bx = U + 5 * nc, *by = U + 6 * nc, *bz = U + 7 * nc;
  const double gm = p.gm, dt = *dtp;
  const double eta = p.hc_kapper * dt * (gm - 1.0) / ro[q] * gm;
  const double bxl = (bx[q - 1] + bx[q]) / 2.0, bxr = (bx[q + 1] + bx[q]) / 2.0;
  const double bxd = (bx[q - ix] + bx[q]) / 2.0, bxu = (bx[q + ix] + bx[q]) / 2.0;
  const double byl = (by[q - 1] + by[q]) / 2.0, byr = (by[q + 1] + by[q]) / 2.0;
  const double byd = (by[q - ix] + by[q]) / 2.0, byu = (by[q + ix] + by[q]) / 2.0;
  const double bzl = (bz[q - 1] + bz[q]) / 2.0, bzr = (bz[q + 1] + bz[q]) / 2.0;
  const double bzd = (bz[q - ix] + bz[q]) / 2.0, bzu = (bz[q + ix] + bz[q]) / 2.0;
  const double al = fmax(sqrt(bxl * bxl + byl * byl + bzl * bzl), kEpsi);
  const double ar = fmax(sqrt(bxr * bxr + byr * byr + bzr * bzr), kEpsi);
  const double ad = fmax(sqrt(bxd * bxd + byd * byd + bzd * bzd), kEpsi);
  const double au = fmax(sqrt(bxu * bxu + byu * byu + bzu * bzu), kEpsi);
  const double nxl = bxl / al, nxr = bxr / ar, nxd = bxd / ad, nxu = bxu / au;
  const double nyl = byl / al, nyr = byr / ar, nyd = byd / ad, nyu = byu / au;
  const double te_xm = 0.5 * (te[q] + te[q - 1]), te_xp = 0.5 * (te[q] + te[q + 1]);
  const double te_ym = 0.5 * (te[q] + te[q - ix]), te_yp = 0.5 * (te[q] + te[q + ix]);
  const double te_xm25 = te_xm * te_xm * sqrt(te_xm), te_xp25 = te_xp * te_xp * sqrt(te_xp);
  const double te_ym25 = te_ym * te_ym * sqrt(te_ym), te_yp25 = te_yp * te_yp * sqrt(te_yp);
  const double dxc = p.dx[i], dyc = p.dy[j];
  const double bxxl = -(eta * te_xm25 * nxl * nxl / dxc / p.dx[i - 1]);
  const double bxxr = -(eta * te_xp25 * nxr * nxr / dxc / p.dx[i]);
  const double byyd = -(eta * te_ym25 * nyd * nyd / dyc / p.dy[j - 1]);
  const double byyu = -(eta * te_yp25 * nyu * nyu / dyc / p.dy[j]);
  const double bxyl = -(eta / 4.0 / dxc / dyc * nxl * nyl * te_xm25);
  const double bxyr = -(eta / 4.0 / dxc / dyc * nxr * nyr * te_xp25);
  const double byxd = -(eta / 4.0 / dxc / dyc * nyd * nxd * te_ym25);
  const double byxu = -(eta / 4.0 / dxc / dyc * nyu * nxu * te_yp25);
  double m[9];
  m[1] = bxxl - (byxu - byxd);
  m[2] = bxxr + (byxu - byxd);
  m[3] = byyd - (bxyr - bxyl);
  m[4] = byyu + (bxyr - bxyl);
  m[5] = bxyl + byxd;
  m[6] = -(bxyr + byxd);
  m[7] = -(bxyl + byxu);
  m[8] = bxyr + byxu;
  m[0] = 1.0 - (m[1] + m[2] + m[3] + m[4]);
  if (i == p.m0) {                 // x-minus
    m[0] = m[1] + m[0]; m[1] = 0.0;
    m[3] = m[3] + m[5]; m[5] = 0.0;
    m[4] = m[4] + m[7]; m[7] = 0.0;
  }
  if (i == p.m0 + p.nx - 1) {      // x-plus
    m[0] = m[2] + m[0]; m[2] = 0.0;
    m[3] = m[3] + m[6]; m[6] = 0.0;
    m[4] = m[4] + m[8]; m[8] = 0.0;
  }
  if (j == p.m1) {                 // y-minus
    m[0] = m[3] + m[0]; m[3] = 0.0;
    m[1] = m[5] + m[1]; m[5] = 0.0;
    m[2] = m[6] + m[2]; m[6] = 0.0;
  }
  if (j == p.m1 + p.ny - 1) {      // y-plus
    m[0] = m[4] + m[0]; m[4] = 0.0;
    m[1] = m[1] + m[7]; m[7] = 0.0;
    m[2] = m[2] + m[8]; m[8] = 0.0;
  }
#pragma unroll
  for (int n = 0; n < 9; ++n) m64[q + n * nc] = m[n];
  if (m32) {
#pragma unroll
    for (int n = 0; n < 9; ++n) m32[q + n * nc] = (float)m[n];
  }
}

// r = b - A x (term by term, as the reference's initial residual), r0 = r, p = r;
// totals (r,r), (b,b); the stop test of the loop head.
template <typename T>
__global__ void __launch_bounds__(NT) init_kernel(const KParams p, const T *__restrict__ m,
                                                   const T *__restrict__ x, const T *__restrict__ b,
                                                   T *r, T *r0, T *pv, double *part, Scal *sc) {
  int i, j;
  double rr = 0.0, bb = 0.0;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (interior_cell(p, t, i, j)) {
    const long long nc = p.nc, ix = p.ix;
    const long long q = (long long)j * ix + i;
    double v = (double)b[q];
    v = v - (double)m[q] * (double)x[q];
    v = v - (double)m[q + nc] * (double)x[q - 1];
    v = v - (double)m[q + 2 * nc] * (double)x[q + 1];
    v = v - (double)m[q + 3 * nc] * (double)x[q - ix];
    v = v - (double)m[q + 4 * nc] * (double)x[q + ix];
    v = v - (double)m[q + 5 * nc] * (double)x[q - 1 - ix];
    v = v - (double)m[q + 6 * nc] * (double)x[q + 1 - ix];
    v = v - (double)m[q + 7 * nc] * (double)x[q - 1 + ix];
    v = v - (double)m[q + 8 * nc] * (double)x[q + 1 + ix];
    const T vt = (T)v;
    r[q] = vt;
    r0[q] = vt;
    pv[q] = vt;
    rr = (double)vt * (double)vt;
    bb = (double)b[q] * (double)b[q];
  }
  double tot[2];
  if (reduce2(rr, bb, part, &sc->blocks_done, tot)) {
    sc->rr = tot[0];
    sc->bb = tot[1];
    sc->count = 0;
    sc->relres = tot[1] > 0.0 ? sqrt(tot[0] / tot[1]) : 0.0;
    sc->done = !(sc->relres > sc->tol && sc->count <= sc->hc_max);
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k0_kernel(const KParams p, const T *__restrict__ r, T *pv,
                                                 const T *__restrict__ ap, const Scal *sc) {
  if (sc->done || sc->count == 0) return;
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long q = (long long)j * p.ix + i;
  const double beta = sc->beta, omega = sc->omega;
  pv[q] = (T)((double)r[q] + beta * ((double)pv[q] - omega * (double)ap[q]));
}

template <typename T>
__global__ void __launch_bounds__(NT) k1_kernel(const KParams p, const T *__restrict__ m,
                                                 const T *__restrict__ pv, const T *__restrict__ r,
                                                 const T *__restrict__ r0, T *ap, double *part, Scal *sc) {
  if (sc->done) return;
  int i, j;
  double au = 0.0, ad = 0.0;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (interior_cell(p, t, i, j)) {
    const long long q = (long long)j * p.ix + i;
    const T a = (T)apply9(m, pv, q, p.nc, p.ix);
    ap[q] = a;
    au = (double)r[q] * (double)r0[q];
    ad = (double)r0[q] * (double)a;
  }
  double tot[2];
  if (reduce2(au, ad, part, &sc->blocks_done, tot)) {
    sc->alphau = tot[0];
    sc->alphad = tot[1];
    sc->alpha = tot[0] / tot[1];
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k2_kernel(const KParams p, const T *__restrict__ m,
                                                 const T *__restrict__ r, const T *__restrict__ ap,
                                                 T *tv, double *part, Scal *sc) {
  if (sc->done) return;
  int i, j;
  double ou = 0.0, od = 0.0;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (interior_cell(p, t, i, j)) {
    const long long nc = p.nc, ix = p.ix;
    const long long q = (long long)j * ix + i;
    const double alpha = sc->alpha;
    // t = r - alpha Ap at the cell and its neighbours (outside the interior the matrix
    // entries are zero and Ap, r are zero)
    auto tt = [&](long long k) { return (T)((double)r[k] - alpha * (double)ap[k]); };
    const T t0 = tt(q);
    tv[q] = t0;
    const double at = (double)m[q] * (double)t0 + (double)m[q + nc] * (double)tt(q - 1) +
                      (double)m[q + 2 * nc] * (double)tt(q + 1) + (double)m[q + 3 * nc] * (double)tt(q - ix) +
                      (double)m[q + 4 * nc] * (double)tt(q + ix) +
                      (double)m[q + 5 * nc] * (double)tt(q - 1 - ix) +
                      (double)m[q + 6 * nc] * (double)tt(q + 1 - ix) +
                      (double)m[q + 7 * nc] * (double)tt(q - 1 + ix) +
                      (double)m[q + 8 * nc] * (double)tt(q + 1 + ix);
    const double atr = (double)(T)at;
    ou = (double)t0 * atr;
    od = atr * atr;
  }
  double tot[2];
  if (reduce2(ou, od, part, &sc->blocks_done, tot)) {
    sc->omegau = tot[0];
    sc->omegad = tot[1];
    sc->omega = tot[0] / tot[1];
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k3_kernel(const KParams p, T *x, const T *__restrict__ pv,
                                                 const T *__restrict__ tv, const Scal *sc) {
  if (sc->done) return;
  int i, j;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (!interior_cell(p, t, i, j)) return;
  const long long q = (long long)j * p.ix + i;
  x[q] = (T)((double)x[q] + sc->alpha * (double)pv[q] + sc->omega * (double)tv[q]);
}

template <typename T>
__global__ void __launch_bounds__(NT) k4_kernel(const KParams p, const T *__restrict__ m,
                                                 const T *__restrict__ x, const T *__restrict__ b,
                                                 const T *__restrict__ r0, T *r, double *part, Scal *sc) {
  if (sc->done) return;
  int i, j;
  double bu = 0.0, rr = 0.0;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (interior_cell(p, t, i, j)) {
    const long long q = (long long)j * p.ix + i;
    const T v = (T)((double)b[q] - apply9(m, x, q, p.nc, p.ix));
    r[q] = v;
    bu = (double)r0[q] * (double)v;
    rr = (double)v * (double)v;
  }
  double tot[2];
  if (reduce2(bu, rr, part, &sc->blocks_done, tot)) {
    sc->betau = tot[0];
    sc->rr = tot[1];
    sc->beta = tot[0] / sc->alphau * sc->alpha / sc->omega;
    sc->count = sc->count + 1;
    sc->relres = sqrt(tot[1] / sc->bb);
    sc->done = !(sc->relres > sc->tol && sc->count <= sc->hc_max);
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

__global__ void set_scal_kernel(Scal *sc, double tol, int hc_max) {
  sc->tol = tol;
  sc->hc_max = hc_max;
  sc->done = 0;
  sc->count = 0;
  sc->blocks_done = 0u;
}

}  // namespace hc

struct HcEngine {
  long long nc = 0;
  int nb = 0;                       // blocks over the interior
  bool mixed = false;
  double *m64 = nullptr, *te = nullptr, *b = nullptr, *kin = nullptr, *mag = nullptr;
  double *r = nullptr, *r0 = nullptr, *p = nullptr, *ap = nullptr, *t = nullptr;
  float *m32 = nullptr, *d = nullptr, *b32 = nullptr, *r32 = nullptr, *r032 = nullptr,
        *p32 = nullptr, *ap32 = nullptr, *t32 = nullptr;
  double *part = nullptr;
  hc::Scal *sc = nullptr, *sc32 = nullptr;
  hc::Scal *h_sc = nullptr;         // pinned
};

void hc_destroy(HcEngine *e) {
  if (!e) return;
  void *bufs[] = {e->m64, e->te, e->b, e->kin, e->mag, e->r, e->r0, e->p, e->ap, e->t,
                  e->m32, e->d, e->b32, e->r32, e->r032, e->p32, e->ap32, e->t32,
                  e->part, e->sc, e->sc32};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (e->h_sc) cudaFreeHost(e->h_sc);
  delete e;
}

cudaError_t hc_create(const KParams &k, bool mixed, HcEngine **out) {
  *out = nullptr;
  HcEngine *e = new (std::nothrow) HcEngine();
  if (!e) return cudaErrorMemoryAllocation;
  e->nc = k.nc;
  e->mixed = mixed;
  const long long n = (long long)k.nx * k.ny;
  e->nb = (int)((n + hc::NT - 1) / hc::NT);
  const size_t dv = sizeof(double) * (size_t)k.nc, fv = sizeof(float) * (size_t)k.nc;
  cudaError_t err = cudaSuccess;
  auto md = [&](double **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes);
    if (err == cudaSuccess) err = cudaMemset(*p, 0, bytes);
  };
  auto mf = [&](float **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes);
    if (err == cudaSuccess) err = cudaMemset(*p, 0, bytes);
  };
  md(&e->m64, 9 * dv);
  md(&e->te, dv); md(&e->b, dv); md(&e->kin, dv); md(&e->mag, dv);
  md(&e->r, dv); md(&e->r0, dv); md(&e->p, dv); md(&e->ap, dv); md(&e->t, dv);
  if (mixed) {
    mf(&e->m32, 9 * fv);
    mf(&e->d, fv); mf(&e->b32, fv); mf(&e->r32, fv); mf(&e->r032, fv);
    mf(&e->p32, fv); mf(&e->ap32, fv); mf(&e->t32, fv);
  }
  md(&e->part, sizeof(double) * 2 * (size_t)e->nb);
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

// BiCGstab on the interior cells until the stop flag of sc is set; the host reads the flag
// every `group` iterations.  Returns the scalars block (count, relres) in *h.
template <typename T>
cudaError_t bicgstab(HcEngine *e, const KParams &k, const T *m, T *x, const T *b, T *r, T *r0, T *pv,
                     T *ap, T *tv, hc::Scal *sc, double tol, int hc_max, cudaStream_t s,
                     hc::Scal *h) {
  using namespace hc;
  const int nb = e->nb;
  set_scal_kernel<<<1, 1, 0, s>>>(sc, tol, hc_max);
  init_kernel<T><<<nb, NT, 0, s>>>(k, m, x, b, r, r0, pv, e->part, sc);
  const int group = 4;
  for (int it = 0; it <= hc_max; it += group) {
    for (int g = 0; g < group; ++g) {
      k0_kernel<T><<<nb, NT, 0, s>>>(k, r, pv, ap, sc);
      k1_kernel<T><<<nb, NT, 0, s>>>(k, m, pv, r, r0, ap, e->part, sc);
      k2_kernel<T><<<nb, NT, 0, s>>>(k, m, r, ap, tv, e->part, sc);
      k3_kernel<T><<<nb, NT, 0, s>>>(k, x, pv, tv, sc);
      k4_kernel<T><<<nb, NT, 0, s>>>(k, m, x, b, r0, r, e->part, sc);
    }
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    err = cudaMemcpyAsync(h, sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return err;
    if (h->done) break;
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t hc_run(HcEngine *e, const KParams &k, double *U, const double *dtp, double tol,
                   int hc_max, cudaStream_t s, int *iters, double *relres, int *status) {
  using namespace hc;
  const long long nc = k.nc;
  const int gu = (int)std::min<long long>((nc + 255) / 256, 148 * 8);
  setup_kernel<<<gu, 256, 0, s>>>(k, U, e->te, e->b, e->kin, e->mag);
  matrix_kernel<<<e->nb, NT, 0, s>>>(k, U, e->te, dtp, e->m64, e->mixed ? e->m32 : nullptr);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  int total = 0;
  Scal *h = e->h_sc;
  if (!e->mixed) {
    err = bicgstab<double>(e, k, e->m64, e->te, e->b, e->r, e->r0, e->p, e->ap, e->t, e->sc, tol,
                           hc_max, s, h);
    if (err != cudaSuccess) return err;
    total = h->count;
  } else {
    // iterative refinement: FP64 residual of the FP64 matrix, FP32 BiCGstab on the
    // correction, FP64 update; at most hc_max inner iterations in total
    const double inner_tol = 1.0e-4;
    for (int outer = 0; outer < 32; ++outer) {
      set_scal_kernel<<<1, 1, 0, s>>>(e->sc, tol, 0);
      init_kernel<double><<<e->nb, NT, 0, s>>>(k, e->m64, e->te, e->b, e->r, e->r0, e->p, e->part,
                                               e->sc);
      err = cudaMemcpyAsync(h, e->sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      if (err != cudaSuccess) return err;
      if (!(h->relres > tol) || total > hc_max) break;
      cast_kernel<<<e->nb, NT, 0, s>>>(k, e->r, e->b32);
      cudaMemsetAsync(e->d, 0, sizeof(float) * (size_t)nc, s);
      err = bicgstab<float>(e, k, e->m32, e->d, e->b32, e->r32, e->r032, e->p32, e->ap32, e->t32,
                            e->sc32, inner_tol, std::max(1, hc_max - total), s, h);
      if (err != cudaSuccess) return err;
      total += h->count;
      correct_kernel<<<e->nb, NT, 0, s>>>(k, e->te, e->d);
    }
    // the FP64 residual of the final iterate
    set_scal_kernel<<<1, 1, 0, s>>>(e->sc, tol, 0);
    init_kernel<double><<<e->nb, NT, 0, s>>>(k, e->m64, e->te, e->b, e->r, e->r0, e->p, e->part,
                                             e->sc);
    err = cudaMemcpyAsync(h, e->sc, sizeof(Scal), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return err;
  }
  writeback_kernel<<<e->nb, NT, 0, s>>>(k, U, e->te, e->kin, e->mag);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  if (iters) *iters = total;
  if (relres) *relres = h->relres;
  if (status) *status = h->relres <= tol ? 0 : 5;  // PIP_ERR_ITER
  return cudaSuccess;
}

}  // namespace pip
