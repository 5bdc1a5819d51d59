// pip_adjoint.cu -- discrete adjoint of the FP64 two-fluid step (include/pip_adjoint.h).
//
// Forward model of one step n (the kernels of pip_run, main.f90:31-68, Solver_rot.f90:42-81):
//   dt_n = CFL(z_n)                             (cfl, Scheme_rot.f90:183-213)
//   U1   = z_n + dt_n/2 * G(z_n)                (stage 1)
//   U2   = z_n + dt_n   * G(U1)                 (stage 2)
//   z_n+1 = fill(rewrite(U2))                   (PIPbnd, cq2pv rewrites of the two cfl calls)
// with G(U) = -div F(MUSCL-minmod(u2v(U))) + S(cq2pv(U)) on interior cells and fill() the
// ghost copy of Boundary_rot.f90.  The reverse sweep of a step, for a cotangent La of z_n+1:
//   fold(La)                                    ghost cotangents -> their interior sources
//   Lb   = (dt_n G'(U1))^T La                   reverse stage 2 (faces, then cells)
//   fold(Lb)
//   La   = La + Lb + (dt_n/2 G'(z_n))^T Lb      reverse stage 1, in place
//   La  += (dL/ddt_n) dCFL/dz_n, dL/dalpha_c   finalize_kernel
// where dL/ddt_n = (<La, G(U1)> + <Lb, G(z_n)>/2) is accumulated by the two stage kernels
// from face fluxes and cell sources, and the CFL derivative is taken at the cell (or the
// collision bound) that set dt_n.  States z_n, U1 of a segment of K steps are recomputed
// from the segment's checkpoint with the recorded dt (bitwise the forward trajectory).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/pip_adjoint.h"
#include "../../include/pip_gpu.h"
#include "pip_adjoint_physics.cuh"
#include "pip_kernels.cuh"

namespace pip {
namespace adjk {

constexpr int NVM = 8, NV = 13;

// Thread-block sizes of the reverse-stage kernels and their minimum resident blocks per SM
// (register budget: 65536 / (threads * blocks) per thread).
#ifndef PIP_ADJ_FACE_MINB
#define PIP_ADJ_FACE_MINB 2
#endif
#ifndef PIP_ADJ_FACEH_MINB
#define PIP_ADJ_FACEH_MINB 2
#endif
#ifndef PIP_ADJ_CELL_MINB
#define PIP_ADJ_CELL_MINB 2
#endif
constexpr int kFaceThreads = 128;   // one face per thread (ion faces)
constexpr int kFaceThreadsH = 256;  // one face per thread (neutral faces)
constexpr int kCellThreads = 256;

// Per-block CFL candidates of stage 1 (the state z_n).
struct CandPart {
  double cmin;
  long long cidx;
  double rmax;
  long long ridx;
  int ckind;  // 0 ions, 1 neutrals
  int rsp;    // species of rmax: 0 ions, 1 neutrals
};

__device__ __forceinline__ bool interior(const KParams &p, int i, int j) {
  return i >= p.m0 && i < p.m0 + p.nx && (p.ndim == 1 || (j >= p.m1 && j < p.m1 + p.ny));
}

// direction 2 swaps (vx, vy) and (bx, by) (set_HLLD_fluxes, HLL_rot.f90:365-383)
__device__ __forceinline__ int perm_m(int n) {
  return n == 1 ? 2 : n == 2 ? 1 : n == 5 ? 6 : n == 6 ? 5 : n;
}
__device__ __forceinline__ int perm_h(int n) { return n == 1 ? 2 : n == 2 ? 1 : n; }

// minmod derivative of the slope at cell 1 of (v0, v1, v2) with respect to v_q
__device__ __forceinline__ double dmm(int mode, int q) {
  if (mode == 1) return q == 1 ? -1.0 : (q == 2 ? 1.0 : 0.0);
  if (mode == 2) return q == 0 ? -1.0 : (q == 1 ? 1.0 : 0.0);
  return 0.0;
}

// Reverse of one face for the ions (SP = 0: HLLD) or the neutrals (SP = 1: HLLC): MUSCL-minmod
// face states from the primitives in shared memory
// (cells a - s, a, a + s, a + 2s along the face normal), the density floors and the
// Riemann solvers.  lamF: cotangent of the face flux (natural variable order).  Writes the
// cotangents of the two face states (gL, gR, natural order, after the floors), the minmod
// branches and returns <F, lamF>.
template <int SP>
__device__ __forceinline__ double face_vjp(const KParams &p, const double *__restrict__ V,
                                           long long a, long long s, bool ydir,
                                           const double (&lamF)[NV], double *gL, double *gR,
                                           long long nf, long long f, unsigned long long &modes) {
  const long long RR = p.nc;  // plane stride of the primitives
  double fdot = 0.0;
  modes = 0ull;
  if (SP == 0) {
    double vl[8], vr[8], af[8], avl[8], avr[8], flx[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const int src = ydir ? perm_m(n) : n;
      const double *v = V + src * RR + a;
      const double v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
      const int mL = adj::minmod_mode(v0, v1, v2), mR = adj::minmod_mode(v1, v2, v3);
      modes |= (unsigned long long)(mL | (mR << 2)) << (4 * src);
      vl[n] = v1 + 0.5 * minmod<double>(v0, v1, v2);
      vr[n] = v2 - 0.5 * minmod<double>(v1, v2, v3);
      af[n] = lamF[src];
      avl[n] = 0.0;
      avr[n] = 0.0;
    }
    const bool fl0 = vl[0] < p.ro_lim, fr0 = vr[0] < p.ro_lim;
    vl[0] = fmax(vl[0], p.ro_lim);
    vr[0] = fmax(vr[0], p.ro_lim);
    adj::hlld_vjp(vl, vr, af, p.gm, p.igm1, avl, avr, flx);
    if (fl0) avl[0] = 0.0;
    if (fr0) avr[0] = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const int src = ydir ? perm_m(n) : n;
      fdot += flx[n] * af[n];
      gL[src * nf + f] = avl[n];
      gR[src * nf + f] = avr[n];
    }
  } else {
    double vl[5], vr[5], af[5], avl[5], avr[5], flx[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int src = ydir ? perm_h(n) : n;
      const double *v = V + (NVM + src) * RR + a;
      const double v0 = v[-s], v1 = v[0], v2 = v[s], v3 = v[2 * s];
      const int mL = adj::minmod_mode(v0, v1, v2), mR = adj::minmod_mode(v1, v2, v3);
      modes |= (unsigned long long)(mL | (mR << 2)) << (4 * (NVM + src));
      vl[n] = v1 + 0.5 * minmod<double>(v0, v1, v2);
      vr[n] = v2 - 0.5 * minmod<double>(v1, v2, v3);
      af[n] = lamF[NVM + src];
      avl[n] = 0.0;
      avr[n] = 0.0;
    }
    const bool fl0 = vl[0] < p.ro_lim, fr0 = vr[0] < p.ro_lim;
    vl[0] = fmax(vl[0], p.ro_lim);
    vr[0] = fmax(vr[0], p.ro_lim);
    adj::hllc_vjp(vl, vr, af, p.gm, p.igm1, avl, avr, flx);
    if (fl0) avl[0] = 0.0;
    if (fr0) avr[0] = 0.0;
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int src = ydir ? perm_h(n) : n;
      fdot += flx[n] * af[n];
      gL[(NVM + src) * nf + f] = avl[n];
      gR[(NVM + src) * nf + f] = avr[n];
    }
  }
  return fdot;
}

// Adds the contributions of the faces k = c-2 .. c+1 of one direction (face k between
// cells k and k+1; face data at index base + k*df, only faces 0 <= k < kmax exist) to the
// primitive cotangents of cell c.
__device__ __forceinline__ void gather_dir(const double *__restrict__ gL, const double *__restrict__ gR,
                                           const unsigned long long *__restrict__ M, long long nf,
                                           long long base, long long df, int c, int kmax,
                                           double (&av)[NV]) {
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int k = c - 2 + r;
    if (k < 0 || k >= kmax) continue;
    const long long f = base + (long long)k * df;
    const unsigned long long m = M[f];
    if (m == 0ull && r != 1 && r != 2) continue;   // slope terms only: nothing to add
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const int sh = 4 * n;
      const int mL = (int)((m >> sh) & 3ull), mR = (int)((m >> (sh + 2)) & 3ull);
      const double l = gL[n * nf + f], rr = gR[n * nf + f];
      double add;
      if (r == 0)        // cell c is k+2: third cell of the right stencil
        add = -0.5 * rr * dmm(mR, 2);
      else if (r == 1)   // cell c is k+1: right cell
        add = rr + 0.5 * l * dmm(mL, 2) - 0.5 * rr * dmm(mR, 1);
      else if (r == 2)   // cell c is k: left cell
        add = l + 0.5 * l * dmm(mL, 1) - 0.5 * rr * dmm(mR, 0);
      else               // cell c is k-1: first cell of the left stencil
        add = 0.5 * l * dmm(mL, 0);
      av[n] += add;
    }
  }
}

// Primitives of every cell (u2v_mhd / u2v_hd, HLL_rot.f90:1136-1186).
__global__ void u2v_kernel(const KParams p, const double *__restrict__ U, double *__restrict__ V) {
  const long long nc = p.nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    double um[8], uh[5], vm[8], vh[5];
#pragma unroll
    for (int n = 0; n < 8; ++n) um[n] = U[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n) uh[n] = U[q + (NVM + n) * nc];
    u2v_mhd<double, 8>(um, vm, p.gm, p.ro_lim, p.pr_lim);
    u2v_hd<double>(uh, vh, p.gm, p.ro_lim, p.pr_lim);
#pragma unroll
    for (int n = 0; n < 8; ++n) V[q + n * nc] = vm[n];
#pragma unroll
    for (int n = 0; n < 5; ++n) V[q + (NVM + n) * nc] = vh[n];
  }
}

// Reverse of the face fluxes of one RK stage for one species (SP = 0 ions, 1 neutrals): one
// thread per face.  x faces (j, i) lie between cells (j, i) and (j, i+1), y faces (j, i)
// between (j, i) and (j+1, i); a face is stored at the index j*ix + i of its lower cell.
// For faces next to an interior cell: the flux cotangent from the cotangent lam of the
// stage output, the reverse of the MUSCL face states and the Riemann solver (face_vjp),
// written as (gL, gR) on the species' planes and its half of the minmod-branch word (the
// ion planes' branches fill bits 0-31, the neutral planes' bits 32-51); other faces are
// written as zero.  Per block: sum of <F, lamF> over the species' planes (the flux part of
// dt_sub <lam, dU/d(dt_sub)>).  The two species run as separate kernels because the HLLD
// reverse needs every register a thread can have and the HLLC reverse far fewer.
template <int SP, int NT>
__global__ void __launch_bounds__(NT, SP == 0 ? PIP_ADJ_FACE_MINB : PIP_ADJ_FACEH_MINB)
face_vjp_kernel(const KParams p, const double *__restrict__ V, const double *__restrict__ lam,
                const double *dtp, double fac, double *gx, unsigned long long *mx, double *gy,
                unsigned long long *my, double *part_dot, double *part_dac) {
  constexpr int N0 = SP == 0 ? 0 : NVM, N1 = SP == 0 ? NVM : NV;
  __shared__ double s_red[NT / 32];
  const long long nc = p.nc;
  const double dt_sub = fac * (*dtp);
  const long long nfx = (long long)p.jx * (p.ix - 1);
  const long long nfy = p.ndim == 2 ? (long long)(p.jx - 1) * p.ix : 0;
  double dot = 0.0;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < nfx + nfy) {
    const bool ydir = t >= nfx;
    int ia, ja, ib, jb;
    if (!ydir) {
      ja = (int)(t / (p.ix - 1));
      ia = (int)(t % (p.ix - 1));
      ib = ia + 1;
      jb = ja;
    } else {
      const long long u = t - nfx;
      ja = (int)(u / p.ix);
      ia = (int)(u % p.ix);
      ib = ia;
      jb = ja + 1;
    }
    const long long qa = (long long)ja * p.ix + ia, qb = (long long)jb * p.ix + ib;
    double *g = ydir ? gy : gx;
    unsigned int *mh = reinterpret_cast<unsigned int *>(ydir ? my : mx) + 2 * qa + SP;
    const bool in_a = interior(p, ia, ja), in_b = interior(p, ib, jb);
    if (!in_a && !in_b) {
#pragma unroll
      for (int n = N0; n < N1; ++n) {
        g[n * nc + qa] = 0.0;
        g[(NV + n) * nc + qa] = 0.0;
      }
      *mh = 0u;
    } else {
      double ca = 0.0, cb = 0.0;
      if (!ydir) {
        if (in_a) ca = dt_sub / p.dx[ia];
        if (in_b) cb = dt_sub / p.dx[ib];
      } else {
        if (in_a) ca = dt_sub / p.dy[ja];
        if (in_b) cb = dt_sub / p.dy[jb];
      }
      double lamF[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        if (n < N0 || n >= N1) {
          lamF[n] = 0.0;
          continue;
        }
        const double la = in_a ? lam[qa + n * nc] : 0.0;
        const double lb = in_b ? lam[qb + n * nc] : 0.0;
        lamF[n] = -ca * la + cb * lb;
      }
      unsigned long long m;
      dot = face_vjp<SP>(p, V, qa, ydir ? (long long)p.ix : 1ll, ydir, lamF, g, g + NV * nc, nc,
                         qa, m);
      *mh = (unsigned int)(m >> (32 * SP));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
  if (threadIdx.x % 32 == 0) s_red[threadIdx.x / 32] = dot;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sd = 0.0;
    for (int k = 0; k < NT / 32; ++k) sd += s_red[k];
    part_dot[blockIdx.x] = sd;
    part_dac[blockIdx.x] = 0.0;
  }
}

// Reverse of one RK stage per cell (every cell of the ghosted array): the face-state
// cotangents of the faces whose MUSCL stencils reach the cell (face_vjp_kernel's output)
// through minmod, u2v, the explicit collision source (interior cells), the U0 terms
// acc + lam of stage 1 (interior cells, when acc is given), and for stage 1 the CFL
// candidates of the cell (cand).  Per block: dt_sub <lam, S>, dS/dalpha_c . lam.
__global__ void __launch_bounds__(kCellThreads, PIP_ADJ_CELL_MINB)
cell_vjp_kernel(const KParams p, const double *__restrict__ Us, const double *__restrict__ lam,
                const double *acc, double *out, const double *dtp, double fac,
                const double *__restrict__ gx, const unsigned long long *__restrict__ mx,
                const double *__restrict__ gy, const unsigned long long *__restrict__ my,
                double *part_dot, double *part_dac, CandPart *cand) {
  constexpr int NT = kCellThreads;
  __shared__ double s_red[4][NT / 32];
  __shared__ long long s_idx[2][NT / 32];
  __shared__ int s_kind[2][NT / 32];
  const int tid = threadIdx.x;
  const double dt_sub = fac * (*dtp);
  const long long nc = p.nc;
  double dot = 0.0, dac = 0.0;
  double cmin = 1.0e300, rmax = -1.0e300;
  long long cidx = -1, ridx = -1;
  int ckind = 0, rsp = 0;
  const long long q = blockIdx.x * (long long)NT + tid;
  if (q < nc) {
    const int gi = (int)(q % p.ix), gj = (int)(q / p.ix);
    double av[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) av[n] = 0.0;
    gather_dir(gx, gx + NV * nc, mx, nc, (long long)gj * p.ix, 1, gi, p.ix - 1, av);
    if (p.ndim == 2) gather_dir(gy, gy + NV * nc, my, nc, gi, p.ix, gj, p.jx - 1, av);
    double um[8], uh[5];
#pragma unroll
    for (int n = 0; n < 8; ++n) um[n] = Us[q + n * nc];
#pragma unroll
    for (int n = 0; n < 5; ++n) uh[n] = Us[q + (NVM + n) * nc];
    double aum[8] = {0, 0, 0, 0, 0, 0, 0, 0}, auh[5] = {0, 0, 0, 0, 0};
    {
      double avm[8], avh[5];
#pragma unroll
      for (int n = 0; n < 8; ++n) avm[n] = av[n];
#pragma unroll
      for (int n = 0; n < 5; ++n) avh[n] = av[NVM + n];
      adj::u2v_mhd_vjp(um, avm, p.gm, p.ro_lim, p.pr_lim, aum);
      adj::u2v_hd_vjp(uh, avh, p.gm, p.ro_lim, p.pr_lim, auh);
    }
    if (interior(p, gi, gj)) {
      double lm[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) lm[n] = lam[q + n * nc];
      double ads[5];
      ads[0] = 0.0;
#pragma unroll
      for (int k = 1; k < 5; ++k) ads[k] = dt_sub * (lm[k] - lm[NVM + k]);
      const double d = adj::collision_vjp(um, uh, ads, p.gm, p.igm1, p.ac, p.ro_lim, p.pr_lim, aum, auh);
      dac += d;
      dot += p.ac * d;
      if (acc) {
#pragma unroll
        for (int n = 0; n < 8; ++n) aum[n] += acc[q + n * nc] + lm[n];
#pragma unroll
        for (int n = 0; n < 5; ++n) auh[n] += acc[q + (NVM + n) * nc] + lm[NVM + n];
      }
      if (cand) {
        double wm[8], wh[5];
#pragma unroll
        for (int n = 0; n < 8; ++n) wm[n] = um[n];
#pragma unroll
        for (int n = 0; n < 5; ++n) wh[n] = uh[n];
        const Prim<double> qm = cq2pv_mhd_rcp<double, 8>(wm, p.gm, p.igm1, p.ro_lim, p.pr_lim);
        const Prim<double> qh = cq2pv_hd_rcp<double>(wh, p.gm, p.igm1, p.ro_lim, p.pr_lim);
        const double gmin = fmin(fmin(p.dx[gi], p.ndim == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
        const double sg = p.safety * gmin;
        const double cm = cfl_mhd_cell<double>(qm, wm[5], wm[6], wm[7], p.gm, sg);
        const double ch = cfl_hd_cell<double>(qh, p.gm, sg);
        cmin = fmin(cm, ch);
        ckind = cm <= ch ? 0 : 1;
        cidx = q;
        const double rm = um[0] * p.ac, rh = uh[0] * p.ac;
        rmax = fmax(rm, rh);
        rsp = rm >= rh ? 0 : 1;
        ridx = q;
      }
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) out[q + n * nc] = aum[n];
#pragma unroll
    for (int n = 0; n < 5; ++n) out[q + (NVM + n) * nc] = auh[n];
  }

  // block reductions (fixed order: deterministic)
  const int w = tid / 32, l = tid % 32;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dot += __shfl_xor_sync(0xffffffffu, dot, o);
    dac += __shfl_xor_sync(0xffffffffu, dac, o);
    if (cand) {
      const double c2 = __shfl_xor_sync(0xffffffffu, cmin, o);
      const long long i2 = __shfl_xor_sync(0xffffffffu, cidx, o);
      const int k2 = __shfl_xor_sync(0xffffffffu, ckind, o);
      if (c2 < cmin || (c2 == cmin && i2 >= 0 && (cidx < 0 || i2 < cidx))) {
        cmin = c2;
        cidx = i2;
        ckind = k2;
      }
      const double r2 = __shfl_xor_sync(0xffffffffu, rmax, o);
      const long long j2 = __shfl_xor_sync(0xffffffffu, ridx, o);
      const int s2 = __shfl_xor_sync(0xffffffffu, rsp, o);
      if (r2 > rmax || (r2 == rmax && j2 >= 0 && (ridx < 0 || j2 < ridx))) {
        rmax = r2;
        ridx = j2;
        rsp = s2;
      }
    }
  }
  if (l == 0) {
    s_red[0][w] = dot;
    s_red[1][w] = dac;
    s_red[2][w] = cmin;
    s_red[3][w] = rmax;
    s_idx[0][w] = cidx;
    s_idx[1][w] = ridx;
    s_kind[0][w] = ckind;
    s_kind[1][w] = rsp;
  }
  __syncthreads();
  if (tid == 0) {
    double sd = 0.0, sa = 0.0;
    for (int k = 0; k < NT / 32; ++k) {
      sd += s_red[0][k];
      sa += s_red[1][k];
    }
    part_dot[blockIdx.x] = sd;
    part_dac[blockIdx.x] = sa;
    if (cand) {
      CandPart c;
      c.cmin = 1.0e300;
      c.cidx = -1;
      c.ckind = 0;
      c.rmax = -1.0e300;
      c.ridx = -1;
      c.rsp = 0;
      for (int k = 0; k < NT / 32; ++k) {
        const long long i2 = s_idx[0][k];
        if (i2 >= 0 && (s_red[2][k] < c.cmin || (s_red[2][k] == c.cmin && (c.cidx < 0 || i2 < c.cidx)))) {
          c.cmin = s_red[2][k];
          c.cidx = i2;
          c.ckind = s_kind[0][k];
        }
        const long long j2 = s_idx[1][k];
        if (j2 >= 0 && (s_red[3][k] > c.rmax || (s_red[3][k] == c.rmax && (c.ridx < 0 || j2 < c.ridx)))) {
          c.rmax = s_red[3][k];
          c.ridx = j2;
          c.rsp = s_kind[1][k];
        }
      }
      cand[blockIdx.x] = c;
    }
  }
}

// Adjoint of the ghost fill (Boundary_rot.f90:54-125 as done by the stage kernels' ghost
// writes): each interior cell that is the source of ghost copies gathers their cotangents
// (x ghosts, then for each of them its corner ghosts, then y ghosts, with the sign tables
// folded into a per-plane sign mask).  The gather list is built on the host (fold_plan);
// one thread per (cell, plane), plane-major so a warp's loads follow the list.  Ghost
// entries are left as they are; consumers read interior cells only, and no ghost read here
// is a fold target.
__global__ void __launch_bounds__(256) fold_kernel(double *lam, long long nc, const int *cells,
                                                   const int *src, const unsigned short *neg,
                                                   int ncells, int nent) {
  const long long total = (long long)ncells * NV;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(t / ncells), k = (int)(t - (long long)n * ncells);
    double add = 0.0;
    for (int e = 0; e < nent; ++e) {
      const int g = src[(long long)e * ncells + k];
      if (g < 0) break;
      const double v = lam[g + n * nc];
      add += ((neg[(long long)e * ncells + k] >> n) & 1) ? -v : v;
    }
    lam[cells[k] + n * nc] += add;
  }
}

// One block: dL/ddt_n from the stage partials, the CFL bound that set dt_n and its
// gradient (added to lamz at that cell), dL/dalpha_c accumulated into *dcol.
__global__ void __launch_bounds__(256) finalize_kernel(const KParams p, int nb, int ncand,
                                                       const double *p1dot, const double *p1dac,
                                                       const double *p2dot, const double *p2dac,
                                                       const CandPart *cand, const double *dtp,
                                                       const double *z, double *lamz, double *dcol,
                                                       double *ldt_out) {
  __shared__ double s_a[256], s_b[256], s_c[256], s_r[256];
  __shared__ long long s_ci[256], s_ri[256];
  __shared__ int s_ck[256], s_rs[256];
  const int t = threadIdx.x;
  double sd = 0.0, sa = 0.0, cm = 1.0e300, rm = -1.0e300;
  long long ci = -1, ri = -1;
  int ck = 0, rs = 0;
  for (int b = t; b < nb; b += 256) {
    sd += p1dot[b] + p2dot[b];
    sa += p1dac[b] + p2dac[b];
  }
  for (int b = t; b < ncand; b += 256) {
    const CandPart c = cand[b];
    if (c.cidx >= 0 && (c.cmin < cm || (c.cmin == cm && (ci < 0 || c.cidx < ci)))) {
      cm = c.cmin;
      ci = c.cidx;
      ck = c.ckind;
    }
    if (c.ridx >= 0 && (c.rmax > rm || (c.rmax == rm && (ri < 0 || c.ridx < ri)))) {
      rm = c.rmax;
      ri = c.ridx;
      rs = c.rsp;
    }
  }
  s_a[t] = sd;
  s_b[t] = sa;
  s_c[t] = cm;
  s_r[t] = rm;
  s_ci[t] = ci;
  s_ri[t] = ri;
  s_ck[t] = ck;
  s_rs[t] = rs;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h) {
      s_a[t] += s_a[t + h];
      s_b[t] += s_b[t + h];
      const long long i2 = s_ci[t + h];
      if (i2 >= 0 && (s_c[t + h] < s_c[t] || (s_c[t + h] == s_c[t] && (s_ci[t] < 0 || i2 < s_ci[t])))) {
        s_c[t] = s_c[t + h];
        s_ci[t] = i2;
        s_ck[t] = s_ck[t + h];
      }
      const long long j2 = s_ri[t + h];
      if (j2 >= 0 && (s_r[t + h] > s_r[t] || (s_r[t + h] == s_r[t] && (s_ri[t] < 0 || j2 < s_ri[t])))) {
        s_r[t] = s_r[t + h];
        s_ri[t] = j2;
        s_rs[t] = s_rs[t + h];
      }
    }
    __syncthreads();
  }
  if (t != 0) return;
  const double dt = *dtp;
  const double ldt = s_a[0] / dt;
  double dac = s_b[0];
  const double cmin = s_c[0];
  const double dtcol = p.col_lim / s_r[0];
  const long long nc = p.nc;
  if (dtcol < cmin && dtcol < 10.0 && s_ri[0] >= 0) {
    // dt = col_lim / (alpha_c * rho) at the densest cell (cfl_pn_col, Scheme_rot.f90:305-313)
    const long long q = s_ri[0];
    const int plane = s_rs[0] == 0 ? 0 : NVM;
    const double rho = z[q + plane * nc];
    lamz[q + plane * nc] += ldt * (-dtcol / rho);
    dac += ldt * (-dtcol / p.ac);
  } else if (cmin < 10.0 && s_ci[0] >= 0) {
    const long long q = s_ci[0];
    const int gi = (int)(q % p.ix), gj = (int)(q / p.ix);
    const double gmin = fmin(fmin(p.dx[gi], p.ndim == 2 ? p.dy[gj] : p.dy[0]), p.dz0);
    const double sg = p.safety * gmin;
    if (s_ck[0] == 0) {
      double u[8], g[8];
      for (int n = 0; n < 8; ++n) u[n] = z[q + n * nc];
      adj::cfl_mhd_grad(u, p.gm, p.ro_lim, p.pr_lim, sg, g);
      for (int n = 0; n < 8; ++n) lamz[q + n * nc] += ldt * g[n];
    } else {
      double u[5], g[5];
      for (int n = 0; n < 5; ++n) u[n] = z[q + (NVM + n) * nc];
      adj::cfl_hd_grad(u, p.gm, p.ro_lim, p.pr_lim, sg, g);
      for (int n = 0; n < 5; ++n) lamz[q + (NVM + n) * nc] += ldt * g[n];
    }
  }
  *dcol += dac;
  if (ldt_out) *ldt_out = ldt;
}

int face_blocks_h(const KParams &p);

// One reverse stage: primitives of Us, faces (ions, then neutrals), cells.  Partial sums: the
// ion face blocks first (nbf), then the neutral face blocks, then the cell blocks.
cudaError_t launch_stage_vjp(const KParams &p, const double *Us, const double *lam, const double *acc,
                             double *out, const double *dtp, double fac, double *V, double *gx,
                             unsigned long long *mx, double *gy, unsigned long long *my,
                             double *pdot, double *pdac, int nbf, CandPart *cand, cudaStream_t s) {
  const long long nc = p.nc;
  const int gu = (int)std::min<long long>((nc + 255) / 256, 148 * 8);
  u2v_kernel<<<gu, 256, 0, s>>>(p, Us, V);
  face_vjp_kernel<0, kFaceThreads><<<nbf, kFaceThreads, 0, s>>>(p, V, lam, dtp, fac, gx, mx, gy,
                                                                my, pdot, pdac);
  const int nbh = face_blocks_h(p);
  face_vjp_kernel<1, kFaceThreadsH><<<nbh, kFaceThreadsH, 0, s>>>(p, V, lam, dtp, fac, gx, mx, gy,
                                                                  my, pdot + nbf, pdac + nbf);
  const int nbc = (int)((nc + kCellThreads - 1) / kCellThreads);
  cell_vjp_kernel<<<nbc, kCellThreads, 0, s>>>(p, Us, lam, acc, out, dtp, fac, gx, mx, gy, my,
                                               pdot + nbf + nbh, pdac + nbf + nbh, cand);
  return cudaGetLastError();
}

long long face_count(const KParams &p) {
  return (long long)p.jx * (p.ix - 1) + (p.ndim == 2 ? (long long)(p.jx - 1) * p.ix : 0);
}
// blocks of the ion and of the neutral face kernel
int face_blocks(const KParams &p) { return (int)((face_count(p) + kFaceThreads - 1) / kFaceThreads); }
int face_blocks_h(const KParams &p) {
  return (int)((face_count(p) + kFaceThreadsH - 1) / kFaceThreadsH);
}
int cell_blocks(const KParams &p) { return (int)((p.nc + kCellThreads - 1) / kCellThreads); }

cudaError_t prepare() { return cudaSuccess; }

}  // namespace adjk
}  // namespace pip

using pip::DevCtrl;
using pip::KParams;
using pip::adjk::CandPart;

struct pip_adj {
  pip_params p{};
  KParams kp{};
  const pip::Launchers *L = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t max_steps = 0, steps = 0;
  int K = 25;
  int nseg_max = 0;
  size_t state_elems = 0;
  double *A = nullptr, *B = nullptr;
  std::vector<double *> ckpt;   // nseg_max states
  std::vector<double *> segz[2];  // two sets of K-1 states (z_1 .. z_K-1 of a segment)
  std::vector<double *> segu[2];  // two sets of K states (U1 of each step of a segment)
  cudaStream_t stream2 = nullptr;  // recomputation of the next segment during a reverse sweep
  cudaEvent_t ev_start = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr};
  double *La = nullptr, *Lb = nullptr;
  double *dt_hist = nullptr;
  double *d_dx = nullptr, *d_dy = nullptr;
  double *p1dot = nullptr, *p1dac = nullptr, *p2dot = nullptr, *p2dac = nullptr;
  CandPart *cand = nullptr;
  double *dcol = nullptr;
  double *d_dt = nullptr;         // dt of the unit-level stage VJP
  double *V = nullptr;            // primitives of the stage state
  double *gx = nullptr, *gy = nullptr;            // face-state cotangents (2*13 planes)
  unsigned long long *mx = nullptr, *my = nullptr; // minmod branches per face
  int nbf = 0, nbc = 0;
  int *d_fold = nullptr;          // interior cells that are the source of ghost copies
  int *d_fsrc = nullptr;          // their ghost cells, entry-major (nfent x nfold, -1 = none)
  unsigned short *d_fneg = nullptr;  // per entry: plane n's sign is negative iff bit n
  int nfold = 0, nfent = 0;
  DevCtrl *ctrl = nullptr;
  DevCtrl *h_ctrl = nullptr;
  int nb = 0;
  bool have_forward = false;
};

#define ACK(call)                                  \
  do {                                             \
    cudaError_t e__ = (call);                      \
    if (e__ != cudaSuccess) {                      \
      pip::record_cuda_error((int)e__);                 \
      return PIP_ERR_CUDA;                         \
    }                                              \
  } while (0)

namespace {

int grid_fold(int n) {
  return std::max(1, std::min((n * pip::adjk::NV + 255) / 256, 148 * 8));
}

// Gather list of the ghost-fill adjoint: for every interior cell within 2*margin of a
// boundary that is the source of ghost copies (gx/gy: the interior column/row each ghost
// column/row copies), its ghost cells in the order x ghosts (each followed by its corner
// ghosts), then y ghosts, with sign masks from the boundary sign tables.
struct FoldPlan {
  std::vector<int> cells, src;
  std::vector<unsigned short> neg;
  int nent = 0;
};

FoldPlan fold_plan(const KParams &k) {
  std::vector<int> cells;
  std::vector<std::vector<std::pair<int, unsigned short>>> ent;
  const int j0 = k.ndim == 2 ? k.m1 : 0, j1 = k.ndim == 2 ? k.m1 + k.ny : 1;
  for (int j = j0; j < j1; ++j)
    for (int i = k.m0; i < k.m0 + k.nx; ++i) {
      if (!(i < 2 * k.m0 || i >= k.ix - 2 * k.m0 ||
            (k.ndim == 2 && (j < 2 * k.m1 || j >= k.jx - 2 * k.m1))))
        continue;
      int tx[2 * pip::kMaxMargin], sx[2 * pip::kMaxMargin], ntx = 0;
      int ty[2 * pip::kMaxMargin], sy[2 * pip::kMaxMargin], nty = 0;
      for (int s = 0; s < 2; ++s)
        for (int l = 0; l < k.m0; ++l)
          if (k.gx[s][l] == i) {
            tx[ntx] = s == 0 ? l : k.ix - k.m0 + l;
            sx[ntx++] = s;
          }
      if (k.ndim == 2)
        for (int s = 0; s < 2; ++s)
          for (int l = 0; l < k.m1; ++l)
            if (k.gy[s][l] == j) {
              ty[nty] = s == 0 ? l : k.jx - k.m1 + l;
              sy[nty++] = s;
            }
      if (ntx == 0 && nty == 0) continue;
      std::vector<std::pair<int, unsigned short>> e;
      auto mask = [&](int gxs, int gys) {
        unsigned short m = 0;
        for (int n = 0; n < pip::adjk::NV; ++n) {
          const int sg = (gxs >= 0 ? k.symx[gxs][n] : 1) * (gys >= 0 ? k.symy[gys][n] : 1);
          if (sg < 0) m = (unsigned short)(m | (1u << n));
        }
        return m;
      };
      for (int a = 0; a < ntx; ++a) {
        e.push_back({j * k.ix + tx[a], mask(sx[a], -1)});
        for (int b = 0; b < nty; ++b) e.push_back({ty[b] * k.ix + tx[a], mask(sx[a], sy[b])});
      }
      for (int b = 0; b < nty; ++b) e.push_back({ty[b] * k.ix + i, mask(-1, sy[b])});
      cells.push_back(j * k.ix + i);
      ent.push_back(e);
    }
  FoldPlan f;
  f.cells = cells;
  for (const auto &e : ent) f.nent = std::max(f.nent, (int)e.size());
  const size_t nf = cells.size();
  f.src.assign((size_t)f.nent * nf, -1);
  f.neg.assign((size_t)f.nent * nf, 0);
  for (size_t c = 0; c < nf; ++c)
    for (size_t q = 0; q < ent[c].size(); ++q) {
      f.src[q * nf + c] = ent[c][q].first;
      f.neg[q * nf + c] = ent[c][q].second;
    }
  return f;
}

void fold(pip_adj *a, double *lam, int grid) {
  if (a->nfold > 0)
    pip::adjk::fold_kernel<<<grid, 256, 0, a->stream>>>(lam, a->kp.nc, a->d_fold, a->d_fsrc,
                                                       a->d_fneg, a->nfold, a->nfent);
}

cudaError_t launch_vjp(pip_adj *a, int stage, const double *Us, const double *lam, const double *acc,
                       double *out, const double *dtp) {
  const double fac = stage == 1 ? 0.5 : 1.0;
  double *pd = stage == 1 ? a->p1dot : a->p2dot;
  double *pa = stage == 1 ? a->p1dac : a->p2dac;
  CandPart *c = stage == 1 ? a->cand : nullptr;
  return pip::adjk::launch_stage_vjp(a->kp, Us, lam, acc, out, dtp, fac, a->V, a->gx, a->mx, a->gy,
                                     a->my, pd, pa, a->nbf, c, a->stream);
}

void reset_slot(DevCtrl &h, int slot) {
  const double ten = 10.0;
  std::memcpy(&h.red_dt[slot], &ten, sizeof(double));
  h.red_rho[slot] = 0ull;
  h.red_gr[slot] = 0ull;
}

}  // namespace

extern "C" {

int pip_adj_create(const pip_params *p, int64_t max_steps, int checkpoint_every, pip_adj **out) {
  if (!out) return PIP_ERR_NULL;
  *out = nullptr;
  if (!p) return PIP_ERR_NULL;
  KParams k;
  int st = pip::kparams_from_params(p, &k);
  if (st != PIP_OK) return st;
  if (p->precision != PIP_FP64 || p->flag_divb != 0 || p->flag_pip_imp != 0 ||
      p->flag_ir != PIP_IR_NONE || p->flag_heat != 0)
    return PIP_ERR_PARAM;
  if (max_steps <= 0) return PIP_ERR_PARAM;
  pip_adj *a = new (std::nothrow) pip_adj();
  if (!a) return PIP_ERR_NOMEM;
  a->p = *p;
  a->p.dx = a->p.dy = a->p.dz = nullptr;
  a->kp = k;
  a->L = p->fp_exact ? &pip::launchers_exact() : &pip::launchers_fast();
  a->max_steps = max_steps;
  a->K = checkpoint_every > 0 ? checkpoint_every : 25;
  a->nseg_max = (int)((max_steps + a->K - 1) / a->K);
  a->state_elems = (size_t)k.nc * (k.nvm + 5);
  const size_t sb = a->state_elems * sizeof(double);
  auto fail = [&](cudaError_t e) {
    pip::record_cuda_error((int)e);
    pip_adj_destroy(a);
    return e == cudaErrorMemoryAllocation ? PIP_ERR_NOMEM : PIP_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaGetDevice(&a->device)) != cudaSuccess) return fail(e);
  if ((e = a->L->prepare()) != cudaSuccess) return fail(e);
  if ((e = pip::adjk::prepare()) != cudaSuccess) return fail(e);
  // the reverse sweep (stream) is the critical path; the recomputation of the next segment
  // (stream2) fills the SMs it leaves idle, so it gets the lower priority
  int prio_lo = 0, prio_hi = 0;
  if ((e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi)) != cudaSuccess) return fail(e);
  if ((e = cudaStreamCreateWithPriority(&a->stream, cudaStreamNonBlocking, prio_hi)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMalloc(&a->A, sb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->B, sb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->La, sb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->Lb, sb)) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(a->B, 0, sb)) != cudaSuccess) return fail(e);
  a->ckpt.assign(a->nseg_max, nullptr);
  for (auto &x : a->ckpt)
    if ((e = cudaMalloc(&x, sb)) != cudaSuccess) return fail(e);
  // the second set lets the recomputation of segment s-1 run beside the reverse sweep of s
  for (int set = 0; set < (a->nseg_max > 1 ? 2 : 1); ++set) {
    a->segz[set].assign(a->K > 1 ? a->K - 1 : 0, nullptr);
    for (auto &x : a->segz[set])
      if ((e = cudaMalloc(&x, sb)) != cudaSuccess) return fail(e);
    a->segu[set].assign(a->K, nullptr);
    for (auto &x : a->segu[set]) {
      if ((e = cudaMalloc(&x, sb)) != cudaSuccess) return fail(e);
      if ((e = cudaMemset(x, 0, sb)) != cudaSuccess) return fail(e);
    }
  }
  if ((e = cudaStreamCreateWithPriority(&a->stream2, cudaStreamNonBlocking, prio_lo)) != cudaSuccess)
    return fail(e);
  if ((e = cudaEventCreateWithFlags(&a->ev_start, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  for (int set = 0; set < 2; ++set) {
    if ((e = cudaEventCreateWithFlags(&a->ev_rec[set], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e);
    if ((e = cudaEventCreateWithFlags(&a->ev_rev[set], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e);
  }
  if ((e = cudaMalloc(&a->dt_hist, sizeof(double) * max_steps)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->d_dx, sizeof(double) * p->ix)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->d_dy, sizeof(double) * p->jx)) != cudaSuccess) return fail(e);
  if ((e = cudaMemcpy(a->d_dx, p->dx, sizeof(double) * p->ix, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemcpy(a->d_dy, p->dy, sizeof(double) * p->jx, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  a->kp.dx = a->d_dx;
  a->kp.dy = a->d_dy;
  a->nbf = pip::adjk::face_blocks(a->kp);
  a->nbc = pip::adjk::cell_blocks(a->kp);
  a->nb = a->nbf + pip::adjk::face_blocks_h(a->kp) + a->nbc;
  if ((e = cudaMalloc(&a->V, sb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->gx, sizeof(double) * 2 * 13 * (size_t)k.nc)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->gy, sizeof(double) * 2 * 13 * (size_t)k.nc)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->mx, sizeof(unsigned long long) * (size_t)k.nc)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->my, sizeof(unsigned long long) * (size_t)k.nc)) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(a->gy, 0, sizeof(double) * 2 * 13 * (size_t)k.nc)) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(a->my, 0, sizeof(unsigned long long) * (size_t)k.nc)) != cudaSuccess) return fail(e);
  {
    const FoldPlan fp = fold_plan(a->kp);
    a->nfold = (int)fp.cells.size();
    a->nfent = fp.nent;
    const size_t ne = std::max<size_t>(1, fp.src.size());
    if ((e = cudaMalloc(&a->d_fold, sizeof(int) * std::max<size_t>(1, fp.cells.size()))) != cudaSuccess)
      return fail(e);
    if ((e = cudaMalloc(&a->d_fsrc, sizeof(int) * ne)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&a->d_fneg, sizeof(unsigned short) * ne)) != cudaSuccess) return fail(e);
    if (!fp.cells.empty()) {
      if ((e = cudaMemcpy(a->d_fold, fp.cells.data(), sizeof(int) * fp.cells.size(),
                          cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
      if ((e = cudaMemcpy(a->d_fsrc, fp.src.data(), sizeof(int) * fp.src.size(),
                          cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
      if ((e = cudaMemcpy(a->d_fneg, fp.neg.data(), sizeof(unsigned short) * fp.neg.size(),
                          cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    }
  }
  if ((e = cudaMalloc(&a->p1dot, sizeof(double) * a->nb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->p1dac, sizeof(double) * a->nb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->p2dot, sizeof(double) * a->nb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->p2dac, sizeof(double) * a->nb)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->cand, sizeof(CandPart) * a->nbc)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->dcol, sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->d_dt, sizeof(double))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&a->ctrl, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&a->h_ctrl, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
  std::memset(a->h_ctrl, 0, sizeof(DevCtrl));
  *out = a;
  return PIP_OK;
}

void pip_adj_destroy(pip_adj *a) {
  if (!a) return;
  cudaSetDevice(a->device);
  if (a->stream) cudaStreamSynchronize(a->stream);
  double *bufs[] = {a->A, a->B, a->La, a->Lb, a->dt_hist, a->d_dx, a->d_dy,
                    a->p1dot, a->p1dac, a->p2dot, a->p2dac, a->dcol, a->d_dt, a->V, a->gx, a->gy};
  for (double *b : bufs)
    if (b) cudaFree(b);
  for (double *b : a->ckpt)
    if (b) cudaFree(b);
  if (a->stream2) cudaStreamSynchronize(a->stream2);
  for (int set = 0; set < 2; ++set) {
    for (double *b : a->segz[set])
      if (b) cudaFree(b);
    for (double *b : a->segu[set])
      if (b) cudaFree(b);
    if (a->ev_rec[set]) cudaEventDestroy(a->ev_rec[set]);
    if (a->ev_rev[set]) cudaEventDestroy(a->ev_rev[set]);
  }
  if (a->ev_start) cudaEventDestroy(a->ev_start);
  if (a->stream2) cudaStreamDestroy(a->stream2);
  if (a->cand) cudaFree(a->cand);
  if (a->d_fold) cudaFree(a->d_fold);
  if (a->d_fsrc) cudaFree(a->d_fsrc);
  if (a->d_fneg) cudaFree(a->d_fneg);
  if (a->mx) cudaFree(a->mx);
  if (a->my) cudaFree(a->my);
  if (a->ctrl) cudaFree(a->ctrl);
  if (a->h_ctrl) cudaFreeHost(a->h_ctrl);
  if (a->stream) cudaStreamDestroy(a->stream);
  delete a;
}

int pip_adj_set_col(pip_adj *a, double col) {
  if (!a) return PIP_ERR_NULL;
  if (!(col >= 0.0) || !std::isfinite(col)) return PIP_ERR_PARAM;
  a->p.col = col;
  a->kp.ac = col;
  a->have_forward = false;
  return PIP_OK;
}

int pip_adj_forward(pip_adj *a, const double *U0, double *UN, int64_t nsteps, float *device_ms) {
  if (!a || !U0 || !UN) return PIP_ERR_NULL;
  if (nsteps <= 0 || nsteps > a->max_steps) return PIP_ERR_PARAM;
  ACK(cudaSetDevice(a->device));
  const size_t sb = a->state_elems * sizeof(double);
  DevCtrl &h = *a->h_ctrl;
  std::memset(&h, 0, sizeof(DevCtrl));
  h.nsteps = nsteps;
  reset_slot(h, 0);
  reset_slot(h, 1);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (device_ms) {
    ACK(cudaEventCreate(&e0));
    ACK(cudaEventCreate(&e1));
  }
  ACK(cudaMemcpyAsync(a->ctrl, a->h_ctrl, sizeof(DevCtrl), cudaMemcpyHostToDevice, a->stream));
  if (device_ms) ACK(cudaEventRecord(e0, a->stream));
  ACK(cudaMemcpyAsync(a->A, U0, sb, cudaMemcpyDeviceToDevice, a->stream));
  // the loop of pip_run: cfl of the first step, then [stage 1, stage 2] per step
  ACK(a->L->cfl(a->kp, a->A, a->ctrl, 0, a->stream));
  for (int64_t n = 0; n < nsteps; ++n) {
    if (n % a->K == 0)
      ACK(cudaMemcpyAsync(a->ckpt[n / a->K], a->A, sb, cudaMemcpyDeviceToDevice, a->stream));
    ACK(a->L->stage(a->kp, 1, a->A, a->A, a->B, a->ctrl, 1, 0, a->stream, nullptr, 0));
    ACK(cudaMemcpyAsync(a->dt_hist + n, &a->ctrl->dt, sizeof(double), cudaMemcpyDeviceToDevice,
                        a->stream));
    ACK(a->L->stage(a->kp, 2, a->B, a->A, a->A, a->ctrl, 1, -1, a->stream, nullptr, 0));
  }
  ACK(cudaMemcpyAsync(UN, a->A, sb, cudaMemcpyDeviceToDevice, a->stream));
  if (device_ms) ACK(cudaEventRecord(e1, a->stream));
  ACK(cudaMemcpyAsync(a->h_ctrl, a->ctrl, sizeof(DevCtrl), cudaMemcpyDeviceToHost, a->stream));
  ACK(cudaStreamSynchronize(a->stream));
  if (device_ms) {
    ACK(cudaEventElapsedTime(device_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  a->steps = h.step;
  a->have_forward = h.step == nsteps && !h.nan_flag && h.status == 0;
  if (h.nan_flag) return PIP_ERR_NAN;
  if (h.status) return h.status;
  if (h.step != nsteps) return PIP_ERR_STATE;
  return PIP_OK;
}

int pip_adj_backward(pip_adj *a, const double *gN, double *g0, double *g_col, float *device_ms) {
  if (!a || !gN || !g0) return PIP_ERR_NULL;
  if (!a->have_forward) return PIP_ERR_STATE;
  ACK(cudaSetDevice(a->device));
  const size_t sb = a->state_elems * sizeof(double);
  const KParams &kp = a->kp;
  DevCtrl &h = *a->h_ctrl;
  std::memset(&h, 0, sizeof(DevCtrl));
  reset_slot(h, 0);
  reset_slot(h, 1);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (device_ms) {
    ACK(cudaEventCreate(&e0));
    ACK(cudaEventCreate(&e1));
  }
  ACK(cudaMemcpyAsync(a->ctrl, a->h_ctrl, sizeof(DevCtrl), cudaMemcpyHostToDevice, a->stream));
  if (device_ms) ACK(cudaEventRecord(e0, a->stream));
  ACK(cudaMemcpyAsync(a->La, gN, sb, cudaMemcpyDeviceToDevice, a->stream));
  ACK(cudaMemsetAsync(a->dcol, 0, sizeof(double), a->stream));
  const int64_t N = a->steps;
  const int nseg = (int)((N + a->K - 1) / a->K);
  const int gf = grid_fold(a->nfold);
  // Segment s is recomputed from its checkpoint into buffer set s % 2 on stream2 while the
  // reverse sweep of segment s + 1 runs on stream: the recomputation waits for the sweep
  // that last used its set (segment s + 2), the sweep of s for the recomputation of s.
  auto zp = [&](int s, int j) -> double * { return j == 0 ? a->ckpt[s] : a->segz[s % 2][j - 1]; };
  auto recompute = [&](int s) -> int {
    const int64_t n0 = (int64_t)s * a->K;
    const int len = (int)std::min<int64_t>(a->K, N - n0);
    if (s + 2 < nseg) ACK(cudaStreamWaitEvent(a->stream2, a->ev_rev[s % 2], 0));
    // z_n, U1_n of the segment with the recorded dt
    for (int j = 0; j < len; ++j) {
      ACK(cudaMemcpyAsync(&a->ctrl->dt, a->dt_hist + n0 + j, sizeof(double), cudaMemcpyDeviceToDevice,
                          a->stream2));
      ACK(a->L->stage(kp, 1, zp(s, j), zp(s, j), a->segu[s % 2][j], a->ctrl, 0, 0, a->stream2, nullptr, 0));
      if (j + 1 < len)
        ACK(a->L->stage(kp, 2, a->segu[s % 2][j], zp(s, j), zp(s, j + 1), a->ctrl, 0, 2, a->stream2, nullptr, 0));
    }
    ACK(cudaEventRecord(a->ev_rec[s % 2], a->stream2));
    return PIP_OK;
  };
  ACK(cudaEventRecord(a->ev_start, a->stream));
  ACK(cudaStreamWaitEvent(a->stream2, a->ev_start, 0));
  int rst = recompute(nseg - 1);
  if (rst != PIP_OK) return rst;
  for (int s = nseg - 1; s >= 0; --s) {
    if (s > 0 && (rst = recompute(s - 1)) != PIP_OK) return rst;
    const int64_t n0 = (int64_t)s * a->K;
    const int len = (int)std::min<int64_t>(a->K, N - n0);
    ACK(cudaStreamWaitEvent(a->stream, a->ev_rec[s % 2], 0));
    // reverse sweep
    for (int j = len - 1; j >= 0; --j) {
      const double *dtp = a->dt_hist + n0 + j;
      fold(a, a->La, gf);
      ACK(cudaGetLastError());
      ACK(launch_vjp(a, 2, a->segu[s % 2][j], a->La, nullptr, a->Lb, dtp));
      fold(a, a->Lb, gf);
      ACK(cudaGetLastError());
      ACK(launch_vjp(a, 1, zp(s, j), a->Lb, a->La, a->La, dtp));
      pip::adjk::finalize_kernel<<<1, 256, 0, a->stream>>>(kp, a->nb, a->nbc, a->p1dot, a->p1dac, a->p2dot,
                                                            a->p2dac, a->cand, dtp, zp(s, j), a->La,
                                                            a->dcol, nullptr);
      ACK(cudaGetLastError());
    }
    ACK(cudaEventRecord(a->ev_rev[s % 2], a->stream));
  }
  ACK(cudaMemcpyAsync(g0, a->La, sb, cudaMemcpyDeviceToDevice, a->stream));
  if (device_ms) ACK(cudaEventRecord(e1, a->stream));
  double dc = 0.0;
  ACK(cudaMemcpyAsync(&a->h_ctrl->dt, a->dcol, sizeof(double), cudaMemcpyDeviceToHost, a->stream));
  ACK(cudaStreamSynchronize(a->stream));
  dc = a->h_ctrl->dt;
  if (g_col) *g_col = dc;
  if (device_ms) {
    ACK(cudaEventElapsedTime(device_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return PIP_OK;
}

int pip_adj_stage_vjp(pip_adj *a, int stage, const double *Us, const double *lam, double *out,
                      double dt, double *dot, double *dcol) {
  if (!a || !Us || !lam || !out) return PIP_ERR_NULL;
  if ((stage != 1 && stage != 2) || !(dt > 0.0)) return PIP_ERR_PARAM;
  ACK(cudaSetDevice(a->device));
  ACK(cudaMemcpyAsync(a->d_dt, &dt, sizeof(double), cudaMemcpyHostToDevice, a->stream));
  ACK(launch_vjp(a, stage, Us, lam, nullptr, out, a->d_dt));
  std::vector<double> pd(a->nb), pa(a->nb);
  ACK(cudaMemcpyAsync(pd.data(), stage == 1 ? a->p1dot : a->p2dot, sizeof(double) * a->nb,
                      cudaMemcpyDeviceToHost, a->stream));
  ACK(cudaMemcpyAsync(pa.data(), stage == 1 ? a->p1dac : a->p2dac, sizeof(double) * a->nb,
                      cudaMemcpyDeviceToHost, a->stream));
  ACK(cudaStreamSynchronize(a->stream));
  double sd = 0.0, sa = 0.0;
  for (int b = 0; b < a->nb; ++b) {
    sd += pd[b];
    sa += pa[b];
  }
  if (dot) *dot = sd;
  if (dcol) *dcol = sa;
  return PIP_OK;
}

int pip_adj_fold(pip_adj *a, double *lam) {
  if (!a || !lam) return PIP_ERR_NULL;
  ACK(cudaSetDevice(a->device));
  fold(a, lam, grid_fold(a->nfold));
  ACK(cudaGetLastError());
  ACK(cudaStreamSynchronize(a->stream));
  return PIP_OK;
}

int pip_adj_dt(pip_adj *a, double *dt, int64_t n, int64_t *steps) {
  if (!a) return PIP_ERR_NULL;
  if (steps) *steps = a->steps;
  if (dt && n > 0) {
    ACK(cudaSetDevice(a->device));
    const int64_t m = std::min(n, a->steps);
    if (m > 0) ACK(cudaMemcpy(dt, a->dt_hist, sizeof(double) * m, cudaMemcpyDeviceToHost));
  }
  return PIP_OK;
}

}  // extern "C"
