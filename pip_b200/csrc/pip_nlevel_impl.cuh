// pip_nlevel_impl.cuh -- FP64 kernels of set_IR type 4, the 6-level hydrogen model
// (PIP_rot.f90:232-311 set_IR, :361-616 get_col_ion_coeff, :919-946 ionexpfitinterp2,
// :1026-1159 hydrogen_excitation_update, :1162-1235 IRgetionpot; Scheme_rot.f90:315-335
// cfl_pip_ir / cfl_pip_ir_nexcite, :692-736 derivative, :1002-1049
// hydrogen_excitation_timestep).  Included by pip_step_impl.cuh inside the flavour's
// namespace, after the cell helpers it uses (get_te, write_ghosts, near_boundary).
//
// HBM layout: Nexcite is 6 planes of ix*jx cells (levels 1-5, then the ions), kept twice
// (the update reads one and writes the other); colrat is 36 planes, plane a + 6*b holding
// colrat(a+1,b+1) as the Fortran (ix,jx,kx,6,6) array does; ion_pot and the rates (irg: Gm_ion
// then Gm_rec) one plane each.  The exponential-integral table (4 doubles per row, 3.2 MB
// for the reference's 100001 rows) stays in L2.
//
// Every kernel works cell by cell, no reduction order depends on the launch shape except the
// maxima (exact), and the arithmetic keeps the Fortran operation order; the FMA-free build
// therefore matches the CPU restatement up to the last bits of exp, log and pow.

// Default-real literals of the Fortran (rounded to float there): kboltz, melec, a0bohr
// (PIP_rot.f90:366-369), 1.0e14 (:591), the 1.e-16 floor (:1138).
constexpr double kNlKb = (double)1.38064852e-23f;
constexpr double kNlMe = (double)9.10938356e-31f;
constexpr double kNlA0 = (double)5.29e-11f;
constexpr double kNlE14 = (double)1.0e14f;
constexpr double kNlFloor = (double)1.e-16f;
constexpr double kNlMehat = 9.10938356, kNlKbhat = 1.38064852, kNlHhat = 6.62607004;
constexpr double kNlPi = 3.1415926535897932;  // Parameters.f90's pi

// Weights of ionexpfitinterp2 (rad = 0) at z: rows xindex..xindex+2 of the table.  The
// reference clamps xindex to 1..n-1 and then reads row n+1 at the top end, past its table;
// here xindex stops at n-2.  Several E_i at the same z share one set of weights (the same
// arithmetic as recomputing them).
struct NlW {
  const double *r0;
  double w0, w1, w2;
};
// The FMA build multiplies by the rows' precomputed reciprocal denominators (nl_rtab) and
// finds the row with a product, falling back to the reference's quotient when the product
// lies within 1e-9 of a row boundary (a few ulps from the quotient), so both pick the same
// row.
__device__ __forceinline__ NlW nl_weights(const KParams &p, double z) {
  const long long n = p.nl_ntab;
#if PIP_RCP
  const double t = (z - p.nl_xmin) * p.nl_xsc;
  double f = floor(t);
  if (t - f < 1.0e-9 || f + 1.0 - t < 1.0e-9) f = floor((z - p.nl_xmin) / p.nl_xrange * (double)n);
#else
  const double f = floor((z - p.nl_xmin) / p.nl_xrange * (double)n);
#endif
  long long xi;
  if (!(f > 0.0)) xi = 1;
  else if (f >= (double)n) xi = n - 1;
  else xi = (long long)f;
  if (xi > n - 2) xi = n - 2;
  NlW w;
  w.r0 = p.nl_tab + 4 * (xi - 1);
  const double x0 = __ldg(w.r0), x1 = __ldg(w.r0 + 4), x2 = __ldg(w.r0 + 8);
#if PIP_RCP
  const double *rt = p.nl_rtab + 4 * (xi - 1);
  w.w0 = ((z - x1) * (z - x2)) * __ldg(rt);
  w.w1 = ((z - x0) * (z - x2)) * __ldg(rt + 1);
  w.w2 = ((z - x0) * (z - x1)) * __ldg(rt + 2);
#else
  w.w0 = ((z - x1) * (z - x2)) / ((x0 - x1) * (x0 - x2));
  w.w1 = ((z - x0) * (z - x2)) / ((x1 - x0) * (x1 - x2));
  w.w2 = ((z - x0) * (z - x1)) / ((x2 - x0) * (x2 - x1));
#endif
  return w;
}
__device__ __forceinline__ double nl_eval(const NlW &w, int i) {
  return w.w0 * __ldg(w.r0 + i + 1) + w.w1 * __ldg(w.r0 + i + 5) + w.w2 * __ldg(w.r0 + i + 9);
}

// get_col_ion_coeff on one cell of electron temperature te [K] and density ne: colrat into
// cr[a*6+b] = colrat(a+1,b+1), the sums gi = sum max(N(ii)*colrat(ii,6),0) and
// gr = sum max(N(6)*colrat(6,ii),0); true where the reference stops on a negative rate.
// The FMA build divides once by kboltz*te and once by each y and z, and multiplies by the
// reciprocal constants (ixrat, gwq, gwh); the rates then differ from the reference's by a
// few ulps.
__device__ __forceinline__ bool nl_cell(const KParams &p, const NlevConst &k, double te,
                                        double ne, const double (&nx)[6], double (&cr)[36],
                                        double &gi, double &gr) {
#if PIP_RCP
  bool bad = false;
  const double s = sqrt(8.0 * kNlKb * te / kNlPi / kNlMe);
  const double ikt = 1.0 / (kNlKb * te);
#pragma unroll
  for (int m = 0; m < 36; ++m) cr[m] = 0.0;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double ri = (double)(a + 1);
    const double pre = ne * s * 2.0 * (ri * ri) * kNlPi * (kNlA0 * kNlA0);
#pragma unroll
    for (int b = a + 1; b < 5; ++b) {
      const double enn = k.enn[a][b];
      const double yhat = enn * ikt;
      const double zhat = k.rnn[a][b] + enn * ikt;
      const double iy = 1.0 / yhat, iz = 1.0 / zhat;
      const NlW wy = nl_weights(p, yhat), wz = nl_weights(p, zhat);
      const double E1y = nl_eval(wy, 1), E1z = nl_eval(wz, 1);
      const double E2y = nl_eval(wy, 2), E2z = nl_eval(wz, 2);
      const double ann = k.ann[a][b];
      const double colex = pre * k.ixrat[a][b] * (yhat * yhat) *
                           (ann * ((iy + 0.5) * E1y - (iz + 0.5) * E1z) +
                            (k.bnn[a][b] - ann * k.lgt[a][b]) * (E2y * iy - E2z * iz));
      cr[a * 6 + b] = k.gwq[a][b] * colex;
      cr[b * 6 + a] = colex * exp(-((k.eion[a] - k.eion[b]) * ikt));
    }
    const double yn = k.eion[a] * ikt;
    const double zn = k.rn[a] + k.eion[a] * ikt;
    const double iyn = 1.0 / yn, izn = 1.0 / zn;
    const NlW wy = nl_weights(p, yn), wz = nl_weights(p, zn);
    const double E1y = nl_eval(wy, 1), E1z = nl_eval(wz, 1);
    const double E2y = nl_eval(wy, 2), E2z = nl_eval(wz, 2);
    const double E0y = nl_eval(wy, 0), E0z = nl_eval(wz, 0);
    const double ziyn = E0y - 2.0 * E1y + E2y, zizn = E0z - 2.0 * E1z + E2z;
    const double an0 = k.an0[a];
    const double colex = pre * (yn * yn) *
                         (an0 * (E1y * iyn - E1z * izn) + (k.bn0[a] - an0 * k.lgi[a]) * (ziyn - zizn));
    bad |= colex < 0.0;
    cr[a * 6 + 5] = colex * exp(-((k.eion[5] - k.eion[a]) * ikt));
  }
  const double saha =
      pow(2.0 * kNlPi * kNlMehat * kNlKbhat * te / kNlHhat / kNlHhat * kNlE14, -3.0 / 2.0);
  double si = 0.0, sr = 0.0;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    cr[30 + a] = ne * cr[a * 6 + 5] * k.gwh[a] * saha * exp(k.eion[a] * ikt);
    si = si + fmax(nx[a] * cr[a * 6 + 5], 0.0);
    sr = sr + fmax(nx[5] * cr[30 + a], 0.0);
  }
#pragma unroll
  for (int m = 0; m < 36; ++m) bad |= cr[m] < 0.0;
  gi = si;
  gr = sr;
  return bad;
#else
  bool bad = false;
  const double s = sqrt(8.0 * kNlKb * te / kNlPi / kNlMe);
#pragma unroll
  for (int m = 0; m < 36; ++m) cr[m] = 0.0;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double ri = (double)(a + 1);
#pragma unroll
    for (int b = a + 1; b < 5; ++b) {
      const double enn = k.enn[a][b];
      const double yhat = enn / kNlKb / te;
      const double zhat = k.rnn[a][b] + enn / kNlKb / te;
      const NlW wy = nl_weights(p, yhat), wz = nl_weights(p, zhat);
      const double E1y = nl_eval(wy, 1), E1z = nl_eval(wz, 1);
      const double E2y = nl_eval(wy, 2), E2z = nl_eval(wz, 2);
      const double ann = k.ann[a][b];
      const double colex = ne * s * 2.0 * (ri * ri) / k.xrat[a][b] * kNlPi * (kNlA0 * kNlA0) *
                           (yhat * yhat) *
                           (ann * ((1.0 / yhat + 0.5) * E1y - (1.0 / zhat + 0.5) * E1z) +
                            (k.bnn[a][b] - ann * k.lgt[a][b]) * (E2y / yhat - E2z / zhat));
      cr[a * 6 + b] = k.gw[a] / k.gw[b] * colex;
      cr[b * 6 + a] = colex * exp(-((k.eion[a] - k.eion[b]) / kNlKb / te));
    }
    const double yn = k.eion[a] / kNlKb / te;
    const double zn = k.rn[a] + k.eion[a] / kNlKb / te;
    const NlW wy = nl_weights(p, yn), wz = nl_weights(p, zn);
    const double E1y = nl_eval(wy, 1), E1z = nl_eval(wz, 1);
    const double E2y = nl_eval(wy, 2), E2z = nl_eval(wz, 2);
    const double E0y = nl_eval(wy, 0), E0z = nl_eval(wz, 0);
    const double ziyn = E0y - 2.0 * E1y + E2y, zizn = E0z - 2.0 * E1z + E2z;
    const double an0 = k.an0[a];
    const double colex = ne * s * 2.0 * (ri * ri) * kNlPi * (kNlA0 * kNlA0) * (yn * yn) *
                         (an0 * (E1y / yn - E1z / zn) + (k.bn0[a] - an0 * k.lgi[a]) * (ziyn - zizn));
    bad |= colex < 0.0;
    cr[a * 6 + 5] = colex * exp(-((k.eion[5] - k.eion[a]) / kNlKb / te));
  }
  const double saha =
      pow(2.0 * kNlPi * kNlMehat * kNlKbhat * te / kNlHhat / kNlHhat * kNlE14, -3.0 / 2.0);
  double si = 0.0, sr = 0.0;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    cr[30 + a] = ne * cr[a * 6 + 5] * k.gw[a] / k.gw[5] / 2.0 * saha * exp(k.eion[a] / kNlKb / te);
    si = si + fmax(nx[a] * cr[a * 6 + 5], 0.0);
    sr = sr + fmax(nx[5] * cr[30 + a], 0.0);
  }
#pragma unroll
  for (int m = 0; m < 36; ++m) bad |= cr[m] < 0.0;
  gi = si;
  gr = sr;
  return bad;
#endif
}

// IRgetionpot (PIP_rot.f90:1162-1235) of one cell.
__device__ __forceinline__ double nl_ionpot(const KParams &p, const NlevConst &k,
                                            const double (&cr)[36], const double (&nx)[6]) {
  double il = 0.0, ig = 0.0;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    il = il + cr[i * 6 + 5] * k.eev[i] * nx[i];
    ig = ig + cr[30 + i] * k.eev[i] * nx[5];
#pragma unroll
    for (int j = 1; j < 5; ++j) {
      il = il + nx[i] * cr[i * 6 + j] * (k.eev[i] - k.eev[j]);
      ig = ig + nx[j] * (cr[j * 6 + i] * (k.eev[i] - k.eev[j]));
    }
  }
  const double en = p.nl_odd ? (il - ig) / p.gm / p.nl_T0 / (double)8.6173e-5f
                             : (il - ig) / p.nl_en_even;
  return en / p.nl_gref * p.nl_tir;
}

// set_IR type 4's reference block (PIP_rot.f90:250-279) on cell (1,1,1): colrat at
// (T_norm, n_norm) and that cell's recombination sum, the normalisation Gm_rec_ref.
__global__ void nlev_ref_kernel(const __grid_constant__ KParams p, double *out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const NlevConst &k = *p.nl_k;
  double nx[6], cr[36], gi, gr;
#pragma unroll
  for (int m = 0; m < 6; ++m) nx[m] = p.nl_nex[m * p.nc];
  nl_cell(p, k, p.nl_T0, p.nl_n0, nx, cr, gi, gr);
  for (int m = 0; m < 36; ++m) out[m] = cr[m];
  out[36] = gr;
}

// set_IR type 4 over every cell of U (ghosts included): get_Te_HD/MHD's energy rewrite
// (after set_collisional's when colrw), colrat from Te_p*T0/tfac and rho_i*n0/n0fac, the
// normalised rates Gm_ion/rho_n/Gm_rec_ref*t_ir and Gm_rec/rho_i/Gm_rec_ref*t_ir.  U itself
// is not written: the kernels that follow make the same rewrites of their copies.
// ipmode 1: ion_pot (source_PIP's IRgetionpot) from the new colrat; 2: from crref (the
// prologue's block).
template <int NVM>
__global__ void __launch_bounds__(128) nlev_rates_kernel(const __grid_constant__ KParams p,
                                                         const double *__restrict__ U, int colrw,
                                                         int ipmode, const double *crref,
                                                         DevCtrl *ctrl) {
  const NlevConst &k = *p.nl_k;
  const long long nc = p.nc;
  bool bad = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    double um[NVM], uh[5];
    load_cell<NVM>(U, q, nc, um, uh);
    double te_m, te_h, rm, rh;
    if (colrw) get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
    get_te<NVM>(um, uh, p, te_m, te_h, rm, rh);
    double nx[6], cr[36], gi, gr;
#pragma unroll
    for (int m = 0; m < 6; ++m) nx[m] = p.nl_nex[q + m * nc];
    bad |= nl_cell(p, k, te_m * p.nl_T0 / p.nl_tfac, um[0] * p.nl_n0 / p.nl_n0fac, nx, cr, gi, gr);
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
      for (int b = 0; b < 6; ++b) p.nl_cr[q + (long long)(a + 6 * b) * nc] = cr[a * 6 + b];
    p.irg[q] = gi / uh[0] / p.nl_gref * p.nl_tir;
    p.irg[nc + q] = gr / um[0] / p.nl_gref * p.nl_tir;
    if (ipmode == 1) {
      p.nl_ip[q] = nl_ionpot(p, k, cr, nx);
    } else if (ipmode == 2) {
      double c0[36];
#pragma unroll
      for (int m = 0; m < 36; ++m) c0[m] = crref[m];
      p.nl_ip[q] = nl_ionpot(p, k, c0, nx);
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(&ctrl->status, 0, 9);  // PIP_ERR_RATE
}

// colrat(a+1,b+1) of cell q.
__device__ __forceinline__ double nl_cr(const KParams &p, long long q, int a, int b) {
  return p.nl_cr[q + (long long)(a + 6 * b) * p.nc];
}

// derivative (Scheme_rot.f90:692-736) of plane v at cell (i, j) along x (dir 1) or y:
// order 4 the five-point form, 1 the two-point one; zero where the stencil leaves the array
// (cells the reference leaves unset) and with order 0.
template <int DIR>
__device__ __forceinline__ double nl_deriv(const KParams &p, const double *v, long long q, int i,
                                           int j) {
  const int order = p.nl_deriv;
  if (order == 0) return 0.0;
  const int w = order == 4 ? 2 : 1;
  const long long s = DIR == 1 ? 1 : p.ix;
  const int c = DIR == 1 ? i : j, n = DIR == 1 ? p.ix : p.jx;
  if (c < w || c >= n - w) return 0.0;
  const double d = DIR == 1 ? p.dx[i] : p.dy[j];
  if (order == 4) return (-v[q + 2 * s] + 8.0 * v[q + s] - 8.0 * v[q - s] + v[q - 2 * s]) / (12.0 * d);
  return (v[q + s] - v[q - s]) / (2.0 * d);
}

// The convective term of level m at cell q: d(Nexcite)/dx*vx_n (+ d/dy*vy_n in 2D).
template <int NDIM, int NVM>
__device__ __forceinline__ double nl_conv(const KParams &p, const double *U, int m, long long q,
                                          int i, int j) {
  const long long nc = p.nc;
  const double *v = p.nl_nex + m * nc;
  const double rh = U[q + NVM * nc];
  double c = nl_deriv<1>(p, v, q, i, j) * U[q + (NVM + 1) * nc] / rh;
  if (NDIM == 2) c = c + nl_deriv<2>(p, v, q, i, j) * U[q + (NVM + 2) * nc] / rh;
  return c;
}

// hydrogen_excitation_update after a stage (Solver_rot.f90:218-220) over the interior cells
// of the updated state U, dt_sub = dt/2 (stage 1) or dt (stage 2): the ion population's sum,
// the neutral levels' sums over the ion and the other levels, minus the convection; the
// 1e-16 floor; the ground level takes up the difference to rho_n; Nexcite(6) = rho_i.
// nl_nex -> nl_nex2; bnd_energy's ghosts (the type mapping of MHDbnd, sign +1) are written by
// the threads of their source cells.
template <int NDIM, int NVM>
__global__ void __launch_bounds__(128) nlev_update_kernel(const __grid_constant__ KParams p,
                                                          const double *__restrict__ U,
                                                          const DevCtrl *ctrl, int stage) {
  // (launched only for a step the stages run: the host loop stops before a step that would
  // not, and the last step's stage 2 sets ctrl->done once it has run)
  const double dt = ctrl->dt;
  const double dts = stage == 1 ? dt / 2.0 : dt / 1.0;
  const long long nc = p.nc, n = (long long)p.nx * p.ny;
  const double g = p.nl_gref, tir = p.nl_tir;
#if PIP_RCP
  const double cg = tir / g;   // x/g*tir as x*cg
#define PIP_NL_GT(x) ((x) * cg)
#else
#define PIP_NL_GT(x) ((x) / g * tir)
#endif
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = p.m0 + (int)(t % p.nx), j = p.m1 + (int)(t / p.nx);
    const long long q = (long long)j * p.ix + i;
    double nx[6], d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < 6; ++m) nx[m] = p.nl_nex[q + m * nc];
#pragma unroll
    for (int jj = 0; jj < 5; ++jj)
      d[5] = d[5] + PIP_NL_GT(nx[jj] * nl_cr(p, q, jj, 5)) - PIP_NL_GT(nx[5] * nl_cr(p, q, 5, jj));
#pragma unroll
    for (int ii = 0; ii < 5; ++ii)
      d[ii] = d[ii] + PIP_NL_GT(nx[5] * nl_cr(p, q, 5, ii)) - PIP_NL_GT(nx[ii] * nl_cr(p, q, ii, 5));
#pragma unroll
    for (int ii = 0; ii < 5; ++ii)
#pragma unroll
      for (int jj = 0; jj < 5; ++jj)
        d[ii] = d[ii] + PIP_NL_GT(nx[jj] * nl_cr(p, q, jj, ii)) - PIP_NL_GT(nx[ii] * nl_cr(p, q, ii, jj));
    double o[6];
#pragma unroll
    for (int ii = 0; ii < 5; ++ii) {
      const double v = nx[ii] + dts * (d[ii] - nl_conv<NDIM, NVM>(p, U, ii, q, i, j));
      o[ii] = v > kNlFloor ? v : kNlFloor;
    }
    const double tot = o[0] + o[1] + o[2] + o[3] + o[4] - U[q + NVM * nc];
    o[0] = o[0] - tot;
    o[5] = U[q];
#pragma unroll
    for (int m = 0; m < 6; ++m) p.nl_nex2[q + m * nc] = o[m];
    if (near_boundary<NDIM>(p, i, j)) write_ghosts<NDIM>(p, i, j, p.nl_nex2, 6, true);
  }
}
#undef PIP_NL_GT

// cfl_pip_ir's type-4 terms and cfl_pip_ir_nexcite (Scheme_rot.f90:315-335) over every cell,
// after the cfl kernel: max of the rates, with flag_IR_type 0 get_Pr_MHD's energy rewrite and
// max(ion_pot/(pr/(gm-1)), 1e-5), and max(dNexcite/dt, 1e-5) over levels 1-5
// (hydrogen_excitation_timestep's sums, Scheme_rot.f90:1017-1046), into slot `slot`.
template <int NDIM, int NVM>
__global__ void __launch_bounds__(256) nlev_cfl_kernel(const __grid_constant__ KParams p,
                                                       double *__restrict__ U, DevCtrl *ctrl,
                                                       int slot) {
  const long long nc = p.nc;
  const double g = p.nl_gref, tir = p.nl_tir, gm = p.gm;
#if PIP_RCP
  const double cg = tir / g;
#define PIP_NL_GT(x) ((x) * cg)
#else
#define PIP_NL_GT(x) ((x) / g * tir)
#endif
  double gmax = 0.0, ipmax = 1.0e-5, nxmax = 1.0e-5;
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < nc; q += (long long)gridDim.x * 256) {
    const int i = (int)(q % p.ix), j = (int)(q / p.ix);
    gmax = fmax(gmax, fmax(p.irg[q], p.irg[nc + q]));
    if (p.ir_type == 0) {
      double u[NVM];
#pragma unroll
      for (int m = 0; m < NVM; ++m) u[m] = U[q + m * nc];
      double pr = (gm - 1.0) * (u[4] - 0.5 * ((u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
                                              u[5] * u[5] + u[6] * u[6] + u[7] * u[7]));
      pr = fmax(pr, p.pr_lim);
      U[q + 4 * nc] = pr / (gm - 1.0) + 0.5 * ((u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
                                               u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
      ipmax = fmax(ipmax, p.nl_ip[q] / (pr / (gm - 1.0)));
    }
    double nx[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) nx[m] = p.nl_nex[q + m * nc];
    for (int ii = 0; ii < 5; ++ii) {
      double d = 0.0;
      for (int jj = 0; jj < 6; ++jj)
        d = d + PIP_NL_GT(nx[jj] * nl_cr(p, q, jj, ii)) - PIP_NL_GT(nx[ii] * nl_cr(p, q, ii, jj));
      nxmax = fmax(nxmax, d - nl_conv<NDIM, NVM>(p, U, ii, q, i, j));
    }
  }
#undef PIP_NL_GT
  // block maxima (exact), then one atomic per block on the ordered bits of the positive values
  __shared__ double red[3][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    gmax = fmax(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
    ipmax = fmax(ipmax, __shfl_xor_sync(0xffffffffu, ipmax, o));
    nxmax = fmax(nxmax, __shfl_xor_sync(0xffffffffu, nxmax, o));
  }
  if (lane == 0) {
    red[0][warp] = gmax;
    red[1][warp] = ipmax;
    red[2][warp] = nxmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) {
      gmax = fmax(gmax, red[0][w]);
      ipmax = fmax(ipmax, red[1][w]);
      nxmax = fmax(nxmax, red[2][w]);
    }
    atomicMax(&ctrl->red_gr[slot], dbits(gmax));
    atomicMax(&ctrl->red_ip[slot], dbits(ipmax));
    atomicMax(&ctrl->red_nx[slot], dbits(nxmax));
  }
}
