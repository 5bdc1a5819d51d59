// pip_kernels.cuh -- kernel parameter blocks shared by the FP64 kernels and the C ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pip {

constexpr int kMaxMargin = 3;
constexpr int kMaxPlanes = 14;   // 9 ion + 5 neutral

// Cell-independent coefficients of the 6-level hydrogen model's collisional rates
// (get_col_ion_coeff, PIP_rot.f90:378-439,507-524), built on the host in the Fortran
// operation order; index a, b = level - 1, entries with a < b used.
struct NlevConst {
  double gw[6], eion[6], rn[6];
  double xrat[5][5], enn[5][5], rnn[5][5], ann[5][5], bnn[5][5], lgt[5][5];
  double an0[5], bn0[5], lgi[5];
  double eev[6];     // IRgetionpot's level energies (eV, default-real literals)
  // reciprocal forms of the FMA build: 1/xrat, gw(a)/gw(b), gw(a)/gw(6)/2
  double ixrat[5][5], gwq[5][5], gwh[5];
};

// Scalars and tables of one simulation, passed by value to every kernel.
struct KParams {
  int ndim;          // 1 or 2
  int ix, jx;        // array extents with ghosts
  int nx, ny;        // interior extents
  int m0, m1;        // ghost layers in x and y
  int nvm;           // ion planes (8 or 9); neutral planes follow
  int imp;           // exponential collision form
  int ir;            // an ionisation/recombination law is active (IR source and cfl bound)
  int irs;           // 2 or 3: set_IR's Popescu law, rates from every stage's state (FP64 form)
  int irl;           // 1, 2 or 3: set_IR runs before each cfl (with get_Te's energy rewrite)
  int irf;           // 1: set_IR type 1, rates frozen in irg between the time loop's set_IR calls
  int ir_type;       // IR energy form 0 (with the ionisation potential, set_IR type 4), 1 or 2
  int irn;           // set_IR type 4: the 6-level hydrogen model (FP64 form; irs = 4 as well)
  long long nc;      // ix*jx
  double gm, ro_lim, pr_lim, ac, safety;
  double igm1;       // 1/(gm-1)
  double c32g;       // 3/gm/2 of the explicit collision energy term
  double sg_all;     // safety*min over all dx, dy, dz (numerator of cmax)
  double col_lim;    // min(safety,0.3) or pip_imp_factor (cfl_pn_col)
  double ir_lim;     // min(safety,0.1) (cfl_pip_ir)
  double ir_chi, ir_ion, ir_rec;
  double decay[2];   // Dedner psi factor exp(-(dt_sub/dt)*safety*db_clean) per stage
  double dz0;        // dz(1)
  double hc_kapper;  // Spitzer coefficient of the implicit conduction (kapper)
  int col_type;      // set_collisional col_type: 0 constant alpha_c, 1..6 per cell (FP64 form)
  double ac_b2g;     // beta/2*gm of col_type 1, 3, 5
  double ac_sb;      // sqrt(beta/2*gm)
  double ir_c136, ir_n6, ir_c291, ir_c291n6;  // 13.6/Te_0, n_norm*1e6, 2.91e-14, their product
  double ir_recfac, ir_fp, ir_tfac, ir_sqtfac, ir_tir;  // rec_fac, f_p, tfac, sqrt(tfac), t_ir
  double ir_factor, ir_ionfac;  // set_IR type 1: factor = exp(-13.2/(T0/11605)), ion_fac
  double *irg;       // type 1: Gm_ion (nc values) then Gm_rec (nc values) of the last set_IR
  double *acf;       // alpha_c per cell of the last set_collisional (col_type >= 1), nc values
  int resi;          // flag_resi 1: resistive flux with the fixed eta field etaf; 2: eta from
                     // the stage state at every RK stage (resi_type), FP64 form
  const double *etaf;  // eta per cell, nc values (resi 1)
  int resi_type;       // resi 2: set_resistivity resi_type 2 (|curl B| switch) or 3 (drift law)
  double eta0, j_cri, vd_cri;  // eta_0 and the thresholds of resi_type 2 and 3
  unsigned long long *resi_bound;  // resi 2: cfl_resi's bound (ordered bits of a positive
                                   // double) of the eta of the last set_resistivity
  double resi_dt;    // cfl_resi's bound min(safety*gmin^2/max(eta,1e-8)) over the interior
                     // cells (+inf without resistivity); seeds the min-CFL reduction slot
  // set_IR type 4 (irn): exponential-integral table rows (yn, E0, E1, E2), its first
  // abscissa and range, the model's coefficients, level populations (6 planes: current and
  // the excitation update's target), colrat (36 planes, plane a + 6*b = colrat(a+1,b+1)),
  // ion_pot, and the normalisation of set_IR type 4 / IRgetionpot
  const double *nl_tab;
  long long nl_ntab;
  double nl_xmin, nl_xrange;
  const double *nl_rtab;  // FMA build: per table row r, 1/((x0-x1)(x0-x2)), 1/((x1-x0)(x1-x2)),
                          // 1/((x2-x0)(x2-x1)) of its rows r, r+1, r+2 (4 doubles a row)
  double nl_xsc;          // ntab / xrange
  const NlevConst *nl_k;
  double *nl_nex, *nl_nex2, *nl_cr, *nl_ip;
  int nl_deriv;      // convective derivative: 0 none, 1 two-point, 4 five-point
  int nl_odd;        // mod(flag_col,2) == 1
  double nl_T0, nl_tfac, nl_n0, nl_n0fac, nl_gref, nl_tir;
  double nl_en_even; // beta/T0/2/8.6173e-5 (even flag_col)
  double nl_lim;     // min(safety,0.01) of cfl_pip_ir_nexcite
  const double *dx, *dy;
  const double *rdx, *rdy;   // 1/dx, 1/dy (FP32-mixed form only; null otherwise)
  // boundary maps: ghost layer q of side s (0 lower, 1 upper) copies interior index g?[s][q]
  int gx[2][kMaxMargin], gy[2][kMaxMargin];
  signed char symx[2][kMaxPlanes], symy[2][kMaxPlanes];
  int typex[2], typey[2];
};

// Device-resident loop state of pip_run (main.f90's time, dt and stop flags).
struct DevCtrl {
  double dt, cmax, time, time_next, t_end;
  long long step, nsteps;
  unsigned long long red_dt[2];   // min CFL candidate (positive doubles as ordered bits)
  unsigned long long red_rho[2];  // max rho*alpha_c
  unsigned long long red_gr[2];   // max IR rate
  unsigned long long red_ip[2];   // set_IR type 4, flag_IR_type 0: max(ion_pot/e_int, 1e-5)
  unsigned long long red_nx[2];   // set_IR type 4: max(dNexcite/dt, 1e-5)
  int last, done, nan_flag, status;
  unsigned int blocks_done;       // last-block-done counter of the stage-2 kernel
};

// Host launchers (one set per arithmetic flavour: FMA-contracted or FMA-free).
struct Launchers {
  cudaError_t (*prepare)();
  // tm: the TMA map of Us for the 2D tiles (tile_map), or null for per-thread loads.  rows
  // (2D): 0 every tile row; 1 the first and the last tile row (those a y-halo exchange
  // sends); 2 the rows between them.  A stage launched as 1 then 2 equals one launch of 0.
  cudaError_t (*stage)(const KParams &p, int stage, const double *Us, const double *U0, double *Uo,
                       DevCtrl *ctrl, int dt_mode, int epi, cudaStream_t s, const CUtensorMap *tm,
                       int rows);
  cudaError_t (*cfl)(const KParams &p, double *U, DevCtrl *ctrl, int slot, cudaStream_t s);
  cudaError_t (*ghosts)(const KParams &p, double *U, cudaStream_t s);
  cudaError_t (*flux)(const KParams &p, const double *U, double *F, int dir, double cmax,
                      cudaStream_t s);
  cudaError_t (*source)(const KParams &p, double *U, double *S, double dt_coll, cudaStream_t s);
  cudaError_t (*nan_scan)(const KParams &p, const double *U, int *flag, cudaStream_t s);
  cudaError_t (*coefficients)(const KParams &p, double *U, cudaStream_t s);
  // the TMA map of a stage source U (nvm+5 FP64 planes) for the 2D stage kernels' tiles;
  // false where the grid or the address breaks the TMA's alignment rules
  bool (*tile_map)(const KParams &p, const double *U, CUtensorMap *map);
  // set_IR type 4.  nlev_ref: colrat at (T_norm, n_norm) with cell (1,1,1)'s populations
  // into out[0..35] (out[a*6+b] = colrat(a+1,b+1)) and that cell's recombination sum
  // (Gm_rec_ref) into out[36].  nlev_rates: set_IR over every cell of U (colrw: a
  // set_collisional rewrite comes first; ipmode 0 no ion_pot, 1 ion_pot from the new colrat,
  // 2 from crref), writing colrat, the rates into irg and ion_pot; status 9 into ctrl on a
  // negative rate.  nlev_update: hydrogen_excitation_update after stage `stage` (dt from
  // ctrl), nl_nex -> nl_nex2 with its ghosts.  nlev_cfl: cfl_pip_ir's type-4 terms and
  // cfl_pip_ir_nexcite into slot `slot`.
  cudaError_t (*nlev_ref)(const KParams &p, double *out, cudaStream_t s);
  cudaError_t (*nlev_rates)(const KParams &p, const double *U, int colrw, int ipmode,
                            const double *crref, DevCtrl *ctrl, cudaStream_t s);
  cudaError_t (*nlev_update)(const KParams &p, const double *U, const DevCtrl *ctrl, int stage,
                             cudaStream_t s);
  cudaError_t (*nlev_cfl)(const KParams &p, double *U, DevCtrl *ctrl, int slot, cudaStream_t s);
};

const Launchers &launchers_fast();
const Launchers &launchers_exact();

}  // namespace pip

struct pip_params;
namespace pip {

// Implicit conduction of the ions (pip_conduction.cu): buffers for one grid; mixed = FP32
// inner BiCGstab with FP64 iterative refinement.  hc_run works on the FP64 state U (ion
// planes first) with dt read from the device; the ghost cells of U are left for the caller
// to fill.  status: 0 or PIP_ERR_ITER.
struct HcEngine;
cudaError_t hc_create(const KParams &k, bool mixed, HcEngine **out);
void hc_destroy(HcEngine *e);
// Polls of a staging mbarrier before a BiCGstab block gives up and flags the solve as
// failed (polls < 0: the default); applies from the next solve.
void hc_set_wait_limit(HcEngine *e, int polls);
void hc_set_loop(HcEngine *e, int device_loop);
// Distributed BiCGstab (BiCGstabMPI) in phases, for a block with neighbouring ranks across
// y faces: hcd_begin sets up te, the matrix (folded on the physical faces only) and the
// residual of the state U (ghost rows holding the neighbours' rows) and returns the local
// sums (r,r), (b,b); hcd_phase runs phase 0 (p = r), 1 (Ap = A p; sums (r,r0), (r0,Ap)), 2
// (t = r - coef[0] Ap, At; sums (t,At), (At,At)), 3 (x += coef[0] p + coef[1] t), 4 (r = b - A x;
// sums (r0,r), (r,r)) or 5 (p = r + coef[0] (p - coef[1] Ap)); hcd_vector gives the device
// plane of vector 0 (x), 1 (r) or 2 (Ap) for the halo rows; hcd_end writes te back into the
// energy of the interior cells.
cudaError_t hcd_begin(HcEngine *e, const KParams &k, double *U, const double *dtp, cudaStream_t s,
                      double sums[2]);
cudaError_t hcd_phase(HcEngine *e, const KParams &k, int phase, const double coef[2], cudaStream_t s,
                      double sums[2]);
double *hcd_vector(HcEngine *e, int vec);
cudaError_t hcd_end(HcEngine *e, const KParams &k, double *U, cudaStream_t s);
cudaError_t hc_run(HcEngine *e, const KParams &k, double *U, const double *dtp, double tol,
                   int hc_max, cudaStream_t s, int *iters, double *relres, int *status);

// Halo messages of mpi_bnd (pip_halo.cu): elements per array of face f's message, and the
// copies between the state arrays (a1 may be null) and a message buffer.
long long halo_elems(const KParams &p, int face);
cudaError_t halo_pack(const KParams &p, int face, const void *a0, const void *a1, int elem_bytes,
                      void *buf, cudaStream_t s);
cudaError_t halo_unpack(const KParams &p, int face, void *a0, void *a1, int elem_bytes,
                        const void *buf, cudaStream_t s);

// Records a CUDA error code for pip_last_cuda_error (pip_capi.cu).
void record_cuda_error(int code);

// The 6-level model's cell-independent coefficients (pip_nlevel.cu).
void nlev_constants(NlevConst *k);

// Validates a parameter block and fills the kernel parameters without allocating
// (pip_capi.cu); dx and dy of the result are left null.
int kparams_from_params(const pip_params *p, KParams *k);

// FP32-mixed form (pip_mixed.cu): A = (hi, lo) FP32 pair, B = FP32 stage state.
cudaError_t mixed_prepare();
cudaError_t mixed_stage(const KParams &p, int stage, const float *Us, const float *U0hi,
                        const float *U0lo, float *Ohi, float *Olo, DevCtrl *ctrl, int dt_mode,
                        int epi, cudaStream_t s, const CUtensorMap *tm = nullptr,
                        int rows = 0);
// The TMA map of the stage source Us (an array of nvm+5 FP32 planes) for the 2D mixed stage
// kernels' tiles; false (use per-thread loads) where the grid or the address breaks the
// TMA's alignment rules.
bool mixed_tile_map(const KParams &p, const float *Us, CUtensorMap *map);
cudaError_t mixed_cfl(const KParams &p, float *hi, float *lo, DevCtrl *ctrl, int slot,
                      cudaStream_t s);
cudaError_t mixed_split(const double *U, float *hi, float *lo, long long n, cudaStream_t s);
cudaError_t mixed_join(const float *hi, const float *lo, double *U, long long n, cudaStream_t s);

}  // namespace pip
