/*
 * pip_gpu.h -- C ABI of the B200 (sm_100a) two-fluid finite-volume step of PIP.
 *
 * The Fortran driver of PIP calls a fixed set of module procedures per time step
 * (main.f90:31-68): cfl, run_solver, and through run_solver set_flux, source_PIP and
 * PIPbnd.  Each entry point below replaces one of those calls.  All arrays crossing this
 * boundary are the Fortran arrays themselves: FP64, column-major U(ix,jx,kx,nvar) with
 * ghost cells included (Globalvar.f90:17), passed by address (c_loc / assumed size).
 * The host keeps ownership of its arrays; the context owns the device copies.
 *
 * Errors: every int-returning call returns PIP_OK (0) or one of pip_status_code.  No call
 * stops the process (the Fortran code's `stop` becomes a status code), mirroring the
 * flag_stop convention of stop_sim (IO_rot.f90:625-674).
 *
 * Threading: one context per MPI rank and per device; calls on one context are not
 * re-entrant.  Calls are synchronous with respect to the host buffers they take.
 */
#ifndef PIP_GPU_H
#define PIP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIP_ABI_VERSION 1

enum pip_status_code {
  PIP_OK = 0,
  PIP_ERR_PARAM = 1,   /* parameter block unsupported or inconsistent (get_parameters checks) */
  PIP_ERR_CUDA = 2,    /* a CUDA runtime call failed; pip_last_cuda_error() has the code */
  PIP_ERR_NAN = 3,     /* NaN in the state (stop_sim, IO_rot.f90:641-668) */
  PIP_ERR_DT = 4,      /* dt <= 1e-12 (stop_sim, IO_rot.f90:636-640) */
  PIP_ERR_ITER = 5,    /* an iterative solver or bounded device loop hit its limit */
  PIP_ERR_STATE = 6,   /* call out of order, e.g. a step before any upload */
  PIP_ERR_NOMEM = 7,   /* device allocation failed */
  PIP_ERR_NULL = 8,    /* a required pointer argument was NULL */
  PIP_ERR_RATE = 9     /* a rate of the 6-level hydrogen model came out negative (where
                          get_col_ion_coeff stops the run, PIP_rot.f90:546-557,592-601) */
};

enum pip_precision {
  PIP_FP64 = 0,        /* plain FP64 path: the drop-in, parity-checked against the oracle */
  PIP_MIXED = 1        /* FP32 fluxes/state, FP64 coupling source and compensated RK sums */
};

/* Ionisation/recombination laws accepted in pip_params.flag_ir. */
enum pip_ir_law {
  PIP_IR_NONE = 0,
  /* set_IR type 1 (PIP_rot.f90:135-149, marked work in progress there): rates from T_norm,
   * n_norm and t_ir; computed by the time loop's set_IR before each cfl (main.f90:32-34,44-46)
   * and at the prologue, after get_Te's energy rewrite, and frozen over the step. */
  PIP_IR_JEFFERY = 1,
  /* set_IR type 2 (PIP_rot.f90:148-170): Popescu et al. 2019 empirical rates with the
   * electron temperature T_norm/1.1604e4 eV and n_norm; recomputed with set_coefficients at
   * every RK stage (Solver_rot.f90:111) and before each cfl (main.f90:32-34,44-46), each time
   * after get_Te's energy rewrite (Scheme_rot.f90:83-128). */
  PIP_IR_POPESCU = 2,
  /* set_IR type 3 (PIP_rot.f90:173-228): the type-2 rates scaled to the ionisation
   * equilibrium of T_norm (f_n, f_p, tfac from flag_col's parity and beta); same calls. */
  PIP_IR_POPESCU_EQ = 3,
  /* set_IR type 4 (PIP_rot.f90:232-311): the 6-level hydrogen atom (Johnson 1972 collisional
   * rates, PIP_rot.f90:361-616) with level populations Nexcite advanced after every RK stage
   * (hydrogen_excitation_update, PIP_rot.f90:1026-1159).  Needs pip_set_nlevel (the
   * exponential-integral table and the model's settings) and pip_set_nexcite; FP64 form. */
  PIP_IR_NLEVEL = 4,
  /* Gm_ion = ir_ion_coef*T^-1/2*exp(-ir_chi/T), Gm_rec = ir_rec_coef*T^-1/2 with
   * T = gm*p_i/(2 rho_i) (get_Te_MHD, Scheme_rot.f90:104-110); the rates are frozen at
   * the start of each step as set_IR is (main.f90:32-34).  This law is new: none of
   * set_IR's types 1-4 (PIP_rot.f90:134-310) has it. */
  PIP_IR_POWERLAW = 5
};

/*
 * Parameter block: mirrors the globalvar module (Globalvar.f90) after get_parameters
 * (Model_rot.f90:39-333) and set_coordinate (Model_rot.f90:394-458) have run.
 * Supported subset (anything else returns PIP_ERR_PARAM):
 *   flag_eqs=PIP (two-fluid), flag_sch=0, flag_hll=2, s_order=2, t_order=2, flag_time=0,
 *   ndim 1 or 2 (kx=1), flag_divb 0/1 (forced 0 in 1D), flag_col 1..7 (2..7 with
 *   precision PIP_FP64 only),
 *   flag_pip_imp 0/1, flag_ir 0, PIP_IR_JEFFERY, PIP_IR_POPESCU, PIP_IR_POPESCU_EQ,
 *   PIP_IR_NLEVEL (FP64 form; T_norm and n_norm > 0) or PIP_IR_POWERLAW, with flag_ir_type
 *   1 or 2 (or 0, the ionisation-potential form, with PIP_IR_NLEVEL),
 *   flag_bnd in {1,2,3,4,5,6,7,10,11}, flag_resi 0, 1 (a fixed eta field) or 2 (eta
 *   recomputed at every RK stage, resi_type 2 or 3; FP64 form, not with flag_heat), no
 *   viscosity/gravity/ambipolar diffusion.
 */
typedef struct pip_params {
  int32_t abi_version;     /* must equal PIP_ABI_VERSION */
  int32_t ndim;            /* 1 or 2 */
  int32_t ix, jx, kx;      /* cells per axis including ghosts: ix = ix0 + 2*margin(1) */
  int32_t margin[3];       /* ghost layers per axis (Model_rot.f90:282-289,319-330) */
  int32_t nvar_h;          /* neutral (hydro) variables: 5 */
  int32_t nvar_m;          /* ion (MHD) variables: 8, or 9 with the Dedner psi */
  int32_t flag_sch;        /* 0: HLL branch */
  int32_t flag_hll;        /* 2: HLLD ions, HLLC neutrals */
  int32_t s_order;         /* 2: minmod MUSCL */
  int32_t t_order;         /* 2: midpoint RK2 */
  int32_t flag_time;       /* 0: standard RK (Solver_rot.f90:203-220) */
  int32_t flag_divb;       /* 1: Dedner 9-wave cleaning */
  int32_t flag_col;        /* 1: alpha_c = col everywhere (set_collisional col_type 0);
                              2..7: col_type 1..6, alpha_c per cell from both species'
                              temperatures (and drift) at the start of every RK stage
                              (PIP_rot.f90:44-97, set_coefficients Solver_rot.f90:95-122) */
  int32_t flag_pip_imp;    /* 0: explicit collision source; 1: exponential form */
  int32_t flag_ir;         /* pip_ir_law */
  int32_t flag_ir_type;    /* IR energy exchange: 1 Khomenko, 2 Singh (PIP_rot.f90:1399-1411),
                              0 with the ionisation potential IRgetionpot (:1381-1397, set_IR
                              type 4 only) */
  int32_t flag_heat;       /* 0 or 1 (implicit anisotropic conduction of the ions) */
  int32_t hc_max;          /* BiCGstab iteration limit */
  int32_t flag_bnd[6];     /* x_l, x_r, y_l, y_r, z_l, z_r boundary codes */
  int32_t precision;       /* pip_precision */
  int32_t fp_exact;        /* 1: FP64 kernels built without FMA contraction (bitwise
                              comparable with an FMA-free CPU build); 0: contracted */
  int32_t flag_resi;       /* 0, or 1: resistive flux with a fixed eta field (resistive_flux,
                              Solver_rot.f90:505-638, flag_sch=0 branch; cfl_resi,
                              Scheme_rot.f90:291-302); eta = eta_0 everywhere unless
                              pip_set_resistivity gives the field (FP64 form only);
                              2: eta from the stage state at the start of every RK stage
                              (set_resistivity resi_type 2 or 3, Res_rot.f90:37-60, called by
                              set_coefficients, Solver_rot.f90:98-101) -- the setting's
                              flag_resi = 22 or 32 */
  int32_t resi_type;       /* flag_resi 2: 2 anomalous eta = 11 eta_0 where |curl B| >= j_cri
                              (else eta_0), 3 eta = eta_0 (|curl B|/rho_i/vd_cri - 1)^2 where
                              |curl B|/rho_i >= vd_cri (else 0) */
  int32_t reserved_i[4];
  double gm;               /* ratio of specific heats: gm_d/gm_n */
  double safety;           /* CFL number */
  double ro_lim, pr_lim;   /* density and pressure floors */
  double col;              /* collision coefficient alpha_c */
  double db_clean;         /* Dedner psi damping ratio */
  double pip_imp_factor;   /* dt bound factor of the exponential collision form */
  double t_ir;             /* unused by PIP_IR_POWERLAW; kept for set_IR parity */
  double ir_chi;           /* ionisation potential in code temperature units */
  double ir_ion_coef;      /* ionisation rate coefficient */
  double ir_rec_coef;      /* recombination rate coefficient */
  double kapper;           /* Spitzer coefficient: kappa_par = kapper*T^2.5 */
  double hc_error;         /* BiCGstab relative residual target */
  double beta;             /* plasma beta of set_collisional col_type 1, 3, 5 (> 0 there) */
  double eta_0;            /* uniform resistivity (set_resistivity resi_type 0) */
  double t_norm, n_norm;   /* T0 (K) and n0 of the normalisation (setting keys T_norm, n_norm;
                              set_IR types 2 and 3) */
  double j_cri, vd_cri;    /* thresholds of resi_type 2 and 3 (setting keys j_cri, vd_cri) */
  double reserved_d[1];
  const double *dx;        /* ix cell widths (dsc(:,1)) */
  const double *dy;        /* jx cell widths (dsc(:,2)); 1D: one entry, the reference sets 100 */
  const double *dz;        /* kx cell widths (dsc(:,3)); one entry, the reference sets 100 */
} pip_params;

typedef struct pip_ctx pip_ctx;

/* Replaces the tail of prologue (Initial_rot.f90:140-160): validates the parameters,
 * allocates the device state and builds the boundary tables (initialize_bnd,
 * Boundary_rot.f90:20-32, set_sym_mhd/hd :239-320). */
int pip_ctx_create(const pip_params *p, pip_ctx **out);

/* Replaces epilogue's release of the state (IO_rot.f90 epilogue). */
void pip_ctx_destroy(pip_ctx *ctx);

/* Host -> device copy of U_h(ix,jx,kx,nvar_h) and U_m(ix,jx,kx,nvar_m) (FP64, with ghosts).
 * Called after the initial condition is set (Initial_rot.f90:46-140) or after restart
 * (IO_rot.f90:405-459). */
int pip_upload(pip_ctx *ctx, const double *U_h, const double *U_m);

/* Device -> host copy of the current state including its ghost cells (every stage and
 * pip_fill_ghosts keep them filled); feeds output() (IO_rot.f90:39-105), whose HDF5
 * layout stays with the Fortran host. */
int pip_download(pip_ctx *ctx, double *U_h, double *U_m);

/* cfl(U_h,U_m,dt) (Scheme_rot.f90:183-213): floors and rewrites the state through
 * primitives (cq2pv_mhd/hd, :132-179), returns the CFL time step (cfl_mhd :245-289,
 * cfl_hd :215-243, cfl_pn_col :305-313) and the Dedner speed
 * cmax = safety*min(dx,dy,dz)/dt (:203-211).  The cmax kept for the next pip_step is the
 * value computed with this dt, as the Fortran global cmax is. Either pointer may be NULL. */
int pip_cfl(pip_ctx *ctx, double *dt, double *cmax);

/* run_solver(U_h,U_m) (Solver_rot.f90:42-81): t_order RK stages of fluxes (HLLD/HLLC),
 * collisional source, conservative update and ghost fill with the given dt. */
int pip_step(pip_ctx *ctx, double dt);

/* Allocation-free run_solver.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a host code whose device memory is owned by
 * someone else (an OpenACC or CUDA Fortran data region, a fixed-size memory pool of the
 * application) or that must not allocate on its stepping path.  Same computation as
 * pip_step with the FP64 kernels (the two RK stages with their ghost fill), on a state the
 * caller already holds on the device:
 * U_dev is the device image of U_m followed by U_h (nvar_m + 5 planes of ix*jx doubles,
 * Fortran order, ghosts included), updated in place.  dt and cmax are what cfl returned
 * (pip_cfl, or the caller's own).  The work is queued on `stream` (a cudaStream_t; NULL for
 * the legacy default stream) and the call returns without waiting for it.
 *
 * The U1 stage buffer, the control block and device copies of dx/dy live in one
 * file-scope device array of PIP_NOALLOC_SCRATCH_BYTES that every GPU loading this
 * library holds until the process exits.  Limits: ix*jx <= PIP_NOALLOC_MAX_CELLS and
 * ix, jx <= PIP_NOALLOC_MAX_AXIS; larger grids, the mixed precision form, implicit
 * conduction (flag_heat = 1: pip_step's BiCGstab after the stages needs a context's
 * buffers), per-cell alpha_c (flag_col >= 2), resistivity, set_IR types 1-3 and any
 * parameter pip_ctx_create would reject return PIP_ERR_PARAM before any GPU work.  The
 * call reads p->dx and p->dy (host arrays) while it runs.  The first call on each
 * device looks up that array's device address and sets the kernels' shared-memory limit;
 * make that first call before any stream capture.  All calls share the one array and it
 * keeps the previous call's contents (the control block is rewritten by every call), so
 * calls whose GPU work overlaps race with each other: serialise them, e.g. on one stream.
 * The call itself allocates nothing on the device or the host. */
#define PIP_NOALLOC_MAX_CELLS 262144
#define PIP_NOALLOC_MAX_AXIS 8192
#define PIP_NOALLOC_SCRATCH_BYTES \
  (256 + 2 * 8 * PIP_NOALLOC_MAX_AXIS + 14 * 8 * (long long)PIP_NOALLOC_MAX_CELLS)
int pip_step_noalloc(const pip_params *p, double *U_dev, double dt, double cmax, void *stream);

/* The time loop of main.f90:31-68 on the device: repeats {cfl; run_solver; cfl;
 * time += dt; stop_sim} until nsteps steps are done (nsteps <= 0: no step limit) or
 * time >= t_end (t_end <= 0: no time limit).  The per-step dt and the stop checks stay on
 * the device.  Returns the status of stop_sim (PIP_ERR_NAN / PIP_ERR_DT) if it fired.
 * time_out and steps_done (either may be NULL) receive the simulation time and the number
 * of steps taken. */
int pip_run(pip_ctx *ctx, int64_t nsteps, double t_end, double *time_out, int64_t *steps_done);

/* Simulation time kept by the context (Globalvar `time`); pip_run advances it. */
int pip_set_time(pip_ctx *ctx, double time);
int pip_get_time(pip_ctx *ctx, double *time);

/* set_flux (Solver_rot.f90:124-159) for one direction dir (1..ndim) of the current state:
 * F_h(ix,jx,kx,nvar_h) and F_m(ix,jx,kx,nvar_m) hold the flux through the face between
 * cells i and i+1 (x) or j and j+1 (y) at index i (j), as in the Fortran F arrays.
 * Faces adjacent to interior cells are computed; the other entries are set to zero.
 * Uses the cmax of the last pip_cfl for the Dedner components. */
int pip_flux(pip_ctx *ctx, int dir, double *F_h, double *F_m);

/* source_PIP (PIP_rot.f90:1309-1429) on the current state with collision sub-step dt_coll.
 * Like the Fortran routine it rewrites the state through primitives (cq2pv).  With
 * flag_pip_imp=0 it returns S_h, S_m (the rates added by add_source); with
 * flag_pip_imp=1 it returns the increments the exponential form adds to U0
 * (-dt_coll*dS for the neutrals, +dt_coll*dS for the ions). */
int pip_source(pip_ctx *ctx, double dt_coll, double *S_h, double *S_m);

/* set_coefficients(U_h,U_m,1) (Solver_rot.f90:95-122), collision part: with flag_col
 * 2..7, set_collisional (PIP_rot.f90:44-97) rewrites both energies through the floored
 * pressure (get_Te_MHD/get_Te_HD, Scheme_rot.f90:83-128) and sets alpha_c per cell from
 * the temperatures and the drift; pip_source then uses that field.  No-op for flag_col 1.
 * pip_step, pip_run and pip_stage make the field themselves at the start of every stage.
 * After pip_upload the first call that needs the field (pip_cfl, pip_step, pip_run,
 * pip_stage, pip_flux, pip_source, pip_dev_begin, pip_get_alpha_c) runs this first, as
 * the prologue's set_coefficients(U_h,U_m,0) (Initial_rot.f90:140) does. */
int pip_coefficients(pip_ctx *ctx);

/* alpha_c per cell (ix*jx doubles, Fortran order; the globalvar `ac` array that output()
 * saves as "ac", IO_rot.f90:235): the field of the last set_collisional, or col
 * everywhere for flag_col 1. */
int pip_get_alpha_c(pip_ctx *ctx, double *ac);

/* Restart's read of the "ac" dataset (reread_variables, IO_rot.f90:570-572): sets the
 * field the first cfl after a pip_upload uses instead of making one from the state.
 * No-op for flag_col 1. */
int pip_set_alpha_c(pip_ctx *ctx, const double *ac);

/* set_resistivity (Res_rot.f90:16-60) for flag_resi 1: the eta field (ix*jx doubles,
 * Fortran order, ghosts included) that resistive_flux and cfl_resi use from the next call
 * on; eta_0 everywhere until called.  PIP_ERR_PARAM without flag_resi 1. */
int pip_set_resistivity(pip_ctx *ctx, const double *eta);

/* cfl_resi's bound (Scheme_rot.f90:291-302) of the current eta: min over the interior cells
 * of safety*min(dx,dy,dz)**2/max(eta,1e-8).  With flag_resi 2 the eta is set_resistivity's
 * of the last RK stage (or of the uploaded state before the first step).  cfl_resi writes
 * the Fortran global dt rather than cfl's argument, so after run_solver the time loop's
 * cfl(U_h,U_m,dtnew) lowers the dt that `time` advances by (main.f90:47,58): a host that
 * steps with pip_step and pip_cfl applies dt = min(dt, bound) before time = time + dt.
 * pip_run does this itself.  PIP_ERR_PARAM without resistivity. */
int pip_resi_dt(pip_ctx *ctx, double *bound);

/* PIPbnd(U_h,U_m,0) (Boundary_rot.f90:34-52) on the device state; with one rank the
 * MPI halo exchange (MPI_rot.f90:128-339) reduces to this ghost fill. */
int pip_fill_ghosts(pip_ctx *ctx);

/* stop_sim's flags for the device state (IO_rot.f90:625-674): *nan_flag = 1 if any
 * variable of either species is NaN or Inf; *stop_flag = 1 if the NaN flag is set or
 * the last dt was <= 1e-12.  Either pointer may be NULL. */
int pip_status(pip_ctx *ctx, int *stop_flag, int *nan_flag);

/* Implicit anisotropic conduction of the ion species over dt: HC(U_m,nvar_m,1)
 * (HC_rot.f90:67-140) with the 9-point matrix (set_matrix_source_MHD2D9, :643-739) and
 * BiCGstab (:187-299).  Returns PIP_ERR_ITER if hc_max iterations did not reach
 * hc_error.  iters and relres (either may be NULL) receive the iteration count and the
 * final relative residual. */
int pip_conduction(pip_ctx *ctx, double dt, int *iters, double *relres);

/* Diagnostic; no counterpart in the reference.  The BiCGstab kernels stage their rows with
 * bulk async copies and wait for each on an mbarrier a bounded number of polls; a block
 * whose wait runs out flags the solve, waits (bounded by the default limit) for its copies
 * still in flight and returns, the remaining kernels of the solve return at once, and
 * pip_conduction / pip_step / pip_run return PIP_ERR_CUDA with pip_last_cuda_error() =
 * cudaErrorLaunchTimeout (702); the context stays usable (upload a state and go on).
 * This sets the number of polls from the next solve on (polls < 0: the default, 2^22);
 * 0 makes every wait run out at once, which exercises that path.  PIP_ERR_PARAM without
 * flag_heat = 1. */
int pip_set_hc_wait_limit(pip_ctx *ctx, int polls);

/* Diagnostic; no counterpart in the reference.  How a BiCGstab solve schedules its
 * iterations: device_loop = 1 (the default) as one device-side loop (a CUDA graph whose
 * conditional while node runs the iterations until the last kernel of an iteration ends it:
 * one host wait per solve; a device or stream that cannot build that graph falls back to
 * 0), 0 in groups of four after each of which the host reads the stop flag.  Both run the
 * same kernels on the same buffers, so the results and iteration counts are identical.
 * PIP_ERR_PARAM without flag_heat = 1 or for another value. */
int pip_set_hc_loop(pip_ctx *ctx, int device_loop);

/*
 * Implicit conduction of a decomposed run: BiCGstabMPI (HC_rot.f90:303-466) for a block
 * whose y faces border other ranks (pip_set_neighbors; x faces stay physical), driven by
 * the caller as the reference's loop with its MPI calls in between.  After stage 2 and its
 * halo exchange (ghost rows hold the neighbours' rows, so te and the matrix next to an
 * exchanged face are the undecomposed ones):
 *   pip_hcd_begin(ctx, dt, s)          te, the matrix (folded on physical faces only),
 *                                      r = b - A te; s = local (r,r), (b,b); SUM over ranks
 *   exchange vector 1 (r), then pip_hcd_phase(ctx, 0, 0, 0)            p = r
 *   while sqrt(R/B) > hc_error and count <= hc_max:
 *     pip_hcd_phase(ctx, 1, 0, s)      Ap = A p; s = (r,r0), (r0,Ap); SUM; alpha = S0/S1;
 *                                      exchange vector 2 (Ap)
 *     pip_hcd_phase(ctx, 2, {alpha}, s) t = r - alpha Ap, At; s = (t,At), (At,At); SUM;
 *                                      omega = S0/S1
 *     pip_hcd_phase(ctx, 3, {alpha, omega}, 0)   x = x + alpha p + omega t
 *     pip_hcd_phase(ctx, 4, 0, s)      r = b - A x; s = (r0,r), (r,r); SUM;
 *                                      beta = S0/(alpha's S0)*alpha/omega, R = S1;
 *                                      exchange vector 1 (r)
 *     pip_hcd_phase(ctx, 5, {beta, omega}, 0)    p = r + beta (p - omega Ap); count += 1
 *   pip_hcd_end(ctx, count)            te back into the ion energy (interior cells), ghosts
 *                                      of the physical faces; then the state's exchange
 * A vector exchange moves one row per face: pip_hcd_pack(ctx, vec, f, send) copies the row
 * the rank across face f (2 = y-, 3 = y+) needs into the device buffer send
 * (pip_hcd_row_bytes), pip_hcd_unpack(ctx, vec, f, recv) stores the row received from it.
 * Every scalar is the global one; the reference takes omega from the rank's own sums
 * (HC_rot.f90:425-427), which makes its iterates depend on the decomposition.  FP64 vectors
 * for either precision form.  PIP_ERR_PARAM without flag_heat = 1.
 */
int pip_hcd_begin(pip_ctx *ctx, double dt, double sums[2]);
int pip_hcd_phase(pip_ctx *ctx, int phase, const double coef[2], double sums[2]);
int64_t pip_hcd_row_bytes(pip_ctx *ctx);
int pip_hcd_pack(pip_ctx *ctx, int vec, int face, void *send);
int pip_hcd_unpack(pip_ctx *ctx, int vec, int face, const void *recv);
int pip_hcd_end(pip_ctx *ctx, int iters);

/*
 * set_IR type 4 (flag_ir = PIP_IR_NLEVEL): the 6-level hydrogen model.
 *
 * The Fortran keeps the model's state in globalvar (Nexcite, colrat, ion_pot, Gm_rec_ref)
 * and reads expintcalc/colexp.dat once (expintread, PIP_rot.f90:315-357, called by the
 * initial condition).  Here:
 *   pip_colexp_table   regenerates that table: colexpintcalc.f90's rows (yn, E0(yn), E1(yn),
 *                      E2(yn)) for yn = ymin + t*(108-ymin)/nsamps, t = 0..nsamps, as a
 *                      (4, nsamps+1) column-major array -- the layout expintread fills
 *                      expinttab with (the reference's file has nsamps = 100000).
 *   pip_set_nlevel     hands the table and the model's settings to the context; the next
 *                      prologue-like call (the first pip_cfl / pip_step / pip_run) runs set_IR
 *                      type 4's fresh-start block (PIP_rot.f90:250-280): Gm_rec_ref from the
 *                      rates at (T_norm, n_norm) with cell (1,1,1)'s populations, and the
 *                      initial ion_pot.
 *   pip_set_nexcite    Nexcite(ix,jx,kx,6): levels 1-5 then the ions, ghosts included, in
 *   pip_get_nexcite    the state's normalisation (the sum of levels 1-5 is rho_n); the
 *                      excitation update keeps Nexcite(6) = rho_i and the sum = rho_n.
 *   pip_get_colrat     colrat(ix,jx,kx,6,6) of the last set_IR.
 *   pip_get_ion_pot    ion_pot(ix,jx,kx) of the last source_PIP (flag_IR_type 0).
 *   pip_nlevel_gm_rec_ref  the normalisation rate Gm_rec_ref.
 * Every RK stage runs set_IR (the rates from the stage state), the stage, then
 * hydrogen_excitation_update over dt_sub (Solver_rot.f90:218-220); every cfl adds
 * cfl_pip_ir's and cfl_pip_ir_nexcite's bounds (Scheme_rot.f90:315-335).  pip_run steps on
 * the host (a launch per kernel), single rank only (pip_set_neighbors and pip_dev_begin return
 * PIP_ERR_PARAM).  Without pip_set_nlevel those calls return PIP_ERR_STATE.  A negative rate
 * (where get_col_ion_coeff stops the run) makes pip_run return PIP_ERR_RATE.
 */
typedef struct pip_nlevel {
  int32_t n_levels;        /* nlevels setting: 5 (the hydrogen atom's levels 1-5, then ions) */
  int32_t flag_rad;        /* 0 or 1: collisional rates only (flag_rad >= 2 adds
                              get_radrat_fixed's radiative rates, not built: PIP_ERR_PARAM) */
  int32_t deriv;           /* convective derivative of the excitation update: 1 the two-point
                              form, 4 the five-point form (derivative, Scheme_rot.f90:692-736,
                              for s_order 1 and 4), 0 none.  For s_order 2, the scheme of this
                              path, the reference's derivative sets nothing and the term reads
                              an uninitialised array, so the form is a setting here. */
  int32_t reserved;
  double n0fac;            /* globalvar n0fac, f_p_ini, f_p_p_ini (set by the initial */
  double f_p_ini;          /* condition, e.g. KHnlev.f90:103-105): electron density */
  double f_p_p_ini;        /* U_m(1)*n_norm/n0fac, tfac of PIP_rot.f90:240-248 */
} pip_nlevel;

int pip_colexp_table(int64_t nsamps, double *out);
int pip_set_nlevel(pip_ctx *ctx, const pip_nlevel *cfg, const double *table, int64_t nrows);
int pip_set_nexcite(pip_ctx *ctx, const double *nexcite);
int pip_get_nexcite(pip_ctx *ctx, double *nexcite);
int pip_get_colrat(pip_ctx *ctx, double *colrat);
int pip_get_ion_pot(pip_ctx *ctx, double *ion_pot);
int pip_nlevel_gm_rec_ref(pip_ctx *ctx, double *gm_rec_ref);

/* Gm_ion and Gm_rec (ix,jx,kx each) of the last set_IR, for output's "ion" and "rec"
 * datasets (IO_rot.f90:297-300): contexts that keep the rates between kernels, set_IR types
 * 1 and 4; PIP_ERR_PARAM for the laws the kernels evaluate in place. */
int pip_get_ir_rates(pip_ctx *ctx, double *gm_ion, double *gm_rec);

/*
 * Domain decomposition over ranks (one context per rank and device, each holding its own
 * block with ghost cells, as the Fortran code does after set_mpi, MPI_rot.f90:11-41).
 *
 * pip_set_neighbors replaces set_mpi_neighbor (MPI_rot.f90:90-126): neighbor[f] for faces
 * f = 0 (x-), 1 (x+), 2 (y-), 3 (y+) is the rank owning the block across the face, or -1
 * where the face is a physical boundary (faces beyond ndim must be -1).  Faces with a
 * neighbour get their ghost layers only from the halo exchange: the stage kernels and
 * pip_fill_ghosts apply flag_bnd to the other faces, as MHDbnd/HDbnd skip faces whose
 * neighbor is not -1 (Boundary_rot.f90:80-90).  With a neighbour on any face, pip_step and
 * pip_run return PIP_ERR_STATE (the exchange must come between the stages: step with
 * pip_stage); with flag_heat = 1 the split is along y and pip_stage(ctx, 2, ...) leaves the
 * conduction to the pip_hcd_* calls (above).
 *
 * pip_stage runs one RK stage of run_solver (Solver_rot.f90:59-71) with the given dt and
 * Dedner speed cmax: stage 1 then stage 2, each followed by PIPbnd's exchange
 * (pip_halo_pack / pip_halo_unpack on every face with a neighbour).  dt is the global one
 * (cfl's MPI_Allreduce MIN of the ranks' pip_cfl values, Scheme_rot.f90:201-202) and cmax
 * the maximum over ranks of safety*min(dx,dy,dz)/dt (:207-209).
 *
 * pip_halo_pack / pip_halo_unpack are the two halves of mpi_bnd (MPI_rot.f90:128-339):
 * pack copies the margin interior layers next to face f (all planes of the state the last
 * stage wrote, ghost cells of the other direction included) into `send`; unpack writes a
 * message received from the neighbour across face f into the ghost layers of face f.  A
 * message packed at face f is unpacked by the neighbour at the opposite face (f ^ 1).
 * send and recv are DEVICE buffers of at least pip_halo_bytes(ctx, f) bytes; *bytes gets
 * the message length, which the receiver passes to unpack (FP64 form: margin x extent x
 * (nvar_m + 5) doubles; FP32-mixed form after stage 1: half of that).
 *
 * pip_stage, pip_halo_pack and pip_halo_unpack queue their work on the context's stream
 * (pip_ctx_stream) and return without waiting for it, so a step needs no host round trip
 * between its stages: issue the message transfer on the same stream (NCCL send/recv on
 * that stream, or a copy queued there), or wait for the stream before touching the buffers
 * from elsewhere.  Errors of queued work surface at the next call that waits (pip_cfl,
 * pip_download, pip_status).
 */
int pip_set_neighbors(pip_ctx *ctx, const int neighbor[4]);
int pip_stage(pip_ctx *ctx, int stage, double dt, double cmax);
int pip_ctx_stream(pip_ctx *ctx, void **stream);

/*
 * Device-driven stepping of a decomposed run: the time loop of pip_run (main.f90:31-68)
 * with dt, cmax, time and the stop flags on the device, and the ranks' cfl reductions done
 * by the caller on device memory between steps -- no host round trip per step.
 *
 *   pip_set_cmax_scale(ctx, s)  once: s = MAX over ranks of safety*min(dx,dy,dz) (cfl's
 *                               cmax allreduce, Scheme_rot.f90:207-209, taken out of dt)
 *   pip_dev_begin(ctx, nsteps, t_end)   state as pip_run starts it; queues the first cfl
 *   reduce the candidates (below), then per step:
 *     pip_dev_stage(ctx, 1); exchange; pip_dev_stage(ctx, 2); exchange; reduce
 *   pip_dev_poll(ctx, &done, &time, &steps)   waits for the queued work and reports
 *
 * pip_dev_begin waits for the first cfl; pip_dev_stage queues on the context stream and
 * returns at once.  Stage 1 takes dt = min(dt_cfl, col_lim/rho_max, ir_lim/max(gr_max,
 * 1e-5)) from the reduced candidates and cmax = s/dt; stage 2 writes the next step's
 * candidates from its updated cells (the cfl after run_solver and the next step's cfl,
 * fused).  pip_dev_candidates gives their device addresses: dt_min is 2 int64 to reduce
 * with MIN, rho_gr_max 4 int64 to reduce with MAX (positive doubles as bit patterns, which
 * order like the doubles; both slots of each, as they lie in memory).  Every rank must
 * issue the same calls; a rank whose state stops (NaN, dt floor, last step) keeps
 * exchanging and reducing while its kernels do nothing, so the collectives stay matched.
 * pip_dev_poll returns PIP_ERR_NAN / PIP_ERR_DT like pip_run; *done is 1 once the loop has
 * ended.  Not with flag_heat = 1 (PIP_ERR_PARAM).
 */
int pip_set_cmax_scale(pip_ctx *ctx, double safety_min_d);
int pip_dev_begin(pip_ctx *ctx, int64_t nsteps, double t_end);
int pip_dev_stage(pip_ctx *ctx, int stage);

/* The y exchange overlapped with the stage (2D; no counterpart in the reference, whose
 * mpi_bnd runs after the whole stage).  pip_dev_stage_split(ctx, k, &bs) queues stage k
 * as two launches: the first and the last row of tiles -- every cell the exchange sends --
 * on a high-priority stream of the context, returned in bs, and the rows between them on
 * the context stream, concurrently; the context stream then waits for the boundary rows.
 * Together they equal pip_dev_stage(ctx, k) bit for bit.  The caller records an event on
 * bs right after the call and runs the exchange (pack, transfer, unpack) on a stream of its
 * own after that event while the middle rows compute; the context stream waits for the
 * exchange before the next stage.  The middle rows neither read nor write what the
 * exchange reads or writes (it reads the boundary rows' cells, it writes the ghost rows of
 * the exchanged faces, and a stage reads only its input array).
 * pip_set_halo_stream(ctx, stream) makes pip_halo_pack / pip_halo_unpack queue on `stream`
 * (NULL: the context stream again). */
int pip_dev_stage_split(pip_ctx *ctx, int stage, void **boundary_stream);
int pip_set_halo_stream(pip_ctx *ctx, void *stream);
int pip_dev_candidates(pip_ctx *ctx, void **dt_min, void **rho_gr_max);
int pip_dev_poll(pip_ctx *ctx, int *done, double *time, int64_t *steps);
int64_t pip_halo_bytes(pip_ctx *ctx, int face);
int pip_halo_pack(pip_ctx *ctx, int face, void *send, int64_t *bytes);
int pip_halo_unpack(pip_ctx *ctx, int face, const void *recv, int64_t bytes);

/* Last CUDA error code seen by any context (cudaError_t as int), 0 if none. */
int pip_last_cuda_error(void);

/* Text for a pip_status_code. */
const char *pip_strerror(int code);

#ifdef __cplusplus
}
#endif

#endif /* PIP_GPU_H */
