/*
 * pip_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of PIP's two-fluid finite-volume step, used as the correctness
 * checker of the CUDA library and as the timed CPU baseline.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity status: UNPINNED by the reference itself.  The reference ships no tests, golden
 * vectors or fixtures for this path and cannot be built here (Fortran 90 + MPI + parallel
 * HDF5, Makefile:29, MPI_rot.f90:7, Globalvar.f90:9; no Fortran compiler in the image).
 * The restatement follows the cited Fortran statement by statement (operation order and
 * parenthesisation kept, no FMA contraction) and is cross-checked by conservation,
 * symmetry and analytic-rate tests and by an independent numpy restatement.
 */
#ifndef PIP_ORACLE_H
#define PIP_ORACLE_H

#include "../include/pip_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const pip_params *p, int *status);
void orc_destroy(orc_ctx *c);
void orc_set_threads(int n);
int orc_get_threads(void);
void orc_set_state(orc_ctx *c, const double *U_h, const double *U_m);
void orc_get_state(const orc_ctx *c, double *U_h, double *U_m);
void orc_set_time(orc_ctx *c, double t);
double orc_get_time(const orc_ctx *c);
double orc_get_cmax(const orc_ctx *c);
void orc_set_cmax(orc_ctx *c, double cmax);

/* Scheme_rot.f90:183-213 (rewrites the state, returns dt and cmax). */
void orc_cfl(orc_ctx *c, double *dt, double *cmax);
/* Solver_rot.f90:42-81 with the given dt and the stored cmax. */
void orc_run_solver(orc_ctx *c, double dt);
/* One stage (1 or 2) of run_solver with the closing PIPbnd of the stage. */
void orc_stage(orc_ctx *c, int istep, double dt);
/* set_mpi_neighbor: faces x-, x+, y-, y+ with a neighbouring rank (>= 0) are skipped by
 * the boundary fill and left to the caller's halo exchange. */
void orc_set_neighbors(orc_ctx *c, const int nb[4]);
/* Solver_rot.f90:124-159 for one direction (1-based), F arrays (ix,jx,kx,nvar). */
void orc_flux(orc_ctx *c, int dir, double *F_h, double *F_m);
/* PIP_rot.f90:1309-1429; returns S (explicit) or the U0 increments (exponential form). */
void orc_source(orc_ctx *c, double dt_coll, double *S_h, double *S_m);
/* set_coefficients (Solver_rot.f90:95-122): with flag_col 2..7, set_collisional
 * (PIP_rot.f90:44-97) rewrites both energies and sets alpha_c per cell; with set_IR types 2
 * and 3, set_IR (PIP_rot.f90:127-228) rewrites them again and sets the rates. */
void orc_coefficients(orc_ctx *c);
/* Gm_ion and Gm_rec of the last set_IR (nc values each). */
void orc_ir_rates(const orc_ctx *c, double *gm_ion, double *gm_rec);
/* alpha_c of every cell (col for flag_col 1), made from the current state when no
 * set_collisional has run yet (Initial_rot.f90:140). */
int orc_alpha_c(orc_ctx *c, double *ac);
/* The eta field of set_resistivity (Res_rot.f90:16-60) for flag_resi 1 (nc values);
 * eta_0 everywhere until called. */
void orc_set_resistivity(orc_ctx *c, const double *eta);
/* The current eta field (nc values): the fixed field, or with flag_resi 2 the one
 * set_resistivity computed at the start of the last RK stage (or of the prologue). */
void orc_resistivity(orc_ctx *c, double *eta);
/* Boundary_rot.f90:34-52. */
void orc_bnd(orc_ctx *c);
/* main.f90:31-68 loop; returns 0, PIP_ERR_NAN or PIP_ERR_DT.  dt_hist (may be NULL)
 * receives up to max_hist per-step dt values. */
int orc_run(orc_ctx *c, long nsteps, double t_end, double *time_out, long *steps_done,
            double *dt_hist, long max_hist);
/* HC(U_m,nvar_m,1) (HC_rot.f90:67-140), 9-point matrix + BiCGstab on one rank, over dt;
 * returns PIP_OK or PIP_ERR_ITER; iters/relres may be NULL. */
int orc_conduction(orc_ctx *c, double dt, int *iters, double *relres);
/* BiCGstabMPI (HC_rot.f90:303-466) in the phases of pip_hcd_* (include/pip_gpu.h) for a
 * block with neighbours: orc_hcd_begin (sums (r,r), (b,b)), orc_hcd_phase 0..5 with coef
 * (alpha; alpha, omega; beta, omega) and sums, rows of vector 0 (x), 1 (r), 2 (Ap) for the
 * exchange, orc_hcd_end (the write-back of orc_conduction, every cell). */
int orc_hcd_begin(orc_ctx *c, double dt, double sums[2]);
int orc_hcd_phase(orc_ctx *c, int phase, const double coef[2], double sums[2]);
void orc_hcd_get_row(const orc_ctx *c, int vec, int row, double *out);
void orc_hcd_set_row(orc_ctx *c, int vec, int row, const double *in);
int orc_hcd_end(orc_ctx *c);
/* stop_sim's NaN scan (IO_rot.f90:641-668) over both species. */
int orc_has_nan(const orc_ctx *c);

/* set_IR type 4, the 6-level hydrogen model (PIP_rot.f90:232-311,361-616,874-946,
 * 1026-1235; Scheme_rot.f90:315-335,692-736,1002-1049).
 * orc_expint_table: colexpintcalc.f90's table, 4*(nsamps+1) values (yn, E0, E1, E2 per row).
 * orc_set_nlevel: deriv 0 (no convective term), 1 or 4 (the two- and five-point forms of
 * derivative); n0fac, f_p_ini, f_p_p_ini of globalvar; table as expintread holds it
 * (4 x nrows, column-major).  Resets the prologue's block (Gm_rec_ref, ion_pot).
 * Nexcite is (ix,jx,kx,6), colrat (ix,jx,kx,6,6), both column-major. */
void orc_expint_table(long nsamps, double *out);
int orc_set_nlevel(orc_ctx *c, int deriv, double n0fac, double f_p_ini, double f_p_p_ini,
                   const double *table, long nrows);
void orc_set_nexcite(orc_ctx *c, const double *nex);
void orc_get_nexcite(const orc_ctx *c, double *nex);
void orc_get_colrat(const orc_ctx *c, double *colrat);
void orc_get_ion_pot(const orc_ctx *c, double *ion_pot);
double orc_gm_rec_ref(const orc_ctx *c);
/* 1 once a rate came out negative (where the reference stops). */
int orc_nlevel_status(const orc_ctx *c);

#ifdef __cplusplus
}
#endif

#endif
