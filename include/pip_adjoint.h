/*
 * pip_adjoint.h -- discrete adjoint of the FP64 two-fluid step.
 *
 * No counterpart in the reference: PIP has no derivatives.  An adjoint handle runs the
 * FP64 time loop (the kernels and the arithmetic of pip_run, main.f90:31-68) forward from
 * a given state for a fixed number of steps, keeping the state every `checkpoint_every`
 * steps and each step's dt; pip_adj_backward then pulls a cotangent of the final state
 * back to the initial state and to alpha_c (pip_params.col), recomputing each segment of
 * steps from its checkpoint.  The derivative is that of the discrete step as executed:
 * every branch (minmod slope, HLLD fan region, HLLC-G fallback, wave-speed min/max,
 * floors inside the fluxes) is differentiated on the side taken, and dt = CFL(state) is
 * differentiated through the cell (or the collision bound) that sets it.  The cq2pv
 * rewrites of cfl (Scheme_rot.f90:153-179) are identities wherever no floor acts and are
 * taken as identities.
 *
 * Supported parameter blocks: precision PIP_FP64, ndim 1 or 2, flag_divb = 0,
 * flag_pip_imp = 0 (explicit collision source), flag_ir = PIP_IR_NONE, flag_heat = 0, any
 * boundary codes pip_ctx_create accepts.
 *
 * State arrays here are DEVICE pointers (on the device current at create time) to the
 * device layout of the context: nvar_m + 5 planes of ix*jx doubles (x fastest), ion
 * planes (ro, mx, my, mz, en, bx, by, bz) first, then neutral planes (ro, mx, my, mz, en).
 * Ghost cells are part of the state: the gradient with respect to the initial state
 * carries separate entries for the ghost cells given as input.
 */
#ifndef PIP_ADJOINT_H
#define PIP_ADJOINT_H

#include <stdint.h>

#include "pip_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pip_adj pip_adj;

/* Allocates device storage for runs of up to max_steps steps with a checkpoint every
 * checkpoint_every steps (<= 0: 25). */
int pip_adj_create(const pip_params *p, int64_t max_steps, int checkpoint_every, pip_adj **out);
void pip_adj_destroy(pip_adj *a);

/* Sets alpha_c for the following forward runs (the derivative is taken at this value). */
int pip_adj_set_col(pip_adj *a, double col);

/* Runs nsteps steps from U0 (device, not modified) and writes the final state to UN
 * (device; may equal U0).  device_ms (may be NULL) receives the device time of the run.
 * Returns PIP_ERR_NAN if the state stopped being finite, PIP_ERR_DT on a dt <= 1e-12. */
int pip_adj_forward(pip_adj *a, const double *U0, double *UN, int64_t nsteps, float *device_ms);

/* Given gN = dL/dUN (device) of the last forward run, writes g0 = dL/dU0 (device; may
 * equal gN) and *g_col = dL/dalpha_c.  device_ms (may be NULL) receives the device time
 * (recomputation included). */
int pip_adj_backward(pip_adj *a, const double *gN, double *g0, double *g_col, float *device_ms);

/* Unit-level pieces of the reverse sweep (for tests).  pip_adj_stage_vjp: for one RK stage
 * (stage 1 advances by dt/2, stage 2 by dt) from the stage state Us, writes the cotangent
 * of Us (every cell, device) for the cotangent lam of the stage output on interior cells
 * (device; ghost entries ignored), with *dot = dt_sub <lam, dU/d(dt_sub)> and
 * *dcol = <lam, dU/dalpha_c>.  pip_adj_fold: the adjoint of the ghost fill in place --
 * the cotangent of every ghost cell is added to the interior cell it copies. */
int pip_adj_stage_vjp(pip_adj *a, int stage, const double *Us, const double *lam, double *out,
                      double dt, double *dot, double *dcol);
int pip_adj_fold(pip_adj *a, double *lam);

/* The dt of each step of the last forward run (host array of n >= steps entries) and the
 * number of steps. */
int pip_adj_dt(pip_adj *a, double *dt, int64_t n, int64_t *steps);

#ifdef __cplusplus
}
#endif

#endif
