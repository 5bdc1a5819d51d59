/*
 * pip_bench.h -- measurement hooks of the B200 two-fluid step library.
 *
 * These calls have no counterpart in the reference (PIP times itself with MPI_Wtime only,
 * IO_rot.f90:48,56,270-273).  They time the device work with CUDA events recorded on the
 * context's own stream, around the kernels themselves.
 */
#ifndef PIP_BENCH_H
#define PIP_BENCH_H

#include <stdint.h>

#include "pip_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* pip_run with the device time of the launched work (events around the whole loop,
 * excluding the final host read of the control block) in *device_ms. */
int pip_run_timed(pip_ctx *ctx, int64_t nsteps, double t_end, double *time_out,
                  int64_t *steps_done, float *device_ms);

/* Runs nsteps steps of the pip_run loop with an event pair around every stage kernel and
 * returns the mean duration of one stage-1 launch, one stage-2 launch and one whole step
 * (ms).  Advances the state like pip_run(ctx, nsteps, 0, ...). */
int pip_bench_stage_ms(pip_ctx *ctx, int nsteps, float *ms_stage1, float *ms_stage2,
                       float *ms_step);

/* Number of kernels pip_run launches for nsteps steps (1 cfl pass + 2 per step; runs with
 * conduction add the BiCGstab kernels, see pip_conduction_iterations). */
int64_t pip_kernels_per_run(pip_ctx *ctx, int64_t nsteps);

/* BiCGstab iterations (inner iterations for the mixed form) of the last pip_run, pip_step
 * or pip_conduction of a flag_heat = 1 context. */
int64_t pip_conduction_iterations(pip_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif
