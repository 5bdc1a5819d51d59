/*
 * pip_ensemble.h -- batched ensembles of independent 1D and 2D two-fluid runs.
 *
 * No counterpart in the reference: PIP runs one simulation per process.  An ensemble holds
 * many runs of different sizes and parameters (each described by its own pip_params,
 * ndim = 1 or 2, precision = PIP_MIXED) and advances all of them to an end time in one
 * persistent kernel launch, captured in a CUDA graph: each thread block takes whole runs
 * from a work queue ordered longest first and steps each with its own dt.  A 1D run is
 * walked in chunks of cells, a 2D run tile by tile (16 x 14 cells) with the single-run
 * stage kernel's tile step.  Per-run arithmetic is that of the single-run FP32-mixed form.
 * An ensemble with a 2D run needs at least 256 threads per block.
 *
 * Each launch first estimates every run's work (interior cells x the steps its current dt
 * gives to the end) and orders the queue by it.  In an ensemble of 1D runs stepped by 256
 * or 512 threads per block, the runs whose work exceeds a quarter of an even share are each
 * shared by a thread-block cluster of 4 or 8 blocks (each block a contiguous part of the
 * cells, the cluster barrier between stages, the dt reduced over the cluster); the rest
 * go one per block.  A shared run takes the same steps as on one block; its state agrees
 * to the rounding that FMA contraction gives each kernel instance.
 */
#ifndef PIP_ENSEMBLE_H
#define PIP_ENSEMBLE_H

#include <stdint.h>

#include "pip_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pip_ensemble pip_ensemble;

/* n parameter blocks, one per run (validated as pip_ctx_create does). */
int pip_ensemble_create(const pip_params *members, int n, pip_ensemble **out);
void pip_ensemble_destroy(pip_ensemble *e);

/* Host -> device copy of one run's U_h, U_m (FP64, Fortran layout, ghosts included); resets
 * that run's time and step count. */
int pip_ensemble_upload(pip_ensemble *e, int member, const double *U_h, const double *U_m);

/* Advances every run to t_end (t_end <= 0: no time limit) or by max_steps steps
 * (max_steps <= 0: no step limit) in one graph launch.  device_ms (may be NULL) receives
 * the device time of the launch. */
int pip_ensemble_run(pip_ensemble *e, double t_end, int64_t max_steps, float *device_ms);

/* One run's state (U_h/U_m may be NULL), time, step count and stop status (0, PIP_ERR_NAN or
 * PIP_ERR_DT). */
int pip_ensemble_member(pip_ensemble *e, int member, double *U_h, double *U_m, double *time,
                        int64_t *steps, int *status);

/* Load-balance record of the last launch: for every run, when a thread block (or cluster)
 * took it from the queue and when it finished, in microseconds of the device's global timer
 * after the earliest start (-1 for runs no launch has advanced); arrays of n.  slots: the
 * thread blocks the launch keeps resident (SMs x blocks per SM, or resident clusters x
 * cluster size). */
int pip_ensemble_timings(pip_ensemble *e, double *start_us, double *end_us);
int pip_ensemble_slots(pip_ensemble *e, int *slots);
/* The thread blocks that stepped each run in the last launch that advanced it (1, or the
 * cluster size for a shared run; 0 for runs no launch has advanced); array of n. */
int pip_ensemble_blocks(pip_ensemble *e, int *blocks);

/* Cluster sharing of long runs: 0 (default) chosen at each launch from the work estimate,
 * 1 off, 4 or 8 blocks per cluster; a run is shared when its work exceeds `share` (default
 * 0.25) times an even share of the total (PIP_ERR_PARAM with a 2D run, with 128 or 1024
 * threads per block, or share <= 0).  pip_ensemble_plan reports the last launch's choice:
 * cluster size (1: none), runs shared, blocks launched. */
int pip_ensemble_set_cluster(pip_ensemble *e, int cluster, double share);
int pip_ensemble_plan(pip_ensemble *e, int *cluster, int *shared_runs, int *grid);

/* Launch configuration: threads per block (128, 256, 512, 1024; not 128 when a run is 2D)
 * and blocks per SM. */
int pip_ensemble_set_config(pip_ensemble *e, int threads, int ctas_per_sm);

/* Autotuner: times every configuration the device can hold on a probe run to t_probe from
 * the current state (restored afterwards), keeps the fastest and reports it. */
int pip_ensemble_tune(pip_ensemble *e, double t_probe, int *threads, int *ctas_per_sm,
                      float *best_ms);

#ifdef __cplusplus
}
#endif

#endif
