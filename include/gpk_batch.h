/*
 * gpk_batch.h — many independent grids advanced together (parameter sweeps).
 *
 * The reference runs a sweep as a loop of GPKGrid objects, one after the
 * other (e.g. the lamellar break-up sweep of demos/gpk.cpp:1119-1200, which
 * builds and steps one GPKGrid per spacing).  A batch advances a set of
 * gpk_grid handles of any sizes and models together: a pool of worker
 * threads, each driving its instances' own CUDA streams, so that the small
 * kernels and host round trips of many instances overlap on one GPU.  Every
 * instance follows exactly the step sequence it would follow alone, so its
 * results are bit-identical to stepping it alone.
 *
 * The batch does not own the grids: create them with gpk_grid_create, load
 * them, and destroy them after the batch.  While a batch call runs, the
 * caller must not use its grids.
 */
#ifndef GPK_BATCH_H
#define GPK_BATCH_H

#include <stddef.h>
#include <stdint.h>

#include "gpk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpk_batch gpk_batch;

/* n >= 1 distinct, non-null grid handles.  workers: threads (0 = one per
 * hardware thread, at most n).  Instances are handed to workers largest
 * first.                                                                   */
int gpk_batch_create(int n, gpk_grid* const* grids, int workers, gpk_batch** out);
int gpk_batch_destroy(gpk_batch* b);
int gpk_batch_set_workers(gpk_batch* b, int workers);
int gpk_batch_workers(const gpk_batch* b, int* workers);
/* Every instance takes `steps` steps of GPKGrid::step(dt, dt_cap) (dt < 0:
 * each instance's own stable dt).  Returns when all work has finished.  On
 * an error the remaining instances are left where they are; the message
 * names the first failing instance.                                        */
int gpk_batch_step(gpk_batch* b, int steps, double dt, double dt_cap);
/* Every instance runs GPKGrid::run(t_end, dt) (at most max_steps steps);
 * steps_out (n entries, may be null) receives each instance's step count. */
int gpk_batch_run(gpk_batch* b, double t_end, double dt, int max_steps, int* steps_out);
/* Picks the worker count: times trial_steps real steps of every instance at
 * each candidate count (1, 2, 4, ... up to n and 64) and keeps the fastest.
 * The trials advance the instances: trial_steps x candidates steps in all
 * (reported in *steps_taken).  *workers_out (may be null) gets the choice. */
int gpk_batch_autotune(gpk_batch* b, int trial_steps, int* workers_out, int* steps_taken);

#ifdef __cplusplus
}
#endif
#endif /* GPK_BATCH_H */
