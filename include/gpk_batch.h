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
/* The same steps with the whole sweep as one captured CUDA graph: every
 * instance's step is captured once (two steps per graph, so that the
 * buffers the step swaps come back to their places), the instance graphs
 * become the independent children of one graph, and each launch of it
 * advances every instance two steps with no host round trip.  A captured
 * step runs the same kernels in the same order as gpk_grid_step, so results
 * are bit-identical to stepping alone.  Supported when every instance's
 * model needs no host decision inside a step (gpk_grid_graph_supported):
 * no region-identity topology certificates, no stochastic noise, no
 * recovery, no global-separable geometry; GPK_ERR_UNSUPPORTED_MODEL names
 * the first instance that does not qualify.  A fresh instance first takes
 * one ordinary step; an odd step left over is ordinary too.  Graphs are
 * captured again when an instance's model, settings or step arguments
 * change.                                                                  */
int gpk_batch_step_graph(gpk_batch* b, int steps, double dt, double dt_cap);
/* The CUDA stream (cudaStream_t) the sweep graph is launched on, for the
 * caller's own events around gpk_batch_step_graph.                        */
int gpk_batch_graph_stream(gpk_batch* b, void** stream);
/* Autotuner of the sweep graph's tile shapes: instances are grouped by side
 * (up to 160, 161..320, above 320 cells), and for each group in turn every
 * 2-D geometry tile height (gpk_grid_set_tile_rows 1, 2, 4) is timed over
 * trial_steps (rounded up to even) graph steps of the whole sweep, keeping
 * the fastest.  The trials advance the instances (*steps_taken steps in
 * all).  choice_out (3 entries, may be null) receives the divisor chosen
 * per group.                                                               */
int gpk_batch_autotune_tiles(gpk_batch* b, int trial_steps, int* choice_out, int* steps_taken);
/* Picks the worker count: times trial_steps real steps of every instance at
 * each candidate count (1, 2, 4, ... up to n and 64) and keeps the fastest.
 * The trials advance the instances: trial_steps x candidates steps in all
 * (reported in *steps_taken).  *workers_out (may be null) gets the choice. */
int gpk_batch_autotune(gpk_batch* b, int trial_steps, int* workers_out, int* steps_taken);

#ifdef __cplusplus
}
#endif
#endif /* GPK_BATCH_H */
