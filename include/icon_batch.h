/*
 * icon_batch.h -- uneven multi-series batches and the autotuner of the B200
 * ICON engine.
 *
 * No counterpart in the reference: ICON-GPU v1.2.9 reconstructs one tilt
 * series per process and one slice at a time (the slice loop of Lib_2D2,
 * ICON-GPU/MainCode.cu:113-162; the per-GPU slice ranges of
 * ICON-GPU/ICONGPU.cu:393-466).  Here a batch holds many series of uneven
 * width, tilt count, thickness and slice count; each series gets a plan whose
 * slices per group and slices per launch come from the autotuner, each
 * series' iteration is captured once into CUDA graphs, and the series'
 * graphs are replayed round-robin on their own streams, so that series of
 * every size run on the GPU at the same time.
 */
#ifndef ICON_BATCH_H
#define ICON_BATCH_H

#include "icon_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One series of a batch: the geometry of icon_geometry and its number of
 * slices (xz-slices, i.e. detector rows y). */
typedef struct {
    int nx;                  /* detector width N0                      */
    int thickness;           /* N1 (0 means nx)                         */
    int ntilt;
    const float *tilt_deg;   /* h_: angles as in the .tlt file          */
    int slices;              /* slices to reconstruct (>= 1)            */
} icon_series;

/* A tuning choice for one series shape: slices per group (the B of the
 * batched layout, 1/2/4/8), slices per launch (the plan's capacity), and the
 * measured device time per slice and iteration.  tuned = 1 when it was timed
 * in this process, 2 when read from the cache file, 0 for the built-in
 * default (no cache entry and tuning off). */
typedef struct {
    int group;
    int chunk;
    double us_per_slice_iteration;
    int tuned;
} icon_tuning;

typedef struct icon_batch icon_batch;

/* Creates a batch on `device` (-1: current) with normal operator `op`
 * (ICON_OPERATOR_*).  For every series the tuning is looked up in
 * `tune_cache` (a text file of lines "nx thickness ntilt slices op group
 * chunk us", slices capped at 256; NULL: none); a shape without an entry is
 * timed when `tune` is
 * nonzero (candidates: every valid group size times up to three chunk
 * sizes, a few iterations each on the device) and appended to the cache
 * file when `tune` is 2; otherwise it gets the default (the plan's group
 * size, chunk = min(slices, 128)).  Creates the plans (device memory for all
 * series at their chunk sizes). */
icon_status icon_batch_create(const icon_series *series, int nseries, int device, int op, const char *tune_cache,
                              int tune, icon_batch **out);
icon_status icon_batch_destroy(icon_batch *batch);

/* The tuning used for series k. */
icon_status icon_batch_tuning(const icon_batch *batch, int k, icon_tuning *out);

/* Reconstructs every series with the schedule cfg (the reference's
 * iteration, Iteration2.cu:42-146, from m = 0): h_rows[k] is series k's
 * rows [slices][ntilt][nx] and h_m[k] receives its slices [slices][N0][N1]
 * (Y fastest, as icon_solve).  With concurrent != 0 the series run at the
 * same time (per series a stream and CUDA graphs of its iteration, replayed
 * round-robin); with 0 one after another with direct launches (the same
 * kernels, for comparison).  Host buffers should be pinned (icon_host_alloc
 * or cudaHostAlloc) so that copies overlap the work.  Returns when every
 * result is in host memory. */
icon_status icon_batch_reconstruct_host(icon_batch *batch, const icon_solve_cfg *cfg, const float *const *h_rows,
                                        float *const *h_m, int concurrent);

#ifdef __cplusplus
}
#endif

#endif /* ICON_BATCH_H */
