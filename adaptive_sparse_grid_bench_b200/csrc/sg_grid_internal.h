/* Internal state of a single-grid handle (sgrid.c), shared with the
 * serving loop (sgrid_server.c). */
#ifndef SG_GRID_INTERNAL_H
#define SG_GRID_INTERNAL_H

#include <cuda_runtime_api.h>
#include <stdint.h>

#include "sg_kernels.h"
#include "sg_layout.h"

#define NOPT 11

/* Device allocator hooks.  A handle made by sg_create uses cudaMalloc and
 * cudaFree; the serving loop hands its grids a sub-allocator over one
 * reserved range instead, so admitting and evicting grids never calls the
 * CUDA allocator (whose frees wait for the whole device).  alloc returns an
 * SG_* code and sets *ptr (256-byte aligned); free accepts NULL. */
typedef int (*sg_dev_alloc_fn)(void *ctx, void **ptr, int64_t bytes);
typedef void (*sg_dev_free_fn)(void *ctx, void *ptr);

struct sg_grid {
    sg_layout L;
    int dev;        /* device of the device state, -1 before it exists */
    int has_values; /* a value array has been stored                   */
    int64_t opt[NOPT];
    float *d_alpha;   /* Npad floats, group-aligned layout         */
    double *d_work;   /* Npad doubles, FP64 hierarchization (lazy) */
    float *d_blk;        /* N floats: surpluses in the block layout    */
    sg_repack *d_repack; /* per-subspace compact -> block descriptors  */
    uint32_t blk3[SG_MAX_LEVELS]; /* block size per level budget        */
    uint32_t blk2[SG_MAX_LEVELS]; /* sub-block size per level budget    */
    int eval_dirty;      /* d_blk is stale                              */
    sg_chain *d_chains[SG_MAX_DIMS];
    uint32_t *d_seg[SG_MAX_DIMS];
    sg_sweep_tables sweep[SG_MAX_DIMS];
    int *d_err;       /* device-side wait timeout flag             */
    void *d_scratch;  /* evaluate: sort scratch + sorted coords + permutation */
    int64_t scratch_bytes;
    void *d_io;       /* host-buffer evaluate: staged coords and results */
    int64_t io_bytes;
    int64_t dev_bytes;
    cudaEvent_t ev[SG_NUM_PHASES][2]; /* profiling: start/stop per phase */
    int ev_used[SG_NUM_PHASES];
    uint32_t *d_walk;    /* evaluation walk tables (split sums only)     */
    int nparts;          /* parts of a split sum in batched launches (0/1: whole) */
    uint32_t split[SG_EVAL_MAX_PARTS + 1];
    sg_dev_alloc_fn alloc; /* NULL: cudaMalloc/cudaFree */
    sg_dev_free_fn free_fn;
    void *alloc_ctx;
};

/* sg_create with the handle's device memory taken from alloc/free_fn. */
int sg_create_with_allocator(int d, int n, const int *limits, sg_dev_alloc_fn alloc, sg_dev_free_fn free_fn,
                             void *ctx, sg_grid **grid);


/* Builds the block layout if the values changed since it was last built. */
int sg_grid_prepare_eval(sg_grid *g, cudaStream_t st);
/* Splits each point's sum over the subspaces into nparts block ranges of
 * about equal work for batched evaluations (d >= 4; otherwise, or for
 * nparts <= 1, whole sums).  Uploads the walk tables on st. */
int sg_grid_set_parts(sg_grid *g, int nparts, cudaStream_t st);
/* Kernel arguments to evaluate grid g at m points (device pointers); a
 * split grid's arguments carry its parts, part_out is left to the caller. */
void sg_grid_eval_args(const sg_grid *g, const float *coords, float *out, int64_t m, sg_eval_args *a);

#endif
