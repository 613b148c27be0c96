/*
 * Launchers of the sm_100a kernels, callable from the C API layer.  All take
 * device pointers and a stream and return cudaError_t values as int.
 */
#ifndef SG_KERNELS_H
#define SG_KERNELS_H

#include <stdint.h>

#include "sg_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-dim sweep tables as the kernels read them. */
typedef struct sg_sweep_tables {
    const sg_chain *chains; /* device */
    const uint32_t *seg;    /* device */
    int64_t nchains;
    int lmax_max;           /* highest lmax over the chains          */
    int64_t cap32;          /* shared-memory elements for one chain (FP32) */
    int64_t cap64;          /* same for FP64                          */
} sg_sweep_tables;

/* Shared-memory bytes a chain-sweep CTA needs, or a negative value if the
 * chains of this grid do not fit and the per-level gather path must run. */
int64_t sgk_chain_smem_bytes(int64_t cap_elems, int elem_bytes);

/* One sweep of dim k over all chains, FP32 in place, staged through shared
 * memory with bulk copies.  err: device int, set nonzero on a wait timeout. */
int sgk_sweep_chains_f32(float *a, const sg_sweep_tables *t, int *err, void *stream);
int sgk_sweep_chains_f64(double *a, const sg_sweep_tables *t, int *err, void *stream);
/* The wait-timeout test of sgk_sweep_chains_f32: the first chain of every
 * CTA announces its copy bytes but issues no copy, so its bounded wait runs
 * out after wait_limit clock cycles (1 .. the default ~2 s limit); every CTA
 * sets *err and returns.  The grid's values are left partly swept. */
int sgk_sweep_chains_stall_f32(float *a, const sg_sweep_tables *t, int *err, long long wait_limit, void *stream);
/* The same sweep as lmax_max launches, finest level first, gathering the
 * parents from global memory (any chain size). */
int sgk_sweep_gather_f32(float *a, const sg_sweep_tables *t, void *stream);
int sgk_sweep_gather_f64(double *a, const sg_sweep_tables *t, void *stream);
/* The same sweep for short chains: one warp per chain, plain loads into a
 * per-warp shared-memory buffer of cap elements (8 warps per CTA).
 * sgk_small_smem_bytes < 0: the chains are too long for it. */
int sgk_sweep_small_f32(float *a, const sg_sweep_tables *t, void *stream);
int sgk_sweep_small_f64(double *a, const sg_sweep_tables *t, void *stream);
int64_t sgk_small_smem_bytes(int64_t cap_elems, int elem_bytes);
int sgk_widen(const float *src, double *dst, int64_t n, void *stream);

/* A run of values at `compact` in a caller's compact array and at `dev` in
 * a device layout.  Runs are cut into pieces of at most SG_COPY_PIECE
 * values (one CTA copies one piece at a time). */
#define SG_COPY_PIECE 8192
typedef struct sg_copy_seg {
    int64_t compact, dev, count;
} sg_copy_seg;
int sgk_copy_segments(const float *src, float *dst, const sg_copy_seg *segs, int64_t nseg, int to_compact,
                      void *stream);
int sgk_narrow(const double *src, float *dst, int64_t n, void *stream);

/* Evaluation. */
typedef struct sg_eval_plan {
    const float *alpha;          /* device grid in the block layout          */
    int d, n;
    int lim[SG_MAX_DIMS];
    uint32_t blk3[SG_MAX_LEVELS]; /* block size for each level budget R      */
    uint32_t blk2[SG_MAX_LEVELS]; /* sub-block size for each level budget r  */
    int ppt;                     /* points per thread (1 or 2)               */
    int blocking;                /* subspace blocking preset, 0 .. SG_EVAL_BLOCKINGS-1
                                    (wide, medium)                            */
} sg_eval_plan;

/* Subspace blocking presets of the evaluation kernels (SG_OPT_EVAL_BLOCKING
 * 1..2 select preset 0..1): how much of the walk runs as fully unrolled
 * blocks of compile-time shape (separate kernel instantiations for
 * 3 <= d <= 12; other d have one form).  Every preset gives bit-identical
 * results. */
#define SG_EVAL_BLOCKINGS 2

/* A point's sum over the subspaces can be split into up to this many
 * parts (ranges of the walk's blocks), evaluated by separate CTAs and added
 * in part order afterwards: bounds the latency of one point on a large grid. */
#define SG_EVAL_MAX_PARTS 8

/* Per-grid arguments of the evaluation kernels (also the element type of
 * the batched launch's grid table). */
typedef struct sg_eval_args {
    const float *alpha;      /* block layout                         */
    const float *coords;     /* num_evals x d                        */
    const int32_t *perm;     /* optional: sorted position -> caller  */
    float *out;
    int64_t num_evals;
    int nm1;                 /* n - 1                                */
    int lim2;                /* min limit of dims d-2, d-1: a sub-block of
                                budget r <= lim2 has the regular shape  */
    int lim3;                /* min limit of dims d-3..d-1 (3-D blocks) */
    int lim[SG_MAX_DIMS];
    uint32_t blk3[SG_MAX_LEVELS]; /* block size per budget R         */
    uint32_t blk2[SG_MAX_LEVELS]; /* sub-block size per budget r     */
    /* split evaluation (batched launch only; nparts 1 = whole sums):
     * part k covers the walk's blocks [split[k], split[k+1]) and writes its
     * sums to part_out[k * num_evals + i]; walk = per (prefix depth K,
     * budget b) the block count and block-layout extent of the subtree
     * (sg_layout_walk_tables), used to skip subtrees outside the range. */
    int nparts;
    uint32_t split[SG_EVAL_MAX_PARTS + 1];
    float *part_out;
    const uint32_t *walk;
} sg_eval_args;

void sgk_fill_eval_args(const sg_eval_plan *p, const float *coords, const int32_t *perm, float *out,
                        int64_t num_evals, sg_eval_args *a);

/* Prepares the evaluation kernels on the current device (their dynamic
 * shared-memory limit); done once per device, before any evaluation launch
 * or stream capture.  The device-state set-up of grids, batches and servers
 * calls it. */
int sgk_eval_setup(void);

/* out[perm ? perm[i] : i] = interpolant at coords[i*d .. i*d+d-1]. */
int sgk_evaluate(const sg_eval_plan *p, const float *coords, const int32_t *perm, float *out,
                 int64_t num_evals, void *stream);
/* Many grids of dimension d in one launch: items (device, 2 ints per CTA) =
 * (index into grids | part << 29, first point); each CTA covers
 * SG_EVAL_CTA_POINTS(ppt) points of its grid (index < 2^29; part selects
 * the block range of a split sum, 0 for whole sums); blocking is the
 * preset index of the launch (0 .. SG_EVAL_BLOCKINGS-1). */
int sgk_evaluate_batch(int d, const sg_eval_args *grids, const int32_t *items, int nitems, int ppt, int blocking,
                       void *stream);

/* out[i] = compensated sum over k < nparts of part_out[k * num_evals + i]
 * (part order) for the split grids: items as for sgk_evaluate_batch, one
 * CTA per 256 points. */
int sgk_combine_parts(const sg_eval_args *grids, const int32_t *items, int nitems, void *stream);

/* Reorders the surpluses from the group-aligned compact layout into the
 * block layout (one descriptor per subspace). */
int sgk_repack(const float *src, float *dst, const sg_repack *rp, int64_t nsub, void *stream);

/* Whole-grid hierarchization in shared memory for small grids, one CTA per
 * grid (all d sweeps between one load and one store). */
typedef struct sg_smem_grid {
    uint32_t base;                  /* first element in the value buffer (multiple of 32) */
    uint32_t npad;                  /* elements (multiple of 32)                         */
    int d;
    uint32_t chain0[SG_MAX_DIMS];   /* first chain of sweep k in the chain array          */
    uint32_t nch[SG_MAX_DIMS];      /* chains of sweep k                                  */
} sg_smem_grid;
#define SG_SMEM_GRID_MAX_BYTES (200 * 1024)
int sgk_hier_smem_grids(float *a, const sg_smem_grid *grids, int ngrids, const sg_chain *chains,
                        const uint32_t *seg, int max_npad, int fp64, void *stream);

/* Spatial ordering of query points: writes the sorted coordinates and the
 * permutation (sorted position -> caller position).  scratch: device bytes
 * of at least sgk_sort_scratch_bytes(num_evals, d). */
int64_t sgk_sort_scratch_bytes(int64_t num_evals, int d);
int sgk_sort_points(const float *coords, int64_t num_evals, int d, void *scratch,
                    float *sorted, int32_t *perm, void *stream);

/* Spatial ordering of a batch's points, each grid's points among
 * themselves: per grid its point count m, point offset, coordinate offset,
 * dimension, Morton key bits (sgk_batch_sort_bits) and first bin.  The
 * grids' bins must be in the order of their point offsets and the point
 * offsets must be the running sum of the m of the grids listed (the sort's
 * positions are counted over exactly these points); items
 * (device, 2 ints per CTA) = (grid, first local point), 256 points per CTA.
 * Writes sorted coordinates at the same offsets and perm[pt_off + sorted
 * local position] = caller's local index.  scratch: device bytes of at
 * least sgk_batch_sort_scratch_bytes(total points, total bins). */
typedef struct sg_bsort_grid {
    int64_t m, pt_off, coff;
    uint32_t bin_base;
    int d, kb;
} sg_bsort_grid;
int sgk_batch_sort_bits(int64_t m, int d);
int64_t sgk_batch_sort_scratch_bytes(int64_t npts, int64_t nbins);
int sgk_batch_sort_points(const float *coords, const sg_bsort_grid *grids, const int32_t *items, int nitems,
                          int64_t npts, int64_t nbins, void *scratch, float *sorted, int32_t *perm, void *stream);

/* Batched bijection on the device. */
int sgk_idx2gp(const sg_layout *L, const int64_t *index, int *levels, int *indices,
               int64_t count, void *stream);
int sgk_gp2idx(const sg_layout *L, const int *levels, const int *indices, int64_t *index,
               int64_t count, void *stream);

/* f at every point of the device grid (group-aligned layout), FP64 -> FP32. */
int sgk_sample(const sg_layout *L, int fn, const double *params, int nparams, float *alpha,
               void *stream);

/* out[q] = bits of max |alpha| over subspace q (subspaces in group order,
 * positions as sg_layout_idx2l), alpha in the group-aligned layout. */
int sgk_subspace_maxabs(const sg_layout *L, const float *alpha, unsigned *out, void *stream);

int sgk_num_sms(void);

/* Device address and size of the fixed no-allocation scratch array on the
 * current device (looked up on the first call per device). */
int sgk_noalloc_scratch(void **ptr, int64_t *bytes);

/* Process-wide count of kernels this library has launched. */
void sgk_count(int launches);
int64_t sgk_launches(void);

#ifdef __cplusplus
}
#endif
#endif
