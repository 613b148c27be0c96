/*
 * sgrid.h - C ABI of the B200 compact sparse-grid library (libsgb200.so).
 *
 * A drop-in for the callable surface of the reference benchmark
 * adaptive_sparse_grid_bench.c (citations "c:LINE" refer to that file):
 *
 *   reference                                   this library
 *   -----------------------------------------   ---------------------------
 *   globals num_dims/num_levels/limits + init()  sg_create / sg_destroy
 *     (c:77-85, c:101-140)
 *   num_grid_points, num_subspaces (c:130-137)   sg_num_points/_subspaces
 *   sg1d filled at the grid points (c:146-152)    sg_set_values
 *   int hierarchizeK(void)  (c:557-1233)          sg_hierarchize
 *   int evaluateK(sg1d, coord_mat, out, n)        sg_evaluate
 *     (c:1237-1722)
 *   int gp2idx(levels, indices)  (c:187-207)      sg_gp2idx
 *   int idx2gp(index, levels, indices) (c:210)    sg_idx2gp
 *   idx2l / l2idx  (c:245-279)                    sg_idx2l / sg_l2idx
 *
 * Conventions are the reference's: levels are 0-based, a grid of n levels
 * holds every level vector l with sum(l) <= n-1 and l[k] <= limits[k]; point
 * (l, i) sits at x = (2i+1)/2^(l+1); values, surpluses and the linear index
 * follow the compact layout (level groups in order, subspaces by l2idx,
 * points row-major with dim 0 most significant).  coord_mat is num_evals x d
 * row-major floats in [0, 1).
 *
 * Every function returns an int status: SG_OK (0, the reference's
 * "return 0") or a negative SG_ERR_* code; sg_last_error() gives the text.
 * Host buffers belong to the caller; device memory belongs to the handle.
 * A handle may be used by one host thread at a time.  sg_create touches no
 * GPU: device storage is created on the current device by the first call
 * that needs it.
 */
#ifndef SGRID_H
#define SGRID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_MAX_DIMS 20   /* the reference's CUDA cap (cu:17) */
#define SG_MAX_LEVELS 16 /* n <= 16 (the reference's CUDA cap is 10, cu:18) */

#define SG_OK 0
#define SG_ERR_ARG (-1)     /* invalid argument                                */
#define SG_ERR_RANGE (-2)   /* size beyond what the library supports           */
#define SG_ERR_CUDA (-3)    /* a CUDA call failed                              */
#define SG_ERR_NOMEM (-4)   /* host or device allocation failed                */
#define SG_ERR_STATE (-5)   /* call out of order (e.g. no values set yet)      */
#define SG_ERR_TIMEOUT (-6) /* a device-side wait gave up; results are invalid */

/* Hierarchization precision (sg_set_option(SG_OPT_HIER_PRECISION, ...)). */
#define SG_HIER_FP32 0 /* FP32 sweeps, bit-identical to hierarchize0 (c:557) */
#define SG_HIER_FP64 1 /* FP64 sweeps, each surplus rounded once to FP32     */

/* Options (sg_set_option / sg_get_option). */
#define SG_OPT_HIER_PRECISION 1 /* SG_HIER_FP32 (default) or SG_HIER_FP64           */
#define SG_OPT_EVAL_SORT 2      /* 1 (default): spatially order points on the GPU   */
                                /* before evaluating; 0: evaluate in caller order    */
#define SG_OPT_EVAL_PPT 3       /* points per thread in evaluate: 0 = auto, 1, 2     */
#define SG_OPT_HIER_KERNEL 5    /* 0 = auto, 1 = shared-memory chains, 2 = gather,   */
                                /* 3 = one warp per chain (batches only)            */
#define SG_OPT_PROFILE 6        /* 1: record CUDA events around each phase            */
#define SG_OPT_USE_GRAPH 7      /* batches: 1 (default) capture launches in a CUDA graph */
#define SG_OPT_SWEEP_GROUP 8    /* batches: values per sweep group (default 2^22): all   */
                                /* sweeps of a group run back to back so it stays in  */
                                /* L2; 0 = every sweep over the whole batch.  Set it  */
                                /* before the batch's first device call.             */
#define SG_OPT_TEST_WAIT 9      /* tests of the device-wait timeout, FP32 grids: k in */
                                /* 1..2048 makes every staged sweep's first copy per  */
                                /* CTA never start, so its bounded wait gives up after */
                                /* k * 2^20 clock cycles (about k/2 ms); the next     */
                                /* sg_sync returns SG_ERR_TIMEOUT and the values are  */
                                /* invalid.  0 (default): off.                       */
#define SG_OPT_EVAL_BLOCKING 10 /* evaluate: how much of the subspace walk runs as   */
                                /* fully unrolled blocks of compile-time shape:      */
                                /* 1 = wide (3-D blocks of level budget <= 6, leaf  */
                                /* subtrees of budget <= 5 at one point per thread  */
                                /* or <= 4 at two), 2 = medium (5, 3); 0 = auto    */
                                /* (wide, or the tuned choice).  Grids of d < 3 or  */
                                /* d > 12 have one form.  Results are bit-identical */
                                /* under every setting.                             */

/* Phases reported by sg_timings (milliseconds of the most recent call). */
#define SG_PHASE_HIERARCHIZE 0  /* all sweeps of the last hierarchization    */
#define SG_PHASE_SORT 1         /* spatial ordering of the last evaluation  */
#define SG_PHASE_EVALUATE 2     /* the evaluation kernel itself             */
#define SG_NUM_PHASES 3

typedef struct sg_grid sg_grid;

/* ---- create / destroy (init(), c:101-140; cu:72-102) ------------------- */

/* limits == NULL gives the regular grid (limits[k] = n-1, as c:1760-1763). */
int sg_create(int d, int n, const int *limits, sg_grid **grid);
int sg_destroy(sg_grid *grid);

int sg_num_points(const sg_grid *grid, int64_t *num_points);       /* c:130-137 */
int sg_num_subspaces(const sg_grid *grid, int64_t *num_subspaces); /* c:130-137 */
int sg_dims(const sg_grid *grid, int *d, int *n, int *limits);

/* dp[d*n]: dp[i*n+s] = number of level vectors over dims 0..i with sum s
 * (dp_mat, c:113-129); lidx[n+1]: first index of each level group
 * (lidx_vect, c:132-140, plus lidx[n] = num_points). */
int sg_tables(const sg_grid *grid, int64_t *dp, int64_t *lidx);

/* ---- index bijection (host; c:187-279) ---------------------------------- */
int sg_gp2idx(const sg_grid *grid, const int *levels, const int *indices, int64_t *index);
int sg_idx2gp(const sg_grid *grid, int64_t index, int *levels, int *indices);
int sg_l2idx(const sg_grid *grid, const int *levels, int64_t *position);
int sg_idx2l(const sg_grid *grid, int64_t position, int level_sum, int *levels);

/* ---- host-buffer calls: synchronous, the reference's calling style ------ */

/* values[num_points] in compact order (the sg1d fill of c:146-152). */
int sg_set_values(sg_grid *grid, const float *values);
/* Reads the grid back (surpluses after sg_hierarchize). */
int sg_get_values(sg_grid *grid, float *values);
/* In-place hierarchization of the stored values (hierarchize0..8, c:557). */
int sg_hierarchize(sg_grid *grid);
/* out[c] = interpolant at coord_mat[c*d .. c*d+d-1] (evaluate0..5, c:1237). */
int sg_evaluate(sg_grid *grid, const float *coord_mat, float *out, int64_t num_evals);

/* ---- device-pointer calls: asynchronous on `stream` (a cudaStream_t; NULL
 *      is the legacy default stream).  Pointers are device memory. -------- */
int sg_set_values_device(sg_grid *grid, const float *values, void *stream);
int sg_get_values_device(sg_grid *grid, float *values, void *stream);
int sg_hierarchize_async(sg_grid *grid, void *stream);
int sg_evaluate_device(sg_grid *grid, const float *coord_mat, float *out,
                       int64_t num_evals, void *stream);
/* Evaluation that allocates no memory, for callers that cannot call
 * cudaMalloc at evaluation time: serving loops whose device memory is
 * reserved up front by their own pool, latency-bound request paths that
 * cannot afford cudaMalloc's device synchronisation, and hosts that forbid
 * plugins from allocating device memory.  No counterpart in the reference.
 * Same meaning and result as sg_evaluate_device, but the point-sorting
 * scratch is a fixed array of SG_NOALLOC_SCRATCH_BYTES in this library that
 * every GPU loading the library holds until the process exits.  Limits: the
 * handle's device state must already exist (created by an earlier
 * sg_set_values*, sg_sample_function or sg_hierarchize* call on this
 * device, else SG_ERR_STATE) and num_evals <= SG_NOALLOC_MAX_POINTS (else
 * SG_ERR_RANGE).  The first call on a device looks up the array's device
 * address, which makes the CUDA runtime place the array on that device;
 * make that first call before capturing work on the stream.  All
 * calls share the one array: calls whose work overlaps on the GPU (other
 * streams, other handles, other host threads) race and must be serialised
 * by the caller.  The looked-up address is cached per device (safe for
 * concurrent host threads); a cudaDeviceReset invalidates it together with
 * every handle on that device. */
#define SG_NOALLOC_MAX_POINTS (1 << 18)
#define SG_NOALLOC_SCRATCH_BYTES (24 << 20)
int sg_evaluate_device_noalloc(sg_grid *grid, const float *coord_mat, float *out,
                               int64_t num_evals, void *stream);

/* Waits for `stream` and reports any device-side error flag of the handle. */
int sg_sync(sg_grid *grid, void *stream);

/* Autotuner (no reference counterpart; the reference tunes its CUDA block
 * size by hand, run.sh).  Times, on the caller's device buffers and stream,
 * the evaluation under every setting of points per thread {1, 2} x spatial
 * ordering {off, on}, then, at the faster of those, under every subspace
 * blocking (SG_OPT_EVAL_BLOCKING 1..2), and the hierarchization with the
 * shared-memory chain sweeps (where they fit) and the gather sweeps; keeps
 * the fastest in the handle's options (SG_OPT_EVAL_PPT, SG_OPT_EVAL_SORT,
 * SG_OPT_EVAL_BLOCKING, SG_OPT_HIER_KERNEL).  No setting changes any result.
 * The grid's values are the same on return (saved and restored); out[] holds
 * the evaluation.  ms (optional, SG_TUNE_TIMINGS entries): evaluation ms for
 * (ppt, sort) = (1,0), (1,1), (2,0), (2,1), then hierarchization ms for
 * chains and gather, then evaluation ms for blocking 1, 2 (-1: not
 * applicable). */
#define SG_TUNE_TIMINGS 8
int sg_autotune(sg_grid *grid, const float *coord_mat, float *out, int64_t num_evals, void *stream, double *ms);

/* Device bijection for batches (no reference counterpart beyond looping
 * gp2idx/idx2gp; used to sample grids on the GPU).  levels/indices are
 * count x d int32 row-major. */
int sg_idx2gp_device(const sg_grid *grid, const int64_t *index, int *levels,
                     int *indices, int64_t count, void *stream);
int sg_gp2idx_device(const sg_grid *grid, const int *levels, const int *indices,
                     int64_t *index, int64_t count, void *stream);

/* Built-in test functions for sg_sample_function (evaluated in FP64 at the
 * grid points, rounded once to FP32).  No reference counterpart beyond the
 * sg1d fill of c:146-152, which samples SG_FN_REFERENCE on the host. */
#define SG_FN_REFERENCE 0 /* sum_k x_k^2 (1 - x_k)^2  (fct, c:87-94)            */
#define SG_FN_PROD4 1     /* prod_k 4 x_k (1 - x_k)                             */
#define SG_FN_GAUSS 2     /* exp(-sum_k x_k^2)                                  */
#define SG_FN_BUMP 3      /* exp(-p[1] sum_k (x_k - p[0])^2)                    */
#define SG_FN_QUAD 4      /* prod_k (p[3k] + p[3k+1] x_k + p[3k+2] x_k^2)       */
#define SG_MAX_FN_PARAMS 64

/* Fills the grid with f at its points, on the device (replaces the value
 * array like sg_set_values). */
int sg_sample_function(sg_grid *grid, int fn, const double *params, int num_params, void *stream);

/* ---- limits-adaptive refinement -----------------------------------------
 * The reference's adaptive grid is the per-dimension limit vector of
 * init() (c:82-83, c:113-129) and nothing refines it.  These calls refine
 * within that family, so every grid they produce is one the reference's
 * init/idx2gp/hierarchize0 reproduce for the same (d, n, limits).
 * Levels are 0-based as in the reference. */
/* maxabs[q] = max |value| over the points of subspace q (subspaces in
 * compact order: level sum s ascending, sg_idx2l positions inside a group);
 * S floats.  Runs on the legacy default stream and waits for it. */
int sg_subspace_maxabs(sg_grid *grid, float *maxabs);
/* One step: a subspace is active if maxabs > tol; every child l + e_k with
 * l_k < max_level of an active subspace must be in the next grid, which is
 * the smallest (n_out, limits_out) containing (n, limits) and those
 * children (n_out capped at SG_MAX_LEVELS).  changed = 0 when it is the
 * same grid.  Host only. */
int sg_refine_step(int d, int n, const int *limits, const float *maxabs, double tol, int max_level,
                   int *n_out, int *limits_out, int *changed);
/* Driver: from (d, n0, limits0 or NULL), sample fn, hierarchize (precision
 * SG_HIER_FP32/FP64), measure, step, until the grid stops changing, after
 * max_iters grids, or before a grid of more than max_points points.
 * Returns the last grid, hierarchized; sg_dims reads its n and limits. */
int sg_refine(int d, int n0, const int *limits0, int fn, const double *params, int num_params, double tol,
              int max_level, int64_t max_points, int max_iters, int precision, sg_grid **grid,
              int *iterations);

/* ---- batches of independent grids -------------------------------------
 * Many grids of mixed d, n and limits held in one device buffer and run
 * through a fixed set of launches (replayed as one CUDA graph).  No
 * reference counterpart: the reference handles one grid per process.
 * Values cross the ABI as the grids' compact arrays concatenated in grid
 * order (offsets from sg_batch_offsets).  limits: NULL, or every grid's d
 * limits concatenated. */
typedef struct sg_batch sg_batch;
int sg_batch_create(int num_grids, const int *dims, const int *levels, const int *limits,
                    sg_batch **batch);
int sg_batch_destroy(sg_batch *batch);
int sg_batch_num_grids(const sg_batch *batch, int *num_grids);
/* value_offsets[num_grids+1]: first value of each grid in the concatenation */
int sg_batch_offsets(const sg_batch *batch, int64_t *value_offsets);
int sg_batch_set_values(sg_batch *batch, const float *values);
int sg_batch_set_values_device(sg_batch *batch, const float *values, void *stream);
int sg_batch_get_values(sg_batch *batch, float *values);
int sg_batch_get_values_device(sg_batch *batch, float *values, void *stream);
/* params: params_per_grid doubles per grid (SG_FN_QUAD: 3*d of them) */
int sg_batch_sample_function(sg_batch *batch, int fn, const double *params, int params_per_grid,
                             void *stream);
/* All grids, one graph launch; bit-identical to sg_hierarchize per grid. */
int sg_batch_hierarchize_async(sg_batch *batch, void *stream);
int sg_batch_hierarchize(sg_batch *batch);
/* Grid g is evaluated at the point_offsets[g+1]-point_offsets[g] points
 * whose coordinates follow each other in `coord_mat` (rows of d_g floats,
 * grid after grid); results land at out[point_offsets[g] ...].  Device
 * pointers; point_offsets is a host array of num_grids+1 entries. */
int sg_batch_evaluate_device(sg_batch *batch, const int64_t *point_offsets, const float *coord_mat,
                             float *out, void *stream);
int sg_batch_sync(sg_batch *batch, void *stream);
/* SG_OPT_HIER_PRECISION, SG_OPT_EVAL_PPT, SG_OPT_USE_GRAPH, SG_OPT_HIER_KERNEL (sweeps),
 * SG_OPT_EVAL_SORT (1, default: each grid's points spatially ordered on the GPU),
 * SG_OPT_EVAL_BLOCKING, SG_OPT_SWEEP_GROUP (before the first device call;
 * SG_ERR_STATE after it) */
int sg_batch_set_option(sg_batch *batch, int option, int64_t value);
/* Autotuner for batches (no reference counterpart): times each
 * dimension's evaluation launch over the caller's points at 1 and at 2
 * points per thread under each subspace blocking (SG_OPT_EVAL_BLOCKING
 * 1..2) and keeps the fastest pair per dimension, and times the
 * hierarchization with each chain size class on the staged chain kernel and
 * on one warp per chain and keeps the faster per class (the values are
 * saved and restored).  Results do not change.  An SG_OPT_EVAL_PPT,
 * SG_OPT_EVAL_BLOCKING or SG_OPT_HIER_KERNEL setting replaces the tuned
 * choice.  ms (optional, SG_BATCH_TUNE_TIMINGS entries):
 * [(blocking-1)*2 + ppt-1][d] launch ms, -1 where no grid has d. */
#define SG_BATCH_TUNE_TIMINGS (4 * (SG_MAX_DIMS + 1))
int sg_batch_autotune(sg_batch *batch, const int64_t *point_offsets, const float *coord_mat, float *out,
                      void *stream, double *ms);
int sg_batch_device_bytes(const sg_batch *batch, int64_t *bytes);

/* ---- serving loop --------------------------------------------------------
 * A pool of hierarchized grids resident on the current device under a byte
 * cap, and a dispatcher thread that batches evaluate requests continuously.
 * Requests are queued in two lanes by their work (points x grid subspaces,
 * SG_SRV_OPT_HEAVY_PAIRS); every request of a lane queued when one of the
 * lane's batch slots frees up goes into one batch (one batched launch per
 * dimension), so batches are assembled while others compute, and light
 * batches run at a higher stream priority than heavy ones.  No reference
 * counterpart. */
typedef struct sg_server sg_server;
/* max_batch_points: points per batch (and the largest single request).
 * Reserves hbm_cap_bytes of device memory at once (SG_ERR_NOMEM if it is not
 * free); every resident grid is sub-allocated from that range, so admission
 * and eviction make no CUDA allocator call. */
int sg_server_create(int64_t hbm_cap_bytes, int64_t max_batch_points, sg_server **server);
/* Stops the dispatcher (running batches finish, queued requests fail) and
 * frees every resident grid. */
int sg_server_destroy(sg_server *server);
/* Admits a grid: create, sample fn (sg_sample_function), hierarchize, build
 * the evaluation layout.  Evicts least recently used grids with no queued or
 * running request while the cap would be exceeded; SG_ERR_NOMEM if that is
 * not enough.  Blocks until the grid is ready. */
int sg_server_add_grid(sg_server *server, int d, int n, const int *limits, int fn, const double *params,
                       int num_params, int64_t *grid_id);
/* Queues out[0..num_evals) = grid at coord_mat (host buffers that must stay
 * valid until sg_server_wait returns for the ticket).  Never blocks on the
 * GPU.  SG_ERR_ARG if the grid is not resident. */
int sg_server_submit(sg_server *server, int64_t grid_id, const float *coord_mat, int64_t num_evals,
                     float *out, int64_t *ticket);
/* Waits for a ticket; latency_ms (optional) = submit -> results in `out`. */
int sg_server_wait(sg_server *server, int64_t ticket, double *latency_ms);
/* sg_server_wait with the request's timeline, ms[5] (optional): milliseconds
 * from submit until it was taken into a batch, until the batch's launches
 * were issued, until the batch's completion was seen, the request's work in
 * point x subspace pairs, and milliseconds until its results were in `out`. */
int sg_server_wait_detail(sg_server *server, int64_t ticket, double *ms);
/* Server options (sg_server_set_option). */
#define SG_SRV_OPT_ZERO_COPY 1 /* 1 (default): batches read coordinates from and write
                                  results to pinned host memory directly (no copy
                                  stages; each request's coordinates are staged into a
                                  pinned ring by sg_server_submit in the caller's
                                  thread); 0: one copy in and one out per batch */
#define SG_SRV_OPT_HEAVY_PAIRS 2 /* requests whose points x grid subspaces reach this
                                    (default 2^27) queue in the heavy lane: its own
                                    batches and slots at a lower stream priority, so
                                    light requests never wait behind them */
#define SG_SRV_OPT_LIGHT_SLOTS 3 /* batches of the light lane in flight at once, 1..3
                                    (default 3); the heavy lane has two */
#define SG_SRV_OPT_SORT_HEAVY 4  /* 1 (default): the points of each heavy request are
                                    put in spatial (Morton) order on the GPU before
                                    evaluation (results scattered back; same values) */
int sg_server_set_option(sg_server *server, int option, int64_t value);
/* stats[7]: batches, requests, points, evictions, resident grids, bytes of
 * the reserved range in use, failed requests */
int sg_server_stats(sg_server *server, int64_t *stats);
/* The request alone through sg_evaluate on the resident grid (the plain
 * one-launch-per-request arrangement; for comparison). */
int sg_server_evaluate_now(sg_server *server, int64_t grid_id, const float *coord_mat, int64_t num_evals,
                           float *out);

/* ---- options and diagnostics ------------------------------------------ */
int sg_set_option(sg_grid *grid, int option, int64_t value);
int sg_get_option(const sg_grid *grid, int option, int64_t *value);
/* Device time of each phase of the most recent calls made with
 * SG_OPT_PROFILE on (waits for them); ms[SG_NUM_PHASES], -1 if not run. */
int sg_timings(sg_grid *grid, double *ms);
/* Number of kernels this library has launched in this process (all
 * handles); a difference of two readings counts the launches in between. */
int sg_kernel_launches(int64_t *count);
/* Bytes of device memory the handle holds (grid, tables and scratch). */
int sg_device_bytes(const sg_grid *grid, int64_t *bytes);
/* Text of the last error raised on the calling thread ("" if none). */
const char *sg_last_error(void);
/* Library version string. */
const char *sg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SGRID_H */
