/*
 * C ABI of the B200 sparse-grid library (include/sgrid.h).  Host code in C:
 * it owns the handle, the index tables and the device memory, and calls the
 * sm_100a kernels through the launchers of sg_kernels.h.  There is no CPU
 * compute path: every grid operation runs on the GPU, and a missing or
 * unusable GPU is reported as SG_ERR_CUDA.
 */
#include <cuda_runtime_api.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sg_kernels.h"
#include "sg_batch_internal.h"
#include "sg_grid_internal.h"
#include "sg_layout.h"

#define SG_API __attribute__((visibility("default")))
#define SG_VERSION "sgb200 0.1.0"

static __thread char g_err[512];

void sg_set_error(const char *fmt, va_list ap) { vsnprintf(g_err, sizeof(g_err), fmt, ap); }

static int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    sg_set_error(fmt, ap);
    va_end(ap);
    return code;
}

static int cuda_fail(cudaError_t e, const char *what)
{
    return fail(SG_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define CU(call, what)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);      \
    } while (0)

SG_API const char *sg_last_error(void) { return g_err; }
SG_API const char *sg_version(void) { return SG_VERSION; }

SG_API int sg_create(int d, int n, const int *limits, sg_grid **grid)
{
    sg_grid *g;
    int r;
    if (!grid) return fail(SG_ERR_ARG, "sg_create: grid is NULL");
    *grid = NULL;
    g = (sg_grid *)calloc(1, sizeof(sg_grid));
    if (!g) return fail(SG_ERR_NOMEM, "sg_create: out of host memory");
    r = sg_layout_init(&g->L, d, n, limits);
    if (r != SG_OK) {
        free(g);
        if (r == SG_ERR_RANGE)
            return fail(r, "sg_create: d=%d n=%d outside 1..%d x 1..%d or grid too large", d, n,
                        SG_MAX_DIMS, SG_MAX_LEVELS);
        return fail(r, "sg_create: invalid arguments d=%d n=%d", d, n);
    }
    g->dev = -1;
    g->opt[SG_OPT_HIER_PRECISION] = SG_HIER_FP32;
    g->opt[SG_OPT_EVAL_SORT] = 1;
    g->opt[SG_OPT_EVAL_PPT] = 0;
    g->opt[SG_OPT_HIER_KERNEL] = 0;
    *grid = g;
    return SG_OK;
}

static void dev_free(sg_grid *g, void *p)
{
    if (!p) return;
    if (g->free_fn) g->free_fn(g->alloc_ctx, p);
    else cudaFree(p);
}

static void free_device(sg_grid *g)
{
    int k;
    if (g->dev < 0) return;
    cudaSetDevice(g->dev);
    for (k = 0; k < SG_NUM_PHASES; k++)
        if (g->ev[k][0]) {
            cudaEventDestroy(g->ev[k][0]);
            cudaEventDestroy(g->ev[k][1]);
            g->ev[k][0] = g->ev[k][1] = NULL;
        }
    dev_free(g, g->d_alpha);
    dev_free(g, g->d_work);
    dev_free(g, g->d_blk);
    dev_free(g, g->d_repack);
    for (k = 0; k < SG_MAX_DIMS; k++) {
        dev_free(g, g->d_chains[k]);
        dev_free(g, g->d_seg[k]);
    }
    dev_free(g, g->d_err);
    dev_free(g, g->d_scratch);
    dev_free(g, g->d_io);
    dev_free(g, g->d_walk);
}

int sg_create_with_allocator(int d, int n, const int *limits, sg_dev_alloc_fn alloc, sg_dev_free_fn free_fn,
                             void *ctx, sg_grid **grid)
{
    int r;
    if (!alloc || !free_fn) return fail(SG_ERR_ARG, "sg_create_with_allocator: allocator hooks are NULL");
    r = sg_create(d, n, limits, grid);
    if (r != SG_OK) return r;
    (*grid)->alloc = alloc;
    (*grid)->free_fn = free_fn;
    (*grid)->alloc_ctx = ctx;
    return SG_OK;
}

SG_API int sg_destroy(sg_grid *g)
{
    if (!g) return SG_OK;
    free_device(g);
    free(g);
    return SG_OK;
}

SG_API int sg_num_points(const sg_grid *g, int64_t *v)
{
    if (!g || !v) return fail(SG_ERR_ARG, "sg_num_points: NULL argument");
    *v = g->L.N;
    return SG_OK;
}

SG_API int sg_num_subspaces(const sg_grid *g, int64_t *v)
{
    if (!g || !v) return fail(SG_ERR_ARG, "sg_num_subspaces: NULL argument");
    *v = g->L.S;
    return SG_OK;
}

SG_API int sg_dims(const sg_grid *g, int *d, int *n, int *limits)
{
    int k;
    if (!g) return fail(SG_ERR_ARG, "sg_dims: NULL grid");
    if (d) *d = g->L.d;
    if (n) *n = g->L.n;
    if (limits)
        for (k = 0; k < g->L.d; k++) limits[k] = g->L.lim[k];
    return SG_OK;
}

SG_API int sg_tables(const sg_grid *g, int64_t *dp, int64_t *lidx)
{
    int i, s;
    if (!g) return fail(SG_ERR_ARG, "sg_tables: NULL grid");
    if (dp)
        for (i = 0; i < g->L.d; i++)
            for (s = 0; s < g->L.n; s++) dp[i * g->L.n + s] = g->L.dp[i][s];
    if (lidx)
        for (s = 0; s <= g->L.n; s++) lidx[s] = g->L.lidx[s];
    return SG_OK;
}

/* ---- bijection (host) ---------------------------------------------------- */

static int check_levels(const sg_grid *g, const int *lv, int *sum)
{
    int k, s = 0;
    for (k = 0; k < g->L.d; k++) {
        if (lv[k] < 0 || lv[k] > g->L.lim[k]) return 0;
        s += lv[k];
    }
    *sum = s;
    return s <= g->L.n - 1;
}

SG_API int sg_gp2idx(const sg_grid *g, const int *lv, const int *ix, int64_t *index)
{
    int k, s;
    if (!g || !lv || !ix || !index) return fail(SG_ERR_ARG, "sg_gp2idx: NULL argument");
    if (!check_levels(g, lv, &s)) return fail(SG_ERR_ARG, "sg_gp2idx: level vector not in the grid");
    for (k = 0; k < g->L.d; k++)
        if (ix[k] < 0 || ix[k] >= (1 << lv[k])) return fail(SG_ERR_ARG, "sg_gp2idx: index out of range");
    *index = sg_layout_gp2idx(&g->L, lv, ix);
    return SG_OK;
}

SG_API int sg_idx2gp(const sg_grid *g, int64_t index, int *lv, int *ix)
{
    if (!g || !lv || !ix) return fail(SG_ERR_ARG, "sg_idx2gp: NULL argument");
    if (index < 0 || index >= g->L.N) return fail(SG_ERR_ARG, "sg_idx2gp: index %lld out of range", (long long)index);
    return sg_layout_idx2gp(&g->L, index, lv, ix);
}

SG_API int sg_l2idx(const sg_grid *g, const int *lv, int64_t *pos)
{
    int s;
    if (!g || !lv || !pos) return fail(SG_ERR_ARG, "sg_l2idx: NULL argument");
    if (!check_levels(g, lv, &s)) return fail(SG_ERR_ARG, "sg_l2idx: level vector not in the grid");
    *pos = sg_layout_l2idx(&g->L, lv);
    return SG_OK;
}

SG_API int sg_idx2l(const sg_grid *g, int64_t pos, int s, int *lv)
{
    if (!g || !lv) return fail(SG_ERR_ARG, "sg_idx2l: NULL argument");
    if (s < 0 || s >= g->L.n || pos < 0 || pos >= g->L.dp[g->L.d - 1][s])
        return fail(SG_ERR_ARG, "sg_idx2l: position out of range");
    sg_layout_idx2l(&g->L, pos, s, lv);
    return SG_OK;
}

/* ---- device state -------------------------------------------------------- */

static int dev_alloc(sg_grid *g, void **p, int64_t bytes, const char *what)
{
    cudaError_t e;
    if (g->alloc) {
        int r = g->alloc(g->alloc_ctx, p, bytes > 0 ? bytes : 16);
        if (r != SG_OK) {
            *p = NULL;
            return fail(r, "allocating %lld bytes for %s from the handle's allocator", (long long)bytes, what);
        }
        g->dev_bytes += bytes;
        return SG_OK;
    }
    e = cudaMalloc(p, (size_t)(bytes > 0 ? bytes : 16));
    if (e != cudaSuccess) {
        *p = NULL;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? SG_ERR_NOMEM : SG_ERR_CUDA,
                    "cudaMalloc(%lld) for %s: %s", (long long)bytes, what, cudaGetErrorString(e));
    }
    g->dev_bytes += bytes;
    return SG_OK;
}

/* Selects the handle's device for the duration of a call. */
static int enter(sg_grid *g, int *prev)
{
    cudaError_t e = cudaGetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (g->dev >= 0 && g->dev != *prev) CU(cudaSetDevice(g->dev), "cudaSetDevice");
    return SG_OK;
}

static void leave(sg_grid *g, int prev)
{
    if (g->dev >= 0 && g->dev != prev) cudaSetDevice(prev);
}

/* Allocates the handle's device state and uploads its tables.  The clears
 * and uploads go on `st` (the stream of the call that needs the state, never
 * the legacy default stream, so a serving loop's streams do not wait on
 * them), and the stream is synchronized before returning, so kernels on any
 * stream may read the tables afterwards. */
static int materialize(sg_grid *g, cudaStream_t st)
{
    const sg_layout *L = &g->L;
    sg_repack *rp = NULL;
    int k, r;
    cudaError_t ce;
    if (g->dev >= 0) return SG_OK;
    CU((cudaError_t)sgk_eval_setup(), "evaluation kernel set-up");
    CU(cudaGetDevice(&g->dev), "cudaGetDevice");
    if ((r = dev_alloc(g, (void **)&g->d_alpha, L->Npad * 4, "grid values")) != SG_OK) goto bad;
    if ((ce = cudaMemsetAsync(g->d_alpha, 0, (size_t)L->Npad * 4, st)) != cudaSuccess) {
        r = cuda_fail(ce, "cudaMemsetAsync");
        goto bad;
    }
    if ((r = dev_alloc(g, (void **)&g->d_err, 16, "error flag")) != SG_OK) goto bad;
    if ((ce = cudaMemsetAsync(g->d_err, 0, 16, st)) != cudaSuccess) {
        r = cuda_fail(ce, "cudaMemsetAsync");
        goto bad;
    }
    if ((r = sg_layout_eval_tables(L, &rp, g->blk3, g->blk2)) != SG_OK) {
        fail(r, "building the evaluation layout tables");
        goto bad;
    }
    if ((r = dev_alloc(g, (void **)&g->d_blk, L->Nblk * 4, "block layout")) != SG_OK) goto bad;
    if ((r = dev_alloc(g, (void **)&g->d_repack, L->S * (int64_t)sizeof(sg_repack), "repack table")) != SG_OK)
        goto bad;
    /* pageable sources: the copy has taken the bytes when the call returns */
    if ((ce = cudaMemcpyAsync(g->d_repack, rp, (size_t)L->S * sizeof(sg_repack), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess) {
        r = cuda_fail(ce, "uploading the repack table");
        goto bad;
    }
    free(rp);
    rp = NULL;
    g->eval_dirty = 1;
    for (k = 0; k < L->d; k++) {
        sg_chain *ch = NULL;
        uint32_t *seg = NULL;
        int64_t nch = 0, nseg = 0, c, cap32 = 0, cap64 = 0;
        int lmax_max = 0;
        if ((r = sg_layout_chains(L, k, &ch, &nch, &seg, &nseg)) != SG_OK) {
            fail(r, "building the sweep tables of dim %d", k);
            goto bad;
        }
        for (c = 0; c < nch; c++) {
            int j;
            int64_t e32 = 0, e64 = 0;
            for (j = 0; j <= ch[c].lmax; j++) {
                int64_t sz = (int64_t)1 << (ch[c].sigma + j);
                e32 += sz < 4 ? 4 : sz;
                e64 += sz < 2 ? 2 : sz;
            }
            if (e32 > cap32) cap32 = e32;
            if (e64 > cap64) cap64 = e64;
            if (ch[c].lmax > lmax_max) lmax_max = ch[c].lmax;
        }
        r = dev_alloc(g, (void **)&g->d_chains[k], nch * (int64_t)sizeof(sg_chain), "sweep chains");
        if (r == SG_OK) r = dev_alloc(g, (void **)&g->d_seg[k], nseg * 4, "sweep segments");
        if (r == SG_OK && nch > 0) {
            cudaError_t e =
                cudaMemcpyAsync(g->d_chains[k], ch, (size_t)nch * sizeof(sg_chain), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(g->d_seg[k], seg, (size_t)nseg * 4, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) r = cuda_fail(e, "uploading sweep tables");
        }
        free(ch);
        free(seg);
        if (r != SG_OK) goto bad;
        g->sweep[k].chains = g->d_chains[k];
        g->sweep[k].seg = g->d_seg[k];
        g->sweep[k].nchains = nch;
        g->sweep[k].lmax_max = lmax_max;
        g->sweep[k].cap32 = cap32;
        g->sweep[k].cap64 = cap64;
    }
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) {
        r = cuda_fail(ce, "uploading the grid tables");
        goto bad;
    }
    return SG_OK;
bad:
    cudaStreamSynchronize(st); /* nothing may still write the ranges freed below */
    free(rp);
    free_device(g);
    memset(g->d_chains, 0, sizeof(g->d_chains));
    memset(g->d_seg, 0, sizeof(g->d_seg));
    g->d_alpha = NULL;
    g->d_work = NULL;
    g->d_blk = NULL;
    g->d_repack = NULL;
    g->d_err = NULL;
    g->d_walk = NULL;
    g->d_scratch = g->d_io = NULL;
    g->scratch_bytes = g->io_bytes = g->dev_bytes = 0;
    g->dev = -1;
    return r;
}

/* Copies the N compact values into (or out of) the group-aligned layout:
 * one contiguous copy per level group. */
static int copy_groups(sg_grid *g, float *dst, const float *src, int to_device, enum cudaMemcpyKind kind,
                       cudaStream_t st)
{
    const sg_layout *L = &g->L;
    int s;
    for (s = 0; s < L->n; s++) {
        int64_t cnt = L->lidx[s + 1] - L->lidx[s];
        const float *sp;
        float *dp;
        if (cnt == 0) continue;
        sp = to_device ? src + L->lidx[s] : src + L->plidx[s];
        dp = to_device ? dst + L->plidx[s] : dst + L->lidx[s];
        CU(cudaMemcpyAsync(dp, sp, (size_t)cnt * 4, kind, st), "cudaMemcpyAsync (grid values)");
    }
    return SG_OK;
}

SG_API int sg_set_values(sg_grid *g, const float *values)
{
    int prev, r;
    if (!g || !values) return fail(SG_ERR_ARG, "sg_set_values: NULL argument");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    if ((r = materialize(g, 0)) == SG_OK &&
        (r = copy_groups(g, g->d_alpha, values, 1, cudaMemcpyHostToDevice, 0)) == SG_OK) {
        cudaError_t e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) r = cuda_fail(e, "sg_set_values");
        else g->has_values = 1, g->eval_dirty = 1;
    }
    leave(g, prev);
    return r;
}

SG_API int sg_set_values_device(sg_grid *g, const float *values, void *stream)
{
    int prev, r;
    if (!g || !values) return fail(SG_ERR_ARG, "sg_set_values_device: NULL argument");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    if ((r = materialize(g, (cudaStream_t)stream)) == SG_OK &&
        (r = copy_groups(g, g->d_alpha, values, 1, cudaMemcpyDeviceToDevice, (cudaStream_t)stream)) == SG_OK)
        g->has_values = 1, g->eval_dirty = 1;
    leave(g, prev);
    return r;
}

SG_API int sg_get_values(sg_grid *g, float *values)
{
    int prev, r;
    if (!g || !values) return fail(SG_ERR_ARG, "sg_get_values: NULL argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_get_values: no values have been set");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    if ((r = copy_groups(g, values, g->d_alpha, 0, cudaMemcpyDeviceToHost, 0)) == SG_OK)
        r = sg_sync(g, 0);
    leave(g, prev);
    return r;
}

SG_API int sg_get_values_device(sg_grid *g, float *values, void *stream)
{
    int prev, r;
    if (!g || !values) return fail(SG_ERR_ARG, "sg_get_values_device: NULL argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_get_values_device: no values have been set");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    r = copy_groups(g, values, g->d_alpha, 0, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    leave(g, prev);
    return r;
}

static void mark(sg_grid *g, int phase, int end, cudaStream_t st)
{
    if (!g->opt[SG_OPT_PROFILE]) return;
    if (!g->ev[phase][0]) {
        if (cudaEventCreate(&g->ev[phase][0]) != cudaSuccess ||
            cudaEventCreate(&g->ev[phase][1]) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
    }
    cudaEventRecord(g->ev[phase][end], st);
    if (end) g->ev_used[phase] = 1;
}

SG_API int sg_timings(sg_grid *g, double *ms)
{
    int k, prev, r;
    if (!g || !ms) return fail(SG_ERR_ARG, "sg_timings: NULL argument");
    for (k = 0; k < SG_NUM_PHASES; k++) ms[k] = -1.0;
    if (g->dev < 0) return SG_OK;
    if ((r = enter(g, &prev)) != SG_OK) return r;
    for (k = 0; k < SG_NUM_PHASES; k++) {
        float t = 0.0f;
        if (!g->ev_used[k]) continue;
        if (cudaEventSynchronize(g->ev[k][1]) != cudaSuccess ||
            cudaEventElapsedTime(&t, g->ev[k][0], g->ev[k][1]) != cudaSuccess) {
            r = cuda_fail(cudaGetLastError(), "sg_timings");
            break;
        }
        ms[k] = t;
    }
    leave(g, prev);
    return r;
}

static int hierarchize_on(sg_grid *g, cudaStream_t st)
{
    const sg_layout *L = &g->L;
    const int prec = (int)g->opt[SG_OPT_HIER_PRECISION];
    const int kern = (int)g->opt[SG_OPT_HIER_KERNEL];
    int k, e;
    if (prec == SG_HIER_FP64) {
        if (!g->d_work) {
            int r = dev_alloc(g, (void **)&g->d_work, L->Npad * 8, "FP64 working grid");
            if (r != SG_OK) return r;
        }
        if ((e = sgk_widen(g->d_alpha, g->d_work, L->Npad, st)) != cudaSuccess)
            return cuda_fail((cudaError_t)e, "widen");
        for (k = 0; k < L->d; k++) {
            const int fits = sgk_chain_smem_bytes(g->sweep[k].cap64, 8) >= 0;
            e = (kern != 2 && fits) ? sgk_sweep_chains_f64(g->d_work, &g->sweep[k], g->d_err, st)
                                    : sgk_sweep_gather_f64(g->d_work, &g->sweep[k], st);
            if (e != cudaSuccess) return cuda_fail((cudaError_t)e, "FP64 sweep");
        }
        if ((e = sgk_narrow(g->d_work, g->d_alpha, L->Npad, st)) != cudaSuccess)
            return cuda_fail((cudaError_t)e, "narrow");
        return SG_OK;
    }
    for (k = 0; k < L->d; k++) {
        const int fits = sgk_chain_smem_bytes(g->sweep[k].cap32, 4) >= 0;
        if (g->opt[SG_OPT_TEST_WAIT] > 0 && fits)
            e = sgk_sweep_chains_stall_f32(g->d_alpha, &g->sweep[k], g->d_err, g->opt[SG_OPT_TEST_WAIT] << 20, st);
        else
            e = (kern != 2 && fits) ? sgk_sweep_chains_f32(g->d_alpha, &g->sweep[k], g->d_err, st)
                                    : sgk_sweep_gather_f32(g->d_alpha, &g->sweep[k], st);
        if (e != cudaSuccess) return cuda_fail((cudaError_t)e, "FP32 sweep");
    }
    return SG_OK;
}

SG_API int sg_hierarchize_async(sg_grid *g, void *stream)
{
    int prev, r;
    if (!g) return fail(SG_ERR_ARG, "sg_hierarchize_async: NULL grid");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_hierarchize: no values have been set");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    mark(g, SG_PHASE_HIERARCHIZE, 0, (cudaStream_t)stream);
    r = hierarchize_on(g, (cudaStream_t)stream);
    g->eval_dirty = 1;
    mark(g, SG_PHASE_HIERARCHIZE, 1, (cudaStream_t)stream);
    leave(g, prev);
    return r;
}

SG_API int sg_hierarchize(sg_grid *g)
{
    int r = sg_hierarchize_async(g, 0);
    if (r != SG_OK) return r;
    return sg_sync(g, 0);
}

/* Device milliseconds of the fastest of `reps` runs of fn on st. */
static int time_best(int (*fn)(sg_grid *, void *), sg_grid *g, void *arg, cudaStream_t st, int reps, double *ms)
{
    cudaEvent_t e0 = NULL, e1 = NULL;
    float t;
    int i, r = SG_OK;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    *ms = 1e30;
    for (i = 0; e == cudaSuccess && r == SG_OK && i < reps; i++) {
        e = cudaEventRecord(e0, st);
        if (e == cudaSuccess) r = fn(g, arg);
        if (e == cudaSuccess && r == SG_OK) e = cudaEventRecord(e1, st);
        if (e == cudaSuccess && r == SG_OK) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess && r == SG_OK) e = cudaEventElapsedTime(&t, e0, e1);
        if (e == cudaSuccess && r == SG_OK && t < *ms) *ms = t;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (r == SG_OK && e != cudaSuccess) r = cuda_fail(e, "sg_autotune timing");
    return r;
}

typedef struct tune_eval_arg {
    const float *coords;
    float *out;
    int64_t m;
    cudaStream_t st;
    const float *saved; /* hierarchization: nodal values to restore first */
} tune_eval_arg;

static int tune_eval_once(sg_grid *g, void *a)
{
    const tune_eval_arg *t = (const tune_eval_arg *)a;
    return sg_evaluate_device(g, t->coords, t->out, t->m, t->st);
}

static int tune_hier_once(sg_grid *g, void *a)
{
    const tune_eval_arg *t = (const tune_eval_arg *)a;
    cudaError_t e = cudaMemcpyAsync(g->d_alpha, t->saved, (size_t)g->L.Npad * 4, cudaMemcpyDeviceToDevice, t->st);
    if (e != cudaSuccess) return cuda_fail(e, "sg_autotune restore");
    return hierarchize_on(g, t->st);
}

SG_API int sg_autotune(sg_grid *g, const float *coords, float *out, int64_t num_evals, void *stream, double *ms)
{
    static const int ppts[2] = {1, 2};
    tune_eval_arg ta;
    double t[SG_TUNE_TIMINGS], best = 1e30;
    float *saved = NULL;
    int prev, r = SG_OK, i, j, k, chains_apply = 0, bi = -1;
    if (!g || !coords || !out || num_evals < 1) return fail(SG_ERR_ARG, "sg_autotune: bad argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_autotune: no values have been set");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    for (i = 0; i < SG_TUNE_TIMINGS; i++) t[i] = -1.0;
    ta.coords = coords;
    ta.out = out;
    ta.m = num_evals;
    ta.st = (cudaStream_t)stream;
    /* evaluation: points per thread x spatial ordering (the per-point
     * arithmetic is the same in every setting, so results do not change) */
    for (i = 0; i < 2 && r == SG_OK; i++)
        for (j = 0; j < 2 && r == SG_OK; j++) {
            g->opt[SG_OPT_EVAL_PPT] = ppts[i];
            g->opt[SG_OPT_EVAL_SORT] = j;
            r = tune_eval_once(g, &ta); /* warm: grows the scratch, builds the block layout */
            if (r == SG_OK) r = time_best(tune_eval_once, g, &ta, ta.st, 2, &t[2 * i + j]);
            if (r == SG_OK && t[2 * i + j] < best) best = t[2 * i + j], bi = 2 * i + j;
        }
    if (r == SG_OK) {
        g->opt[SG_OPT_EVAL_PPT] = ppts[bi / 2];
        g->opt[SG_OPT_EVAL_SORT] = bi % 2;
    }
    /* subspace blocking at that setting (scratch and layout are built) */
    for (i = 0, best = 1e30, bi = -1; i < SG_EVAL_BLOCKINGS && r == SG_OK; i++) {
        g->opt[SG_OPT_EVAL_BLOCKING] = i + 1;
        r = time_best(tune_eval_once, g, &ta, ta.st, 2, &t[6 + i]);
        if (r == SG_OK && t[6 + i] < best) best = t[6 + i], bi = i;
    }
    if (r == SG_OK) g->opt[SG_OPT_EVAL_BLOCKING] = bi + 1;
    /* hierarchization: shared-memory chains (where they fit) vs gather; the
     * values are saved first and restored at the end */
    for (k = 0; k < g->L.d; k++)
        if (sgk_chain_smem_bytes(g->opt[SG_OPT_HIER_PRECISION] == SG_HIER_FP64 ? g->sweep[k].cap64 : g->sweep[k].cap32,
                                 g->opt[SG_OPT_HIER_PRECISION] == SG_HIER_FP64 ? 8 : 4) >= 0)
            chains_apply = 1;
    if (r == SG_OK) r = dev_alloc(g, (void **)&saved, g->L.Npad * 4, "sg_autotune saved values");
    if (r == SG_OK) {
        cudaError_t e = cudaMemcpyAsync(saved, g->d_alpha, (size_t)g->L.Npad * 4, cudaMemcpyDeviceToDevice, ta.st);
        if (e != cudaSuccess) r = cuda_fail(e, "sg_autotune save");
        ta.saved = saved;
        for (k = chains_apply ? 1 : 2; k <= 2 && r == SG_OK; k++) {
            g->opt[SG_OPT_HIER_KERNEL] = k;
            r = tune_hier_once(g, &ta);
            if (r == SG_OK) r = time_best(tune_hier_once, g, &ta, ta.st, 2, &t[3 + k]);
        }
        if (r == SG_OK) g->opt[SG_OPT_HIER_KERNEL] = (t[4] >= 0.0 && t[4] <= t[5]) ? 1 : 2;
        e = cudaMemcpyAsync(g->d_alpha, saved, (size_t)g->L.Npad * 4, cudaMemcpyDeviceToDevice, ta.st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ta.st);
        if (r == SG_OK && e != cudaSuccess) r = cuda_fail(e, "sg_autotune restore");
        g->eval_dirty = 1;
    }
    if (saved) dev_free(g, saved);
    if (saved) g->dev_bytes -= g->L.Npad * 4;
    if (ms)
        for (i = 0; i < SG_TUNE_TIMINGS; i++) ms[i] = t[i];
    leave(g, prev);
    return r == SG_OK ? sg_sync(g, stream) : r;
}

SG_API int sg_sync(sg_grid *g, void *stream)
{
    int prev, r = SG_OK, flag = 0;
    cudaError_t e;
    if (!g) return fail(SG_ERR_ARG, "sg_sync: NULL grid");
    if (g->dev < 0) return SG_OK;
    if ((r = enter(g, &prev)) != SG_OK) return r;
    e = cudaMemcpyAsync(&flag, g->d_err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) r = cuda_fail(e, "sg_sync");
    else if (flag) {
        cudaMemsetAsync(g->d_err, 0, sizeof(int), (cudaStream_t)stream);
        cudaStreamSynchronize((cudaStream_t)stream);
        r = fail(SG_ERR_TIMEOUT, "a device-side wait gave up; the grid values are not valid");
    }
    leave(g, prev);
    return r;
}

static int ensure(sg_grid *g, void **buf, int64_t *have, int64_t need, const char *what)
{
    int r;
    if (*have >= need) return SG_OK;
    if (*buf) {
        dev_free(g, *buf);
        g->dev_bytes -= *have;
        *buf = NULL;
        *have = 0;
    }
    need = (need + 0xFFFFF) & ~(int64_t)0xFFFFF;
    if ((r = dev_alloc(g, buf, need, what)) != SG_OK) return r;
    *have = need;
    return SG_OK;
}

static int eval_ppt(const sg_grid *g)
{
    if (g->opt[SG_OPT_EVAL_PPT] == 1 || g->opt[SG_OPT_EVAL_PPT] == 2) return (int)g->opt[SG_OPT_EVAL_PPT];
    return 2;
}

/* The evaluation plan of the grid's block layout at `ppt` points per
 * thread and the grid's blocking setting (0 = auto: wide). */
static void grid_plan(const sg_grid *g, int ppt, sg_eval_plan *p)
{
    int k;
    p->alpha = g->d_blk;
    p->d = g->L.d;
    p->n = g->L.n;
    for (k = 0; k < SG_MAX_DIMS; k++) p->lim[k] = k < g->L.d ? g->L.lim[k] : 0;
    for (k = 0; k < SG_MAX_LEVELS; k++) {
        p->blk3[k] = g->blk3[k];
        p->blk2[k] = g->blk2[k];
    }
    p->ppt = ppt;
    p->blocking = g->opt[SG_OPT_EVAL_BLOCKING] > 0 ? (int)g->opt[SG_OPT_EVAL_BLOCKING] - 1 : 0;
}

static int evaluate_on(sg_grid *g, const float *coords, float *out, int64_t m, cudaStream_t st)
{
    sg_eval_plan p;
    int e;
    if (g->eval_dirty) {
        if ((e = sgk_repack(g->d_alpha, g->d_blk, g->d_repack, g->L.S, st)) != cudaSuccess)
            return cuda_fail((cudaError_t)e, "repacking surpluses");
        g->eval_dirty = 0;
    }
    grid_plan(g, eval_ppt(g), &p);
    if (g->opt[SG_OPT_EVAL_SORT] && m > 1) {
        const int64_t sort_b = (sgk_sort_scratch_bytes(m, p.d) + 255) & ~(int64_t)255;
        const int64_t coords_b = (m * p.d * 4 + 255) & ~(int64_t)255;
        int r = ensure(g, &g->d_scratch, &g->scratch_bytes, sort_b + coords_b + m * 4, "evaluate scratch");
        char *base = (char *)g->d_scratch;
        float *sorted = (float *)(base + sort_b);
        int32_t *perm = (int32_t *)(base + sort_b + coords_b);
        if (r != SG_OK) return r;
        mark(g, SG_PHASE_SORT, 0, st);
        if ((e = sgk_sort_points(coords, m, p.d, base, sorted, perm, st)) != cudaSuccess)
            return cuda_fail((cudaError_t)e, "sorting query points");
        mark(g, SG_PHASE_SORT, 1, st);
        mark(g, SG_PHASE_EVALUATE, 0, st);
        e = sgk_evaluate(&p, sorted, perm, out, m, st);
        mark(g, SG_PHASE_EVALUATE, 1, st);
    } else {
        mark(g, SG_PHASE_EVALUATE, 0, st);
        e = sgk_evaluate(&p, coords, NULL, out, m, st);
        mark(g, SG_PHASE_EVALUATE, 1, st);
    }
    if (e != cudaSuccess) return cuda_fail((cudaError_t)e, "evaluate");
    return SG_OK;
}

SG_API int sg_evaluate_device(sg_grid *g, const float *coords, float *out, int64_t m, void *stream)
{
    int prev, r;
    if (!g || (m > 0 && (!coords || !out)) || m < 0) return fail(SG_ERR_ARG, "sg_evaluate_device: bad argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_evaluate: no values have been set");
    if (m > 0x7fffffffLL) return fail(SG_ERR_RANGE, "sg_evaluate: at most 2^31-1 points per call");
    if (m == 0) return SG_OK;
    if ((r = enter(g, &prev)) != SG_OK) return r;
    r = evaluate_on(g, coords, out, m, (cudaStream_t)stream);
    leave(g, prev);
    return r;
}

/* The no-allocation evaluation: as evaluate_on with sorting, but every
 * scratch region is carved from the library's fixed device array and no
 * device memory, event or other resource is created. */
SG_API int sg_evaluate_device_noalloc(sg_grid *g, const float *coords, float *out, int64_t m, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    sg_eval_plan p;
    int prev, r = SG_OK, e, k;
    void *scratch = NULL;
    int64_t have = 0, sort_b, coords_b;
    if (!g || m < 0 || (m > 0 && (!coords || !out))) return fail(SG_ERR_ARG, "sg_evaluate_device_noalloc: bad argument");
    if (!g->has_values || g->dev < 0)
        return fail(SG_ERR_STATE, "sg_evaluate_device_noalloc: the grid has no device state yet (set values first)");
    if (m > SG_NOALLOC_MAX_POINTS)
        return fail(SG_ERR_RANGE, "sg_evaluate_device_noalloc: %lld points exceed SG_NOALLOC_MAX_POINTS (%d)",
                    (long long)m, SG_NOALLOC_MAX_POINTS);
    if (m == 0) return SG_OK;
    sort_b = (sgk_sort_scratch_bytes(m, g->L.d) + 255) & ~(int64_t)255;
    coords_b = (m * g->L.d * 4 + 255) & ~(int64_t)255;
    if ((r = enter(g, &prev)) != SG_OK) return r;
    if ((e = sgk_noalloc_scratch(&scratch, &have)) != cudaSuccess) {
        r = cuda_fail((cudaError_t)e, "sg_evaluate_device_noalloc: scratch address");
    } else if (sort_b + coords_b + m * 4 > have) {
        r = fail(SG_ERR_RANGE, "sg_evaluate_device_noalloc: %lld points in %d dims need more than the %lld-byte scratch",
                 (long long)m, g->L.d, (long long)have);
    } else {
        char *base = (char *)scratch;
        float *sorted = (float *)(base + sort_b);
        int32_t *perm = (int32_t *)(base + sort_b + coords_b);
        if (g->eval_dirty) {
            if ((e = sgk_repack(g->d_alpha, g->d_blk, g->d_repack, g->L.S, st)) != cudaSuccess)
                r = cuda_fail((cudaError_t)e, "repacking surpluses");
            else
                g->eval_dirty = 0;
        }
        if (r == SG_OK) {
            grid_plan(g, eval_ppt(g), &p);
            /* the histogram is cleared inside the sort, so nothing left in
             * the shared array by an earlier call is read */
            if ((e = sgk_sort_points(coords, m, p.d, base, sorted, perm, st)) != cudaSuccess)
                r = cuda_fail((cudaError_t)e, "sorting query points");
            else if ((e = sgk_evaluate(&p, sorted, perm, out, m, st)) != cudaSuccess)
                r = cuda_fail((cudaError_t)e, "evaluate");
        }
    }
    leave(g, prev);
    return r;
}

SG_API int sg_evaluate(sg_grid *g, const float *coords, float *out, int64_t m)
{
    int prev, r;
    int64_t cb, need;
    float *dc, *dout;
    if (!g || (m > 0 && (!coords || !out)) || m < 0) return fail(SG_ERR_ARG, "sg_evaluate: bad argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_evaluate: no values have been set");
    if (m > 0x7fffffffLL) return fail(SG_ERR_RANGE, "sg_evaluate: at most 2^31-1 points per call");
    if (m == 0) return SG_OK;
    if ((r = enter(g, &prev)) != SG_OK) return r;
    cb = (m * g->L.d * 4 + 255) & ~(int64_t)255;
    need = cb + m * 4;
    if ((r = ensure(g, &g->d_io, &g->io_bytes, need, "evaluate staging")) == SG_OK) {
        dc = (float *)g->d_io;
        dout = (float *)((char *)g->d_io + cb);
        if (cudaMemcpyAsync(dc, coords, (size_t)(m * g->L.d * 4), cudaMemcpyHostToDevice, 0) != cudaSuccess)
            r = cuda_fail(cudaGetLastError(), "sg_evaluate: copying coordinates");
        else if ((r = evaluate_on(g, dc, dout, m, 0)) == SG_OK) {
            if (cudaMemcpyAsync(out, dout, (size_t)(m * 4), cudaMemcpyDeviceToHost, 0) != cudaSuccess)
                r = cuda_fail(cudaGetLastError(), "sg_evaluate: copying results");
            else
                r = sg_sync(g, 0);
        }
    }
    leave(g, prev);
    return r;
}

SG_API int sg_subspace_maxabs(sg_grid *g, float *maxabs)
{
    int prev, r;
    cudaError_t e;
    if (!g || !maxabs) return fail(SG_ERR_ARG, "sg_subspace_maxabs: NULL argument");
    if (!g->has_values) return fail(SG_ERR_STATE, "sg_subspace_maxabs: no values have been set");
    if ((r = enter(g, &prev)) != SG_OK) return r;
    r = ensure(g, &g->d_scratch, &g->scratch_bytes, g->L.S * 4, "subspace statistics");
    if (r == SG_OK) {
        e = (cudaError_t)sgk_subspace_maxabs(&g->L, g->d_alpha, (unsigned *)g->d_scratch, 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(maxabs, g->d_scratch, (size_t)g->L.S * 4, cudaMemcpyDeviceToHost, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) r = cuda_fail(e, "sg_subspace_maxabs");
    }
    leave(g, prev);
    return r;
}

SG_API int sg_sample_function(sg_grid *g, int fn, const double *params, int np, void *stream)
{
    int prev, r, e, need = 0;
    if (!g || np < 0 || np > SG_MAX_FN_PARAMS || (np > 0 && !params))
        return fail(SG_ERR_ARG, "sg_sample_function: bad argument");
    switch (fn) {
    case SG_FN_REFERENCE: case SG_FN_PROD4: case SG_FN_GAUSS: need = 0; break;
    case SG_FN_BUMP: need = 2; break;
    case SG_FN_QUAD: need = 3 * g->L.d; break;
    default: return fail(SG_ERR_ARG, "sg_sample_function: unknown function %d", fn);
    }
    if (np < need) return fail(SG_ERR_ARG, "sg_sample_function: function %d needs %d parameters", fn, need);
    if ((r = enter(g, &prev)) != SG_OK) return r;
    if ((r = materialize(g, (cudaStream_t)stream)) == SG_OK) {
        if ((e = sgk_sample(&g->L, fn, params, np, g->d_alpha, stream)) != cudaSuccess)
            r = cuda_fail((cudaError_t)e, "sg_sample_function");
        else
            g->has_values = 1, g->eval_dirty = 1;
    }
    leave(g, prev);
    return r;
}

SG_API int sg_idx2gp_device(const sg_grid *g, const int64_t *index, int *levels, int *indices, int64_t count,
                            void *stream)
{
    int e;
    if (!g || count < 0 || (count > 0 && (!index || !levels || !indices)))
        return fail(SG_ERR_ARG, "sg_idx2gp_device: bad argument");
    if ((e = sgk_idx2gp(&g->L, index, levels, indices, count, stream)) != cudaSuccess)
        return cuda_fail((cudaError_t)e, "sg_idx2gp_device");
    return SG_OK;
}

SG_API int sg_gp2idx_device(const sg_grid *g, const int *levels, const int *indices, int64_t *index, int64_t count,
                            void *stream)
{
    int e;
    if (!g || count < 0 || (count > 0 && (!index || !levels || !indices)))
        return fail(SG_ERR_ARG, "sg_gp2idx_device: bad argument");
    if ((e = sgk_gp2idx(&g->L, levels, indices, index, count, stream)) != cudaSuccess)
        return cuda_fail((cudaError_t)e, "sg_gp2idx_device");
    return SG_OK;
}

SG_API int sg_set_option(sg_grid *g, int option, int64_t value)
{
    if (!g) return fail(SG_ERR_ARG, "sg_set_option: NULL grid");
    switch (option) {
    case SG_OPT_HIER_PRECISION:
        if (value != SG_HIER_FP32 && value != SG_HIER_FP64) return fail(SG_ERR_ARG, "bad precision %lld", (long long)value);
        break;
    case SG_OPT_EVAL_SORT:
        if (value != 0 && value != 1) return fail(SG_ERR_ARG, "SG_OPT_EVAL_SORT is 0 or 1");
        break;
    case SG_OPT_EVAL_PPT:
        if (value < 0 || value > 2) return fail(SG_ERR_ARG, "SG_OPT_EVAL_PPT is 0, 1 or 2");
        break;
    case SG_OPT_HIER_KERNEL:
        if (value < 0 || value > 2) return fail(SG_ERR_ARG, "SG_OPT_HIER_KERNEL is 0, 1 or 2");
        break;
    case SG_OPT_PROFILE:
        if (value != 0 && value != 1) return fail(SG_ERR_ARG, "SG_OPT_PROFILE is 0 or 1");
        break;
    case SG_OPT_TEST_WAIT:
        if (value < 0 || value > 2048) return fail(SG_ERR_ARG, "SG_OPT_TEST_WAIT is 0 .. 2048");
        break;
    case SG_OPT_EVAL_BLOCKING:
        if (value < 0 || value > SG_EVAL_BLOCKINGS) return fail(SG_ERR_ARG, "SG_OPT_EVAL_BLOCKING is 0 .. %d", SG_EVAL_BLOCKINGS);
        break;
    default:
        return fail(SG_ERR_ARG, "unknown option %d", option);
    }
    g->opt[option] = value;
    return SG_OK;
}

SG_API int sg_get_option(const sg_grid *g, int option, int64_t *value)
{
    if (!g || !value || option < 1 || option >= NOPT) return fail(SG_ERR_ARG, "sg_get_option: bad argument");
    *value = g->opt[option];
    return SG_OK;
}

SG_API int sg_kernel_launches(int64_t *count)
{
    if (!count) return fail(SG_ERR_ARG, "sg_kernel_launches: NULL argument");
    *count = sgk_launches();
    return SG_OK;
}

SG_API int sg_device_bytes(const sg_grid *g, int64_t *bytes)
{
    if (!g || !bytes) return fail(SG_ERR_ARG, "sg_device_bytes: NULL argument");
    *bytes = g->dev_bytes;
    return SG_OK;
}

/* ---- internal, for the serving loop ------------------------------------- */

int sg_grid_prepare_eval(sg_grid *g, cudaStream_t st)
{
    int e;
    if (!g->eval_dirty) return SG_OK;
    if ((e = sgk_repack(g->d_alpha, g->d_blk, g->d_repack, g->L.S, st)) != cudaSuccess)
        return cuda_fail((cudaError_t)e, "repacking surpluses");
    g->eval_dirty = 0;
    return SG_OK;
}

int sg_grid_set_parts(sg_grid *g, int nparts, cudaStream_t st)
{
    const sg_layout *L = &g->L;
    uint32_t *tab;
    int64_t words;
    int r;
    cudaError_t e;
    if (nparts > SG_EVAL_MAX_PARTS) nparts = SG_EVAL_MAX_PARTS;
    if (L->d < 4 || nparts <= 1 || g->dev < 0) {
        g->nparts = 1;
        return SG_OK;
    }
    words = 2 * (int64_t)(L->d - 2) * L->n;
    tab = (uint32_t *)malloc((size_t)words * sizeof(uint32_t));
    if (!tab) return fail(SG_ERR_NOMEM, "sg_grid_set_parts: out of host memory");
    r = sg_layout_walk_tables(L, g->blk3, tab);
    if (r == SG_OK) r = sg_layout_walk_split(L, nparts, g->split);
    if (r == SG_OK && !g->d_walk) r = dev_alloc(g, (void **)&g->d_walk, words * 4, "walk tables");
    if (r == SG_OK) {
        /* pageable source: the copy has taken the bytes when the call returns */
        e = cudaMemcpyAsync(g->d_walk, tab, (size_t)words * 4, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) r = cuda_fail(e, "uploading the walk tables");
    }
    free(tab);
    if (r != SG_OK) return r;
    g->nparts = nparts;
    return SG_OK;
}

void sg_grid_eval_args(const sg_grid *g, const float *coords, float *out, int64_t m, sg_eval_args *a)
{
    sg_eval_plan p;
    int k;
    grid_plan(g, 2, &p);
    sgk_fill_eval_args(&p, coords, NULL, out, m, a);
    if (g->nparts > 1) {
        a->nparts = g->nparts;
        for (k = 0; k <= g->nparts; k++) a->split[k] = g->split[k];
        a->walk = g->d_walk;
    }
}
