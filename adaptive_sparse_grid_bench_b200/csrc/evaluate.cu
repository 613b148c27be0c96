/*
 * Evaluation support on sm_100a: the compact -> block layout repack, the
 * spatial (Morton) ordering of query points, and the launchers of the
 * evaluation kernels.  The kernels themselves (one instantiation per d,
 * eval_d*.cu) are in eval_impl.cuh, which describes the walk; reference
 * algorithm: evaluate0 in adaptive_sparse_grid_bench.c:1237-1274 and
 * evaluate5 (c:1558-1688).
 *
 * Query points are put in Morton order on the GPU first (counting sort over
 * 2^20 cells: keys, a three-level scan, a stable scatter), so the 32 points
 * of a warp land in few cells of each subspace: their gathers touch few
 * sectors and the grid is served from L1/L2.  Results are scattered back to
 * the caller's order by the permutation.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "eval_args.h"
#include "sg_kernels.h"

namespace {

constexpr int kThreads = 256;

/* Adds the parts of split sums in part order with Kahan compensation; CTA
 * b covers kThreads points of request items[b].x from point items[b].y
 * (sorted positions when the request has a permutation: the sum of point i
 * goes to out[perm[i]]). */
__global__ void __launch_bounds__(kThreads) k_combine_parts(const sg_eval_args *__restrict__ grids,
                                                            const int2 *__restrict__ items)
{
    const int2 item = items[blockIdx.x];
    const sg_eval_args *A = grids + item.x;
    const int64_t m = A->num_evals, i = (int64_t)item.y + threadIdx.x;
    if (i >= m) return;
    const int np = A->nparts;
    const float *src = A->part_out;
    float s = 0.0f, c = 0.0f;
    for (int k = 0; k < np; ++k) {
        const float y = __fsub_rn(src[k * m + i], c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    A->out[A->perm ? A->perm[i] : i] = __fsub_rn(s, c);
}

/* compact (group-aligned) layout -> block layout: every value of level b
 * of dim B goes to slot b of the 2^(L-b) paths of its pole that pass
 * through its cell */
__global__ void k_repack(const float *__restrict__ src, float *__restrict__ dst,
                         const sg_repack *__restrict__ rp, int64_t nsub)
{
    /* one warp per subspace: most subspaces hold a few values, and a warp
     * per subspace keeps many descriptor loads in flight */
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t q = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); q < nsub; q += nw) {
        const sg_repack r = rp[q];
        const int ab = r.a + r.b, cab = r.c + ab;
        const int rep = r.L - r.b; /* the value fills slot b of 2^rep paths */
        const int n = 1 << (r.s + rep);
        const uint32_t w = (uint32_t)SG_PATH_WIDTH(r.L + 1);
        for (int f = threadIdx.x & 31; f < n; f += 32) {
            const uint32_t e = (uint32_t)f >> rep, j = (uint32_t)f & ((1u << rep) - 1u);
            const uint32_t I = e >> cab;
            const uint32_t tc = (e >> ab) & ((1u << r.c) - 1u);
            const uint32_t ta = (e >> r.b) & ((1u << r.a) - 1u);
            const uint32_t tb = e & ((1u << r.b) - 1u);
            const uint32_t path = (tb << rep) | j; /* finest cell t_L of the path */
            dst[r.dst + I * r.blk + tc * r.sub + ta * r.plen + path * w] = src[r.src + e];
        }
    }
}

/* ---- spatial ordering of the query points ------------------------------ */

struct SortGeom {
    int key_bits; /* total Morton bits                   */
};

__device__ __forceinline__ uint32_t morton_key(const float *x, int d, int key_bits)
{
    uint32_t key = 0;
    for (int b = 0; b < key_bits; ++b) {
        const int k = b % d;
        const int lvl = b / d; /* bit lvl (from the top) of coordinate k */
        float v = x[k];
        v = v >= 0.0f ? (v < 1.0f ? v : 0.99999994f) : 0.0f;
        const uint32_t q = (uint32_t)(v * 16777216.0f); /* 24 fraction bits */
        key = (key << 1) | ((q >> (23 - lvl)) & 1u);
    }
    return key;
}

__global__ void k_sort_keys(const float *__restrict__ coords, int64_t n, int d, int key_bits,
                            uint32_t *__restrict__ keys, uint32_t *__restrict__ hist)
{
    float x[SG_MAX_DIMS];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        for (int k = 0; k < d; ++k) x[k] = coords[i * d + k];
        const uint32_t key = morton_key(x, d, key_bits);
        keys[i] = key;
        atomicAdd(hist + key, 1u);
    }
}

/* Exclusive scan of `n` counters in blocks of 2 * kThreads; block totals out. */
__global__ void k_scan_blocks(uint32_t *__restrict__ v, int64_t n, uint32_t *__restrict__ totals)
{
    __shared__ uint32_t warp_sums[kThreads / 32];
    const int64_t i0 = (blockIdx.x * (int64_t)kThreads + threadIdx.x) * 2;
    const uint32_t a = i0 < n ? v[i0] : 0u;
    const uint32_t b = i0 + 1 < n ? v[i0 + 1] : 0u;
    uint32_t s = a + b, incl = s;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint32_t ws = lane < kThreads / 32 ? warp_sums[lane] : 0u, wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < kThreads / 32) warp_sums[lane] = wi - ws;
        if (lane == kThreads / 32 - 1 && totals) totals[blockIdx.x] = wi;
    }
    __syncthreads();
    const uint32_t excl = incl - s + warp_sums[w];
    if (i0 < n) v[i0] = excl;
    if (i0 + 1 < n) v[i0 + 1] = excl + a;
}

__global__ void k_scan_add(uint32_t *__restrict__ v, int64_t n, const uint32_t *__restrict__ offs)
{
    const int64_t i0 = (blockIdx.x * (int64_t)kThreads + threadIdx.x) * 2;
    const uint32_t o = offs[blockIdx.x];
    if (i0 < n) v[i0] += o;
    if (i0 + 1 < n) v[i0 + 1] += o;
}

__global__ void k_sort_scatter(const float *__restrict__ coords, int64_t n, int d,
                               const uint32_t *__restrict__ keys, uint32_t *__restrict__ cursor,
                               float *__restrict__ sorted, int32_t *__restrict__ perm)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t pos = atomicAdd(cursor + keys[i], 1u);
        for (int k = 0; k < d; ++k) sorted[(int64_t)pos * d + k] = coords[i * d + k];
        perm[pos] = (int32_t)i;
    }
}

/* Batched form: CTA b handles 256 points of grid items[b].x from local
 * point items[b].y; the key of a point is its grid's bin base plus its
 * Morton cell, so the bins of one grid are contiguous and, after one scan
 * over all bins, a grid's points land inside its own point range. */
__global__ void __launch_bounds__(256) k_bsort_keys(const float *__restrict__ coords,
                                                    const sg_bsort_grid *__restrict__ grids,
                                                    const int2 *__restrict__ items, uint32_t *__restrict__ keys,
                                                    uint32_t *__restrict__ hist)
{
    const int2 it = items[blockIdx.x];
    const sg_bsort_grid G = grids[it.x];
    const int64_t i = (int64_t)it.y + threadIdx.x;
    if (i >= G.m) return;
    float x[SG_MAX_DIMS];
    for (int k = 0; k < G.d; ++k) x[k] = coords[G.coff + i * G.d + k];
    const uint32_t key = G.bin_base + morton_key(x, G.d, G.kb);
    keys[G.pt_off + i] = key;
    atomicAdd(hist + key, 1u);
}

__global__ void __launch_bounds__(256) k_bsort_scatter(const float *__restrict__ coords,
                                                       const sg_bsort_grid *__restrict__ grids,
                                                       const int2 *__restrict__ items,
                                                       const uint32_t *__restrict__ keys,
                                                       uint32_t *__restrict__ cursor, float *__restrict__ sorted,
                                                       int32_t *__restrict__ perm)
{
    const int2 it = items[blockIdx.x];
    const sg_bsort_grid G = grids[it.x];
    const int64_t i = (int64_t)it.y + threadIdx.x;
    if (i >= G.m) return;
    const int64_t pos = (int64_t)atomicAdd(cursor + keys[G.pt_off + i], 1u) - G.pt_off; /* local position */
    for (int k = 0; k < G.d; ++k) sorted[G.coff + pos * G.d + k] = coords[G.coff + i * G.d + k];
    perm[G.pt_off + pos] = (int32_t)i;
}

int sort_key_bits(int64_t n, int d)
{
    int kb = 0;
    while (kb < 20 && ((int64_t)16 << kb) < n) ++kb;
    if (kb < 1) kb = 1;
    (void)d;
    return kb;
}

/* Scan of m counters: at most two levels of blocks (m <= 512 * 512 * 2 * 2). */
int64_t scan_tmp_words(int64_t m)
{
    const int64_t per = 2 * kThreads;
    const int64_t b1 = (m + per - 1) / per;
    const int64_t b2 = (b1 + per - 1) / per;
    return b1 + b2 + 1;
}

int scan_exclusive(uint32_t *v, int64_t m, uint32_t *tmp, cudaStream_t st)
{
    const int64_t per = 2 * kThreads;
    const int64_t b1 = (m + per - 1) / per;
    uint32_t *t1 = tmp;
    k_scan_blocks<<<(unsigned)b1, kThreads, 0, st>>>(v, m, t1);
    sgk_count(1);
    if (b1 > 1) {
        const int64_t b2 = (b1 + per - 1) / per;
        uint32_t *t2 = tmp + b1;
        k_scan_blocks<<<(unsigned)b2, kThreads, 0, st>>>(t1, b1, t2);
        sgk_count(1);
        if (b2 > 1) {
            if (b2 > per) return cudaErrorInvalidValue;
            k_scan_blocks<<<1, kThreads, 0, st>>>(t2, b2, nullptr);
            sgk_count(1);
            k_scan_add<<<(unsigned)b2, kThreads, 0, st>>>(t1, b1, t2);
            sgk_count(1);
        }
        k_scan_add<<<(unsigned)b1, kThreads, 0, st>>>(v, m, t1);
        sgk_count(1);
    }
    return cudaGetLastError();
}

} // namespace

extern "C" {

void sgk_fill_eval_args(const sg_eval_plan *p, const float *coords, const int32_t *perm, float *out,
                        int64_t num_evals, sg_eval_args *A)
{
    A->alpha = p->alpha;
    A->coords = coords;
    A->perm = perm;
    A->out = out;
    A->num_evals = num_evals;
    A->nm1 = p->n - 1;
    for (int k = 0; k < SG_MAX_DIMS; ++k) A->lim[k] = k < p->d ? p->lim[k] : 0;
    for (int r = 0; r < SG_MAX_LEVELS; ++r) {
        A->blk3[r] = p->blk3[r];
        A->blk2[r] = p->blk2[r];
    }
    const int la = p->d >= 2 ? p->lim[p->d - 2] : 0, lb = p->lim[p->d - 1], lc = p->d >= 3 ? p->lim[p->d - 3] : 0;
    A->lim2 = p->d >= 2 ? (la < lb ? la : lb) : 0;
    A->lim3 = p->d >= 3 ? (lc < A->lim2 ? lc : A->lim2) : 0;
    A->nparts = 1;
    for (int k = 0; k <= SG_EVAL_MAX_PARTS; ++k) A->split[k] = k ? 0xFFFFFFFFu : 0u;
    A->part_out = NULL;
    A->walk = NULL;
}

int sgk_eval_setup(void)
{
    /* once per device: the attribute calls are host-side and must not run
     * inside a stream capture, so they come before any evaluation launch */
    static std::atomic<int> done[64];
    int dev = 0, e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (done[dev].load(std::memory_order_acquire)) return cudaSuccess;
#define SG_D(DD) \
    if ((e = eval_setup<DD>()) != cudaSuccess) return e;
    SG_D(1) SG_D(2) SG_D(3) SG_D(4) SG_D(5) SG_D(6) SG_D(7) SG_D(8) SG_D(9) SG_D(10)
    SG_D(11) SG_D(12) SG_D(13) SG_D(14) SG_D(15) SG_D(16) SG_D(17) SG_D(18) SG_D(19) SG_D(20)
#undef SG_D
    done[dev].store(1, std::memory_order_release);
    return cudaSuccess;
}

int sgk_evaluate(const sg_eval_plan *p, const float *coords, const int32_t *perm, float *out,
                 int64_t num_evals, void *stream)
{
    if (num_evals <= 0) return cudaSuccess;
    EvalArgs A;
    sgk_fill_eval_args(p, coords, perm, out, num_evals, &A);
    const int ppt = p->ppt, bl = p->blocking >= 0 && p->blocking < SG_EVAL_BLOCKINGS ? p->blocking : 0;
    switch (p->d) {
#define SG_D(DD) \
    case DD: return eval_launch<DD>(A, ppt, bl, stream);
        SG_D(1) SG_D(2) SG_D(3) SG_D(4) SG_D(5) SG_D(6) SG_D(7) SG_D(8) SG_D(9) SG_D(10)
        SG_D(11) SG_D(12) SG_D(13) SG_D(14) SG_D(15) SG_D(16) SG_D(17) SG_D(18) SG_D(19)
        SG_D(20)
#undef SG_D
    default: return cudaErrorInvalidValue;
    }
}

int sgk_evaluate_batch(int d, const sg_eval_args *grids, const int32_t *items, int nitems, int ppt, int blocking,
                       void *stream)
{
    const int2 *it = reinterpret_cast<const int2 *>(items);
    const int bl = blocking >= 0 && blocking < SG_EVAL_BLOCKINGS ? blocking : 0;
    switch (d) {
#define SG_D(DD) \
    case DD: return eval_batch_launch<DD>(grids, it, nitems, ppt, bl, stream);
        SG_D(1) SG_D(2) SG_D(3) SG_D(4) SG_D(5) SG_D(6) SG_D(7) SG_D(8) SG_D(9) SG_D(10)
        SG_D(11) SG_D(12) SG_D(13) SG_D(14) SG_D(15) SG_D(16) SG_D(17) SG_D(18) SG_D(19)
        SG_D(20)
#undef SG_D
    default: return cudaErrorInvalidValue;
    }
}

int sgk_combine_parts(const sg_eval_args *grids, const int32_t *items, int nitems, void *stream)
{
    if (nitems <= 0) return cudaSuccess;
    k_combine_parts<<<nitems, kThreads, 0, (cudaStream_t)stream>>>(grids, reinterpret_cast<const int2 *>(items));
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_repack(const float *src, float *dst, const sg_repack *rp, int64_t nsub, void *stream)
{
    if (nsub <= 0) return cudaSuccess;
    int64_t g = (nsub + 7) / 8;
    if (g > 148 * 16) g = 148 * 16;
    k_repack<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(src, dst, rp, nsub);
    sgk_count(1);
    return cudaGetLastError();
}

int64_t sgk_sort_scratch_bytes(int64_t num_evals, int d)
{
    const int64_t bins = (int64_t)1 << sort_key_bits(num_evals, d);
    (void)d;
    return (num_evals + bins + scan_tmp_words(bins)) * 4 + 256;
}

int sgk_batch_sort_bits(int64_t m, int d) { return sort_key_bits(m, d); }

int64_t sgk_batch_sort_scratch_bytes(int64_t npts, int64_t nbins)
{
    return (npts + nbins + scan_tmp_words(nbins)) * 4 + 256;
}

int sgk_batch_sort_points(const float *coords, const sg_bsort_grid *grids, const int32_t *items, int nitems,
                          int64_t npts, int64_t nbins, void *scratch, float *sorted, int32_t *perm, void *stream)
{
    if (nitems <= 0 || npts <= 0) return cudaSuccess;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *keys = (uint32_t *)scratch;
    uint32_t *hist = keys + npts;
    uint32_t *tmp = hist + nbins;
    const int2 *it = reinterpret_cast<const int2 *>(items);
    cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)nbins * 4, st);
    if (e != cudaSuccess) return e;
    k_bsort_keys<<<nitems, 256, 0, st>>>(coords, grids, it, keys, hist);
    sgk_count(1);
    int r = scan_exclusive(hist, nbins, tmp, st);
    if (r != cudaSuccess) return r;
    k_bsort_scatter<<<nitems, 256, 0, st>>>(coords, grids, it, keys, hist, sorted, perm);
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_sort_points(const float *coords, int64_t n, int d, void *scratch, float *sorted,
                    int32_t *perm, void *stream)
{
    if (n <= 0) return cudaSuccess;
    cudaStream_t st = (cudaStream_t)stream;
    const int kb = sort_key_bits(n, d);
    const int64_t bins = (int64_t)1 << kb;
    uint32_t *keys = (uint32_t *)scratch;
    uint32_t *hist = keys + n;
    uint32_t *tmp = hist + bins;
    cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)bins * 4, st);
    if (e != cudaSuccess) return e;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_sort_keys<<<(unsigned)g, 256, 0, st>>>(coords, n, d, kb, keys, hist);
    sgk_count(1);
    int r = scan_exclusive(hist, bins, tmp, st);
    if (r != cudaSuccess) return r;
    k_sort_scatter<<<(unsigned)g, 256, 0, st>>>(coords, n, d, keys, hist, sorted, perm);
    sgk_count(1);
    return cudaGetLastError();
}

} // extern "C"
