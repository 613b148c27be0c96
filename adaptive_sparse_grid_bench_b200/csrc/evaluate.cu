/*
 * Evaluation kernels for sm_100a.
 *
 * Reference algorithm: evaluate0 in adaptive_sparse_grid_bench.c:1237-1274
 * (definition) and evaluate5 (c:1558-1688): for a query point x,
 *     u(x) = sum over subspaces l of  a[off(l) + idx(x, l)] * prod_k hat_k
 * with t_k = floor(x_k 2^l_k), idx(x, l) = row-major (t_0, ..., t_{d-1}) over
 * the subspace (dim 0 most significant) and hat_k = 1 - |x_k 2^(l_k+1) - (2t_k+1)|.
 *
 * B200 design.  One thread owns PPT query points; every warp walks the same
 * depth-first tree over level vectors (dims 0..d-1, each dim's level
 * ascending, sum(l) <= n-1, l_k <= limits[k]), so the loop structure is
 * uniform across the warp and partial products / partial cell indices are
 * shared between all subspaces of a subtree:
 *   - at depth k the next level's fractional part, cell index and hat come
 *     from the previous level's with a doubling (exact in FP32), so no
 *     division, no float->int conversion and no table appears in the walk;
 *   - the innermost dim's hats and cell indices are precomputed once per
 *     point in registers; its loop (one subspace per iteration) is one
 *     shift-add, one gather and one FMA per point;
 *   - subspace offsets come from a depth-first offset table (one broadcast
 *     load per subspace, shared by the whole warp);
 *   - the innermost partial sum is folded into a Kahan-compensated
 *     accumulator (compensated summation over subspaces).
 * Query points are first put in spatial (Morton) order on the GPU so that
 * the 32 points of a warp land in few cells of each subspace: the gathers
 * then touch few sectors and the grid is served from L1/L2.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kNL = SG_MAX_LEVELS; /* register arrays sized for any n */

struct EvalArgs {
    const float *__restrict__ alpha;
    const uint32_t *__restrict__ leaf;
    const float *__restrict__ coords;
    const int32_t *__restrict__ perm;
    float *__restrict__ out;
    int64_t num_evals;
    int nm1;
    int lim[SG_MAX_DIMS];
};

__device__ __forceinline__ void kahan_add(float &s, float &c, float v)
{
    const float y = __fsub_rn(v, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

/* hat at the current level from the fractional part y = frac(x 2^l) */
__device__ __forceinline__ float hat_of(float y)
{
    return 1.0f - fabsf(fmaf(2.0f, y, -1.0f));
}

template <int D, int K, int P>
struct Walk {
    static __device__ __forceinline__ void run(const EvalArgs &A, int budget, int &leaf,
                                               const float (&x)[P][D], const uint32_t (&T)[P],
                                               const float (&hl)[P][kNL], const float (&pin)[P],
                                               const uint32_t (&iin)[P], float (&sum)[P],
                                               float (&comp)[P])
    {
        if constexpr (K == D - 1) {
            /* innermost dim: one subspace per level j */
            const int jmax = min(A.lim[K], budget);
            float s[P];
#pragma unroll
            for (int p = 0; p < P; ++p) s[p] = 0.0f;
#pragma unroll
            for (int j = 0; j < kNL; ++j) {
                if (j > jmax) break;
                const uint32_t off = __ldg(A.leaf + leaf + j);
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const uint32_t idx = (iin[p] << j) + (T[p] >> (kNL - 1 - j));
                    s[p] = fmaf(hl[p][j], __ldg(A.alpha + off + idx), s[p]);
                }
            }
            leaf += jmax + 1;
#pragma unroll
            for (int p = 0; p < P; ++p) kahan_add(sum[p], comp[p], pin[p] * s[p]);
        } else {
            const int lmax = min(A.lim[K], budget);
            float y[P];
            uint32_t t[P], J[P];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                y[p] = x[p][K];
                t[p] = 0;
                J[p] = iin[p];
            }
            for (int l = 0; l <= lmax; ++l) {
                if (l) {
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const float y2 = y[p] + y[p];
                        const bool b = y2 >= 1.0f;
                        y[p] = b ? y2 - 1.0f : y2;
                        t[p] = (t[p] << 1) | (uint32_t)b;
                        J[p] <<= 1;
                    }
                }
                float pn[P];
                uint32_t in[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    pn[p] = pin[p] * hat_of(y[p]);
                    in[p] = J[p] + t[p];
                }
                Walk<D, K + 1, P>::run(A, budget - l, leaf, x, T, hl, pn, in, sum, comp);
            }
        }
    }
};

template <int D, int P>
__global__ void __launch_bounds__(kThreads) k_evaluate(const EvalArgs A)
{
    const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t base = warp * (32 * P) + lane;

    float x[P][D];
    bool valid[P], nan_in[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int64_t i = base + 32 * p;
        valid[p] = i < A.num_evals;
        nan_in[p] = false;
        bool inside = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float v = valid[p] ? A.coords[i * D + k] : 0.0f;
            nan_in[p] |= (v != v);
            inside &= (v >= 0.0f) && (v < 1.0f);
            x[p][k] = v;
        }
        /* outside [0,1)^d every basis function is 0: walk at x = 0 (always
         * in range) and write 0 (NaN for NaN input) instead */
        if (!inside) {
#pragma unroll
            for (int k = 0; k < D; ++k) x[p][k] = 0.0f;
        }
        valid[p] = valid[p] && inside;
    }

    /* innermost dim: hats and cell indices of every level */
    uint32_t T[P];
    float hl[P][kNL];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float y = x[p][D - 1];
        T[p] = (uint32_t)(y * (float)(1u << (kNL - 1)));
#pragma unroll
        for (int j = 0; j < kNL; ++j) {
            hl[p][j] = hat_of(y);
            const float y2 = y + y;
            y = y2 >= 1.0f ? y2 - 1.0f : y2;
        }
    }

    float pin[P], sum[P], comp[P];
    uint32_t iin[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        pin[p] = 1.0f;
        iin[p] = 0;
        sum[p] = 0.0f;
        comp[p] = 0.0f;
    }
    int leaf = 0;
    Walk<D, 0, P>::run(A, A.nm1, leaf, x, T, hl, pin, iin, sum, comp);

#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int64_t i = base + 32 * p;
        if (i < A.num_evals) {
            const float r = valid[p] ? __fsub_rn(sum[p], comp[p]) : (nan_in[p] ? __int_as_float(0x7fc00000) : 0.0f);
            A.out[A.perm ? A.perm[i] : i] = r;
        }
    }
}

template <int D, int P>
int launch_eval(const EvalArgs &A, void *stream)
{
    const int64_t per_block = (int64_t)kThreads * P;
    const int64_t blocks = (A.num_evals + per_block - 1) / per_block;
    if (blocks > 0x7fffffff) return cudaErrorInvalidValue;
    k_evaluate<D, P><<<(unsigned)blocks, kThreads, 0, (cudaStream_t)stream>>>(A);
    return cudaGetLastError();
}

template <int D>
int dispatch_ppt(const EvalArgs &A, int ppt, void *stream)
{
    if (ppt == 2) return launch_eval<D, 2>(A, stream);
    return launch_eval<D, 1>(A, stream);
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
    if (b1 > 1) {
        const int64_t b2 = (b1 + per - 1) / per;
        uint32_t *t2 = tmp + b1;
        k_scan_blocks<<<(unsigned)b2, kThreads, 0, st>>>(t1, b1, t2);
        if (b2 > 1) {
            if (b2 > per) return cudaErrorInvalidValue;
            k_scan_blocks<<<1, kThreads, 0, st>>>(t2, b2, nullptr);
            k_scan_add<<<(unsigned)b2, kThreads, 0, st>>>(t1, b1, t2);
        }
        k_scan_add<<<(unsigned)b1, kThreads, 0, st>>>(v, m, t1);
    }
    return cudaGetLastError();
}

} // namespace

extern "C" {

int sgk_evaluate(const sg_eval_plan *p, const float *coords, const int32_t *perm, float *out,
                 int64_t num_evals, void *stream)
{
    if (num_evals <= 0) return cudaSuccess;
    EvalArgs A;
    A.alpha = p->alpha;
    A.leaf = p->leaf;
    A.coords = coords;
    A.perm = perm;
    A.out = out;
    A.num_evals = num_evals;
    A.nm1 = p->n - 1;
    for (int k = 0; k < SG_MAX_DIMS; ++k) A.lim[k] = k < p->d ? p->lim[k] : 0;
    const int ppt = p->ppt;
    switch (p->d) {
#define SG_D(DD) \
    case DD: return dispatch_ppt<DD>(A, ppt, stream);
        SG_D(1) SG_D(2) SG_D(3) SG_D(4) SG_D(5) SG_D(6) SG_D(7) SG_D(8) SG_D(9) SG_D(10)
        SG_D(11) SG_D(12) SG_D(13) SG_D(14) SG_D(15) SG_D(16) SG_D(17) SG_D(18) SG_D(19)
        SG_D(20)
#undef SG_D
    default: return cudaErrorInvalidValue;
    }
}

int64_t sgk_sort_scratch_bytes(int64_t num_evals, int d)
{
    const int64_t bins = (int64_t)1 << sort_key_bits(num_evals, d);
    (void)d;
    return (num_evals + bins + scan_tmp_words(bins)) * 4 + 256;
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
    int r = scan_exclusive(hist, bins, tmp, st);
    if (r != cudaSuccess) return r;
    k_sort_scatter<<<(unsigned)g, 256, 0, st>>>(coords, n, d, keys, hist, sorted, perm);
    return cudaGetLastError();
}

} // extern "C"
