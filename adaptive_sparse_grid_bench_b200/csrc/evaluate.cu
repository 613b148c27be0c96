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
 * depth-first tree over the level vectors of the prefix dims 0..d-3 (each
 * dim's level ascending, sum(l) <= n-1, l_k <= limits[k]), so control flow is
 * uniform across the warp and partial products / partial cell indices are
 * shared by all subspaces below a node.  At depth d-2 the walk reaches a
 * block: every subspace of the two innermost dims (A = d-2, B = d-1) under
 * that prefix, stored contiguously per prefix cell in the block layout (see
 * sg_layout.h), with dim B's levels as a 1-D heap.  The surplus of (a, b) is
 * then at base + aoff(a) + t_a*plen(a) + (2^b - 1 + t_b):
 *   - base is one multiply-add per block and point; the row offset one
 *     multiply-add per row; 2^b - 1 + t_b and the hats of dims A and B are
 *     precomputed per point in registers, so each subspace costs one add,
 *     one gather and one FMA;
 *   - blocks of budget R < 12 (all of them in regular grids up to n = 12)
 *     run fully unrolled, so a block's gathers issue back to back;
 *   - hats of the prefix dims come from the previous level's with a doubling
 *     (exact in FP32), so no division or table appears in the walk;
 *   - each block's partial sum enters a Kahan-compensated accumulator.
 * Query points are first put in spatial (Morton) order on the GPU so that
 * the 32 points of a warp land in few cells of each subspace: the gathers
 * then touch few sectors and the grid is served from L1/L2.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kNB = 12; /* blocks with level budget R < kNB run fully unrolled */
constexpr int kTB = 15; /* T = floor(x 2^15) holds the cells of levels 0..15  */

struct EvalArgs {
    const float *__restrict__ alpha;          /* block layout                 */
    const uint32_t *__restrict__ prefix_base; /* one block base per prefix    */
    const float *__restrict__ coords;
    const int32_t *__restrict__ perm;
    float *__restrict__ out;
    int64_t num_evals;
    int nm1;                                  /* n - 1                        */
    int regular2;                             /* last two dims unrestricted   */
    int lim[SG_MAX_DIMS];
    uint32_t blk[SG_MAX_LEVELS];              /* block size per budget R      */
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

/* next level: y <- frac(2y), t <- 2t + floor(2y); exact in FP32 */
__device__ __forceinline__ void step_level(float &y, uint32_t &t)
{
    const float y2 = y + y;
    const bool b = y2 >= 1.0f;
    y = b ? y2 - 1.0f : y2;
    t = (t << 1) | (uint32_t)b;
}

/* Per-point values of the two innermost dims (A = d-2, B = d-1). */
template <int P>
struct Inner {
    float hB[P][kNB];    /* hat of dim B at level b                      */
    uint32_t cB[P][kNB]; /* heap index 2^b - 1 + t_b of dim B            */
    float hA[P][kNB];    /* hat of dim A at level a                      */
    uint32_t TA[P];      /* floor(x_A 2^15): t_a = TA >> (15 - a)        */
};

__host__ __device__ constexpr uint32_t aoff_reg(int R, int a)
{
    uint32_t o = 0;
    for (int q = 0; q < a; ++q) o += (1u << q) * ((2u << (R - q)) - 1u);
    return o;
}

/* One block of budget R of a grid whose last two dims are unrestricted:
 * rows a = 0..R, row a holds 2^a poles of R-a+1 levels.  Fully unrolled:
 * one add, one gather and one FMA per subspace and point. */
template <int R, int P>
__device__ __forceinline__ void block_fixed(const float *__restrict__ alpha, const uint32_t (&base)[P],
                                            const Inner<P> &in, float (&s)[P])
{
#pragma unroll
    for (int a = 0; a <= R; ++a) {
        const uint32_t plen = (2u << (R - a)) - 1u;
        const uint32_t ao = aoff_reg(R, a);
        uint32_t rb[P];
        float sr[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            rb[p] = base[p] + ao + (in.TA[p] >> (kTB - a)) * plen;
            sr[p] = 0.0f;
        }
#pragma unroll
        for (int b = 0; b <= R - a; ++b)
#pragma unroll
            for (int p = 0; p < P; ++p)
                sr[p] = fmaf(in.hB[p][b], __ldg(alpha + rb[p] + in.cB[p][b]), sr[p]);
#pragma unroll
        for (int p = 0; p < P; ++p) s[p] = fmaf(in.hA[p][a], sr[p], s[p]);
    }
}

template <int R, int P>
__device__ __forceinline__ bool block_dispatch(int r, const float *__restrict__ alpha, const uint32_t (&base)[P],
                                               const Inner<P> &in, float (&s)[P])
{
    if (r == R) {
        block_fixed<R, P>(alpha, base, in, s);
        return true;
    }
    if constexpr (R + 1 < kNB) return block_dispatch<R + 1, P>(r, alpha, base, in, s);
    return false;
}

/* Any block: runtime loops, hats stepped level by level (limits on the last
 * two dims, budgets R >= kNB, and d = 1 where dim A is absent). */
template <int D, int P>
__device__ __forceinline__ void block_generic(const EvalArgs &A, int R, const float (&x)[P][D],
                                              const uint32_t (&base)[P], float (&s)[P])
{
    const int limA = D >= 2 ? A.lim[D - 2] : 0;
    const int limB = A.lim[D - 1];
    const int amax = min(R, limA);
    uint32_t aoff = 0;
    float yA[P];
    uint32_t tA[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        yA[p] = D >= 2 ? x[p][D >= 2 ? D - 2 : 0] : 0.0f;
        tA[p] = 0;
    }
    for (int a = 0; a <= amax; ++a) {
        if (a) {
#pragma unroll
            for (int p = 0; p < P; ++p) step_level(yA[p], tA[p]);
        }
        const int rl = min(R - a, limB) + 1;
        const uint32_t plen = (1u << rl) - 1u;
        float yB[P], sr[P];
        uint32_t tB[P], rb[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            yB[p] = x[p][D - 1];
            tB[p] = 0;
            sr[p] = 0.0f;
            rb[p] = base[p] + aoff + tA[p] * plen;
        }
        for (int b = 0; b < rl; ++b) {
            if (b) {
#pragma unroll
                for (int p = 0; p < P; ++p) step_level(yB[p], tB[p]);
            }
#pragma unroll
            for (int p = 0; p < P; ++p)
                sr[p] = fmaf(hat_of(yB[p]), __ldg(A.alpha + rb[p] + (1u << b) - 1u + tB[p]), sr[p]);
        }
#pragma unroll
        for (int p = 0; p < P; ++p) s[p] = fmaf(D >= 2 ? hat_of(yA[p]) : 1.0f, sr[p], s[p]);
        aoff += (1u << a) * plen;
    }
}

/* Depth-first walk over the prefix dims 0..D-3; at depth D-2 one block. */
template <int D, int K, int P>
struct Walk {
    static __device__ __forceinline__ void run(const EvalArgs &A, int budget, int &pc, const float (&x)[P][D],
                                               const Inner<P> &in, const float (&pin)[P],
                                               const uint32_t (&iin)[P], float (&sum)[P], float (&comp)[P])
    {
        if constexpr (K >= D - 2) {
            const int R = budget;
            const uint32_t bb = __ldg(A.prefix_base + pc);
            ++pc;
            const uint32_t blk = A.blk[R];
            uint32_t base[P];
            float s[P];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                base[p] = bb + iin[p] * blk;
                s[p] = 0.0f;
            }
            bool done = false;
            if (D >= 2 && A.regular2) done = block_dispatch<0, P>(R, A.alpha, base, in, s);
            if (!done) block_generic<D, P>(A, R, x, base, s);
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
                        step_level(y[p], t[p]);
                        J[p] <<= 1;
                    }
                }
                float pn[P];
                uint32_t ix[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    pn[p] = pin[p] * hat_of(y[p]);
                    ix[p] = J[p] + t[p];
                }
                Walk<D, K + 1, P>::run(A, budget - l, pc, x, in, pn, ix, sum, comp);
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

    Inner<P> in;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float y = x[p][D - 1];
        uint32_t t = 0;
#pragma unroll
        for (int j = 0; j < kNB; ++j) {
            if (j) step_level(y, t);
            in.hB[p][j] = hat_of(y);
            in.cB[p][j] = ((1u << j) - 1u) + t;
        }
        const float xa = D >= 2 ? x[p][D >= 2 ? D - 2 : 0] : 0.0f;
        in.TA[p] = (uint32_t)(xa * (float)(1u << kTB));
        y = xa;
#pragma unroll
        for (int j = 0; j < kNB; ++j) {
            if (j) y = (y + y >= 1.0f) ? y + y - 1.0f : y + y;
            in.hA[p][j] = hat_of(y);
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
    int pc = 0;
    Walk<D, 0, P>::run(A, A.nm1, pc, x, in, pin, iin, sum, comp);

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

/* compact (group-aligned) layout -> block layout, one CTA per subspace */
__global__ void k_repack(const float *__restrict__ src, float *__restrict__ dst,
                         const sg_repack *__restrict__ rp, int64_t nsub)
{
    for (int64_t q = blockIdx.x; q < nsub; q += gridDim.x) {
        const sg_repack r = rp[q];
        const int n = 1 << r.s;
        const int ab = r.a + r.b;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const uint32_t I = (uint32_t)e >> ab;
            const uint32_t ta = ((uint32_t)e >> r.b) & ((1u << r.a) - 1u);
            const uint32_t tb = (uint32_t)e & ((1u << r.b) - 1u);
            dst[r.dst + I * r.blk + ta * r.plen + tb] = src[r.src + e];
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
    A.prefix_base = p->prefix_base;
    A.coords = coords;
    A.perm = perm;
    A.out = out;
    A.num_evals = num_evals;
    A.nm1 = p->n - 1;
    for (int k = 0; k < SG_MAX_DIMS; ++k) A.lim[k] = k < p->d ? p->lim[k] : 0;
    for (int r = 0; r < SG_MAX_LEVELS; ++r) A.blk[r] = p->blk[r];
    A.regular2 = p->d >= 2 && p->lim[p->d - 2] >= p->n - 1 && p->lim[p->d - 1] >= p->n - 1;
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

int sgk_repack(const float *src, float *dst, const sg_repack *rp, int64_t nsub, void *stream)
{
    if (nsub <= 0) return cudaSuccess;
    int64_t g = nsub < 148 * 64 ? nsub : 148 * 64;
    k_repack<<<(unsigned)g, 128, 0, (cudaStream_t)stream>>>(src, dst, rp, nsub);
    return cudaGetLastError();
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
