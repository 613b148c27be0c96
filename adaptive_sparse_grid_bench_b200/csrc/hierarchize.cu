/*
 * Hierarchization kernels for sm_100a.
 *
 * Reference algorithm: hierarchize0 in adaptive_sparse_grid_bench.c:557-571
 * (definition) and its loop-interchanged form hierarchize7 (c:1009-1090):
 * d sweeps, dim 0 first; in sweep k every point (l, i) with l_k >= 1 becomes
 *     a[l,i] - (a[left parent] + a[right parent]) * 0.5f
 * where the parents are its 1-D hierarchical ancestors in dim k (c:828-854)
 * and a missing parent (domain boundary) counts as 0.  All parents of a sweep
 * are read before they are updated, so one sweep is a pure gather from the
 * pre-sweep values; doing exactly the same three FP32 operations per point
 * makes the result bit-identical to hierarchize0 in any execution order.
 *
 * B200 design: the unit of work is a chain (all subspaces that differ only in
 * l_k, i.e. 2^sigma complete 1-D poles).  Each segment of a chain is a whole
 * subspace, contiguous in the group-aligned layout, so a CTA moves a chain
 * into shared memory with one bulk copy (cp.async.bulk, the TMA engine's 1-D
 * form) per segment, completes the 1-D updates from shared memory and writes
 * the changed segments back with 16-byte stores: 2 x 4 bytes of HBM traffic
 * per updated point per sweep.  Subspaces with l_k = 0 are read (they are
 * parents) but never written.  CTAs are persistent and double-buffered: the
 * next chain's copies are in flight while the current one is computed.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxStages = 2;
constexpr long long kWaitCycles = 4000000000LL; /* ~2 s at 1.9 GHz: the default wait limit */

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

/* Bounded wait: gives up after `limit` clock cycles and reports false. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/* The reference expression a - (L + R) * 0.5 with every rounding explicit, so
 * the compiler can neither contract nor reorder it. */
__device__ __forceinline__ float upd(float a, float l, float r)
{
    return __fsub_rn(a, __fmul_rn(__fadd_rn(l, r), 0.5f));
}
__device__ __forceinline__ double upd(double a, double l, double r)
{
    return __dsub_rn(a, __dmul_rn(__dadd_rn(l, r), 0.5));
}

/* Shared-memory start (elements) of segment j: segments are packed in level
 * order, each rounded up to 16 bytes (A elements, a power of two). */
template <int A>
__device__ __forceinline__ int seg_soff(int sigma, int j)
{
    if ((1 << sigma) >= A) return ((1 << j) - 1) << sigma;
    int o = 0;
    for (int q = 0; q < j; ++q) o += max(1 << (sigma + q), A);
    return o;
}

template <typename T>
struct Vec;
template <>
struct Vec<float> {
    using type = float4;
    static constexpr int W = 4;
};
template <>
struct Vec<double> {
    using type = double2;
    static constexpr int W = 2;
};

/* Value of one updated point: local index p of segment j in a chain whose
 * segments sit in `buf`.  i_k is bits [lo, lo+j) of p. */
template <typename T, int A>
__device__ __forceinline__ T chain_point(const T *buf, int sigma, int lo, int j, int p)
{
    const int ik = (p >> lo) & ((1 << j) - 1);
    const int hi = p >> (lo + j);
    const int lw = p & ((1 << lo) - 1);
    T lft = T(0), rgt = T(0);
    if (ik != 0) {
        const int tz = __ffs(ik) - 1;
        const int pl = j - 1 - tz;
        const int pi = ik >> (tz + 1);
        lft = buf[seg_soff<A>(sigma, pl) + ((((hi << pl) | pi) << lo) | lw)];
    }
    const int ik1 = ik + 1;
    if (ik1 != (1 << j)) {
        const int tz = __ffs(ik1) - 1;
        const int pl = j - 1 - tz;
        const int pi = ik1 >> (tz + 1);
        rgt = buf[seg_soff<A>(sigma, pl) + ((((hi << pl) | pi) << lo) | lw)];
    }
    return upd(buf[seg_soff<A>(sigma, j) + p], lft, rgt);
}

/* Shared-memory index of the 1-D node at position m / 2^j of pole (hi, lw):
 * m odd-multiple of 2^tz is the point of level j-1-tz, index m >> (tz+1).
 * Valid for 0 < m < 2^j (the ends of the pole are the domain boundary). */
__device__ __forceinline__ int node_index(int sigma, int lo, int j, int hi, int lw, int m)
{
    const int tz = __ffs(m) - 1;
    const int pl = j - 1 - tz;
    return seg_soff<4>(sigma, pl) + ((((hi << pl) | (m >> (tz + 1))) << lo) | lw);
}

__device__ __forceinline__ float node_value(const float *buf, int sigma, int lo, int j, int hi, int lw, int m)
{
    return (m == 0 || m == (1 << j)) ? 0.0f : buf[node_index(sigma, lo, j, hi, lw, m)];
}

/* Four consecutive updated points p..p+3 of segment j (FP32, sigma >= 2, so
 * p is a multiple of 4 and the group lies in one segment).  Each output is
 * upd(self, V(i_k), V(i_k + 1)) with V the pre-sweep value at the point's
 * left/right 1-D neighbour, exactly as chain_point computes it; the groups
 * only share the loads:
 *   lo >= 2: the 4 points differ in the low dims only -> 4-wide loads;
 *   lo == 1: two i_k values x two low cells -> 2-wide loads;
 *   lo == 0: four consecutive i_k of one pole (j >= 2) -> 5 neighbours. */
__device__ __forceinline__ float4 chain_group4(const float *buf, int sigma, int lo, int j, int p)
{
    const float4 self = *reinterpret_cast<const float4 *>(buf + seg_soff<4>(sigma, j) + p);
    float4 o;
    if (lo >= 2) {
        const int ik = (p >> lo) & ((1 << j) - 1);
        const int hi = p >> (lo + j);
        const int lw = p & ((1 << lo) - 1);
        float4 L = make_float4(0.f, 0.f, 0.f, 0.f), R = L;
        if (ik != 0) L = *reinterpret_cast<const float4 *>(buf + node_index(sigma, lo, j, hi, lw, ik));
        if (ik + 1 != (1 << j)) R = *reinterpret_cast<const float4 *>(buf + node_index(sigma, lo, j, hi, lw, ik + 1));
        o.x = upd(self.x, L.x, R.x);
        o.y = upd(self.y, L.y, R.y);
        o.z = upd(self.z, L.z, R.z);
        o.w = upd(self.w, L.w, R.w);
    } else if (lo == 1) {
        const int ik = (p >> 1) & ((1 << j) - 1); /* even */
        const int hi = p >> (1 + j);
        float2 v0 = make_float2(0.f, 0.f), v2 = v0;
        if (ik != 0) v0 = *reinterpret_cast<const float2 *>(buf + node_index(sigma, 1, j, hi, 0, ik));
        const float2 v1 = *reinterpret_cast<const float2 *>(buf + node_index(sigma, 1, j, hi, 0, ik + 1));
        if (ik + 2 != (1 << j)) v2 = *reinterpret_cast<const float2 *>(buf + node_index(sigma, 1, j, hi, 0, ik + 2));
        o.x = upd(self.x, v0.x, v1.x);
        o.y = upd(self.y, v0.y, v1.y);
        o.z = upd(self.z, v1.x, v2.x);
        o.w = upd(self.w, v1.y, v2.y);
    } else if (j >= 2) {
        const int ik = p & ((1 << j) - 1); /* multiple of 4 */
        const int hi = p >> j;
        const float2 odd = *reinterpret_cast<const float2 *>(buf + seg_soff<4>(sigma, j - 1) + (hi << (j - 1)) + (ik >> 1));
        const float mid = buf[seg_soff<4>(sigma, j - 2) + (hi << (j - 2)) + (ik >> 2)];
        const float v0 = node_value(buf, sigma, 0, j, hi, 0, ik);
        const float v4 = node_value(buf, sigma, 0, j, hi, 0, ik + 4);
        o.x = upd(self.x, v0, odd.x);
        o.y = upd(self.y, odd.x, mid);
        o.z = upd(self.z, mid, odd.y);
        o.w = upd(self.w, odd.y, v4);
    } else {
        o.x = chain_point<float, 4>(buf, sigma, lo, j, p);
        o.y = chain_point<float, 4>(buf, sigma, lo, j, p + 1);
        o.z = chain_point<float, 4>(buf, sigma, lo, j, p + 2);
        o.w = chain_point<float, 4>(buf, sigma, lo, j, p + 3);
    }
    return o;
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_sweep_chains(T *__restrict__ a,
                                                          const sg_chain *__restrict__ chains,
                                                          const uint32_t *__restrict__ seg,
                                                          int nch, int cap, int nst, int *__restrict__ err,
                                                          long long wait_limit, int stall)
{
    constexpr int A = 16 / sizeof(T); /* elements per 16 bytes */
    using V = typename Vec<T>::type;
    constexpr int W = Vec<T>::W;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar[kMaxStages];
    __shared__ int s_abort;
    T *const stage0 = reinterpret_cast<T *>(smem_raw);
    const int G = gridDim.x;
    const int tid = threadIdx.x;

    /* chain c goes to stage b; the stage's barrier completes when all its
     * bulk copies have landed.  With `stall` (the wait-timeout test), the
     * first chain of every CTA announces its bytes (at least 16) but issues
     * no copy, so its wait can only run out: no copy is ever in flight
     * towards that stage. */
    auto issue = [&](int c, int b) {
        const sg_chain ch = chains[c];
        T *dst = stage0 + (size_t)b * cap;
        uint32_t bytes = 0;
        for (int j = 0; j <= ch.lmax; ++j) {
            const uint32_t sz = (uint32_t)sizeof(T) << (ch.sigma + j);
            if (sz >= 16) bytes += sz;
        }
        fence_proxy_async();
        if (stall && c == (int)blockIdx.x) {
            mbar_arrive_expect_tx(&bar[b], bytes < 16 ? 16u : bytes);
            return;
        }
        mbar_arrive_expect_tx(&bar[b], bytes);
        for (int j = 0; j <= ch.lmax; ++j) {
            const uint32_t sz = (uint32_t)sizeof(T) << (ch.sigma + j);
            if (sz >= 16) bulk_load(dst + seg_soff<A>(ch.sigma, j), a + seg[ch.seg + j], sz, &bar[b]);
        }
    };

    if (tid == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        s_abort = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int b = 0; b < nst; ++b)
            if (blockIdx.x + b * G < nch) issue(blockIdx.x + b * G, b);

    int it = 0, abort_it = -1;
    for (int c = blockIdx.x; c < nch; c += G, ++it) {
        const int b = it % nst;
        const uint32_t parity = (it / nst) & 1;
        const sg_chain ch = chains[c];
        const int sigma = ch.sigma, lo = ch.lo, lmax = ch.lmax;
        T *buf = stage0 + (size_t)b * cap;
        if (!mbar_wait(&bar[b], parity, wait_limit)) {
            atomicExch(err, 1);
            s_abort = 1;
        }
        /* segments under 16 bytes cannot be bulk-copied */
        for (int j = 0; j <= lmax; ++j) {
            const int n = 1 << (sigma + j);
            if (n * (int)sizeof(T) < 16 && tid < n)
                buf[seg_soff<A>(sigma, j) + tid] = a[seg[ch.seg + j] + tid];
        }
        __syncthreads();
        if (s_abort) {
            abort_it = it;
            break;
        }

        /* updated points: segments 1..lmax, flattened; segment j starts at
         * q = 2^sigma (2^j - 2) */
        const int U = (((2 << lmax) - 2) << sigma);
        if ((1 << sigma) >= W) {
            for (int v = tid; v < U / W; v += NT) {
                const int q = v * W;
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                V out;
                if constexpr (W == 4) {
                    out = chain_group4(buf, sigma, lo, j, p);
                } else {
                    out = make_double2(chain_point<T, A>(buf, sigma, lo, j, p),
                                       chain_point<T, A>(buf, sigma, lo, j, p + 1));
                }
                *reinterpret_cast<V *>(a + seg[ch.seg + j] + p) = out;
            }
        } else {
            for (int q = tid; q < U; q += NT) {
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                a[seg[ch.seg + j] + p] = chain_point<T, A>(buf, sigma, lo, j, p);
            }
        }
        __syncthreads(); /* every read of stage b is done */
        if (tid == 0 && c + nst * G < nch) issue(c + nst * G, b);
    }
    if (abort_it >= 0 && tid == 0) {
        /* let the copies still in flight land before the CTA exits: every
         * stage issued for iterations abort_it .. abort_it+nst-1 (bounded) */
        for (int q = abort_it; q < abort_it + nst; ++q)
            if (blockIdx.x + q * G < nch) (void)mbar_wait(&bar[q % nst], (q / nst) & 1, wait_limit);
    }
}

/* Fallback for chains larger than shared memory: level j of every chain,
 * parents read from global memory.  Launched for j = lmax_max .. 1 so that
 * the parents (levels < j) still hold pre-sweep values. */
template <typename T>
__global__ void __launch_bounds__(kThreads) k_sweep_gather(T *__restrict__ a,
                                                          const sg_chain *__restrict__ chains,
                                                          const uint32_t *__restrict__ seg,
                                                          int nch, int j)
{
    for (int c = blockIdx.x; c < nch; c += gridDim.x) {
        const sg_chain ch = chains[c];
        if (ch.lmax < j) continue;
        const int sigma = ch.sigma, lo = ch.lo;
        const int n = 1 << (sigma + j);
        T *dst = a + seg[ch.seg + j];
        for (int p = threadIdx.x; p < n; p += blockDim.x) {
            const int ik = (p >> lo) & ((1 << j) - 1);
            const int hi = p >> (lo + j);
            const int lw = p & ((1 << lo) - 1);
            T lft = T(0), rgt = T(0);
            if (ik != 0) {
                const int tz = __ffs(ik) - 1, pl = j - 1 - tz, pi = ik >> (tz + 1);
                lft = a[seg[ch.seg + pl] + ((((hi << pl) | pi) << lo) | lw)];
            }
            const int ik1 = ik + 1;
            if (ik1 != (1 << j)) {
                const int tz = __ffs(ik1) - 1, pl = j - 1 - tz, pi = ik1 >> (tz + 1);
                rgt = a[seg[ch.seg + pl] + ((((hi << pl) | pi) << lo) | lw)];
            }
            dst[p] = upd(dst[p], lft, rgt);
        }
    }
}

__global__ void k_widen(const float *__restrict__ s, double *__restrict__ d, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}

__global__ void k_narrow(const double *__restrict__ s, float *__restrict__ d, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = __double2float_rn(s[i]);
}

/* dst[seg.dst + i] = src[seg.src + i] for i < seg.count, one segment per
 * CTA iteration (moves values between the caller's compact concatenation
 * and a batch's group-aligned layout in one launch). */
__global__ void k_copy_segments(const float *__restrict__ src, float *__restrict__ dst,
                                const sg_copy_seg *__restrict__ segs, int64_t nseg, int to_compact)
{
    for (int64_t q = blockIdx.x; q < nseg; q += gridDim.x) {
        const sg_copy_seg sgm = segs[q];
        const int64_t from = to_compact ? sgm.dev : sgm.compact;
        const int64_t to = to_compact ? sgm.compact : sgm.dev;
        for (int64_t i = threadIdx.x; i < sgm.count; i += blockDim.x) dst[to + i] = src[from + i];
    }
}

int g_num_sms = 0;
long long g_launches = 0;

template <typename T, int NT>
int launch_chains_nt(T *a, const sg_sweep_tables *t, int64_t cap, int *err, long long wait_limit, int stall,
                     void *stream)
{
    const int64_t stage_bytes = (cap * (int64_t)sizeof(T) + 127) / 128 * 128;
    /* as many stages (2..kMaxStages) as fit in 96 KB */
    int nst = (int)((96 * 1024) / stage_bytes);
    nst = nst < 2 ? 2 : (nst > kMaxStages ? kMaxStages : nst);
    const int64_t smem = nst * stage_bytes;
    const int capi = (int)(stage_bytes / (int64_t)sizeof(T));
    cudaError_t e = cudaFuncSetAttribute(k_sweep_chains<T, NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chains<T, NT>, NT, (size_t)smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)sgk_num_sms() * per_sm;
    if (grid > t->nchains) grid = t->nchains;
    k_sweep_chains<T, NT><<<(unsigned)grid, NT, (size_t)smem, (cudaStream_t)stream>>>(
        a, t->chains, t->seg, (int)t->nchains, capi, nst, err, wait_limit, stall);
    sgk_count(1);
    return cudaGetLastError();
}

/* CTA size follows the chain size: up to 12 elements (three 16-byte groups)
 * per thread, between 128 and 512 threads. */
template <typename T>
int launch_chains(T *a, const sg_sweep_tables *t, int *err, void *stream, long long wait_limit = kWaitCycles,
                  int stall = 0)
{
    if (t->nchains == 0) return cudaSuccess;
    const int64_t cap = sizeof(T) == 4 ? t->cap32 : t->cap64;
    if (sgk_chain_smem_bytes(cap, (int)sizeof(T)) < 0) return cudaErrorInvalidValue;
    if (cap <= 128 * 12) return launch_chains_nt<T, 128>(a, t, cap, err, wait_limit, stall, stream);
    if (cap <= 256 * 12) return launch_chains_nt<T, 256>(a, t, cap, err, wait_limit, stall, stream);
    return launch_chains_nt<T, 512>(a, t, cap, err, wait_limit, stall, stream);
}

/* Small chains (the many short chains of batched grids): one warp per
 * chain.  The warp loads the chain's segments into its own shared-memory
 * buffer with coalesced 16-byte loads (no bulk copies, barriers or CTA-wide
 * synchronisation, whose fixed cost dominates a chain of a few hundred
 * values), then writes the updated points straight to global memory, four
 * FP32 values (two FP64) per lane and 16-byte store wherever 2^sigma holds
 * a whole group: the updates read only the pre-sweep values in the buffer,
 * with the same arithmetic as k_sweep_chains, so results are bit-identical.
 * The one-value-per-lane form spent most of its time issuing index
 * arithmetic (issue-bound at a fifth of the DRAM bandwidth). */
template <typename T>
__global__ void __launch_bounds__(256) k_sweep_small(T *__restrict__ a, const sg_chain *__restrict__ chains,
                                                     const uint32_t *__restrict__ seg, int nch, int cap)
{
    constexpr int A = 16 / sizeof(T);
    using V = typename Vec<T>::type;
    constexpr int W = Vec<T>::W;
    extern __shared__ __align__(16) unsigned char smem_small[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T *buf = reinterpret_cast<T *>(smem_small) + (size_t)w * cap;
    const int nw = gridDim.x * (blockDim.x >> 5);
    /* the chain index is the same for all lanes: every loop below is
     * warp-uniform */
    for (int c = blockIdx.x * (blockDim.x >> 5) + w; c < nch; c += nw) {
        const sg_chain ch = chains[c];
        const int sigma = ch.sigma, lo = ch.lo, lmax = ch.lmax;
        /* a subspace of 2^s values starts on a multiple of 2^s in the
         * group-aligned layout, so every segment of at least 16 bytes moves
         * with 16-byte loads; its shared-memory slot is 16-byte aligned too
         * (cap and the segment starts are multiples of A) */
        for (int j = 0; j <= lmax; ++j) {
            const int n = 1 << (sigma + j);
            const T *src = a + seg[ch.seg + j];
            T *dst = buf + seg_soff<A>(sigma, j);
            if (n >= W) {
                for (int v = lane; v < n / W; v += 32)
                    reinterpret_cast<V *>(dst)[v] = reinterpret_cast<const V *>(src)[v];
            } else if (lane < n) {
                dst[lane] = src[lane];
            }
        }
        __syncwarp();
        /* updated points: segments 1..lmax flattened, segment j starting at
         * q = 2^sigma (2^j - 2); W at a time when a pole group holds W
         * consecutive values, with the arithmetic of k_sweep_chains */
        const int U = (((2 << lmax) - 2) << sigma);
        if ((1 << sigma) >= W) {
            for (int v = lane; v < U / W; v += 32) {
                const int q = v * W;
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                V o;
                if constexpr (W == 4) {
                    o = chain_group4(buf, sigma, lo, j, p);
                } else {
                    o = make_double2(chain_point<T, A>(buf, sigma, lo, j, p),
                                     chain_point<T, A>(buf, sigma, lo, j, p + 1));
                }
                *reinterpret_cast<V *>(a + seg[ch.seg + j] + p) = o;
            }
        } else {
            for (int q = lane; q < U; q += 32) {
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                a[seg[ch.seg + j] + p] = chain_point<T, A>(buf, sigma, lo, j, p);
            }
        }
        __syncwarp();
    }
}

template <typename T>
int launch_small(T *a, const sg_sweep_tables *t, void *stream)
{
    if (t->nchains == 0) return cudaSuccess;
    const int64_t cap = sizeof(T) == 4 ? t->cap32 : t->cap64;
    const int64_t smem = 8 * cap * (int64_t)sizeof(T); /* 8 warps per CTA */
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_sweep_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_small<T>, 256, (size_t)smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (t->nchains + 7) / 8;
    if (grid > (int64_t)sgk_num_sms() * per_sm) grid = (int64_t)sgk_num_sms() * per_sm;
    k_sweep_small<T><<<(unsigned)grid, 256, (size_t)smem, (cudaStream_t)stream>>>(a, t->chains, t->seg,
                                                                                (int)t->nchains, (int)cap);
    sgk_count(1);
    return cudaGetLastError();
}

template <typename T>
int launch_gather(T *a, const sg_sweep_tables *t, void *stream)
{
    if (t->nchains == 0) return cudaSuccess;
    int64_t grid = (int64_t)sgk_num_sms() * 8;
    if (grid > t->nchains) grid = t->nchains;
    for (int j = t->lmax_max; j >= 1; --j) {
        k_sweep_gather<T><<<(unsigned)grid, kThreads, 0, (cudaStream_t)stream>>>(
            a, t->chains, t->seg, (int)t->nchains, j);
        sgk_count(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

} // namespace

extern "C" {

void sgk_count(int launches) { __atomic_fetch_add(&g_launches, (long long)launches, __ATOMIC_RELAXED); }
int64_t sgk_launches(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int sgk_num_sms(void)
{
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

int64_t sgk_chain_smem_bytes(int64_t cap_elems, int elem_bytes)
{
    const int64_t stage = (cap_elems * elem_bytes + 127) / 128 * 128;
    const int64_t total = 2 * stage;
    return total <= 200 * 1024 ? total : -1;
}

int sgk_sweep_chains_f32(float *a, const sg_sweep_tables *t, int *err, void *stream)
{
    return launch_chains<float>(a, t, err, stream);
}
int sgk_sweep_chains_f64(double *a, const sg_sweep_tables *t, int *err, void *stream)
{
    return launch_chains<double>(a, t, err, stream);
}
int sgk_sweep_chains_stall_f32(float *a, const sg_sweep_tables *t, int *err, long long wait_limit, void *stream)
{
    if (wait_limit < 1 || wait_limit > kWaitCycles) return cudaErrorInvalidValue;
    return launch_chains<float>(a, t, err, stream, wait_limit, 1);
}
int sgk_sweep_small_f32(float *a, const sg_sweep_tables *t, void *stream)
{
    return launch_small<float>(a, t, stream);
}
int sgk_sweep_small_f64(double *a, const sg_sweep_tables *t, void *stream)
{
    return launch_small<double>(a, t, stream);
}
int64_t sgk_small_smem_bytes(int64_t cap_elems, int elem_bytes)
{
    const int64_t b = 8 * cap_elems * elem_bytes;
    return b <= 200 * 1024 ? b : -1;
}
int sgk_sweep_gather_f32(float *a, const sg_sweep_tables *t, void *stream)
{
    return launch_gather<float>(a, t, stream);
}
int sgk_sweep_gather_f64(double *a, const sg_sweep_tables *t, void *stream)
{
    return launch_gather<double>(a, t, stream);
}

int sgk_widen(const float *src, double *dst, int64_t n, void *stream)
{
    if (n <= 0) return cudaSuccess;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    k_widen<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(src, dst, n);
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_copy_segments(const float *src, float *dst, const sg_copy_seg *segs, int64_t nseg, int to_compact,
                      void *stream)
{
    if (nseg <= 0) return cudaSuccess;
    int64_t g = nseg < 148 * 32 ? nseg : 148 * 32;
    k_copy_segments<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(src, dst, segs, nseg, to_compact);
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_narrow(const double *src, float *dst, int64_t n, void *stream)
{
    if (n <= 0) return cudaSuccess;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    k_narrow<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(src, dst, n);
    sgk_count(1);
    return cudaGetLastError();
}

} // extern "C"
