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
constexpr long long kWaitCycles = 4000000000LL; /* ~2 s at 1.9 GHz */

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

/* Bounded wait: gives up after kWaitCycles and reports false. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kWaitCycles) return false;
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

template <typename T>
__global__ void __launch_bounds__(kThreads) k_sweep_chains(T *__restrict__ a,
                                                          const sg_chain *__restrict__ chains,
                                                          const uint32_t *__restrict__ seg,
                                                          int nch, int cap, int *__restrict__ err)
{
    constexpr int A = 16 / sizeof(T); /* elements per 16 bytes */
    using V = typename Vec<T>::type;
    constexpr int W = Vec<T>::W;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar[2];
    __shared__ int s_abort;
    T *stage[2] = {reinterpret_cast<T *>(smem_raw), reinterpret_cast<T *>(smem_raw) + cap};
    const int G = gridDim.x;
    const int tid = threadIdx.x;

    auto issue = [&](int c, int b) {
        const sg_chain ch = chains[c];
        uint32_t bytes = 0;
        for (int j = 0; j <= ch.lmax; ++j) {
            const uint32_t sz = (uint32_t)sizeof(T) << (ch.sigma + j);
            if (sz >= 16) bytes += sz;
        }
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[b], bytes);
        for (int j = 0; j <= ch.lmax; ++j) {
            const uint32_t sz = (uint32_t)sizeof(T) << (ch.sigma + j);
            if (sz >= 16)
                bulk_load(stage[b] + seg_soff<A>(ch.sigma, j), a + seg[ch.seg + j], sz, &bar[b]);
        }
    };

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_abort = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        if (blockIdx.x < nch) issue(blockIdx.x, 0);
        if (blockIdx.x + G < nch) issue(blockIdx.x + G, 1);
    }

    int it = 0, abort_it = -1;
    for (int c = blockIdx.x; c < nch; c += G, ++it) {
        const int b = it & 1;
        const uint32_t parity = (it >> 1) & 1;
        const sg_chain ch = chains[c];
        const int sigma = ch.sigma, lo = ch.lo, lmax = ch.lmax;
        T *buf = stage[b];
        if (!mbar_wait(&bar[b], parity)) {
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
            for (int v = tid; v < U / W; v += kThreads) {
                const int q = v * W;
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                T r[W];
#pragma unroll
                for (int e = 0; e < W; ++e) r[e] = chain_point<T, A>(buf, sigma, lo, j, p + e);
                V out;
                if constexpr (W == 4) {
                    out = make_float4(r[0], r[1], r[2], r[3]);
                } else {
                    out = make_double2(r[0], r[1]);
                }
                *reinterpret_cast<V *>(a + seg[ch.seg + j] + p) = out;
            }
        } else {
            for (int q = tid; q < U; q += kThreads) {
                const int j = 31 - __clz((q >> sigma) + 2);
                const int p = q - (((1 << j) - 2) << sigma);
                a[seg[ch.seg + j] + p] = chain_point<T, A>(buf, sigma, lo, j, p);
            }
        }
        __syncthreads(); /* every read of stage b is done */
        if (tid == 0 && c + 2 * G < nch) issue(c + 2 * G, b);
    }
    if (abort_it >= 0 && tid == 0) {
        /* let the copies still in flight land before the CTA exits: the stage
         * that timed out and, if it was issued, the next one (bounded) */
        (void)mbar_wait(&bar[abort_it & 1], (abort_it >> 1) & 1);
        if (blockIdx.x + (abort_it + 1) * G < nch)
            (void)mbar_wait(&bar[(abort_it + 1) & 1], ((abort_it + 1) >> 1) & 1);
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

int g_num_sms = 0;
long long g_launches = 0;

template <typename T>
int launch_chains(T *a, const sg_sweep_tables *t, int *err, void *stream)
{
    if (t->nchains == 0) return cudaSuccess;
    const int64_t cap = sizeof(T) == 4 ? t->cap32 : t->cap64;
    const int64_t smem = sgk_chain_smem_bytes(cap, (int)sizeof(T));
    if (smem < 0) return cudaErrorInvalidValue;
    const int capi = (int)((smem / 2) / (int64_t)sizeof(T));
    cudaError_t e = cudaFuncSetAttribute(k_sweep_chains<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chains<T>, kThreads,
                                                      (size_t)smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)sgk_num_sms() * per_sm;
    if (grid > t->nchains) grid = t->nchains;
    k_sweep_chains<T><<<(unsigned)grid, kThreads, (size_t)smem, (cudaStream_t)stream>>>(
        a, t->chains, t->seg, (int)t->nchains, capi, err);
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
