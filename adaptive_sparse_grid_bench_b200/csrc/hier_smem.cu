/*
 * Whole-grid hierarchization in shared memory, for batches of small grids.
 *
 * Same arithmetic as hierarchize0 (adaptive_sparse_grid_bench.c:557-571):
 * d sweeps, dim 0 first; in sweep k every point with l_k >= 1 becomes
 * a - (a_left + a_right) * 0.5 from pre-sweep values.  A grid that fits in
 * shared memory (<= SG_SMEM_GRID_MAX_BYTES, n <= 9) is loaded once by one
 * CTA, swept d times in place, and stored once: 2 x 4 bytes of HBM traffic
 * per point for the whole hierarchization instead of 8 per point per sweep.
 * Within a sweep each warp owns whole chains (the subspaces that differ only
 * in l_k); a warp computes every updated point of its chain into registers
 * before writing any of them back (__syncwarp between), so every update reads
 * pre-sweep values, and chains are disjoint, so warps never race.
 *
 * FP64 mode keeps the grid in shared memory as doubles (widened once on load,
 * rounded once on store): bit-identical to the FP64 oracle rounded to FP32.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxUpdated = 512; /* updated points per chain for n <= 9: < 2^9 */
constexpr int kPerLane = kMaxUpdated / 32;

__device__ __forceinline__ float upd(float a, float l, float r)
{
    return __fsub_rn(a, __fmul_rn(__fadd_rn(l, r), 0.5f));
}
__device__ __forceinline__ double upd(double a, double l, double r)
{
    return __dsub_rn(a, __dmul_rn(__dadd_rn(l, r), 0.5));
}

/* Updated point p of segment j of a chain whose segment j starts at
 * buf + seg[j] (seg: grid-relative offsets of the chain's subspaces). */
template <typename T>
__device__ __forceinline__ T point_update(const T *buf, const uint32_t *__restrict__ seg, int lo, int j, int p,
                                          int *where)
{
    const int ik = (p >> lo) & ((1 << j) - 1);
    const int hi = p >> (lo + j);
    const int lw = p & ((1 << lo) - 1);
    T lft = T(0), rgt = T(0);
    if (ik != 0) {
        const int tz = __ffs(ik) - 1, pl = j - 1 - tz, pi = ik >> (tz + 1);
        lft = buf[__ldg(seg + pl) + ((((hi << pl) | pi) << lo) | lw)];
    }
    const int ik1 = ik + 1;
    if (ik1 != (1 << j)) {
        const int tz = __ffs(ik1) - 1, pl = j - 1 - tz, pi = ik1 >> (tz + 1);
        rgt = buf[__ldg(seg + pl) + ((((hi << pl) | pi) << lo) | lw)];
    }
    const int w = __ldg(seg + j) + p;
    *where = w;
    return upd(buf[w], lft, rgt);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_hier_smem(float *__restrict__ a, const sg_smem_grid *__restrict__ grids,
                                                       const sg_chain *__restrict__ chains,
                                                       const uint32_t *__restrict__ seg)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *buf = reinterpret_cast<T *>(smem_raw);
    const sg_smem_grid g = grids[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nwarps = kThreads / 32;
    float *src = a + g.base;

    /* load (npad and base are multiples of 32: 16-byte vector loads) */
    for (int i = tid * 4; i < (int)g.npad; i += kThreads * 4) {
        const float4 v = *reinterpret_cast<const float4 *>(src + i);
        buf[i] = (T)v.x;
        buf[i + 1] = (T)v.y;
        buf[i + 2] = (T)v.z;
        buf[i + 3] = (T)v.w;
    }
    __syncthreads();

    for (int k = 0; k < g.d; ++k) {
        for (int c = warp; c < (int)g.nch[k]; c += nwarps) {
            const sg_chain ch = chains[g.chain0[k] + c];
            const int U = (((2 << ch.lmax) - 2) << ch.sigma);
            const uint32_t *cs = seg + ch.seg;
            T r[kPerLane];
            int w[kPerLane];
#pragma unroll
            for (int t = 0; t < kPerLane; ++t) {
                const int q = lane + 32 * t;
                if (q < U) {
                    const int j = 31 - __clz((q >> ch.sigma) + 2);
                    const int p = q - (((1 << j) - 2) << ch.sigma);
                    r[t] = point_update<T>(buf, cs, ch.lo, j, p, &w[t]);
                }
            }
            __syncwarp();
#pragma unroll
            for (int t = 0; t < kPerLane; ++t)
                if (lane + 32 * t < U) buf[w[t]] = r[t];
            __syncwarp();
        }
        __syncthreads();
    }

    for (int i = tid * 4; i < (int)g.npad; i += kThreads * 4) {
        float4 v;
        if constexpr (sizeof(T) == 8) {
            v = make_float4(__double2float_rn(buf[i]), __double2float_rn(buf[i + 1]),
                            __double2float_rn(buf[i + 2]), __double2float_rn(buf[i + 3]));
        } else {
            v = make_float4(buf[i], buf[i + 1], buf[i + 2], buf[i + 3]);
        }
        *reinterpret_cast<float4 *>(src + i) = v;
    }
}

template <typename T>
int launch(float *a, const sg_smem_grid *grids, int ngrids, const sg_chain *chains, const uint32_t *seg,
           int max_npad, void *stream)
{
    if (ngrids <= 0) return cudaSuccess;
    const size_t smem = (size_t)max_npad * sizeof(T);
    if (smem > SG_SMEM_GRID_MAX_BYTES) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_hier_smem<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_hier_smem<T><<<ngrids, kThreads, smem, (cudaStream_t)stream>>>(a, grids, chains, seg);
    sgk_count(1);
    return cudaGetLastError();
}

} // namespace

extern "C" int sgk_hier_smem_grids(float *a, const sg_smem_grid *grids, int ngrids, const sg_chain *chains,
                                   const uint32_t *seg, int max_npad, int fp64, void *stream)
{
    return fp64 ? launch<double>(a, grids, ngrids, chains, seg, max_npad, stream)
                : launch<float>(a, grids, ngrids, chains, seg, max_npad, stream);
}
