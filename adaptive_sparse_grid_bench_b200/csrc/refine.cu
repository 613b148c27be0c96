// Per-subspace maximum |surplus| on the device: the statistic the
// limits-adaptive refinement driver (sgrid_refine.c) decides on.
//
// In the group-aligned compact layout every subspace of level group s holds
// 2^s consecutive values, and each group starts on a 32-element boundary, so
// a 32-element warp chunk lies inside one group and a subspace of s < 5 lies
// inside one warp.  One pass over the values, HBM-bound: 4 bytes read per
// value, 4 bytes written per subspace.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

struct MaxAbsTables {
    int n;
    int64_t plidx[SG_MAX_LEVELS + 1]; // device offset of group s
    int64_t len[SG_MAX_LEVELS];       // values in group s (multiple of 2^s)
    int64_t sbase[SG_MAX_LEVELS];     // subspaces before group s
};

__global__ void __launch_bounds__(256) k_subspace_maxabs(MaxAbsTables T, const float *__restrict__ a, int64_t npad,
                                                         unsigned *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // e0 is the warp's first element: the loop trip count is warp-uniform
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); e0 < npad; e0 += stride) {
        int s = 0;
        while (s + 1 < T.n && T.plidx[s + 1] <= e0) ++s;
        const int64_t rel = e0 + lane - T.plidx[s];
        const bool valid = rel < T.len[s];
        float v = valid ? fabsf(__ldg(a + e0 + lane)) : 0.f;
        if (s < 5) {
            // subspaces of 2^s lanes: reduce inside each aligned lane group
            for (int off = 1; off < (1 << s); off <<= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
            if (valid && (lane & ((1 << s) - 1)) == 0) out[T.sbase[s] + (rel >> s)] = __float_as_uint(v);
        } else {
            for (int off = 16; off; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
            // non-negative floats order like their bit patterns
            if (valid && lane == 0) atomicMax(out + T.sbase[s] + (rel >> s), __float_as_uint(v));
        }
    }
}

} // namespace

extern "C" int sgk_subspace_maxabs(const sg_layout *L, const float *alpha, unsigned *out, void *stream)
{
    MaxAbsTables T;
    int64_t sb = 0;
    cudaError_t e;
    T.n = L->n;
    for (int s = 0; s <= SG_MAX_LEVELS; ++s) T.plidx[s] = s <= L->n ? L->plidx[s] : L->Npad;
    for (int s = 0; s < SG_MAX_LEVELS; ++s) {
        T.len[s] = s < L->n ? L->lidx[s + 1] - L->lidx[s] : 0;
        T.sbase[s] = sb;
        sb += T.len[s] >> s;
    }
    if (L->S <= 0 || L->Npad <= 0) return cudaSuccess;
    e = cudaMemsetAsync(out, 0, (size_t)L->S * sizeof(unsigned), (cudaStream_t)stream);
    if (e != cudaSuccess) return e;
    int64_t g = (L->Npad + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    k_subspace_maxabs<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(T, alpha, L->Npad, out);
    sgk_count(1);
    return cudaGetLastError();
}
