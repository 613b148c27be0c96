/*
 * Batched index bijection on the device: the reference's idx2gp
 * (adaptive_sparse_grid_bench.c:210-243) and gp2idx (c:187-207), one thread
 * per point, with the index tables passed as kernel parameters (constant
 * bank).  Used to sample functions at grid points without a host round trip.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "sg_kernels.h"

namespace {

struct Tables {
    int d, n;
    int lim[SG_MAX_DIMS];
    int64_t dp[SG_MAX_DIMS][SG_MAX_LEVELS];
    int64_t lidx[SG_MAX_LEVELS + 1];
    int64_t plidx[SG_MAX_LEVELS + 1];
};

__global__ void k_idx2gp(const Tables T, const int64_t *__restrict__ index, int *__restrict__ lv_out,
                         int *__restrict__ ix_out, int64_t count)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count;
         q += (int64_t)gridDim.x * blockDim.x) {
        int64_t idx = index[q];
        int *lv = lv_out + q * T.d, *ix = ix_out + q * T.d;
        if (idx < 0 || idx >= T.lidx[T.n]) {
            for (int k = 0; k < T.d; ++k) lv[k] = ix[k] = -1;
            continue;
        }
        int s = 0;
        while (s < T.n && idx >= T.lidx[s]) ++s;
        --s;
        idx -= T.lidx[s];
        int64_t rest = idx & (((int64_t)1 << s) - 1);
        int64_t pos = idx >> s;
        int lvl[SG_MAX_DIMS];
        int ss = s;
        for (int i = T.d - 1; i >= 1; --i) {
            int level = 0;
            while (pos >= T.dp[i - 1][ss - level]) {
                pos -= T.dp[i - 1][ss - level];
                ++level;
            }
            lvl[i] = level;
            ss -= level;
        }
        lvl[0] = ss;
        for (int i = T.d - 1; i >= 0; --i) {
            lv[i] = lvl[i];
            ix[i] = (int)(rest & (((int64_t)1 << lvl[i]) - 1));
            rest >>= lvl[i];
        }
    }
}

__global__ void k_gp2idx(const Tables T, const int *__restrict__ lv_in, const int *__restrict__ ix_in,
                         int64_t *__restrict__ index, int64_t count)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int *lv = lv_in + q * T.d, *ix = ix_in + q * T.d;
        int s = 0;
        bool ok = true;
        for (int k = 0; k < T.d; ++k) {
            ok &= lv[k] >= 0 && lv[k] <= T.lim[k] && ix[k] >= 0 && ix[k] < (1 << lv[k]);
            s += lv[k];
        }
        if (!ok || s >= T.n) {
            index[q] = -1;
            continue;
        }
        int64_t in_sub = ix[0], pos = 0;
        int sum = lv[0];
        for (int i = 1; i < T.d; ++i) {
            in_sub = (in_sub << lv[i]) + ix[i];
            sum += lv[i];
            for (int j = 0; j < lv[i]; ++j) pos += T.dp[i - 1][sum - j];
        }
        index[q] = T.lidx[s] + (pos << s) + in_sub;
    }
}

struct FnParams {
    int fn, np;
    double p[SG_MAX_FN_PARAMS];
};

/* One thread per device element; padding elements between groups are set
 * to 0.  x_k = (2 i_k + 1) / 2^(l_k+1) is exact in FP32 and FP64. */
__global__ void k_sample(const Tables T, const FnParams F, float *__restrict__ alpha, int64_t npad)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < npad;
         j += (int64_t)gridDim.x * blockDim.x) {
        int s = 0;
        while (s < T.n && j >= T.plidx[s + 1]) ++s;
        if (s >= T.n) {
            alpha[j] = 0.0f;
            continue;
        }
        const int64_t local = j - T.plidx[s];
        const int64_t gsize = (T.lidx[s + 1] - T.lidx[s]);
        if (local >= gsize) {
            alpha[j] = 0.0f;
            continue;
        }
        int64_t pos = local >> s, rest = local & (((int64_t)1 << s) - 1);
        int lvl[SG_MAX_DIMS];
        int ss = s;
        for (int i = T.d - 1; i >= 1; --i) {
            int level = 0;
            while (pos >= T.dp[i - 1][ss - level]) {
                pos -= T.dp[i - 1][ss - level];
                ++level;
            }
            lvl[i] = level;
            ss -= level;
        }
        lvl[0] = ss;
        double acc = (F.fn == SG_FN_PROD4 || F.fn == SG_FN_QUAD) ? 1.0 : 0.0;
        for (int k = T.d - 1; k >= 0; --k) {
            const int64_t ik = rest & (((int64_t)1 << lvl[k]) - 1);
            rest >>= lvl[k];
            const double x = (double)(2 * ik + 1) / (double)((int64_t)2 << lvl[k]);
            switch (F.fn) {
            case SG_FN_REFERENCE: acc += x * x * (1.0 - x) * (1.0 - x); break;
            case SG_FN_PROD4: acc *= 4.0 * x * (1.0 - x); break;
            case SG_FN_GAUSS: acc += x * x; break;
            case SG_FN_BUMP: acc += (x - F.p[0]) * (x - F.p[0]); break;
            case SG_FN_QUAD: acc *= F.p[3 * k] + F.p[3 * k + 1] * x + F.p[3 * k + 2] * x * x; break;
            default: break;
            }
        }
        double v = acc;
        if (F.fn == SG_FN_GAUSS) v = exp(-acc);
        if (F.fn == SG_FN_BUMP) v = exp(-F.p[1] * acc);
        alpha[j] = __double2float_rn(v);
    }
}

Tables make_tables(const sg_layout *L)
{
    Tables T;
    T.d = L->d;
    T.n = L->n;
    for (int i = 0; i < SG_MAX_DIMS; ++i) T.lim[i] = i < L->d ? L->lim[i] : 0;
    for (int i = 0; i < SG_MAX_DIMS; ++i)
        for (int s = 0; s < SG_MAX_LEVELS; ++s) T.dp[i][s] = L->dp[i][s];
    for (int s = 0; s <= SG_MAX_LEVELS; ++s) T.lidx[s] = L->lidx[s];
    for (int s = 0; s <= SG_MAX_LEVELS; ++s) T.plidx[s] = L->plidx[s];
    return T;
}

} // namespace

extern "C" {

int sgk_idx2gp(const sg_layout *L, const int64_t *index, int *levels, int *indices, int64_t count,
               void *stream)
{
    if (count <= 0) return cudaSuccess;
    int64_t g = (count + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_idx2gp<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(make_tables(L), index, levels, indices,
                                                           count);
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_gp2idx(const sg_layout *L, const int *levels, const int *indices, int64_t *index,
               int64_t count, void *stream)
{
    if (count <= 0) return cudaSuccess;
    int64_t g = (count + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_gp2idx<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(make_tables(L), levels, indices, index,
                                                           count);
    sgk_count(1);
    return cudaGetLastError();
}

int sgk_sample(const sg_layout *L, int fn, const double *params, int nparams, float *alpha, void *stream)
{
    FnParams F;
    F.fn = fn;
    F.np = nparams;
    for (int i = 0; i < SG_MAX_FN_PARAMS; ++i) F.p[i] = i < nparams ? params[i] : 0.0;
    if (L->Npad <= 0) return cudaSuccess;
    int64_t g = (L->Npad + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    k_sample<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(make_tables(L), F, alpha, L->Npad);
    sgk_count(1);
    return cudaGetLastError();
}

} // extern "C"
