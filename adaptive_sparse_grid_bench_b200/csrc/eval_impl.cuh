/*
 * Evaluation kernels for sm_100a (instantiated per dimension in eval_d*.cu).
 *
 * Reference algorithm: evaluate0 in adaptive_sparse_grid_bench.c:1237-1274
 * (definition) and evaluate5 (c:1558-1688): for a query point x,
 *     u(x) = sum over subspaces l of  a[off(l) + idx(x, l)] * prod_k hat_k
 * with t_k = floor(x_k 2^l_k), idx(x, l) = row-major (t_0, ..., t_{d-1}) over
 * the subspace (dim 0 most significant) and hat_k = 1 - |x_k 2^(l_k+1) - (2t_k+1)|.
 *
 * B200 design.  One thread owns P query points; every warp walks the same
 * depth-first tree over the level vectors of the prefix dims 0..d-4 (each
 * dim's level ascending, sum(l) <= n-1, l_k <= limits[k]), so control flow is
 * uniform across the warp and partial products / partial cell indices are
 * shared by all subspaces below a node.  Below a prefix cell the walk reads
 * one block: every subspace of the three innermost dims (C = d-3, A = d-2,
 * B = d-1), stored contiguously in the block layout (sg_layout.h) with dim
 * B's levels as paths: per finest cell t_L of a row, the L+1 surpluses a
 * point in that cell needs, side by side.  The surplus of (c, a, b) sits at
 *     base + coff(c) + t_c sub(R-c) + aoff(a) + t_a plen(a) + t_L (L+1) + b:
 *   - blocks follow each other in walk order, so the block base is a running
 *     counter plus one multiply-add per point (no table);
 *   - a row's L+1 loads share one address (the point's path) and differ by
 *     a constant, so each subspace costs one gather and one FMA, the row one
 *     address; the hats of dim B are precomputed per point in registers,
 *     those of dims A and C in this thread's column of shared memory;
 *   - the two points of a thread are computed with Blackwell's packed FP32x2
 *     instructions (FFMA2, FADD2, FMUL2 through __ffma2_rn, __fadd2_rn,
 *     __fmul2_rn): one instruction does both points' FMA, product or
 *     compensated add, with each point's rounding exactly as in scalar code,
 *     so results are bit-identical to one point per thread;
 *   - blocks of budget R <= kRFof<BL> run fully unrolled; larger blocks
 *     loop over their planes and run each plane's 2-D sub-block fully
 *     unrolled behind a jump table.  A block or sub-block whose budget is within the limits of
 *     its dims has the regular shape whatever the limits, so limit-vector
 *     (adaptive) grids take the unrolled code too; a generic loop covers
 *     budgets above the limits, budgets >= kNB and d = 1;
 *   - most blocks sit under walk nodes of small remaining budget (at d=10,
 *     n=10, 8,008 of 11,440 blocks hold at most 4 subspaces), where loop and
 *     dispatch cost more than the gathers: the last prefix dim with budget
 *     <= kLGof<P, BL> (levels and blocks) and the last two with budget
 *     <= kLG2 run as fully unrolled code with compile-time block sizes, in
 *     walk order, so results are bit-identical to the loop (d <= kMaxUnrollD);
 *   - BL is the subspace blocking preset, a template parameter (wide = 0,
 *     medium = 1; the autotuner picks one per grid or per dimension of a
 *     batch): more unrolled code saves loop and dispatch work but raises
 *     register pressure, and the best trade depends on the grid and on the
 *     kernel (the batched kernel holds more state);
 *   - per prefix dim the walk keeps three values per point: the fractional
 *     part y = frac(x 2^l) (next level: doubling, exact in FP32), the cell
 *     index of the prefix (next level: 2*ix + bit) and the parent's product;
 *   - block sums of one prefix node are accumulated with FMAs and the node's
 *     total enters a Kahan-compensated accumulator.
 * Query points are put in spatial (Morton) order beforehand so the 32 points
 * of a warp share cells of the coarse subspaces and the gathers of a warp
 * touch few sectors; the grid is then served from L1/L2.
 */
#ifndef SG_EVAL_IMPL_CUH
#define SG_EVAL_IMPL_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "eval_args.h"

namespace sgeval {

constexpr int kThreads = 256;
constexpr int kNB = 10; /* 2-D sub-blocks of budget r < kNB run fully unrolled */
constexpr int kRF = SG_EVAL_MAX_RF; /* 3-D blocks of budget R <= kRF can run unrolled */
static_assert(kRF == 6, "block_sum's jump table covers budgets 0..6");
/* largest budget of an unrolled 3-D block under blocking preset BL */
template <int BL>
constexpr int kRFof = BL == 0 ? kRF : 5;
constexpr int kTB = 15; /* T = floor(x 2^15) holds the cells of levels 0..15   */

/* P floats of one thread's points: float2 (packed FP32x2 instructions) for
 * P = 2, a plain float for P = 1. */
template <int P>
struct FV;
template <>
struct FV<1> {
    float v;
    __device__ __forceinline__ float get(int) const { return v; }
    __device__ __forceinline__ void set(int, float x) { v = x; }
    static __device__ __forceinline__ FV all(float x) { return FV{x}; }
};
template <>
struct FV<2> {
    float2 v;
    __device__ __forceinline__ float get(int p) const { return p ? v.y : v.x; }
    __device__ __forceinline__ void set(int p, float x)
    {
        if (p) v.y = x;
        else v.x = x;
    }
    static __device__ __forceinline__ FV all(float x) { return FV{make_float2(x, x)}; }
};
__device__ __forceinline__ FV<1> vfma(FV<1> a, FV<1> b, FV<1> c) { return FV<1>{fmaf(a.v, b.v, c.v)}; }
__device__ __forceinline__ FV<1> vmul(FV<1> a, FV<1> b) { return FV<1>{__fmul_rn(a.v, b.v)}; }
__device__ __forceinline__ FV<1> vadd(FV<1> a, FV<1> b) { return FV<1>{__fadd_rn(a.v, b.v)}; }
__device__ __forceinline__ FV<1> vsub(FV<1> a, FV<1> b) { return FV<1>{__fsub_rn(a.v, b.v)}; }
__device__ __forceinline__ FV<2> vfma(FV<2> a, FV<2> b, FV<2> c) { return FV<2>{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ FV<2> vmul(FV<2> a, FV<2> b) { return FV<2>{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ FV<2> vadd(FV<2> a, FV<2> b) { return FV<2>{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ FV<2> vsub(FV<2> a, FV<2> b)
{
    return FV<2>{__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))};
}

/* compensated (Kahan) s += v, c holding the running rounding error */
template <int P>
__device__ __forceinline__ void kahan_add(FV<P> &s, FV<P> &c, FV<P> v)
{
    const FV<P> y = vsub(v, c);
    const FV<P> t = vadd(s, y);
    c = vsub(vsub(t, s), y);
    s = t;
}

/* cell index at level l (0..15) from T = floor(x 2^15): T >> (15 - l).
 * Level 0 has one cell and T < 2^15 for every x in [0,1) (x 2^15 is exact),
 * so its index is 0; that is written out as a constant because the compiler
 * cannot bound T, which comes from a float conversion, and would otherwise
 * shift and multiply a zero in every row and plane of level 0. */
__device__ __forceinline__ uint32_t cell_at(uint32_t T, int l) { return l == 0 ? 0u : T >> (kTB - l); }

/* hat at the current level from the fractional part y = frac(x 2^l) */
__device__ __forceinline__ float hat_of(float y) { return 1.0f - fabsf(fmaf(2.0f, y, -1.0f)); }

/* next level: y <- frac(2y) (exact), returns floor(2y) */
__device__ __forceinline__ uint32_t step_y(float &y)
{
    const float y2 = y + y;
    const bool b = y2 >= 1.0f;
    y = b ? y2 - 1.0f : y2;
    return (uint32_t)b;
}

template <int P>
__device__ __forceinline__ FV<P> hats(const FV<P> &y)
{
    FV<P> h;
#pragma unroll
    for (int p = 0; p < P; ++p) h.set(p, hat_of(y.get(p)));
    return h;
}

/* Per-point values of the three innermost dims. */
template <int P>
struct Inner {
    FV<P> hB[kNB];        /* hat of dim B at level b                 */
    uint32_t TB[P];       /* floor(x_B 2^15): the path t_L = TB >> (15 - L) */
    const FV<P> *sh;      /* this thread's hats of dims A, C in smem */
    uint32_t TA[P];       /* floor(x_A 2^15): t_a = TA >> (15 - a)   */
    uint32_t TC[P];       /* floor(x_C 2^15)                         */
    __device__ __forceinline__ FV<P> hA(int a) const { return sh[a * kThreads]; }
    __device__ __forceinline__ FV<P> hC(int c) const { return sh[(kNB + c) * kThreads]; }
};
constexpr int kHatSlots = kNB + kRF + 1;

/* Regular shapes: blocks whose budget is within the innermost limits. */
__host__ __device__ constexpr uint32_t plen_reg(int r, int a) { return (1u << (r - a)) * (uint32_t)SG_PATH_WIDTH(r - a + 1); }
__host__ __device__ constexpr uint32_t aoff_reg(int r, int a)
{
    uint32_t o = 0;
    for (int q = 0; q < a; ++q) o += (1u << q) * plen_reg(r, q);
    return o;
}
__host__ __device__ constexpr uint32_t blk2_reg(int r) { return aoff_reg(r, r + 1); }
__host__ __device__ constexpr uint32_t coff_reg(int R, int c)
{
    uint32_t o = 0;
    for (int q = 0; q < c; ++q) o += (1u << q) * blk2_reg(R - q);
    return o;
}

/* 2-D sub-block of budget r: rows a = 0..r, row a holds 2^a poles of r-a+1
 * levels.  Returns sum_a hA[a] sum_b hB[b] alpha[...]. */
template <int r, int P>
__device__ __forceinline__ void block2_fixed(const float *__restrict__ alpha, const uint32_t (&base)[P],
                                             const Inner<P> &in, FV<P> &s)
{
#pragma unroll
    for (int a = 0; a <= r; ++a) {
        const int L = r - a; /* compile-time after unrolling */
        const float *path[P]; /* the point's path: its L+1 surpluses of this row */
#pragma unroll
        for (int p = 0; p < P; ++p)
            path[p] = alpha + (base[p] + aoff_reg(r, a) + cell_at(in.TA[p], a) * plen_reg(r, a) +
                               cell_at(in.TB[p], L) * (uint32_t)SG_PATH_WIDTH(L + 1));
        FV<P> sr = FV<P>::all(0.0f);
        /* slots 2j, 2j+1 in one 8-byte load (paths of L >= 1 start even) */
#pragma unroll
        for (int b = 0; b + 1 <= L; b += 2) {
            float2 w[P];
#pragma unroll
            for (int p = 0; p < P; ++p) w[p] = __ldg(reinterpret_cast<const float2 *>(path[p] + b));
            FV<P> v0, v1;
#pragma unroll
            for (int p = 0; p < P; ++p) {
                v0.set(p, w[p].x);
                v1.set(p, w[p].y);
            }
            sr = vfma(in.hB[b], v0, sr);
            sr = vfma(in.hB[b + 1], v1, sr);
        }
        if ((L & 1) == 0) {
            FV<P> v;
#pragma unroll
            for (int p = 0; p < P; ++p) v.set(p, __ldg(path[p] + L));
            sr = vfma(in.hB[L], v, sr);
        }
        s = (a == 0) ? vmul(in.hA(0), sr) : vfma(in.hA(a), sr, s);
    }
}

/* planes C..R of a fully unrolled 3-D block of budget R */
template <int R, int C, int P>
__device__ __forceinline__ void block3_planes(const float *__restrict__ alpha, const uint32_t (&base)[P],
                                              const Inner<P> &in, FV<P> &s)
{
    uint32_t sb[P];
    FV<P> s2;
#pragma unroll
    for (int p = 0; p < P; ++p) sb[p] = base[p] + coff_reg(R, C) + cell_at(in.TC[p], C) * blk2_reg(R - C);
    block2_fixed<R - C, P>(alpha, sb, in, s2);
    s = (C == 0) ? vmul(in.hC(0), s2) : vfma(in.hC(C), s2, s);
    if constexpr (C < R) block3_planes<R, C + 1, P>(alpha, base, in, s);
}

/* Generic sub-block of budget r (limits, r >= kNB): runtime loops. */
template <int P>
__device__ __forceinline__ void block2_generic(const float *__restrict__ alpha, int r, int limA, int limB,
                                               const float (&xA)[P], const float (&xB)[P], bool hasA,
                                               const uint32_t (&base)[P], FV<P> &s)
{
    const int amax = min(r, limA);
    uint32_t aoff = 0;
    FV<P> yA;
    uint32_t tA[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        yA.set(p, xA[p]);
        tA[p] = 0;
    }
    s = FV<P>::all(0.0f);
    for (int a = 0; a <= amax; ++a) {
        if (a) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                float y = yA.get(p);
                tA[p] = 2 * tA[p] + step_y(y);
                yA.set(p, y);
            }
        }
        const int rl = min(r - a, limB) + 1;
        const uint32_t plen = (1u << (rl - 1)) * (uint32_t)SG_PATH_WIDTH(rl);
        FV<P> yB, sr = FV<P>::all(0.0f);
        uint32_t rb[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            yB.set(p, xB[p]);
            /* path of the finest cell t_L = floor(x_B 2^L), exact */
            rb[p] = base[p] + aoff + tA[p] * plen +
                    (uint32_t)(xB[p] * (float)(1u << (rl - 1))) * (uint32_t)SG_PATH_WIDTH(rl);
        }
        for (int b = 0; b < rl; ++b) {
            if (b) {
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    float y = yB.get(p);
                    (void)step_y(y);
                    yB.set(p, y);
                }
            }
            FV<P> v;
#pragma unroll
            for (int p = 0; p < P; ++p) v.set(p, __ldg(alpha + rb[p] + b));
            sr = vfma(hats(yB), v, sr);
        }
        s = vfma(hasA ? hats(yA) : FV<P>::all(1.0f), sr, s);
        aoff += (1u << a) * plen;
    }
}

/* Sub-block of budget r: unrolled (r within the limits, r < kNB) or generic. */
template <int D, int P>
__device__ __forceinline__ void block2_any(const EvalArgs &A, int r, const Inner<P> &in, const float (&xA)[P],
                                           const float (&xB)[P], const uint32_t (&base)[P], FV<P> &s)
{
    if (D >= 2 && r <= A.lim2) {
        switch (r) {
#define SG_BLK2(RR) \
    case RR: block2_fixed<RR, P>(A.alpha, base, in, s); return;
            SG_BLK2(0) SG_BLK2(1) SG_BLK2(2) SG_BLK2(3) SG_BLK2(4)
            SG_BLK2(5) SG_BLK2(6) SG_BLK2(7) SG_BLK2(8) SG_BLK2(9)
#undef SG_BLK2
        default: break;
        }
    }
    block2_generic<P>(A.alpha, r, D >= 2 ? A.lim[D >= 2 ? D - 2 : 0] : 0, A.lim[D - 1], xA, xB, D >= 2, base, s);
}

/* Sum over the block of budget R at `base` for every point. */
template <int D, int P, int BL>
__device__ __forceinline__ void block_sum(const EvalArgs &A, int R, const Inner<P> &in, const float (&xC)[P],
                                          const float (&xA)[P], const float (&xB)[P], const uint32_t (&base)[P],
                                          FV<P> &s)
{
    if constexpr (D >= 3) {
        if (R <= kRFof<BL> && R <= A.lim3) {
            switch (R) {
            case 0: block3_planes<0, 0, P>(A.alpha, base, in, s); return;
            case 1: block3_planes<1, 0, P>(A.alpha, base, in, s); return;
            case 2: block3_planes<2, 0, P>(A.alpha, base, in, s); return;
            case 3: block3_planes<3, 0, P>(A.alpha, base, in, s); return;
            case 4: block3_planes<4, 0, P>(A.alpha, base, in, s); return;
            case 5:
                if constexpr (kRFof<BL> > 5) {
                    block3_planes<5, 0, P>(A.alpha, base, in, s);
                    return;
                }
                [[fallthrough]];
            default: block3_planes<kRFof<BL>, 0, P>(A.alpha, base, in, s); return;
            }
        }
    }
    /* plane loop; dim C is absent (limit 0) for d < 3 */
    const int cmax = D >= 3 ? min(R, A.lim[D >= 3 ? D - 3 : 0]) : 0;
    uint32_t coff = 0;
    FV<P> yC;
    uint32_t tC[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        yC.set(p, xC[p]);
        tC[p] = 0;
    }
    s = FV<P>::all(0.0f);
    for (int c = 0; c <= cmax; ++c) {
        if (c) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                float y = yC.get(p);
                tC[p] = 2 * tC[p] + step_y(y);
                yC.set(p, y);
            }
        }
        const uint32_t sub = A.blk2[R - c];
        uint32_t sb[P];
        FV<P> s2;
#pragma unroll
        for (int p = 0; p < P; ++p) sb[p] = base[p] + coff + tC[p] * sub;
        block2_any<D, P>(A, R - c, in, xA, xB, sb, s2);
        s = vfma(D >= 3 ? hats(yC) : FV<P>::all(1.0f), s2, s);
        coff += (1u << c) * sub;
    }
}

/* level state (y, cell index, parent product) of the upper prefix dims
 * K < kUpper (K <= D-6, at most 7 of them so that two CTAs still fit an SM
 * at d = 20), kept in shared memory while the subtree below runs */
template <int D>
constexpr int kUpper = D >= 6 ? (D - 5 < 7 ? D - 5 : 7) : 0;

/* The walk's block range of a split evaluation: blocks are numbered in
 * walk order; only [lo, hi) are summed (all of them when !partial). */
struct Range {
    uint32_t leaf, lo, hi;
    bool partial;
};

/* largest budget of an unrolled leaf subtree: of the last prefix dim
 * (kLGof, per points per thread under the wide preset: two points need
 * twice the registers), of the last two (kLG2) */
template <int P, int BL>
constexpr int kLGof = BL == 0 ? (P == 1 ? SG_EVAL_MAX_LEAF_P1 : SG_EVAL_MAX_LEAF_P2) : 3;
constexpr int kLG2 = SG_EVAL_MAX_LEAF2;
static_assert(SG_EVAL_MAX_LEAF_P1 <= 5 && SG_EVAL_MAX_LEAF_P2 <= 5 && kLG2 <= 3,
              "the walk's jump tables cover leaf budgets 0..5 and 0..3");
/* unrolled subtrees are instantiated for d <= kMaxUnrollD only (their code
 * grows with d; grids of more dims keep the loop) */
constexpr int kMaxUnrollD = 12;

/* next level of one prefix dim for every point: y doubles, the cell index
 * takes the next bit */
template <int P>
__device__ __forceinline__ void step_all(FV<P> &y, uint32_t (&ix)[P])
{
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float t = y.get(p);
        ix[p] = 2 * ix[p] + step_y(t);
        y.set(p, t);
    }
}

/* Levels l = L..B of the last prefix dim and their 3-D blocks of budget
 * B - l, fully unrolled (every shape regular: B within the limits). */
template <int D, int P, int B, int L>
__device__ __forceinline__ void leaf_group(const EvalArgs &A, uint32_t &cur, const Inner<P> &in, const FV<P> &pin,
                                           FV<P> &y, uint32_t (&ix)[P], FV<P> &acc)
{
    if constexpr (L > 0) step_all<P>(y, ix);
    constexpr int R = B - L;
    constexpr uint32_t blk = coff_reg(R, R + 1);
    uint32_t base[P];
    FV<P> s;
#pragma unroll
    for (int p = 0; p < P; ++p) base[p] = cur + ix[p] * blk;
    cur += blk << (A.nm1 - R);
    block3_planes<R, 0, P>(A.alpha, base, in, s);
    acc = vfma(vmul(pin, hats(y)), s, acc);
    if constexpr (L < B) leaf_group<D, P, B, L + 1>(A, cur, in, pin, y, ix, acc);
}

/* the coordinates of prefix dim K of this thread's points */
template <int P>
__device__ __forceinline__ FV<P> load_y(const float *sx, int K, int tid)
{
    FV<P> y;
#pragma unroll
    for (int p = 0; p < P; ++p) y.set(p, sx[(K * P + p) * kThreads + tid]);
    return y;
}

/* Levels l = L..B of prefix dim K = D-5, each followed by the unrolled
 * leaf group of dim D-4 with budget B - l (one compensated add per group,
 * as in the walk). */
template <int D, int K, int P, int B, int L>
__device__ __forceinline__ void leaf_group2(const EvalArgs &A, const float *sx, int tid, uint32_t &cur,
                                            const Inner<P> &in, const FV<P> &pin, FV<P> &y, uint32_t (&ix)[P],
                                            FV<P> &sum, FV<P> &comp)
{
    if constexpr (L > 0) step_all<P>(y, ix);
    const FV<P> pn = vmul(pin, hats(y));
    FV<P> y2 = load_y<P>(sx, K + 1, tid);
    FV<P> acc = FV<P>::all(0.0f);
    uint32_t ix2[P];
#pragma unroll
    for (int p = 0; p < P; ++p) ix2[p] = ix[p];
    leaf_group<D, P, B - L, 0>(A, cur, in, pn, y2, ix2, acc);
    kahan_add(sum, comp, acc);
    if constexpr (L < B) leaf_group2<D, K, P, B, L + 1>(A, sx, tid, cur, in, pin, y, ix, sum, comp);
}

/* Walk over prefix dim K (K <= D-4); children of depth D-4 are blocks.
 * M = mode: bit 0 (SPLIT) = the caller may ask for a block range (batched
 * launches), bits 1.. (BL) = the blocking preset. */
template <int D, int K, int P, int M>
struct Walk {
    static constexpr bool SPLIT = (M & 1) != 0;
    static constexpr int BL = M >> 1;
    static __device__ __forceinline__ void run(const EvalArgs &A, const float *sx, int tid, int budget,
                                               uint32_t &cur, Range &rg, const Inner<P> &in, const float (&xC)[P],
                                               const float (&xA)[P], const float (&xB)[P], const FV<P> &pin,
                                               const uint32_t (&ixin)[P], FV<P> &sum, FV<P> &comp)
    {
        if constexpr (K + 6 <= D && K < kUpper<D>) {
            /* upper prefix dim: its level state lives in this thread's
             * shared-memory slots while the subtree below runs, so it holds
             * no registers there */
            constexpr int NPX = D >= 4 ? D - 3 : 1;
            volatile float *ws = const_cast<float *>(sx) + NPX * P * kThreads + (K * 3 * P) * kThreads + tid;
            const int lmax = min(A.lim[K], budget);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                ws[(0 * P + p) * kThreads] = sx[(K * P + p) * kThreads + tid];
                ws[(1 * P + p) * kThreads] = __uint_as_float(ixin[p]);
                ws[(2 * P + p) * kThreads] = pin.get(p);
            }
            for (int l = 0; l <= lmax; ++l) {
                FV<P> y, pp;
                uint32_t ix[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    y.set(p, ws[(0 * P + p) * kThreads]);
                    ix[p] = __float_as_uint(ws[(1 * P + p) * kThreads]);
                    pp.set(p, ws[(2 * P + p) * kThreads]);
                }
                if (l) {
                    step_all<P>(y, ix);
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        ws[(0 * P + p) * kThreads] = y.get(p);
                        ws[(1 * P + p) * kThreads] = __uint_as_float(ix[p]);
                    }
                }
                if (SPLIT && rg.partial) {
                    const uint32_t *w = A.walk + 2 * ((K + 1) * (A.nm1 + 1) + (budget - l));
                    const uint32_t nb = __ldg(w);
                    if (rg.leaf + nb <= rg.lo || rg.leaf >= rg.hi) {
                        rg.leaf += nb;
                        cur += __ldg(w + 1);
                        continue;
                    }
                }
                const FV<P> pn = vmul(pp, hats(y));
                Walk<D, K + 1, P, M>::run(A, sx, tid, budget - l, cur, rg, in, xC, xA, xB, pn, ix, sum, comp);
            }
            return;
        }
        const int lmax = min(A.lim[K], budget);
        FV<P> y = load_y<P>(sx, K, tid);
        FV<P> acc = FV<P>::all(0.0f);
        uint32_t ix[P];
#pragma unroll
        for (int p = 0; p < P; ++p) ix[p] = ixin[p];
        if constexpr (D <= kMaxUnrollD && K + 1 == D - 4) {
            if (!(SPLIT && rg.partial) && budget <= kLG2 && budget <= A.lim[K] && budget <= A.lim[K + 1] &&
                budget <= A.lim3) {
                switch (budget) {
                case 0: leaf_group2<D, K, P, 0, 0>(A, sx, tid, cur, in, pin, y, ix, sum, comp); break;
                case 1: leaf_group2<D, K, P, 1, 0>(A, sx, tid, cur, in, pin, y, ix, sum, comp); break;
                case 2: leaf_group2<D, K, P, 2, 0>(A, sx, tid, cur, in, pin, y, ix, sum, comp); break;
                case 3: leaf_group2<D, K, P, 3, 0>(A, sx, tid, cur, in, pin, y, ix, sum, comp); break;
                default: break;
                }
                return;
            }
        }
        if constexpr (D <= kMaxUnrollD && K == D - 4) {
            if (!(SPLIT && rg.partial) && budget <= kLGof<P, BL> && budget <= A.lim[K] && budget <= A.lim3) {
                switch (budget) {
                case 0: leaf_group<D, P, 0, 0>(A, cur, in, pin, y, ix, acc); break;
                case 1: leaf_group<D, P, 1, 0>(A, cur, in, pin, y, ix, acc); break;
                case 2: leaf_group<D, P, 2, 0>(A, cur, in, pin, y, ix, acc); break;
                case 3: leaf_group<D, P, 3, 0>(A, cur, in, pin, y, ix, acc); break;
                case 4:
                    if constexpr (kLGof<P, BL> >= 4) leaf_group<D, P, 4, 0>(A, cur, in, pin, y, ix, acc);
                    break;
                case 5:
                    if constexpr (kLGof<P, BL> >= 5) leaf_group<D, P, 5, 0>(A, cur, in, pin, y, ix, acc);
                    break;
                default: break;
                }
                kahan_add(sum, comp, acc);
                return;
            }
        }
        for (int l = 0; l <= lmax; ++l) {
            if (l) step_all<P>(y, ix);
            if (SPLIT && rg.partial) {
                /* the child subtree (depth K+1, budget - l) holds blocks
                 * [leaf, leaf + nb): skip it whole when outside [lo, hi) */
                const uint32_t *w = A.walk + 2 * ((K + 1) * (A.nm1 + 1) + (budget - l));
                const uint32_t nb = __ldg(w);
                if (rg.leaf + nb <= rg.lo || rg.leaf >= rg.hi) {
                    rg.leaf += nb;
                    cur += __ldg(w + 1);
                    continue;
                }
            }
            const FV<P> pn = vmul(pin, hats(y));
            if constexpr (K == D - 4) {
                const int R = budget - l;
                const uint32_t blk = A.blk3[R];
                uint32_t base[P];
                FV<P> s;
#pragma unroll
                for (int p = 0; p < P; ++p) base[p] = cur + ix[p] * blk;
                cur += blk << (A.nm1 - R);
                if (SPLIT) ++rg.leaf;
                block_sum<D, P, BL>(A, R, in, xC, xA, xB, base, s);
                acc = vfma(pn, s, acc);
            } else {
                Walk<D, K + 1, P, M>::run(A, sx, tid, budget - l, cur, rg, in, xC, xA, xB, pn, ix, sum, comp);
            }
        }
        if constexpr (K == D - 4) kahan_add(sum, comp, acc);
    }
};

/* Evaluates this thread's points first, first + 32, ..., first + 32(P-1)
 * (those below `end`) against grid A; sx is this CTA's shared coordinate
 * buffer, shat its shared hats of dims A and C. */
template <int D, int P, int M>
__device__ __forceinline__ void eval_points(const EvalArgs &A, float *sx, FV<P> *shat, int tid, int64_t first,
                                            int64_t end, int part)
{
    constexpr bool SPLIT = (M & 1) != 0;
    float xC[P], xA[P], xB[P];
    bool valid[P], nan_in[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int64_t i = first + 32 * p;
        float x[D];
        valid[p] = i < end;
        nan_in[p] = false;
        bool inside = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float v = valid[p] ? A.coords[i * D + k] : 0.0f;
            nan_in[p] |= (v != v);
            inside &= (v >= 0.0f) && (v < 1.0f);
            x[k] = v;
        }
        /* outside [0,1)^d every basis function is 0: walk at x = 0 (always
         * in range) and write 0 (NaN for NaN input) instead */
        if (!inside) {
#pragma unroll
            for (int k = 0; k < D; ++k) x[k] = 0.0f;
        }
        valid[p] = valid[p] && inside;
#pragma unroll
        for (int k = 0; k + 3 < D; ++k) sx[(k * P + p) * kThreads + tid] = x[k];
        xC[p] = D >= 3 ? x[D >= 3 ? D - 3 : 0] : 0.0f;
        xA[p] = D >= 2 ? x[D >= 2 ? D - 2 : 0] : 0.0f;
        xB[p] = x[D - 1];
    }

    Inner<P> in;
    in.sh = shat + tid;
    FV<P> *const shw = shat + tid;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float y = xB[p];
#pragma unroll
        for (int j = 0; j < kNB; ++j) {
            if (j) (void)step_y(y);
            in.hB[j].set(p, hat_of(y));
        }
        in.TB[p] = (uint32_t)(xB[p] * (float)(1u << kTB));
        in.TA[p] = (uint32_t)(xA[p] * (float)(1u << kTB));
        in.TC[p] = (uint32_t)(xC[p] * (float)(1u << kTB));
    }
    {
        FV<P> yA, yC;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            yA.set(p, xA[p]);
            yC.set(p, xC[p]);
        }
#pragma unroll
        for (int j = 0; j < kNB; ++j) {
            if (j)
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    float y = yA.get(p);
                    (void)step_y(y);
                    yA.set(p, y);
                }
            shw[j * kThreads] = hats(yA);
        }
#pragma unroll
        for (int j = 0; j <= kRF; ++j) {
            if (j)
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    float y = yC.get(p);
                    (void)step_y(y);
                    yC.set(p, y);
                }
            shw[(kNB + j) * kThreads] = hats(yC);
        }
    }

    FV<P> sum = FV<P>::all(0.0f), comp = FV<P>::all(0.0f);
    uint32_t cur = 0;
    if constexpr (D >= 4) {
        const FV<P> pin = FV<P>::all(1.0f);
        uint32_t ix[P];
#pragma unroll
        for (int p = 0; p < P; ++p) ix[p] = 0;
        Range rg;
        rg.leaf = 0;
        rg.partial = SPLIT && A.nparts > 1;
        rg.lo = rg.partial ? A.split[part] : 0u;
        rg.hi = rg.partial ? A.split[part + 1] : 0xFFFFFFFFu;
        Walk<D, 0, P, M>::run(A, sx, tid, A.nm1, cur, rg, in, xC, xA, xB, pin, ix, sum, comp);
    } else {
        uint32_t base[P];
        FV<P> s;
#pragma unroll
        for (int p = 0; p < P; ++p) base[p] = 0;
        block_sum<D, P, (M >> 1)>(A, A.nm1, in, xC, xA, xB, base, s);
        kahan_add(sum, comp, s);
    }

    const FV<P> res = vsub(sum, comp);
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int64_t i = first + 32 * p;
        if (i < end) {
            const float r = valid[p] ? res.get(p) : (nan_in[p] ? __int_as_float(0x7fc00000) : 0.0f);
            if (SPLIT && A.nparts > 1)
                A.part_out[(int64_t)part * A.num_evals + i] = r;
            else
                A.out[A.perm ? A.perm[i] : i] = r;
        }
    }
}

/* Dynamic shared memory of one CTA: the hats of dims A and C (kHatSlots
 * FV<P> per thread), then the prefix coordinates (NPX * P floats per thread). */
template <int D, int P>
constexpr int kSmemBytes = kHatSlots * kThreads * (int)sizeof(FV<P>) + (D >= 4 ? D - 3 : 1) * P * kThreads * 4 +
                           kUpper<D> * 3 * P * kThreads * 4;

/* blocking presets instantiated for dimension D: both where the leaf
 * groups and 3-D blocks exist (3 <= D <= kMaxUnrollD); elsewhere one,
 * kBaseBL<D>: medium above kMaxUnrollD (no leaf groups; the wide preset's
 * larger 3-D blocks only add spills to those kernels' large walk state),
 * wide below 3 (no 3-D blocks: the presets are the same code) */
template <int D>
constexpr int kBlockings = (D >= 3 && D <= kMaxUnrollD) ? SG_EVAL_BLOCKINGS : 1;
template <int D>
constexpr int kBaseBL = D > kMaxUnrollD ? 1 : 0;
static_assert(SG_EVAL_BLOCKINGS == 2, "presets: wide (0) and medium (1)");

template <int D, int P, int BL>
__global__ void __launch_bounds__(kThreads, (P == 2 ? 2 : 3)) k_evaluate(const EvalArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_ev[];
    FV<P> *shat = reinterpret_cast<FV<P> *>(smem_ev);
    float *sx = reinterpret_cast<float *>(smem_ev + kHatSlots * kThreads * sizeof(FV<P>));
    const int tid = threadIdx.x;
    const int64_t warp = (blockIdx.x * (int64_t)kThreads + tid) >> 5;
    eval_points<D, P, 2 * BL>(A, sx, shat, tid, warp * (32 * P) + (tid & 31), A.num_evals, 0);
}

/* Many grids of the same dimension in one launch: CTA b evaluates the
 * kThreads*P points of grid items[b].x & (2^29-1) starting at point
 * items[b].y; bits 29..31 of items[b].x select the part of a split sum. */
template <int D, int P, int BL>
__global__ void __launch_bounds__(kThreads, (P == 2 ? 2 : 3))
    k_evaluate_batch(const EvalArgs *__restrict__ grids, const int2 *__restrict__ items)
{
    extern __shared__ __align__(16) unsigned char smem_ev[];
    FV<P> *shat = reinterpret_cast<FV<P> *>(smem_ev);
    float *sx = reinterpret_cast<float *>(smem_ev + kHatSlots * kThreads * sizeof(FV<P>));
    __shared__ EvalArgs sA;
    const int tid = threadIdx.x;
    const int2 item = items[blockIdx.x];
    const int q = item.x & 0x1FFFFFFF, part = (int)((unsigned)item.x >> 29);
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(grids + q);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&sA);
        for (int w = tid; w < (int)(sizeof(EvalArgs) / 4); w += kThreads) dst[w] = src[w];
    }
    __syncthreads();
    const int64_t start = item.y;
    const int64_t end = min(start + (int64_t)kThreads * P, sA.num_evals);
    eval_points<D, P, 2 * BL + 1>(sA, sx, shat, tid, start + (tid >> 5) * (32 * P) + (tid & 31), end, part);
}

template <int D, int P, int BL>
int launch_eval(const EvalArgs &A, void *stream)
{
    const int64_t per_block = (int64_t)kThreads * P;
    const int64_t blocks = (A.num_evals + per_block - 1) / per_block;
    if (blocks > 0x7fffffff) return cudaErrorInvalidValue;
    k_evaluate<D, P, BL><<<(unsigned)blocks, kThreads, kSmemBytes<D, P>, (cudaStream_t)stream>>>(A);
    sgk_count(1);
    return cudaGetLastError();
}

template <int D, int P, int BL>
int launch_eval_batch(const EvalArgs *grids, const int2 *items, int nitems, void *stream)
{
    k_evaluate_batch<D, P, BL><<<nitems, kThreads, kSmemBytes<D, P>, (cudaStream_t)stream>>>(grids, items);
    sgk_count(1);
    return cudaGetLastError();
}

template <int D, int BL>
int set_smem(void)
{
    int e = cudaFuncSetAttribute(k_evaluate<D, 1, BL>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes<D, 1>);
    if (!e) e = cudaFuncSetAttribute(k_evaluate<D, 2, BL>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes<D, 2>);
    if (!e)
        e = cudaFuncSetAttribute(k_evaluate_batch<D, 1, BL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemBytes<D, 1>);
    if (!e)
        e = cudaFuncSetAttribute(k_evaluate_batch<D, 2, BL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemBytes<D, 2>);
    return e;
}

} // namespace sgeval

/* Lets the kernels of dimension D use their dynamic shared memory (above
 * 48 KB for d >= 8 at two points per thread) on the current device; called
 * once per device before the first launch (outside any stream capture). */
template <int D>
int eval_setup()
{
    int e = sgeval::set_smem<D, sgeval::kBaseBL<D>>();
    if constexpr (sgeval::kBlockings<D> > 1)
        if (!e) e = sgeval::set_smem<D, 1>();
    return e;
}

/* blocking: preset index; dimensions with one form take kBaseBL<D> */
template <int D>
int eval_launch(const EvalArgs &A, int ppt, int blocking, void *stream)
{
    constexpr int B0 = sgeval::kBaseBL<D>;
    if constexpr (sgeval::kBlockings<D> > 1)
        if (blocking == 1) return ppt == 1 ? sgeval::launch_eval<D, 1, 1>(A, stream) : sgeval::launch_eval<D, 2, 1>(A, stream);
    return ppt == 1 ? sgeval::launch_eval<D, 1, B0>(A, stream) : sgeval::launch_eval<D, 2, B0>(A, stream);
}

template <int D>
int eval_batch_launch(const EvalArgs *grids, const int2 *items, int nitems, int ppt, int blocking, void *stream)
{
    if (nitems <= 0) return cudaSuccess;
    if constexpr (sgeval::kBlockings<D> > 1)
        if (blocking == 1)
            return ppt == 1 ? sgeval::launch_eval_batch<D, 1, 1>(grids, items, nitems, stream)
                            : sgeval::launch_eval_batch<D, 2, 1>(grids, items, nitems, stream);
    constexpr int B0 = sgeval::kBaseBL<D>;
    return ppt == 1 ? sgeval::launch_eval_batch<D, 1, B0>(grids, items, nitems, stream)
                    : sgeval::launch_eval_batch<D, 2, B0>(grids, items, nitems, stream);
}

#endif
