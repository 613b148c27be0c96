/*
 * CPU oracle for the compact sparse-grid hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only the test suite,
 * the smoke check and the CPU-baseline leg of the benchmark load it.  The
 * product library (adaptive_sparse_grid_bench_b200/libsgb200.so) never links
 * or calls it, and nothing here is a fallback for the CUDA path.
 *
 * It is a plain-C restatement, written for this project, of the algorithm in
 * the reference benchmark adaptive_sparse_grid_bench.c (file:line citations
 * below are to that file):
 *   - index tables dp/lidx            c:101-140  (limit-aware counting, as the
 *                                     CUDA host code cu:79-102 computes it)
 *   - gp2idx / idx2gp / idx2l / l2idx c:187-279
 *   - left/right 1-D parents          c:282-344, c:828-854
 *   - hierarchize0 (definition)       c:557-571  (FP32 and FP64 versions)
 *   - evaluate0 (definition)          c:1237-1274 (FP32 and FP64 versions)
 * It is pinned against the reference itself compiled in place (oracle/_ref,
 * built by oracle/Makefile from the reference sources) and against the
 * golden fixtures in tests/golden/.
 *
 * Conventions: levels are 0-based; a grid of "n levels" holds every level
 * vector l with l_k <= limits[k] and sum(l) <= n-1; point (l,i) sits at
 * x = (2i+1)/2^(l+1).  Linear indices are int64 here (the reference uses int).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAXD 32
#define OR_MAXN 32

#ifdef _WIN32
#define OR_API __declspec(dllexport)
#else
#define OR_API __attribute__((visibility("default")))
#endif

typedef struct {
    int d, n;
    int lim[OR_MAXD];
    int64_t dp[OR_MAXD][OR_MAXN]; /* dp[i][s]: #level vectors over dims 0..i with sum s */
    int64_t lidx[OR_MAXN + 1];    /* lidx[s]: first linear index of level group s       */
    int64_t N, S;
} or_layout;

OR_API int or_layout_size(void) { return (int)sizeof(or_layout); }

/* Tables of c:101-140.  dp[i][s] = sum_{k=0..min(s,lim_i)} dp[i-1][s-k]. */
OR_API int or_layout_init(or_layout *L, int d, int n, const int *limits)
{
    int i, s, k;
    if (d < 1 || d > OR_MAXD || n < 1 || n > OR_MAXN) return -1;
    memset(L, 0, sizeof(*L));
    L->d = d;
    L->n = n;
    for (i = 0; i < d; i++) {
        L->lim[i] = limits ? limits[i] : n - 1;
        if (L->lim[i] < 0) return -1;
        if (L->lim[i] > n - 1) L->lim[i] = n - 1;
    }
    for (s = 0; s < n; s++) L->dp[0][s] = (s <= L->lim[0]) ? 1 : 0;
    for (i = 1; i < d; i++)
        for (s = 0; s < n; s++) {
            int64_t c = 0;
            for (k = 0; k <= s && k <= L->lim[i]; k++) c += L->dp[i - 1][s - k];
            L->dp[i][s] = c;
        }
    L->N = 0;
    L->S = 0;
    for (s = 0; s < n; s++) {
        L->lidx[s] = L->N;
        L->N += L->dp[d - 1][s] << s;
        L->S += L->dp[d - 1][s];
    }
    L->lidx[n] = L->N;
    return 0;
}

/* l2idx, c:266-279: position of level vector lv inside its level group. */
OR_API int64_t or_l2idx(const or_layout *L, const int *lv)
{
    int64_t pos = 0;
    int i, j, sum = lv[0];
    for (i = 1; i < L->d; i++) {
        sum += lv[i];
        for (j = 0; j < lv[i]; j++) pos += L->dp[i - 1][sum - j];
    }
    return pos;
}

/* idx2l, c:245-264: level vector of position pos inside group s. */
OR_API void or_idx2l(const or_layout *L, int64_t pos, int s, int *lv)
{
    int i, level;
    for (i = L->d - 1; i >= 1; i--) {
        level = 0;
        while (pos >= L->dp[i - 1][s - level]) {
            pos -= L->dp[i - 1][s - level];
            level++;
        }
        lv[i] = level;
        s -= level;
    }
    lv[0] = s;
}

/* gp2idx, c:187-207: (levels, indices) -> linear index in the compact layout. */
OR_API int64_t or_gp2idx(const or_layout *L, const int *lv, const int *ix)
{
    int64_t in_sub = ix[0];
    int i, s = lv[0];
    for (i = 1; i < L->d; i++) {
        in_sub = (in_sub << lv[i]) + ix[i];
        s += lv[i];
    }
    return L->lidx[s] + (or_l2idx(L, lv) << s) + in_sub;
}

/* idx2gp, c:210-243: linear index -> (levels, indices). */
OR_API int or_idx2gp(const or_layout *L, int64_t idx, int *lv, int *ix)
{
    int s = 0, i;
    int64_t rest, pos;
    if (idx < 0 || idx >= L->N) return -1;
    while (s < L->n && idx >= L->lidx[s]) s++;
    s--;
    idx -= L->lidx[s];
    rest = idx & ((1LL << s) - 1);
    pos = idx >> s;
    or_idx2l(L, pos, s, lv);
    for (i = L->d - 1; i >= 0; i--) {
        ix[i] = (int)(rest & ((1LL << lv[i]) - 1));
        rest >>= lv[i];
    }
    return 0;
}

/* 1-D hierarchical parents, c:828-854 (get_left_li / get_right_li). */
static int left_parent(int l, int i, int *pl, int *pi)
{
    if (i == 0) return 0;
    *pl = l - 1;
    *pi = i;
    while ((*pi & 1) == 0) { *pi >>= 1; (*pl)--; }
    *pi >>= 1;
    return 1;
}
static int right_parent(int l, int i, int *pl, int *pi)
{
    if (i == (1 << l) - 1) return 0;
    *pl = l - 1;
    *pi = i + 1;
    while ((*pi & 1) == 0) { *pi >>= 1; (*pl)--; }
    *pi >>= 1;
    return 1;
}

/* Value of the dim-k parent of point (lv, ix); 0 at the domain boundary.
 * c:282-344 (get_left_parent_val / get_right_parent_val). */
#define PARENT_VAL(T, name)                                                   \
    static T name(const or_layout *L, const T *a, int *lv, int *ix, int k,   \
                  int right)                                                  \
    {                                                                         \
        int pl, pi, sl = lv[k], si = ix[k];                                   \
        T v;                                                                  \
        if (!(right ? right_parent(sl, si, &pl, &pi)                          \
                    : left_parent(sl, si, &pl, &pi)))                         \
            return (T)0;                                                      \
        lv[k] = pl;                                                           \
        ix[k] = pi;                                                           \
        v = a[or_gp2idx(L, lv, ix)];                                          \
        lv[k] = sl;                                                           \
        ix[k] = si;                                                           \
        return v;                                                             \
    }
PARENT_VAL(float, parent_f32)
PARENT_VAL(double, parent_f64)

/* hierarchize0, c:557-571: for each dim, walk indices downward (parents have
 * smaller indices, so they still hold pre-sweep values) and subtract half the
 * sum of the two parents.  The FP32 version keeps the reference's expression
 * shape a - (L + R) * 0.5f exactly. */
OR_API void or_hierarchize_f32(const or_layout *L, float *a)
{
    int lv[OR_MAXD], ix[OR_MAXD], k;
    int64_t j;
    for (k = 0; k < L->d; k++)
        for (j = L->N - 1; j >= 0; j--) {
            float lft, rgt;
            or_idx2gp(L, j, lv, ix);
            lft = parent_f32(L, a, lv, ix, k, 0);
            rgt = parent_f32(L, a, lv, ix, k, 1);
            a[j] -= (lft + rgt) * 0.5f;
        }
}

OR_API void or_hierarchize_f64(const or_layout *L, double *a)
{
    int lv[OR_MAXD], ix[OR_MAXD], k;
    int64_t j;
    for (k = 0; k < L->d; k++)
        for (j = L->N - 1; j >= 0; j--) {
            double lft, rgt;
            or_idx2gp(L, j, lv, ix);
            lft = parent_f64(L, a, lv, ix, k, 0);
            rgt = parent_f64(L, a, lv, ix, k, 1);
            a[j] -= (lft + rgt) * 0.5;
        }
}

/* The same FP64 hierarchization, organised per subspace so that large grids
 * finish in seconds: every point of subspace lv finds its dim-k parents in the
 * parent subspaces' offsets (the loop structure of c:613-655, hierarchize2).
 * Each point sees exactly the arithmetic of or_hierarchize_f64; groups are
 * walked finest first so parents are still pre-sweep. */
OR_API void or_hierarchize_f64_fast(const or_layout *L, double *a)
{
    int lv[OR_MAXD], ix[OR_MAXD], k, s, m, d = L->d;
    int64_t pos, p, npts;
    int64_t par_off[OR_MAXN];
    for (k = 0; k < d; k++)
        for (s = L->n - 1; s >= 0; s--)
            for (pos = 0; pos < L->dp[d - 1][s]; pos++) {
                int lk, l;
                int64_t base = L->lidx[s] + (pos << s);
                or_idx2l(L, pos, s, lv);
                lk = lv[k];
                if (lk == 0) continue; /* no parents in dim k: a - 0 == a */
                for (l = 0; l < lk; l++) {
                    lv[k] = l;
                    par_off[l] = L->lidx[s - lk + l] + (or_l2idx(L, lv) << (s - lk + l));
                }
                lv[k] = lk;
                npts = (int64_t)1 << s;
                for (p = 0; p < npts; p++) {
                    int64_t rest = p, in_sub;
                    int pl, pi;
                    double lft = 0.0, rgt = 0.0;
                    for (m = d - 1; m >= 0; m--) {
                        ix[m] = (int)(rest & ((1LL << lv[m]) - 1));
                        rest >>= lv[m];
                    }
                    if (left_parent(lk, ix[k], &pl, &pi)) {
                        in_sub = 0;
                        for (m = 0; m < d; m++)
                            in_sub = m == k ? (in_sub << pl) + pi : (in_sub << lv[m]) + ix[m];
                        lft = a[par_off[pl] + in_sub];
                    }
                    if (right_parent(lk, ix[k], &pl, &pi)) {
                        in_sub = 0;
                        for (m = 0; m < d; m++)
                            in_sub = m == k ? (in_sub << pl) + pi : (in_sub << lv[m]) + ix[m];
                        rgt = a[par_off[pl] + in_sub];
                    }
                    a[base + p] -= (lft + rgt) * 0.5;
                }
            }
}

/* evaluate0, c:1237-1274, FP32 with the reference's exact expression order:
 * subspaces in memory order, prod = 1*hat_0*...*hat_{d-1}, then *surplus,
 * then out += prod (plain recursive summation). */
OR_API void or_evaluate_f32(const or_layout *L, const float *a, const float *X,
                            float *out, int64_t m)
{
    int lv[OR_MAXD], s, k, d = L->d;
    int64_t c, pos;
    for (c = 0; c < m; c++) {
        const float *x = X + c * d;
        float acc = 0.0f;
        int64_t base = 0;
        for (s = 0; s < L->n; s++)
            for (pos = 0; pos < L->dp[d - 1][s]; pos++) {
                float prod = 1.0f;
                int64_t in_sub = 0;
                or_idx2l(L, pos, s, lv);
                for (k = 0; k < d; k++) {
                    float div = 1.0f / (float)(1 << lv[k]);
                    int t = (int)(x[k] / div);
                    float left = (float)t * div;
                    float mm = (2.0f * (x[k] - left) - div) / div;
                    in_sub = in_sub * (1 << lv[k]) + t;
                    prod *= 1.0f + mm * (1.0f - (float)((mm >= 0.0f) << 1));
                }
                prod *= a[base + in_sub];
                acc += prod;
                base += (int64_t)1 << s;
            }
        out[c] = acc;
    }
}

/* FP64 statement of the interpolant (the error reference): same traversal,
 * hat = 1 - |x*2^(l+1) - (2t+1)| and the sum accumulated in double. */
OR_API void or_evaluate_f64(const or_layout *L, const double *a, const float *X,
                            double *out, int64_t m)
{
    int lv[OR_MAXD], s, k, d = L->d;
    int64_t c, pos;
    for (c = 0; c < m; c++) {
        const float *x = X + c * d;
        double acc = 0.0;
        int64_t base = 0;
        for (s = 0; s < L->n; s++)
            for (pos = 0; pos < L->dp[d - 1][s]; pos++) {
                double prod = 1.0;
                int64_t in_sub = 0;
                or_idx2l(L, pos, s, lv);
                for (k = 0; k < d; k++) {
                    double sc = ldexp(1.0, lv[k]);
                    double xs = (double)x[k] * sc;
                    int64_t t = (int64_t)xs;
                    double mm = 2.0 * (xs - (double)t) - 1.0;
                    in_sub = (in_sub << lv[k]) + t;
                    prod *= 1.0 - fabs(mm);
                }
                acc += prod * a[base + in_sub];
                base += (int64_t)1 << s;
            }
        out[c] = acc;
    }
}

/* or_evaluate_f64 for large grids and many points: the level vectors of all
 * subspaces are computed once (memory order, as the loop above visits them)
 * and the points are split over OpenMP threads.  Every point sees exactly
 * the arithmetic of or_evaluate_f64, so the results are bit-identical. */
OR_API int or_evaluate_f64_par(const or_layout *L, const double *a, const float *X,
                               double *out, int64_t m)
{
    int d = L->d, s;
    int64_t S = L->S, q = 0, pos, c;
    int *lvs = (int *)malloc((size_t)S * (size_t)d * sizeof(int));
    double *scs = (double *)malloc((size_t)S * (size_t)d * sizeof(double));
    int64_t *bases = (int64_t *)malloc((size_t)S * sizeof(int64_t));
    if (!lvs || !scs || !bases) {
        free(lvs);
        free(scs);
        free(bases);
        return -1;
    }
    {
        int64_t base = 0;
        for (s = 0; s < L->n; s++)
            for (pos = 0; pos < L->dp[d - 1][s]; pos++, q++) {
                int k;
                or_idx2l(L, pos, s, lvs + q * d);
                for (k = 0; k < d; k++) scs[q * d + k] = ldexp(1.0, lvs[q * d + k]);
                bases[q] = base;
                base += (int64_t)1 << s;
            }
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (c = 0; c < m; c++) {
        const float *x = X + c * d;
        double acc = 0.0;
        int64_t t2;
        for (t2 = 0; t2 < S; t2++) {
            const int *lv = lvs + t2 * d;
            const double *sc = scs + t2 * d;
            double prod = 1.0;
            int64_t in_sub = 0;
            int k;
            for (k = 0; k < d; k++) {
                double xs = (double)x[k] * sc[k];
                int64_t t = (int64_t)xs;
                double mm = 2.0 * (xs - (double)t) - 1.0;
                in_sub = (in_sub << lv[k]) + t;
                prod *= 1.0 - fabs(mm);
            }
            acc += prod * a[bases[t2] + in_sub];
        }
        out[c] = acc;
    }
    free(lvs);
    free(scs);
    free(bases);
    return 0;
}

/* Coordinates of every grid point in compact order (N x d, row-major). */
OR_API void or_grid_points(const or_layout *L, float *X)
{
    int lv[OR_MAXD], ix[OR_MAXD], k;
    int64_t j;
    for (j = 0; j < L->N; j++) {
        or_idx2gp(L, j, lv, ix);
        for (k = 0; k < L->d; k++)
            X[j * L->d + k] = (float)(2 * ix[k] + 1) / (float)(1LL << (lv[k] + 1));
    }
}
