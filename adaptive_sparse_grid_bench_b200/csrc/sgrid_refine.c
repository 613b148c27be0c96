/*
 * Limits-adaptive refinement (sg_refine_step, sg_refine in include/sgrid.h).
 * Host code in C over the public API.
 *
 * The reference's adaptive grid is a per-dimension level limit vector
 * (adaptive_sparse_grid_bench.c:82-83, used by init() c:113-129): a grid
 * (d, n, limits) holds every subspace l with sum_k l_k <= n-1 and
 * l_k <= limits[k], stored whole in the compact layout.  It has no
 * refinement of its own.  This driver refines within that family, so every
 * grid it produces is one the reference's init()/idx2gp()/hierarchize0()
 * accept and reproduce:
 *   a subspace is active when max |surplus| over its points exceeds tol;
 *   every child l + e_k (l_k < max_level) of an active subspace must be in
 *   the grid;
 *   the next grid is the smallest (n', limits') holding the current grid and
 *   all those children: n' = max(n, max |child| + 1), limits'[k] =
 *   max(limits[k], max child_k).
 * The driver samples f, hierarchizes, measures and steps until nothing
 * changes, an iteration cap or a point cap is reached.
 */
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include "sg_batch_internal.h"
#include "sg_grid_internal.h"
#include "sg_layout.h"

#define SG_API __attribute__((visibility("default")))

static int rfail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    sg_set_error(fmt, ap);
    va_end(ap);
    return code;
}

/* sg_refine_step, on a layout whose limits are already normalised */
static int refine_step(const sg_layout *L, const float *maxabs, double tol, int max_level, int *n_out,
                       int *limits_out, int *changed)
{
    int lv[SG_MAX_DIMS];
    int k, s, nn = L->n;
    int64_t pos, q = 0;
    for (k = 0; k < L->d; k++) limits_out[k] = L->lim[k];
    for (s = 0; s < L->n; s++) {
        const int64_t cnt = (L->lidx[s + 1] - L->lidx[s]) >> s;
        for (pos = 0; pos < cnt; pos++, q++) {
            if (!((double)maxabs[q] > tol)) continue;
            sg_layout_idx2l(L, pos, s, lv);
            for (k = 0; k < L->d; k++) {
                if (lv[k] >= max_level) continue;
                /* the child l + e_k has level sum s + 1 and l_k + 1 in dim k */
                if (lv[k] + 1 > limits_out[k]) limits_out[k] = lv[k] + 1;
                if (s + 2 > nn) nn = s + 2;
            }
        }
    }
    if (nn > SG_MAX_LEVELS) nn = SG_MAX_LEVELS;
    for (k = 0; k < L->d; k++)
        if (limits_out[k] > nn - 1) limits_out[k] = nn - 1;
    *n_out = nn;
    *changed = nn != L->n;
    for (k = 0; k < L->d; k++)
        if (limits_out[k] != L->lim[k]) *changed = 1;
    return SG_OK;
}

SG_API int sg_refine_step(int d, int n, const int *limits, const float *maxabs, double tol, int max_level,
                          int *n_out, int *limits_out, int *changed)
{
    sg_layout L;
    int r;
    if (!maxabs || !n_out || !limits_out || !changed || max_level < 0 || !(tol >= 0.0))
        return rfail(SG_ERR_ARG, "sg_refine_step: bad argument");
    if ((r = sg_layout_init(&L, d, n, limits)) != SG_OK) return rfail(r, "sg_refine_step: bad grid shape");
    return refine_step(&L, maxabs, tol, max_level, n_out, limits_out, changed);
}

/* A grid of (d, n, limits) with f sampled at its points and hierarchized. */
static int build(int d, int n, const int *lim, int fn, const double *params, int np, int precision, sg_grid **out)
{
    sg_grid *g = NULL;
    int r = sg_create(d, n, lim, &g);
    if (r == SG_OK) r = sg_set_option(g, SG_OPT_HIER_PRECISION, precision);
    if (r == SG_OK) r = sg_sample_function(g, fn, params, np, 0);
    if (r == SG_OK) r = sg_hierarchize_async(g, 0);
    if (r == SG_OK) r = sg_sync(g, 0);
    if (r != SG_OK) {
        sg_destroy(g);
        return r;
    }
    *out = g;
    return SG_OK;
}

SG_API int sg_refine(int d, int n0, const int *limits0, int fn, const double *params, int num_params, double tol,
                     int max_level, int64_t max_points, int max_iters, int precision, sg_grid **grid,
                     int *iterations)
{
    sg_grid *g = NULL;
    sg_layout next;
    float *stat = NULL;
    int lim[SG_MAX_DIMS], nl[SG_MAX_DIMS];
    int n = n0, nn, changed, it, r, k;
    if (!grid || max_iters < 1 || max_points < 1 || max_level < 0 || !(tol >= 0.0))
        return rfail(SG_ERR_ARG, "sg_refine: bad argument");
    *grid = NULL;
    if (iterations) *iterations = 0;
    if ((r = sg_layout_init(&next, d, n0, limits0)) != SG_OK) return rfail(r, "sg_refine: bad starting grid");
    for (k = 0; k < d; k++) lim[k] = next.lim[k];
    for (it = 1;; it++) {
        if ((r = build(d, n, lim, fn, params, num_params, precision, &g)) != SG_OK) break;
        if (iterations) *iterations = it;
        if (it == max_iters) break;
        free(stat);
        stat = (float *)malloc((size_t)(g->L.S > 0 ? g->L.S : 1) * sizeof(float));
        if (!stat) {
            r = rfail(SG_ERR_NOMEM, "sg_refine: out of host memory");
            break;
        }
        if ((r = sg_subspace_maxabs(g, stat)) != SG_OK) break;
        refine_step(&g->L, stat, tol, max_level, &nn, nl, &changed);
        if (!changed) break;
        /* stop before a grid above the point cap */
        if (sg_layout_init(&next, d, nn, nl) != SG_OK || next.N > max_points) break;
        sg_destroy(g);
        g = NULL;
        n = nn;
        memcpy(lim, nl, sizeof(int) * (size_t)d);
    }
    free(stat);
    if (r != SG_OK) {
        sg_destroy(g);
        return r;
    }
    *grid = g;
    return SG_OK;
}
