/*
 * Harness that compiles the REFERENCE benchmark's own C code in place and
 * exports a small C ABI over its global-state functions.  TEST
 * INFRASTRUCTURE ONLY: it is built by oracle/Makefile into oracle/_ref/ (never
 * committed), used to pin the oracle restatement (sg_oracle.c), to generate
 * the golden fixtures, and as the timed CPU baseline.  No reference source is
 * copied into this repository; REF_SRC names the file where it lies.
 *
 * Two build-level adjustments, neither of which changes the reference's
 * arithmetic:
 *   - main() is renamed so the file links as a library;
 *   - malloc is routed to calloc, because init() (c:113-129) reads dp_mat[0][j]
 *     for j > limits[0] without writing it; zero is the value the recurrence
 *     needs there, and fresh calloc memory guarantees it.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define main asgb_reference_main
#define malloc(sz) calloc(1, (sz))
#include REF_SRC
#undef malloc
#undef main

#define REF_API __attribute__((visibility("default")))

static void free_state(void)
{
    int i;
    if (dp_mat) {
        for (i = 0; i < num_dims; i++) free(dp_mat[i]);
        free(dp_mat);
        dp_mat = NULL;
    }
    if (par_lili) {
        for (i = 0; i < num_levels; i++) free(par_lili[i]);
        free(par_lili);
        par_lili = NULL;
    }
    free(lidx_vect);
    lidx_vect = NULL;
    free(sg1d);
    sg1d = NULL;
    free(limits);
    limits = NULL;
}

/* Sets num_dims/num_levels/limits and runs the reference init() (c:101-183).
 * limits == NULL means the reference default limits[i] = n-1 (c:1760-1763). */
REF_API int ref_init(int d, int n, const int *lim)
{
    int i;
    free_state();
    num_dims = d;
    num_levels = n;
    num_evals = 0;
    limits = (int *)calloc(d, sizeof(int));
    for (i = 0; i < d; i++) limits[i] = lim ? lim[i] : n - 1;
    init();
    return 0;
}

REF_API int ref_num_points(void) { return num_grid_points; }
REF_API int ref_num_subspaces(void) { return num_subspaces; }

REF_API void ref_tables(int *dp_out, int *lidx_out)
{
    int i, j;
    for (i = 0; i < num_dims; i++)
        for (j = 0; j < num_levels; j++) dp_out[i * num_levels + j] = dp_mat[i][j];
    for (j = 0; j < num_levels; j++) lidx_out[j] = lidx_vect[j];
}

REF_API void ref_get_values(float *out) { memcpy(out, sg1d, (size_t)num_grid_points * sizeof(float)); }
REF_API void ref_set_values(const float *in) { memcpy(sg1d, in, (size_t)num_grid_points * sizeof(float)); }

REF_API int ref_gp2idx(int *lv, int *ix) { return gp2idx(lv, ix); }
REF_API int ref_idx2gp(int idx, int *lv, int *ix) { return idx2gp(idx, lv, ix); }

/* variant: 0..8 = hierarchize0..8 (c:557-1176), 9 = omp_hierarchize3 (c:1180) */
REF_API int ref_hierarchize(int variant)
{
    switch (variant) {
    case 0: return hierarchize0();
    case 1: return hierarchize1();
    case 2: return hierarchize2();
    case 3: return hierarchize3();
    case 4: return hierarchize4();
    case 5: return hierarchize5();
    case 6: return hierarchize6();
    case 7: return hierarchize7();
    case 8: return hierarchize8();
    case 9: return omp_hierarchize3();
    default: return -1;
    }
}

/* variant: 0..5 = evaluate0..5 (c:1237-1688), 6 = omp_evaluate2, 7 = omp_evaluate5.
 * Evaluates against the current sg1d.  The SSE variants keep the coordinates
 * in a stack array (c:1323, c:1562), so callers pass modest chunks. */
REF_API int ref_evaluate(int variant, float *coords, float *out, int m)
{
    switch (variant) {
    case 0: return evaluate0(sg1d, coords, out, m);
    case 1: return evaluate1(sg1d, coords, out, m);
    case 2: return evaluate2(sg1d, coords, out, m);
    case 3: return evaluate3(sg1d, coords, out, m);
    case 4: return evaluate4(sg1d, coords, out, m);
    case 5: return evaluate5(sg1d, coords, out, m);
    case 6: return omp_evaluate2(sg1d, coords, out, m);
    case 7: return omp_evaluate5(sg1d, coords, out, m);
    default: return -1;
    }
}

REF_API int ref_max_threads(void) { return omp_get_max_threads(); }
