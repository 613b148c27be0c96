/*
 * Host-side index algebra of the compact sparse-grid layout and the device
 * layout derived from it.  Plain C, shared by the API (sgrid.c) and the CUDA
 * launchers.
 *
 * Device layout ("group-aligned compact layout"): exactly the reference's
 * compact order (adaptive_sparse_grid_bench.c:130-140, 187-207), except that
 * each level group starts on a 32-element boundary.  A subspace of group
 * s >= 2 therefore starts on a 16-byte boundary (FP32), which is what the
 * bulk-copy engine and vector loads need.  Compact index j of group s maps to
 * device index j - lidx[s] + plidx[s].
 */
#ifndef SG_LAYOUT_H
#define SG_LAYOUT_H

#include <stdint.h>

#include "../../include/sgrid.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SG_GROUP_ALIGN 32 /* elements */

typedef struct sg_layout {
    int d, n;
    int lim[SG_MAX_DIMS];
    int64_t dp[SG_MAX_DIMS][SG_MAX_LEVELS]; /* dp[i][s], c:113-129          */
    int64_t lidx[SG_MAX_LEVELS + 1];        /* compact group offsets        */
    int64_t plidx[SG_MAX_LEVELS + 1];       /* device (padded) group offsets */
    int64_t N, S, Npad;
} sg_layout;

/* One 1-D "chain" of sweep k: the subspaces that differ only in l_k.  They
 * hold 2^sigma independent poles (one per index combination of the other
 * dims); segment j (l_k = j) is the whole subspace, 2^(sigma+j) values. */
typedef struct sg_chain {
    uint32_t seg;   /* first entry of this chain in the segment-offset array */
    uint8_t sigma;  /* sum of the other dims' levels                         */
    uint8_t lmax;   /* highest l_k in the chain (>= 1; lmax 0 needs no work) */
    uint8_t lo;     /* sum of the levels of dims k+1..d-1 (index bits below) */
    uint8_t pad;
} sg_chain;

int sg_layout_init(sg_layout *L, int d, int n, const int *limits);
int64_t sg_layout_l2idx(const sg_layout *L, const int *lv);
void sg_layout_idx2l(const sg_layout *L, int64_t pos, int s, int *lv);
int64_t sg_layout_gp2idx(const sg_layout *L, const int *lv, const int *ix);
int sg_layout_idx2gp(const sg_layout *L, int64_t idx, int *lv, int *ix);
/* Device offset of the subspace with level vector lv. */
int64_t sg_layout_subspace_offset(const sg_layout *L, const int *lv);

/* Chains of sweep k with lmax >= 1, largest first.  *chains and *seg_off are
 * malloc'd; seg_off[c.seg + j] is the device offset of segment j. */
int sg_layout_chains(const sg_layout *L, int k, sg_chain **chains, int64_t *nchains,
                     uint32_t **seg_off, int64_t *nseg);

/* Device offsets of all subspaces in evaluation (depth-first) order: dims
 * 0..d-1 outermost to innermost, each dim's level ascending.  *off is
 * malloc'd with S entries. */
int sg_layout_dfs_offsets(const sg_layout *L, uint32_t **off);

#ifdef __cplusplus
}
#endif
#endif
