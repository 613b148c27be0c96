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


/*
 * Evaluation layout ("block layout").  The same surpluses, ordered for the
 * evaluation walk: for every prefix level vector p of dims 0..d-3 (depth-
 * first order, level ascending), for every cell I of p (row-major over those
 * dims), one block holding all subspaces (p, a, b) with a = l_{d-2},
 * b = l_{d-1}: rows a = 0..amax, each row 2^a poles (one per cell t_a of dim
 * d-2), each pole the 1-D heap of dim d-1's levels b = 0..rowlen(a)-1 with
 * cell t_b of level b at heap index 2^b - 1 + t_b.  A query point therefore
 * finds every surplus of a block at base + aoff(a) + t_a*plen(a) + 2^b-1 + t_b.
 * For d = 1 the "block" is the single pole of dim 0 (one row, a = 0).
 */
typedef struct sg_eval_shape {
    int R;         /* level budget n-1-sigma left for the last two dims */
    int amax;      /* last row: min(R, lim_{d-2}) (0 for d = 1)          */
    int rowlen[SG_MAX_LEVELS]; /* levels of dim d-1 in row a             */
    uint32_t aoff[SG_MAX_LEVELS + 1]; /* row starts; aoff[amax+1] = block size */
} sg_eval_shape;

void sg_layout_eval_shape(const sg_layout *L, int R, sg_eval_shape *sh);

/* Per-subspace repack descriptor (compact layout -> block layout). */
typedef struct sg_repack {
    uint32_t src;  /* device offset of the subspace in the group-aligned layout */
    uint32_t dst;  /* block-layout offset of its element (I=0, t_a=0, t_b=0)    */
    uint32_t blk;  /* block size: stride between prefix cells I                */
    uint32_t plen; /* pole length of its row: stride between cells t_a         */
    uint8_t a, b, s, pad;
} sg_repack;

/* Block bases (one per prefix, depth-first order) and the repack table (one
 * entry per subspace).  Both malloc'd. */
int sg_layout_eval_tables(const sg_layout *L, uint32_t **prefix_base, int64_t *nprefix,
                          sg_repack **repack);

#ifdef __cplusplus
}
#endif
#endif
