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
    int64_t Nblk; /* values of the evaluation (block) layout */
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
 * evaluation walk.  Dims 0..d-4 form the prefix; the three innermost dims are
 * C = d-3, A = d-2, B = d-1 (for d < 3 the missing leading ones are treated
 * as dims with limit 0).  For every prefix level vector p (depth-first
 * order, level ascending) and every cell I of p (row-major over the prefix
 * dims) one block holds all subspaces (p, c, a, b) below the level budget
 * R = n-1-|p|:
 *   planes c = 0..cmax, each 2^c sub-blocks (one per cell t_c of dim C);
 *   a sub-block of budget r = R-c has rows a = 0..amax(r), each 2^a poles
 *   (one per cell t_a of dim A);
 *   a pole holds dim B's levels b = 0..L (L = rowlen-1) as 2^L paths, one
 *   per finest cell t_L: path t_L is the L+1 surpluses a query point in that
 *   cell needs, level b's cell t_L >> (L-b) in slot b, in W = L+1 rounded up
 *   to even slots (SG_PATH_WIDTH).  A surplus of level b therefore appears
 *   in 2^(L-b) paths (Nblk >= N values in all).
 * A query point finds the surplus of (c, a, b) at
 *   base + coff(c) + t_c * sub(R-c) + aoff(R-c, a) + t_a * plen + t_L * W + b,
 * so the loads of a row share one address and differ by a constant; every
 * row with L >= 1 starts at an even offset (all sizes before it in a block
 * are even), so slots 2j, 2j+1 move with one 8-byte load.
 */
/* Slots of a path of `levels` levels: rounded up to an even count (two
 * levels per 8-byte load), a single level alone. */
#define SG_PATH_WIDTH(levels) ((levels) <= 1 ? (levels) : (((levels) + 1) & ~1))

typedef struct sg_eval_sub {
    int amax;                         /* last row: min(r, lim_A)           */
    int rowlen[SG_MAX_LEVELS];        /* levels of dim B in row a           */
    uint32_t aoff[SG_MAX_LEVELS + 1]; /* row starts; aoff[amax+1] = size    */
} sg_eval_sub;

typedef struct sg_eval_shape {
    int R, cmax;                      /* budget, last plane min(R, lim_C)   */
    uint32_t coff[SG_MAX_LEVELS + 1]; /* plane starts; coff[cmax+1] = size  */
} sg_eval_shape;

void sg_layout_eval_sub(const sg_layout *L, int r, sg_eval_sub *sh);
void sg_layout_eval_shape(const sg_layout *L, int R, sg_eval_shape *sh);

/* Walk tables of the evaluation (d >= 4; the walk visits prefix dims
 * 0..d-4, blocks sit at depth d-3).  For depth K = 0..d-3 and budget
 * b = 0..n-1: walk[2*(K*n + b)] = number of blocks of the subtree entered at
 * depth K with budget b, walk[2*(K*n + b) + 1] = their extent in the block
 * layout (sum of blk3[R] << (n-1-R)).  walk has 2*(d-2)*n entries. */
int sg_layout_walk_tables(const sg_layout *L, const uint32_t *blk3, uint32_t *walk);
/* bounds[0..nparts]: block ranges of the walk with about equal work each
 * (subspaces per block plus a per-block overhead); d >= 4. */
int sg_layout_walk_split(const sg_layout *L, int nparts, uint32_t *bounds);

/* Per-subspace repack descriptor (compact layout -> block layout). */
typedef struct sg_repack {
    uint32_t src;  /* device offset of the subspace in the group-aligned layout */
    uint32_t dst;  /* block-layout offset of its element with I = t = 0 (slot b) */
    uint32_t blk;  /* block size: stride of the prefix cell I                   */
    uint32_t sub;  /* sub-block size: stride of t_c                             */
    uint32_t plen; /* pole length: stride of t_a                                */
    uint8_t c, a, b, s;
    uint8_t L;     /* last level of dim B in the row: paths of L+1 slots        */
    uint8_t pad[3];
} sg_repack;

/* The repack table (one entry per subspace, malloc'd) and the block sizes
 * blk3[R] (3-D block) and blk2[r] (sub-block) for every budget. */
int sg_layout_eval_tables(const sg_layout *L, sg_repack **repack, uint32_t *blk3, uint32_t *blk2);

#ifdef __cplusplus
}
#endif
#endif
