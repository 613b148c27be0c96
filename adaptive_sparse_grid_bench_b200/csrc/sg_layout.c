/*
 * Host-side index algebra (C).  Follows the reference benchmark
 * adaptive_sparse_grid_bench.c: tables c:101-140 (with the limit handling of
 * the CUDA host code, adaptive_sparse_grid_bench_cuda.cu:79-102), bijection
 * c:187-279.  Also builds the per-sweep chain tables and the evaluation
 * order table that the kernels walk.
 */
#include "sg_layout.h"

#include <stdlib.h>
#include <string.h>

static int64_t block_layout_size(const sg_layout *L);

int sg_layout_init(sg_layout *L, int d, int n, const int *limits)
{
    int i, s, k;
    if (!L || d < 1 || n < 1) return SG_ERR_ARG;
    if (d > SG_MAX_DIMS || n > SG_MAX_LEVELS) return SG_ERR_RANGE;
    memset(L, 0, sizeof(*L));
    L->d = d;
    L->n = n;
    for (i = 0; i < d; i++) {
        int v = limits ? limits[i] : n - 1;
        if (v < 0) return SG_ERR_ARG;
        L->lim[i] = v > n - 1 ? n - 1 : v;
    }
    /* dp[i][s] = sum_{k <= min(s, lim_i)} dp[i-1][s-k]  (c:113-129) */
    for (s = 0; s < n; s++) L->dp[0][s] = s <= L->lim[0];
    for (i = 1; i < d; i++)
        for (s = 0; s < n; s++) {
            int64_t c = 0;
            for (k = 0; k <= s && k <= L->lim[i]; k++) c += L->dp[i - 1][s - k];
            L->dp[i][s] = c;
        }
    /* group offsets (c:132-140), compact and padded */
    L->N = L->S = L->Npad = 0;
    for (s = 0; s < n; s++) {
        int64_t sz = L->dp[d - 1][s] << s;
        L->lidx[s] = L->N;
        L->plidx[s] = L->Npad;
        L->N += sz;
        L->S += L->dp[d - 1][s];
        L->Npad += (sz + SG_GROUP_ALIGN - 1) / SG_GROUP_ALIGN * SG_GROUP_ALIGN;
    }
    L->lidx[n] = L->N;
    L->plidx[n] = L->Npad;
    /* kernels index the device grid with 32-bit offsets */
    if (L->Npad >= ((int64_t)1 << 31)) return SG_ERR_RANGE;
    L->Nblk = block_layout_size(L);
    if (L->Nblk >= ((int64_t)1 << 32) - 64) return SG_ERR_RANGE;
    return SG_OK;
}

/* c:266-279 */
int64_t sg_layout_l2idx(const sg_layout *L, const int *lv)
{
    int64_t pos = 0;
    int i, j, sum = lv[0];
    for (i = 1; i < L->d; i++) {
        sum += lv[i];
        for (j = 0; j < lv[i]; j++) pos += L->dp[i - 1][sum - j];
    }
    return pos;
}

/* c:245-264 */
void sg_layout_idx2l(const sg_layout *L, int64_t pos, int s, int *lv)
{
    int i;
    for (i = L->d - 1; i >= 1; i--) {
        int level = 0;
        while (pos >= L->dp[i - 1][s - level]) {
            pos -= L->dp[i - 1][s - level];
            level++;
        }
        lv[i] = level;
        s -= level;
    }
    lv[0] = s;
}

/* c:187-207 */
int64_t sg_layout_gp2idx(const sg_layout *L, const int *lv, const int *ix)
{
    int64_t in_sub = ix[0];
    int i, s = lv[0];
    for (i = 1; i < L->d; i++) {
        in_sub = (in_sub << lv[i]) + ix[i];
        s += lv[i];
    }
    return L->lidx[s] + (sg_layout_l2idx(L, lv) << s) + in_sub;
}

/* c:210-243 */
int sg_layout_idx2gp(const sg_layout *L, int64_t idx, int *lv, int *ix)
{
    int s = 0, i;
    int64_t rest;
    if (idx < 0 || idx >= L->N) return SG_ERR_ARG;
    while (s < L->n && idx >= L->lidx[s]) s++;
    s--;
    idx -= L->lidx[s];
    rest = idx & (((int64_t)1 << s) - 1);
    sg_layout_idx2l(L, idx >> s, s, lv);
    for (i = L->d - 1; i >= 0; i--) {
        ix[i] = (int)(rest & (((int64_t)1 << lv[i]) - 1));
        rest >>= lv[i];
    }
    return SG_OK;
}

int64_t sg_layout_subspace_offset(const sg_layout *L, const int *lv)
{
    int i, s = 0;
    for (i = 0; i < L->d; i++) s += lv[i];
    return L->plidx[s] + (sg_layout_l2idx(L, lv) << s);
}

/* Odometer over level vectors of the dims in `dims` (count m) with sum <= cap
 * and per-dim limits; calls back with the vector written into lv. */
typedef void (*lv_visit)(void *ctx, int *lv, int sum);

static void enum_levels(const sg_layout *L, const int *dims, int m, int idx, int cap,
                        int sum, int *lv, lv_visit fn, void *ctx)
{
    int l, k;
    if (idx == m) {
        fn(ctx, lv, sum);
        return;
    }
    k = dims[idx];
    for (l = 0; l <= L->lim[k] && sum + l <= cap; l++) {
        lv[k] = l;
        enum_levels(L, dims, m, idx + 1, cap, sum + l, lv, fn, ctx);
    }
    lv[k] = 0;
}

typedef struct {
    const sg_layout *L;
    int k;
    sg_chain *chains;
    int64_t nch, cap_ch;
    uint32_t *seg;
    int64_t nseg, cap_seg;
    int err;
} chain_ctx;

static void chain_visit(void *vctx, int *lv, int sigma)
{
    chain_ctx *c = (chain_ctx *)vctx;
    const sg_layout *L = c->L;
    int k = c->k, j, m, lo = 0;
    int lmax = L->n - 1 - sigma;
    if (lmax > L->lim[k]) lmax = L->lim[k];
    if (lmax < 1 || c->err) return;
    if (c->nch == c->cap_ch) {
        c->cap_ch = c->cap_ch ? 2 * c->cap_ch : 1024;
        c->chains = (sg_chain *)realloc(c->chains, (size_t)c->cap_ch * sizeof(sg_chain));
        if (!c->chains) { c->err = SG_ERR_NOMEM; return; }
    }
    while (c->nseg + lmax + 1 > c->cap_seg) {
        c->cap_seg = c->cap_seg ? 2 * c->cap_seg : 4096;
        c->seg = (uint32_t *)realloc(c->seg, (size_t)c->cap_seg * sizeof(uint32_t));
        if (!c->seg) { c->err = SG_ERR_NOMEM; return; }
    }
    for (m = k + 1; m < L->d; m++) lo += lv[m];
    c->chains[c->nch].seg = (uint32_t)c->nseg;
    c->chains[c->nch].sigma = (uint8_t)sigma;
    c->chains[c->nch].lmax = (uint8_t)lmax;
    c->chains[c->nch].lo = (uint8_t)lo;
    c->chains[c->nch].pad = 0;
    c->nch++;
    for (j = 0; j <= lmax; j++) {
        lv[k] = j;
        c->seg[c->nseg++] = (uint32_t)sg_layout_subspace_offset(L, lv);
    }
    lv[k] = 0;
}

static int chain_size_cmp(const void *a, const void *b)
{
    const sg_chain *x = (const sg_chain *)a, *y = (const sg_chain *)b;
    /* size = 2^sigma * (2^(lmax+1) - 1); compare exactly */
    int64_t sx = ((int64_t)1 << x->sigma) * (((int64_t)2 << x->lmax) - 1);
    int64_t sy = ((int64_t)1 << y->sigma) * (((int64_t)2 << y->lmax) - 1);
    if (sx != sy) return sx > sy ? -1 : 1;
    return x->seg < y->seg ? -1 : (x->seg > y->seg);
}

int sg_layout_chains(const sg_layout *L, int k, sg_chain **chains, int64_t *nchains,
                     uint32_t **seg_off, int64_t *nseg)
{
    int dims[SG_MAX_DIMS], lv[SG_MAX_DIMS], m = 0, i;
    chain_ctx c;
    memset(&c, 0, sizeof(c));
    memset(lv, 0, sizeof(lv));
    c.L = L;
    c.k = k;
    for (i = 0; i < L->d; i++)
        if (i != k) dims[m++] = i;
    enum_levels(L, dims, m, 0, L->n - 1, 0, lv, chain_visit, &c);
    if (c.err) {
        free(c.chains);
        free(c.seg);
        return c.err;
    }
    if (c.nch > 1) qsort(c.chains, (size_t)c.nch, sizeof(sg_chain), chain_size_cmp);
    *chains = c.chains;
    *nchains = c.nch;
    *seg_off = c.seg;
    *nseg = c.nseg;
    return SG_OK;
}

/* ---- evaluation (block) layout ------------------------------------------ */

static int lim_of(const sg_layout *L, int k) { return k >= 0 ? L->lim[k] : 0; }

void sg_layout_eval_sub(const sg_layout *L, int r, sg_eval_sub *sh)
{
    const int limA = lim_of(L, L->d - 2), limB = L->lim[L->d - 1];
    int a;
    uint32_t off = 0;
    memset(sh, 0, sizeof(*sh));
    sh->amax = r < limA ? r : limA;
    for (a = 0; a <= sh->amax; a++) {
        int rl = r - a < limB ? r - a : limB;
        sh->rowlen[a] = rl + 1;
        sh->aoff[a] = off;
        /* 2^a poles of 2^rl paths of rl+1 slots */
        off += ((uint32_t)1 << a) * (((uint32_t)1 << rl) * (uint32_t)SG_PATH_WIDTH(rl + 1));
    }
    sh->aoff[sh->amax + 1] = off;
}

void sg_layout_eval_shape(const sg_layout *L, int R, sg_eval_shape *sh)
{
    const int limC = lim_of(L, L->d - 3);
    int c;
    uint32_t off = 0;
    memset(sh, 0, sizeof(*sh));
    sh->R = R;
    sh->cmax = R < limC ? R : limC;
    for (c = 0; c <= sh->cmax; c++) {
        sg_eval_sub sub;
        sg_layout_eval_sub(L, R - c, &sub);
        sh->coff[c] = off;
        off += ((uint32_t)1 << c) * sub.aoff[sub.amax + 1];
    }
    sh->coff[sh->cmax + 1] = off;
}

/* Values of the block layout: every prefix level vector's cells times the
 * block size of its remaining budget. */
static int64_t block_layout_size(const sg_layout *L)
{
    const int np_dims = L->d >= 3 ? L->d - 3 : 0;
    int64_t sz[SG_MAX_DIMS + 1][SG_MAX_LEVELS];
    int k, R;
    for (R = 0; R < L->n; R++) {
        sg_eval_shape sh;
        sg_layout_eval_shape(L, R, &sh);
        sz[np_dims][R] = sh.coff[sh.cmax + 1];
    }
    for (k = np_dims - 1; k >= 0; k--)
        for (R = 0; R < L->n; R++) {
            int l;
            int64_t w = 0;
            for (l = 0; l <= R && l <= L->lim[k]; l++) w += sz[k + 1][R - l] << l;
            sz[k][R] = w;
        }
    return sz[0][L->n - 1];
}

int sg_layout_eval_tables(const sg_layout *L, sg_repack **repack, uint32_t *blk3, uint32_t *blk2)
{
    const int d = L->d;
    const int np_dims = d >= 3 ? d - 3 : 0; /* dims 0..d-4 form the prefix */
    int lv[SG_MAX_DIMS], k, s, R;
    int64_t pos, r = 0;
    /* cnt[k][R]: level vectors over prefix dims k..np_dims-1 with sum <= R;
     * sz[k][R]: total block-layout size of their blocks (all cells) */
    int64_t cnt[SG_MAX_DIMS + 1][SG_MAX_LEVELS], sz[SG_MAX_DIMS + 1][SG_MAX_LEVELS];
    sg_repack *rp;
    for (R = 0; R < L->n; R++) {
        sg_eval_shape sh;
        sg_eval_sub sub;
        sg_layout_eval_shape(L, R, &sh);
        sg_layout_eval_sub(L, R, &sub);
        blk3[R] = sh.coff[sh.cmax + 1];
        blk2[R] = sub.aoff[sub.amax + 1];
        cnt[np_dims][R] = 1;
        sz[np_dims][R] = blk3[R];
    }
    for (k = np_dims - 1; k >= 0; k--)
        for (R = 0; R < L->n; R++) {
            int l;
            int64_t v = 0, w = 0;
            for (l = 0; l <= R && l <= L->lim[k]; l++) {
                v += cnt[k + 1][R - l];
                w += sz[k + 1][R - l] << l; /* 2^l cells of this dim */
            }
            cnt[k][R] = v;
            sz[k][R] = w;
        }
    if (sz[0][L->n - 1] != L->Nblk) return SG_ERR_STATE;
    rp = (sg_repack *)malloc((size_t)(L->S > 0 ? L->S : 1) * sizeof(sg_repack));
    if (!rp) return SG_ERR_NOMEM;
    memset(lv, 0, sizeof(lv));
    for (s = 0; s < L->n; s++)
        for (pos = 0; pos < L->dp[d - 1][s]; pos++) {
            int c, a, b, rem = L->n - 1, sigma = 0;
            int64_t base = 0, scale = 1;
            sg_eval_shape sh;
            sg_eval_sub sub;
            sg_layout_idx2l(L, pos, s, lv);
            /* block-layout start of this prefix: the sizes of all prefixes
             * that precede it in the depth-first walk */
            for (k = 0; k < np_dims; k++) {
                int l;
                for (l = 0; l < lv[k]; l++) base += (sz[k + 1][rem - l] << l) * scale;
                scale <<= lv[k];
                rem -= lv[k];
                sigma += lv[k];
            }
            c = d >= 3 ? lv[d - 3] : 0;
            a = d >= 2 ? lv[d - 2] : 0;
            b = lv[d - 1];
            sg_layout_eval_shape(L, L->n - 1 - sigma, &sh);
            sg_layout_eval_sub(L, L->n - 1 - sigma - c, &sub);
            rp[r].src = (uint32_t)(L->plidx[s] + (pos << s));
            rp[r].dst = (uint32_t)base + sh.coff[c] + sub.aoff[a] + (uint32_t)b;
            rp[r].blk = sh.coff[sh.cmax + 1];
            rp[r].sub = sub.aoff[sub.amax + 1];
            rp[r].plen = ((uint32_t)1 << (sub.rowlen[a] - 1)) * (uint32_t)SG_PATH_WIDTH(sub.rowlen[a]);
            rp[r].L = (uint8_t)(sub.rowlen[a] - 1);
            rp[r].pad[0] = rp[r].pad[1] = rp[r].pad[2] = 0;
            rp[r].c = (uint8_t)c;
            rp[r].a = (uint8_t)a;
            rp[r].b = (uint8_t)b;
            rp[r].s = (uint8_t)s;
            r++;
        }
    *repack = rp;
    return SG_OK;
}

/* ---- walk tables and split evaluation ----------------------------------- */

int sg_layout_walk_tables(const sg_layout *L, const uint32_t *blk3, uint32_t *walk)
{
    const int d = L->d, n = L->n;
    int K, b, l;
    if (d < 4) return SG_ERR_ARG;
    for (b = 0; b < n; b++) {
        walk[2 * ((d - 3) * n + b)] = 1;
        walk[2 * ((d - 3) * n + b) + 1] = blk3[b] << (n - 1 - b);
    }
    for (K = d - 4; K >= 0; K--)
        for (b = 0; b < n; b++) {
            uint64_t cnt = 0, ext = 0;
            for (l = 0; l <= b && l <= L->lim[K]; l++) {
                cnt += walk[2 * ((K + 1) * n + b - l)];
                ext += walk[2 * ((K + 1) * n + b - l) + 1];
            }
            walk[2 * (K * n + b)] = (uint32_t)cnt;
            walk[2 * (K * n + b) + 1] = (uint32_t)ext;
        }
    return SG_OK;
}

/* subspaces (c, a, b) of the innermost dims with c + a + b <= R, in limits */
static double block_subspaces(const sg_layout *L, int R)
{
    const int lc = L->lim[L->d - 3], la = L->lim[L->d - 2], lb = L->lim[L->d - 1];
    double cnt = 0.0;
    int c, a;
    for (c = 0; c <= R && c <= lc; c++)
        for (a = 0; a <= R - c && a <= la; a++) cnt += (R - c - a < lb ? R - c - a : lb) + 1;
    return cnt;
}

#define SG_BLOCK_OVERHEAD 3.0 /* per-block walk cost in subspace-equivalents */

int sg_layout_walk_split(const sg_layout *L, int nparts, uint32_t *bounds)
{
    const int d = L->d, n = L->n;
    double *W;
    uint32_t *cnt;
    int K, b, l, j;
    if (d < 4 || nparts < 1) return SG_ERR_ARG;
    W = (double *)malloc(sizeof(double) * (size_t)(d - 2) * (size_t)n);
    cnt = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(d - 2) * (size_t)n);
    if (!W || !cnt) {
        free(W);
        free(cnt);
        return SG_ERR_NOMEM;
    }
    for (b = 0; b < n; b++) {
        W[(d - 3) * n + b] = block_subspaces(L, b) + SG_BLOCK_OVERHEAD;
        cnt[(d - 3) * n + b] = 1;
    }
    for (K = d - 4; K >= 0; K--)
        for (b = 0; b < n; b++) {
            double w = 0.0;
            uint64_t c = 0;
            for (l = 0; l <= b && l <= L->lim[K]; l++) {
                w += W[(K + 1) * n + b - l];
                c += cnt[(K + 1) * n + b - l];
            }
            W[K * n + b] = w;
            cnt[K * n + b] = (uint32_t)c;
        }
    bounds[0] = 0;
    bounds[nparts] = cnt[n - 1];
    for (j = 1; j < nparts; j++) {
        /* descend to the block holding work position j/nparts of the total */
        const double t = W[n - 1] * j / nparts;
        double acc = 0.0;
        uint32_t leaf = 0;
        K = 0;
        b = n - 1;
        while (K < d - 3) {
            const int lmax = b < L->lim[K] ? b : L->lim[K];
            for (l = 0; l <= lmax; l++) {
                const double w = W[(K + 1) * n + b - l];
                if (acc + w > t) break;
                acc += w;
                leaf += cnt[(K + 1) * n + b - l];
            }
            if (l > lmax) break; /* rounding: t at the very end */
            K++;
            b -= l;
        }
        bounds[j] = leaf < bounds[j - 1] ? bounds[j - 1] : leaf;
        if (bounds[j] > bounds[nparts]) bounds[j] = bounds[nparts];
    }
    free(W);
    free(cnt);
    return SG_OK;
}
