/*
 * Batches of independent grids (sg_batch_* in include/sgrid.h).  Host code in
 * C.  A batch holds many grids of mixed d, n and limits in one device buffer
 * (each grid in the group-aligned compact layout, 32-element aligned), and
 * runs all of them through a fixed set of launches:
 *   hierarchize: grids that fit in shared memory (n <= 9, <= 200 KB) are
 *     hierarchized whole, one CTA per grid, in a few size classes; the
 *     others share one chain-sweep launch per sweep index k across grids
 *     (sweeps of different grids are independent);
 *   evaluate: the surpluses are repacked into the block layout by one launch
 *     over all subspaces of all grids, then one evaluation launch per
 *     distinct d covers every grid of that d, 256*ppt points per CTA.
 * Both sequences can be captured once in a CUDA graph and replayed.
 */
#include <cuda_runtime_api.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sg_batch_internal.h"
#include "sg_kernels.h"
#include "sg_layout.h"

#define SG_API __attribute__((visibility("default")))

/* values per sweep group (SG_OPT_SWEEP_GROUP): measured on 4096 mixed grids
 * (5.1e8 values), smaller groups lose more to launch latency than they
 * gain from L2 */
#define SG_SWEEP_GROUP_DEFAULT (1 << 23)

/* size classes of the shared-memory path (bytes of the larger of FP32/FP64) */
static const int64_t k_class_bytes[SG_BATCH_CLASSES] = {8 * 1024, 32 * 1024, 96 * 1024, SG_SMEM_GRID_MAX_BYTES};

static int bfail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    sg_set_error(fmt, ap);
    va_end(ap);
    return code;
}

static int bcuda(cudaError_t e, const char *what)
{
    return bfail(SG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define BCU(call, what)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return bcuda(e_, what);    \
    } while (0)

SG_API int sg_batch_create(int num_grids, const int *dims, const int *levels, const int *limits,
                           sg_batch **out)
{
    sg_batch *b;
    int g, r;
    int64_t lim_at = 0, doff = 0, voff = 0, boff = 0;
    if (!out || num_grids < 1 || num_grids >= (1 << 29) || !dims || !levels)
        return bfail(SG_ERR_ARG, "sg_batch_create: bad argument");
    *out = NULL;
    b = (sg_batch *)calloc(1, sizeof(sg_batch));
    if (!b) return bfail(SG_ERR_NOMEM, "sg_batch_create: out of host memory");
    b->ng = num_grids;
    b->L = (sg_layout *)calloc((size_t)num_grids, sizeof(sg_layout));
    b->voff = (int64_t *)calloc((size_t)num_grids + 1, sizeof(int64_t));
    b->doff = (int64_t *)calloc((size_t)num_grids + 1, sizeof(int64_t));
    b->boff = (int64_t *)calloc((size_t)num_grids + 1, sizeof(int64_t));
    if (!b->L || !b->voff || !b->doff || !b->boff) {
        sg_batch_destroy(b);
        return bfail(SG_ERR_NOMEM, "sg_batch_create: out of host memory");
    }
    for (g = 0; g < num_grids; g++) {
        r = sg_layout_init(&b->L[g], dims[g], levels[g], limits ? limits + lim_at : NULL);
        if (r != SG_OK) {
            sg_batch_destroy(b);
            return bfail(r, "sg_batch_create: grid %d (d=%d n=%d) rejected", g, dims[g], levels[g]);
        }
        lim_at += dims[g];
        b->voff[g] = voff;
        b->doff[g] = doff;
        b->boff[g] = boff;
        voff += b->L[g].N;
        doff += b->L[g].Npad;
        boff += (b->L[g].Nblk + 1) & ~(int64_t)1; /* grids start even: 8-byte path loads */
    }
    b->voff[num_grids] = voff;
    b->doff[num_grids] = doff;
    b->boff[num_grids] = boff;
    if (boff >= ((int64_t)1 << 32) - 64) {
        sg_batch_destroy(b);
        return bfail(SG_ERR_RANGE, "sg_batch_create: %lld evaluation-layout values exceed 32-bit offsets",
                     (long long)boff);
    }
    if (doff >= ((int64_t)1 << 32) - 64) {
        sg_batch_destroy(b);
        return bfail(SG_ERR_RANGE, "sg_batch_create: %lld values exceed 32-bit offsets", (long long)doff);
    }
    b->dev = -1;
    b->ppt = 2;
    b->precision = SG_HIER_FP32;
    b->use_graph = 1;
    b->sort = 1;
    b->sweep_group = SG_SWEEP_GROUP_DEFAULT;
    *out = b;
    return SG_OK;
}

static void free_dev(sg_batch *b)
{
    int k;
    if (b->dev < 0) return;
    cudaSetDevice(b->dev);
    if (b->hier_graph) cudaGraphExecDestroy(b->hier_graph);
    if (b->eval_graph) cudaGraphExecDestroy(b->eval_graph);
    b->hier_graph = b->eval_graph = NULL;
    cudaFree(b->d_alpha);
    cudaFree(b->d_work);
    cudaFree(b->d_blk);
    cudaFree(b->d_repack);
    cudaFree(b->d_smem_grids);
    cudaFree(b->d_smem_chains);
    cudaFree(b->d_smem_seg);
    for (k = 0; k < SG_MAX_DIMS; k++) {
        cudaFree(b->d_chB[k]);
        cudaFree(b->d_segB[k]);
        b->d_chB[k] = NULL;
        b->d_segB[k] = NULL;
    }
    free(b->sweepG);
    b->sweepG = NULL;
    b->ngroups = 0;
    cudaFree(b->d_sgrids);
    cudaFree(b->d_sitems);
    cudaFree(b->d_sscratch);
    cudaFree(b->d_sorted);
    cudaFree(b->d_perm);
    b->d_sgrids = NULL;
    b->d_sitems = NULL;
    b->d_sscratch = NULL;
    b->d_sorted = NULL;
    b->d_perm = NULL;
    cudaFree(b->d_eval_args);
    cudaFree(b->d_items);
    cudaFree(b->d_err);
    cudaFree(b->d_segs);
    cudaFree(b->d_stage);
    free(b->h_eval_args);
    free(b->h_items);
    b->h_eval_args = NULL;
    b->h_items = NULL;
    for (k = 0; k <= SG_MAX_DIMS; k++) {
        if (b->dst[k]) cudaStreamDestroy(b->dst[k]);
        if (b->ev_d[k]) cudaEventDestroy(b->ev_d[k]);
        b->dst[k] = NULL;
        b->ev_d[k] = NULL;
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    b->ev_fork = NULL;
}

SG_API int sg_batch_destroy(sg_batch *b)
{
    if (!b) return SG_OK;
    free_dev(b);
    free(b->L);
    free(b->voff);
    free(b->doff);
    free(b->boff);
    free(b->eval_pt_off);
    free(b->order);
    free(b);
    return SG_OK;
}

SG_API int sg_batch_offsets(const sg_batch *b, int64_t *value_offsets)
{
    int g;
    if (!b || !value_offsets) return bfail(SG_ERR_ARG, "sg_batch_offsets: NULL argument");
    for (g = 0; g <= b->ng; g++) value_offsets[g] = b->voff[g];
    return SG_OK;
}

SG_API int sg_batch_num_grids(const sg_batch *b, int *num_grids)
{
    if (!b || !num_grids) return bfail(SG_ERR_ARG, "sg_batch_num_grids: NULL argument");
    *num_grids = b->ng;
    return SG_OK;
}

static int balloc(sg_batch *b, void **p, int64_t bytes, const char *what)
{
    cudaError_t e = cudaMalloc(p, (size_t)(bytes > 0 ? bytes : 16));
    if (e != cudaSuccess) {
        *p = NULL;
        cudaGetLastError();
        return bfail(e == cudaErrorMemoryAllocation ? SG_ERR_NOMEM : SG_ERR_CUDA, "cudaMalloc(%lld) for %s: %s",
                     (long long)bytes, what, cudaGetErrorString(e));
    }
    b->dev_bytes += bytes;
    return SG_OK;
}

static int upload(sg_batch *b, void **dst, const void *src, int64_t bytes, const char *what)
{
    int r = balloc(b, dst, bytes, what);
    if (r != SG_OK) return r;
    if (bytes > 0) BCU(cudaMemcpy(*dst, src, (size_t)bytes, cudaMemcpyHostToDevice), what);
    return SG_OK;
}

static int make_fork_streams(sg_batch *b);

/* shared-memory elements one chain needs (segments padded to 16 bytes) */
static int64_t chain_elems(const sg_chain *c, int elem_bytes)
{
    const int64_t minsz = 16 / elem_bytes;
    int64_t e = 0;
    int j;
    for (j = 0; j <= c->lmax; j++) {
        const int64_t sz = (int64_t)1 << (c->sigma + j);
        e += sz < minsz ? minsz : sz;
    }
    return e;
}

static int cmp_chain_desc(const void *x, const void *y)
{
    const int64_t a = chain_elems((const sg_chain *)x, 4), c = chain_elems((const sg_chain *)y, 4);
    if (a != c) return a > c ? -1 : 1;
    return ((const sg_chain *)x)->seg < ((const sg_chain *)y)->seg ? -1 : 1;
}

/* grids that take the shared-memory path, and their size class */
static int smem_class(const sg_layout *L)
{
    int c;
    const int64_t bytes = L->Npad * 8; /* sized for FP64 so both precisions fit */
    if (L->n > 9) return -1;
    for (c = 0; c < SG_BATCH_CLASSES; c++)
        if (bytes <= k_class_bytes[c]) return c;
    return -1;
}

static int cmp_by_size_desc(const void *x, const void *y, void *ctx)
{
    const sg_batch *b = (const sg_batch *)ctx;
    const int gx = *(const int *)x, gy = *(const int *)y;
    if (b->L[gx].Npad != b->L[gy].Npad) return b->L[gx].Npad > b->L[gy].Npad ? -1 : 1;
    return gx - gy;
}

static int materialize(sg_batch *b)
{
    int g, k, c, r = SG_OK;
    int *order = NULL;
    sg_smem_grid *sg = NULL;
    sg_chain *sch = NULL;
    uint32_t *sseg = NULL;
    int64_t nsg = 0, nsch = 0, nsseg = 0, cap_sch = 0, cap_sseg = 0;
    sg_chain *chB[SG_MAX_DIMS];
    uint32_t *segB[SG_MAX_DIMS];
    int64_t nchB[SG_MAX_DIMS], nsegB[SG_MAX_DIMS], capchB[SG_MAX_DIMS], capsegB[SG_MAX_DIMS];
    sg_repack *rp = NULL;
    int64_t nrp = 0;
    int64_t (*gfirst)[SG_MAX_DIMS] = NULL; /* first chain of each sweep group per sweep, ngroups+1 rows */
    int ngr = 0, capgr = 0, q;
    int64_t gacc = 0;
    if (b->dev >= 0) return SG_OK;
    memset(chB, 0, sizeof(chB));
    memset(segB, 0, sizeof(segB));
    memset(nchB, 0, sizeof(nchB));
    memset(nsegB, 0, sizeof(nsegB));
    memset(capchB, 0, sizeof(capchB));
    memset(capsegB, 0, sizeof(capsegB));
    BCU((cudaError_t)sgk_eval_setup(), "evaluation kernel set-up");
    BCU(cudaGetDevice(&b->dev), "cudaGetDevice");
    if ((r = balloc(b, (void **)&b->d_alpha, b->doff[b->ng] * 4, "batch values")) != SG_OK) goto done;
    BCU(cudaMemset(b->d_alpha, 0, (size_t)b->doff[b->ng] * 4), "cudaMemset");
    if ((r = balloc(b, (void **)&b->d_blk, b->boff[b->ng] * 4, "batch block layout")) != SG_OK) goto done;
    if ((r = balloc(b, (void **)&b->d_err, 16, "error flag")) != SG_OK) goto done;
    BCU(cudaMemset(b->d_err, 0, 16), "cudaMemset");

    /* level-group runs for moving values in one launch, cut into pieces of
     * at most SG_COPY_PIECE values so that one CTA's share stays bounded */
    {
        int64_t ns = 0;
        sg_copy_seg *segs;
        for (g = 0; g < b->ng; g++) ns += b->L[g].n + b->L[g].N / SG_COPY_PIECE;
        segs = (sg_copy_seg *)malloc((size_t)ns * sizeof(sg_copy_seg));
        if (!segs) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
        ns = 0;
        for (g = 0; g < b->ng; g++) {
            int s;
            const sg_layout *L = &b->L[g];
            for (s = 0; s < L->n; s++) {
                int64_t at;
                for (at = L->lidx[s]; at < L->lidx[s + 1]; at += SG_COPY_PIECE) {
                    const int64_t left = L->lidx[s + 1] - at;
                    segs[ns].compact = b->voff[g] + at;
                    segs[ns].dev = b->doff[g] + L->plidx[s] + (at - L->lidx[s]);
                    segs[ns].count = left < SG_COPY_PIECE ? left : SG_COPY_PIECE;
                    ns++;
                }
            }
        }
        b->nsegs = ns;
        r = upload(b, (void **)&b->d_segs, segs, ns * (int64_t)sizeof(sg_copy_seg), "batch value runs");
        free(segs);
        if (r != SG_OK) goto done;
    }

    /* shared-memory path: grids in size classes, largest first inside each */
    order = (int *)malloc((size_t)b->ng * sizeof(int));
    sg = (sg_smem_grid *)calloc((size_t)b->ng, sizeof(sg_smem_grid));
    if (!order || !sg) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
    for (g = 0; g < b->ng; g++) order[g] = g;
    qsort_r(order, (size_t)b->ng, sizeof(int), cmp_by_size_desc, b);
    for (c = SG_BATCH_CLASSES - 1; c >= 0; c--) {
        b->cls_first[c] = (int)nsg;
        b->cls_max_npad[c] = 0;
        for (int q = 0; q < b->ng; q++) {
            const int gg = order[q];
            const sg_layout *L = &b->L[gg];
            if (smem_class(L) != c) continue;
            sg[nsg].base = (uint32_t)b->doff[gg];
            sg[nsg].npad = (uint32_t)L->Npad;
            sg[nsg].d = L->d;
            if ((int)L->Npad > b->cls_max_npad[c]) b->cls_max_npad[c] = (int)L->Npad;
            for (k = 0; k < L->d; k++) {
                sg_chain *ch = NULL;
                uint32_t *sgo = NULL;
                int64_t nch = 0, nseg = 0, i;
                if ((r = sg_layout_chains(L, k, &ch, &nch, &sgo, &nseg)) != SG_OK) goto done;
                while (nsch + nch > cap_sch) {
                    cap_sch = cap_sch ? 2 * cap_sch : 4096;
                    sch = (sg_chain *)realloc(sch, (size_t)cap_sch * sizeof(sg_chain));
                }
                while (nsseg + nseg > cap_sseg) {
                    cap_sseg = cap_sseg ? 2 * cap_sseg : 16384;
                    sseg = (uint32_t *)realloc(sseg, (size_t)cap_sseg * sizeof(uint32_t));
                }
                if (!sch || !sseg) { free(ch); free(sgo); r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
                sg[nsg].chain0[k] = (uint32_t)nsch;
                sg[nsg].nch[k] = (uint32_t)nch;
                for (i = 0; i < nch; i++) {
                    sch[nsch + i] = ch[i];
                    sch[nsch + i].seg = (uint32_t)(ch[i].seg + nsseg);
                }
                /* offsets relative to the grid: the shared-memory copy of a
                 * grid has its device layout */
                for (i = 0; i < nseg; i++) sseg[nsseg + i] = sgo[i];
                nsch += nch;
                nsseg += nseg;
                free(ch);
                free(sgo);
            }
            nsg++;
        }
        b->cls_count[c] = (int)nsg - b->cls_first[c];
    }
    b->n_smem = (int)nsg;
    if ((r = upload(b, (void **)&b->d_smem_grids, sg, nsg * (int64_t)sizeof(sg_smem_grid), "batch grid table")) != SG_OK) goto done;
    if ((r = upload(b, (void **)&b->d_smem_chains, sch, nsch * (int64_t)sizeof(sg_chain), "batch chains")) != SG_OK) goto done;
    if ((r = upload(b, (void **)&b->d_smem_seg, sseg, nsseg * 4, "batch segments")) != SG_OK) goto done;

    /* chain-sweep path: the other grids, in sweep groups of consecutive
     * grids; sweep k of every grid of a group in one launch per class */
    for (g = 0; g < b->ng; g++) {
        const sg_layout *L = &b->L[g];
        if (smem_class(L) >= 0) continue;
        b->has_sweep_grids = 1;
        if (ngr == 0 || (b->sweep_group > 0 && gacc > 0 && gacc + L->Npad > b->sweep_group)) {
            if (ngr + 1 >= capgr) {
                void *ng2;
                capgr = capgr ? 2 * capgr : 64;
                ng2 = realloc(gfirst, (size_t)capgr * sizeof(*gfirst));
                if (!ng2) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
                gfirst = (int64_t(*)[SG_MAX_DIMS])ng2;
            }
            for (k = 0; k < SG_MAX_DIMS; k++) gfirst[ngr][k] = nchB[k];
            ngr++;
            gacc = 0;
        }
        gacc += L->Npad;
        for (k = 0; k < L->d; k++) {
            sg_chain *ch = NULL;
            uint32_t *sgo = NULL;
            int64_t nch = 0, nseg = 0, i;
            if ((r = sg_layout_chains(L, k, &ch, &nch, &sgo, &nseg)) != SG_OK) goto done;
            while (nchB[k] + nch > capchB[k]) {
                capchB[k] = capchB[k] ? 2 * capchB[k] : 4096;
                chB[k] = (sg_chain *)realloc(chB[k], (size_t)capchB[k] * sizeof(sg_chain));
            }
            while (nsegB[k] + nseg > capsegB[k]) {
                capsegB[k] = capsegB[k] ? 2 * capsegB[k] : 16384;
                segB[k] = (uint32_t *)realloc(segB[k], (size_t)capsegB[k] * sizeof(uint32_t));
            }
            if (!chB[k] || !segB[k]) { free(ch); free(sgo); r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
            for (i = 0; i < nch; i++) {
                chB[k][nchB[k] + i] = ch[i];
                chB[k][nchB[k] + i].seg = (uint32_t)(ch[i].seg + nsegB[k]);
            }
            for (i = 0; i < nseg; i++) segB[k][nsegB[k] + i] = (uint32_t)(sgo[i] + b->doff[g]);
            nchB[k] += nch;
            nsegB[k] += nseg;
            free(ch);
            free(sgo);
        }
    }
    if (ngr == 0) ngr = 1; /* no sweep grids: one empty group */
    if (!gfirst) {
        gfirst = (int64_t(*)[SG_MAX_DIMS])calloc(2, sizeof(*gfirst));
        if (!gfirst) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
    }
    for (k = 0; k < SG_MAX_DIMS; k++) gfirst[ngr][k] = nchB[k];
    b->ngroups = ngr;
    b->sweepG = (sg_sweep_tables *)calloc((size_t)ngr * SG_MAX_DIMS * SG_SWEEP_CLASSES, sizeof(sg_sweep_tables));
    if (!b->sweepG) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
    for (k = 0; k < SG_MAX_DIMS; k++) {
        if ((r = upload(b, (void **)&b->d_segB[k], segB[k], nsegB[k] * 4, "sweep segments")) != SG_OK) goto done;
        /* per group: largest chains first, then split by the CTA size they
         * need (the chains of a group are contiguous: its grids are) */
        for (q = 0; q < ngr; q++) {
            const int64_t lo = gfirst[q][k], cnt = gfirst[q + 1][k] - gfirst[q][k];
            if (cnt > 1) qsort(chB[k] + lo, (size_t)cnt, sizeof(sg_chain), cmp_chain_desc);
        }
        if ((r = upload(b, (void **)&b->d_chB[k], chB[k], nchB[k] * (int64_t)sizeof(sg_chain), "sweep chains")) != SG_OK)
            goto done;
        for (q = 0; q < ngr; q++) {
            int64_t i, first[SG_SWEEP_CLASSES + 1];
            int cls;
            const int64_t lo = gfirst[q][k], hi_q = gfirst[q + 1][k];
            /* classes are contiguous (sorted by size): count, then prefix sums */
            for (cls = 0; cls <= SG_SWEEP_CLASSES; cls++) first[cls] = lo;
            for (i = lo; i < hi_q; i++) {
                const int64_t e32 = chain_elems(&chB[k][i], 4);
                first[1 + (e32 > 256 * 12 ? 0 : (e32 > 128 * 12 ? 1 : 2))]++;
            }
            for (cls = 1; cls <= SG_SWEEP_CLASSES; cls++) first[cls] += first[cls - 1] - lo;
            for (cls = 0; cls < SG_SWEEP_CLASSES; cls++) {
                sg_sweep_tables *t = &b->sweepG[((int64_t)q * SG_MAX_DIMS + k) * SG_SWEEP_CLASSES + cls];
                const int64_t hi = cls + 1 < SG_SWEEP_CLASSES ? first[cls + 1] : hi_q;
                t->chains = b->d_chB[k] + first[cls];
                t->seg = b->d_segB[k];
                t->nchains = hi - first[cls];
                t->cap32 = t->cap64 = 0;
                t->lmax_max = 0;
                for (i = first[cls]; i < hi; i++) {
                    const int64_t e32 = chain_elems(&chB[k][i], 4), e64 = chain_elems(&chB[k][i], 8);
                    if (e32 > t->cap32) t->cap32 = e32;
                    if (e64 > t->cap64) t->cap64 = e64;
                    if (chB[k][i].lmax > t->lmax_max) t->lmax_max = chB[k][i].lmax;
                }
            }
        }
    }

    /* evaluation: repack table over all grids, per-grid block sizes */
    for (g = 0; g < b->ng; g++) nrp += b->L[g].S;
    rp = (sg_repack *)malloc((size_t)nrp * sizeof(sg_repack));
    if (!rp) { r = bfail(SG_ERR_NOMEM, "out of host memory"); goto done; }
    nrp = 0;
    for (g = 0; g < b->ng; g++) {
        sg_repack *one = NULL;
        uint32_t blk3[SG_MAX_LEVELS], blk2[SG_MAX_LEVELS];
        int64_t i;
        if ((r = sg_layout_eval_tables(&b->L[g], &one, blk3, blk2)) != SG_OK) goto done;
        for (i = 0; i < b->L[g].S; i++) {
            rp[nrp + i] = one[i];
            rp[nrp + i].src = (uint32_t)(one[i].src + b->doff[g]);
            rp[nrp + i].dst = (uint32_t)(one[i].dst + b->boff[g]);
        }
        nrp += b->L[g].S;
        free(one);
    }
    b->nrepack = nrp;
    r = upload(b, (void **)&b->d_repack, rp, nrp * (int64_t)sizeof(sg_repack), "batch repack table");
done:
    free(gfirst);
    free(order);
    free(sg);
    free(sch);
    free(sseg);
    free(rp);
    for (k = 0; k < SG_MAX_DIMS; k++) {
        free(chB[k]);
        free(segB[k]);
    }
    if (r != SG_OK) {
        free_dev(b);
        b->dev = -1;
    }
    return r;
}

static int enter(sg_batch *b, int *prev)
{
    BCU(cudaGetDevice(prev), "cudaGetDevice");
    if (b->dev >= 0 && b->dev != *prev) BCU(cudaSetDevice(b->dev), "cudaSetDevice");
    return SG_OK;
}

static void leave(sg_batch *b, int prev)
{
    if (b->dev >= 0 && b->dev != prev) cudaSetDevice(prev);
}

/* compact concatenation (device) <-> group-aligned batch layout, one launch */
static int move_values(sg_batch *b, const float *src, float *dst, int to_compact, cudaStream_t st)
{
    int e = sgk_copy_segments(src, dst, b->d_segs, b->nsegs, to_compact, st);
    return e == cudaSuccess ? SG_OK : bcuda((cudaError_t)e, "batch value move");
}

static int ensure_stage(sg_batch *b)
{
    return b->d_stage ? SG_OK : balloc(b, (void **)&b->d_stage, b->voff[b->ng] * 4, "batch transfer staging");
}

SG_API int sg_batch_set_values(sg_batch *b, const float *values)
{
    int prev, r;
    if (!b || !values) return bfail(SG_ERR_ARG, "sg_batch_set_values: NULL argument");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if ((r = materialize(b)) == SG_OK && (r = ensure_stage(b)) == SG_OK) {
        cudaError_t e = cudaMemcpy(b->d_stage, values, (size_t)b->voff[b->ng] * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) r = bcuda(e, "sg_batch_set_values");
        else if ((r = move_values(b, b->d_stage, b->d_alpha, 0, 0)) == SG_OK) {
            e = cudaStreamSynchronize(0);
            if (e != cudaSuccess) r = bcuda(e, "sg_batch_set_values");
            else b->has_values = 1, b->eval_dirty = 1;
        }
    }
    leave(b, prev);
    return r;
}

SG_API int sg_batch_set_values_device(sg_batch *b, const float *values, void *stream)
{
    int prev, r;
    if (!b || !values) return bfail(SG_ERR_ARG, "sg_batch_set_values_device: NULL argument");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if ((r = materialize(b)) == SG_OK && (r = move_values(b, values, b->d_alpha, 0, (cudaStream_t)stream)) == SG_OK)
        b->has_values = 1, b->eval_dirty = 1;
    leave(b, prev);
    return r;
}

SG_API int sg_batch_get_values(sg_batch *b, float *values)
{
    int prev, r;
    if (!b || !values) return bfail(SG_ERR_ARG, "sg_batch_get_values: NULL argument");
    if (!b->has_values) return bfail(SG_ERR_STATE, "sg_batch_get_values: no values have been set");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if ((r = ensure_stage(b)) == SG_OK && (r = move_values(b, b->d_alpha, b->d_stage, 1, 0)) == SG_OK) {
        cudaError_t e = cudaMemcpy(values, b->d_stage, (size_t)b->voff[b->ng] * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) r = bcuda(e, "sg_batch_get_values");
    }
    leave(b, prev);
    return r;
}

SG_API int sg_batch_get_values_device(sg_batch *b, float *values, void *stream)
{
    int prev, r;
    if (!b || !values) return bfail(SG_ERR_ARG, "sg_batch_get_values_device: NULL argument");
    if (!b->has_values) return bfail(SG_ERR_STATE, "sg_batch_get_values_device: no values have been set");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    r = move_values(b, b->d_alpha, values, 1, (cudaStream_t)stream);
    leave(b, prev);
    return r;
}

SG_API int sg_batch_sample_function(sg_batch *b, int fn, const double *params, int params_per_grid, void *stream)
{
    int prev, r, g, e;
    if (!b || params_per_grid < 0 || params_per_grid > SG_MAX_FN_PARAMS || (params_per_grid > 0 && !params))
        return bfail(SG_ERR_ARG, "sg_batch_sample_function: bad argument");
    if (fn < SG_FN_REFERENCE || fn > SG_FN_QUAD) return bfail(SG_ERR_ARG, "sg_batch_sample_function: unknown function");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if ((r = materialize(b)) == SG_OK) {
        for (g = 0; g < b->ng && r == SG_OK; g++) {
            const int need = fn == SG_FN_BUMP ? 2 : (fn == SG_FN_QUAD ? 3 * b->L[g].d : 0);
            if (params_per_grid < need) {
                r = bfail(SG_ERR_ARG, "sg_batch_sample_function: grid %d needs %d parameters", g, need);
                break;
            }
            e = sgk_sample(&b->L[g], fn, params ? params + (size_t)g * params_per_grid : NULL, params_per_grid,
                           b->d_alpha + b->doff[g], stream);
            if (e != cudaSuccess) r = bcuda((cudaError_t)e, "sg_batch_sample_function");
        }
        if (r == SG_OK) b->has_values = 1, b->eval_dirty = 1;
    }
    leave(b, prev);
    return r;
}

/* The hierarchization launches (also what the graph captures). */
static const sg_sweep_tables *sweep_table(const sg_batch *b, int q, int k, int c)
{
    return &b->sweepG[((int64_t)q * SG_MAX_DIMS + k) * SG_SWEEP_CLASSES + c];
}

/* One chain-size class of one sweep on stream cs.  Kernel: 2 gather; 3 (or
 * 0 for the shortest chains) one warp per chain; otherwise the staged chain
 * kernel where it fits. */
static int sweep_class(sg_batch *b, const sg_sweep_tables *t, int c, int fp64, cudaStream_t cs)
{
    int e;
    const int kern = b->hier_kernel[c] ? b->hier_kernel[c] : (c == SG_SWEEP_CLASSES - 1 ? 3 : 1);
    const int64_t cap = fp64 ? t->cap64 : t->cap32;
    const int eb = fp64 ? 8 : 4;
    if (kern == 3 && sgk_small_smem_bytes(cap, eb) >= 0)
        e = fp64 ? sgk_sweep_small_f64(b->d_work, t, cs) : sgk_sweep_small_f32(b->d_alpha, t, cs);
    else if (kern != 2 && sgk_chain_smem_bytes(cap, eb) >= 0)
        e = fp64 ? sgk_sweep_chains_f64(b->d_work, t, b->d_err, cs) : sgk_sweep_chains_f32(b->d_alpha, t, b->d_err, cs);
    else
        e = fp64 ? sgk_sweep_gather_f64(b->d_work, t, cs) : sgk_sweep_gather_f32(b->d_alpha, t, cs);
    return e == cudaSuccess ? SG_OK : bcuda((cudaError_t)e, "batch sweep");
}

/* The shared-memory hierarchization of the small grids, one launch per size
 * class, on stream hs. */
static int smem_launches(sg_batch *b, int fp64, cudaStream_t hs)
{
    int c;
    for (c = 0; c < SG_BATCH_CLASSES; c++) {
        cudaError_t e;
        if (!b->cls_count[c]) continue;
        e = (cudaError_t)sgk_hier_smem_grids(b->d_alpha, b->d_smem_grids + b->cls_first[c], b->cls_count[c],
                                             b->d_smem_chains, b->d_smem_seg, b->cls_max_npad[c], fp64, hs);
        if (e != cudaSuccess) return bcuda(e, "batch shared-memory hierarchization");
    }
    return SG_OK;
}

static int hier_launches(sg_batch *b, cudaStream_t st)
{
    int k, c, q, r, any_smem = 0;
    cudaError_t e;
    const int fp64 = b->precision == SG_HIER_FP64;
    /* FP32: the sweeps touch only their own grids' values, so the small
     * grids' shared-memory launches run on a stream of their own beside them
     * (joined back at the end); FP64 runs them after the sweeps, whose
     * widen/narrow round trip rewrites the whole buffer */
    const cudaStream_t hs = b->dst[SG_MAX_DIMS];
    for (c = 0; c < SG_BATCH_CLASSES; c++) any_smem |= b->cls_count[c] > 0;
    const int beside = !fp64 && any_smem && b->has_sweep_grids;
    if (beside) {
        BCU(cudaEventRecord(b->ev_fork, st), "cudaEventRecord");
        BCU(cudaStreamWaitEvent(hs, b->ev_fork, 0), "cudaStreamWaitEvent");
        if ((r = smem_launches(b, fp64, hs)) != SG_OK) return r;
        BCU(cudaEventRecord(b->ev_d[SG_MAX_DIMS], hs), "cudaEventRecord");
    }
    if (b->has_sweep_grids) {
        if (fp64 && (e = (cudaError_t)sgk_widen(b->d_alpha, b->d_work, b->doff[b->ng], st)) != cudaSuccess)
            return bcuda(e, "widen");
        if (b->ngroups == 1) {
            for (k = 0; k < SG_MAX_DIMS; k++) {
                /* the size classes of sweep k are independent: fork them
                 * onto their own streams and join before sweep k+1 */
                int any = 0;
                for (c = 0; c < SG_SWEEP_CLASSES; c++) any |= sweep_table(b, 0, k, c)->nchains > 0;
                if (!any) continue;
                BCU(cudaEventRecord(b->ev_fork, st), "cudaEventRecord");
                for (c = 0; c < SG_SWEEP_CLASSES; c++) {
                    const sg_sweep_tables *t = sweep_table(b, 0, k, c);
                    cudaStream_t cs = b->dst[1 + c];
                    if (!t->nchains) continue;
                    BCU(cudaStreamWaitEvent(cs, b->ev_fork, 0), "cudaStreamWaitEvent");
                    if ((r = sweep_class(b, t, c, fp64, cs)) != SG_OK) return r;
                    BCU(cudaEventRecord(b->ev_d[1 + c], cs), "cudaEventRecord");
                    BCU(cudaStreamWaitEvent(st, b->ev_d[1 + c], 0), "cudaStreamWaitEvent");
                }
            }
        } else {
            /* groups round-robin over SG_SWEEP_STREAMS streams; on its
             * stream a group runs sweep 0..d-1, class after class, so its
             * values stay in L2 from one sweep to the next while the other
             * streams' groups fill the GPU */
            const int ns = b->ngroups < SG_SWEEP_STREAMS ? b->ngroups : SG_SWEEP_STREAMS;
            BCU(cudaEventRecord(b->ev_fork, st), "cudaEventRecord");
            for (q = 0; q < ns; q++) BCU(cudaStreamWaitEvent(b->dst[1 + q], b->ev_fork, 0), "cudaStreamWaitEvent");
            for (q = 0; q < b->ngroups; q++) {
                cudaStream_t cs = b->dst[1 + q % ns];
                for (k = 0; k < SG_MAX_DIMS; k++)
                    for (c = 0; c < SG_SWEEP_CLASSES; c++) {
                        const sg_sweep_tables *t = sweep_table(b, q, k, c);
                        if (t->nchains && (r = sweep_class(b, t, c, fp64, cs)) != SG_OK) return r;
                    }
            }
            for (q = 0; q < ns; q++) {
                BCU(cudaEventRecord(b->ev_d[1 + q], b->dst[1 + q]), "cudaEventRecord");
                BCU(cudaStreamWaitEvent(st, b->ev_d[1 + q], 0), "cudaStreamWaitEvent");
            }
        }
        if (fp64 && (e = (cudaError_t)sgk_narrow(b->d_work, b->d_alpha, b->doff[b->ng], st)) != cudaSuccess)
            return bcuda(e, "narrow");
    }
    if (beside) {
        BCU(cudaStreamWaitEvent(st, b->ev_d[SG_MAX_DIMS], 0), "cudaStreamWaitEvent");
        return SG_OK;
    }
    /* after the sweeps: their FP64 round trip rewrites the whole buffer with
     * the (unchanged) nodal values of the shared-memory grids */
    return smem_launches(b, fp64, st);
}

/* Replays *exec, capturing body into it first.  The library's launch
 * counter counts kernels as they launch, so a replay adds the kernels the
 * capture recorded (*kernels). */
static int run_graph(cudaGraphExec_t *exec, int64_t *kernels, int (*body)(sg_batch *, cudaStream_t), sg_batch *b,
                     cudaStream_t st)
{
    cudaGraph_t graph = NULL;
    cudaError_t e;
    int r;
    int64_t before;
    if (*exec) {
        BCU(cudaGraphLaunch(*exec, st), "cudaGraphLaunch");
        sgk_count((int)*kernels);
        return SG_OK;
    }
    if (st == 0) return body(b, st); /* the legacy stream cannot be captured */
    BCU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    before = sgk_launches();
    r = body(b, st);
    /* captured kernels do not run yet: counted at each replay instead */
    *kernels = sgk_launches() - before;
    sgk_count((int)-*kernels);
    e = cudaStreamEndCapture(st, &graph);
    if (r != SG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return r;
    }
    if (e != cudaSuccess) return bcuda(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        *exec = NULL;
        return bcuda(e, "cudaGraphInstantiate");
    }
    BCU(cudaGraphLaunch(*exec, st), "cudaGraphLaunch");
    sgk_count((int)*kernels);
    return SG_OK;
}

SG_API int sg_batch_hierarchize_async(sg_batch *b, void *stream)
{
    int prev, r;
    cudaStream_t st = (cudaStream_t)stream;
    if (!b) return bfail(SG_ERR_ARG, "sg_batch_hierarchize_async: NULL batch");
    if (!b->has_values) return bfail(SG_ERR_STATE, "sg_batch_hierarchize: no values have been set");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if (b->precision == SG_HIER_FP64 && b->has_sweep_grids && !b->d_work)
        r = balloc(b, (void **)&b->d_work, b->doff[b->ng] * 8, "batch FP64 working values");
    if (r == SG_OK) r = make_fork_streams(b);
    if (r == SG_OK) r = b->use_graph ? run_graph(&b->hier_graph, &b->hier_graph_kernels, hier_launches, b, st) : hier_launches(b, st);
    b->eval_dirty = 1;
    leave(b, prev);
    return r;
}

SG_API int sg_batch_sync(sg_batch *b, void *stream)
{
    int prev, r = SG_OK, flag = 0;
    cudaError_t e;
    if (!b) return bfail(SG_ERR_ARG, "sg_batch_sync: NULL batch");
    if (b->dev < 0) return SG_OK;
    if ((r = enter(b, &prev)) != SG_OK) return r;
    e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) r = bcuda(e, "sg_batch_sync");
    else if (flag) {
        cudaMemset(b->d_err, 0, sizeof(int));
        r = bfail(SG_ERR_TIMEOUT, "a device-side wait gave up; the batch values are not valid");
    }
    leave(b, prev);
    return r;
}

SG_API int sg_batch_hierarchize(sg_batch *b)
{
    int r = sg_batch_hierarchize_async(b, 0);
    return r == SG_OK ? sg_batch_sync(b, 0) : r;
}

/* Evaluation plan: per-grid kernel arguments and per-dimension CTA items for
 * the caller's point offsets and buffers (kept, so an identical call replays
 * the captured graph). */
static int ppt_of(const sg_batch *b, int d) { return b->ppt_d[d] ? b->ppt_d[d] : b->ppt; }
/* blocking preset index (0 .. SG_EVAL_BLOCKINGS-1) of dimension d */
static int blk_of(const sg_batch *b, int d)
{
    const int v = b->blk_d[d] ? b->blk_d[d] : b->blocking;
    return v > 0 ? v - 1 : 0;
}

static int cmp_dim_then_subspaces(const void *x, const void *y, void *ctx)
{
    const sg_batch *b = (const sg_batch *)ctx;
    const sg_layout *a = &b->L[*(const int *)x], *c = &b->L[*(const int *)y];
    if (a->d != c->d) return a->d < c->d ? -1 : 1;
    if (a->S != c->S) return a->S > c->S ? -1 : 1;
    return *(const int *)x - *(const int *)y;
}

/* Spatial ordering of every grid's points (among themselves): per-grid
 * geometry, CTA items and buffers; points the evaluation arguments at the
 * sorted coordinates and the permutation. */
static int plan_sort(sg_batch *b, const int64_t *pt_off)
{
    sg_bsort_grid *sg = NULL;
    int32_t *items = NULL;
    int64_t coff = 0, nbins = 0, ni = 0, cap = 0, ncoord = 0, npts = pt_off[b->ng];
    int g, r = SG_OK;
    const int64_t before = b->dev_bytes;
    b->dev_bytes -= b->sort_bytes;
    cudaFree(b->d_sgrids);
    cudaFree(b->d_sitems);
    cudaFree(b->d_sscratch);
    cudaFree(b->d_sorted);
    cudaFree(b->d_perm);
    b->d_sgrids = NULL;
    b->d_sitems = NULL;
    b->d_sscratch = NULL;
    b->d_sorted = NULL;
    b->d_perm = NULL;
    b->nsitems = 0;
    for (g = 0; g < b->ng; g++) {
        cap += (pt_off[g + 1] - pt_off[g] + 255) / 256;
        ncoord += (pt_off[g + 1] - pt_off[g]) * b->L[g].d;
    }
    sg = (sg_bsort_grid *)malloc(sizeof(sg_bsort_grid) * (size_t)b->ng);
    items = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)(cap > 0 ? cap : 1));
    if (!sg || !items) {
        r = bfail(SG_ERR_NOMEM, "out of host memory");
        goto out;
    }
    for (g = 0; g < b->ng; g++) {
        const int64_t m = pt_off[g + 1] - pt_off[g];
        int64_t p;
        sg[g].m = m;
        sg[g].pt_off = pt_off[g];
        sg[g].coff = coff;
        sg[g].d = b->L[g].d;
        sg[g].kb = sgk_batch_sort_bits(m, b->L[g].d);
        sg[g].bin_base = (uint32_t)nbins;
        nbins += (int64_t)1 << sg[g].kb;
        coff += m * b->L[g].d;
        for (p = 0; p < m; p += 256) {
            items[2 * ni] = g;
            items[2 * ni + 1] = (int32_t)p;
            ni++;
        }
    }
    if (nbins >= ((int64_t)1 << 31)) {
        r = bfail(SG_ERR_RANGE, "sg_batch_evaluate: too many sort bins");
        goto out;
    }
    if ((r = upload(b, (void **)&b->d_sgrids, sg, b->ng * (int64_t)sizeof(sg_bsort_grid), "sort geometry")) != SG_OK ||
        (r = upload(b, (void **)&b->d_sitems, items, ni * 8, "sort items")) != SG_OK ||
        (r = balloc(b, &b->d_sscratch, sgk_batch_sort_scratch_bytes(npts, nbins), "sort scratch")) != SG_OK ||
        (r = balloc(b, (void **)&b->d_sorted, ncoord * 4, "sorted coordinates")) != SG_OK ||
        (r = balloc(b, (void **)&b->d_perm, npts * 4, "sort permutation")) != SG_OK)
        goto out;
    b->nsitems = (int)ni;
    b->sort_bytes = b->dev_bytes - before + b->sort_bytes;
    b->sort_npts = npts;
    b->sort_nbins = nbins;
    for (g = 0; g < b->ng; g++) {
        b->h_eval_args[g].coords = b->d_sorted + sg[g].coff;
        b->h_eval_args[g].perm = b->d_perm + pt_off[g];
    }
out:
    free(sg);
    free(items);
    return r;
}

static int plan_eval(sg_batch *b, const int64_t *pt_off, const float *coords, float *out)
{
    int g, k, r, q;
    int64_t coff = 0, ni = 0, cap_items = 0;
    int same = b->h_eval_args && b->eval_coords == coords && b->eval_out == out && b->eval_sort == b->sort;
    for (k = 0; same && k <= SG_MAX_DIMS; k++) same = b->eval_ppt_d[k] == ppt_of(b, k) && b->eval_blk_d[k] == blk_of(b, k);
    for (g = 0; same && g <= b->ng; g++) same = b->eval_pt_off[g] == pt_off[g];
    if (same) return SG_OK;
    if (b->eval_graph) {
        cudaGraphExecDestroy(b->eval_graph);
        b->eval_graph = NULL;
    }
    if (!b->h_eval_args) {
        b->h_eval_args = (sg_eval_args *)calloc((size_t)b->ng, sizeof(sg_eval_args));
        b->eval_pt_off = (int64_t *)calloc((size_t)b->ng + 1, sizeof(int64_t));
        if (!b->h_eval_args || !b->eval_pt_off) return bfail(SG_ERR_NOMEM, "out of host memory");
        if ((r = balloc(b, (void **)&b->d_eval_args, b->ng * (int64_t)sizeof(sg_eval_args), "batch eval args")) != SG_OK)
            return r;
    }
    for (k = 0; k <= SG_MAX_DIMS; k++) b->items_first[k] = b->items_count[k] = 0;
    for (g = 0; g < b->ng; g++) {
        const int64_t m = pt_off[g + 1] - pt_off[g];
        if (m < 0) return bfail(SG_ERR_ARG, "sg_batch_evaluate: point offsets decrease at grid %d", g);
        cap_items += (m + 255) / 256; /* enough for one point per thread */
    }
    if (!b->order) {
        b->order = (int *)malloc(sizeof(int) * (size_t)b->ng);
        if (!b->order) return bfail(SG_ERR_NOMEM, "out of host memory");
        for (g = 0; g < b->ng; g++) b->order[g] = g;
        qsort_r(b->order, (size_t)b->ng, sizeof(int), cmp_dim_then_subspaces, b);
    }
    free(b->h_items);
    b->h_items = (int32_t *)malloc((size_t)(cap_items > 0 ? cap_items : 1) * 2 * sizeof(int32_t));
    if (!b->h_items) return bfail(SG_ERR_NOMEM, "out of host memory");
    for (g = 0; g < b->ng; g++) {
        const sg_layout *L = &b->L[g];
        sg_eval_plan p;
        sg_eval_shape sh;
        sg_eval_sub sub;
        int s;
        p.alpha = b->d_blk + b->boff[g];
        p.d = L->d;
        p.n = L->n;
        for (k = 0; k < SG_MAX_DIMS; k++) p.lim[k] = k < L->d ? L->lim[k] : 0;
        for (s = 0; s < SG_MAX_LEVELS; s++) {
            if (s < L->n) {
                sg_layout_eval_shape(L, s, &sh);
                sg_layout_eval_sub(L, s, &sub);
                p.blk3[s] = sh.coff[sh.cmax + 1];
                p.blk2[s] = sub.aoff[sub.amax + 1];
            } else {
                p.blk3[s] = p.blk2[s] = 0;
            }
        }
        p.ppt = ppt_of(b, L->d);
        p.blocking = blk_of(b, L->d);
        sgk_fill_eval_args(&p, coords + coff, NULL, out + pt_off[g], pt_off[g + 1] - pt_off[g], &b->h_eval_args[g]);
        coff += (pt_off[g + 1] - pt_off[g]) * L->d;
    }
    if (b->sort && (r = plan_sort(b, pt_off)) != SG_OK) return r;
    /* items grouped by dimension, grids with the most subspaces first (their
     * CTAs are the longest) */
    for (k = 1; k <= SG_MAX_DIMS; k++) {
        const int cta = 256 * ppt_of(b, k);
        b->items_first[k] = (int)ni;
        for (q = 0; q < b->ng; q++) {
            int64_t st;
            g = b->order[q];
            if (b->L[g].d != k) continue;
            for (st = pt_off[g]; st < pt_off[g + 1]; st += cta) {
                b->h_items[2 * ni] = g;
                b->h_items[2 * ni + 1] = (int32_t)(st - pt_off[g]);
                ni++;
            }
        }
        b->items_count[k] = (int)ni - b->items_first[k];
    }
    if (ni > b->items_cap) {
        cudaFree(b->d_items);
        b->d_items = NULL;
        if ((r = balloc(b, (void **)&b->d_items, ni * 2 * 4, "batch eval items")) != SG_OK) return r;
        b->items_cap = ni;
    }
    BCU(cudaMemcpy(b->d_eval_args, b->h_eval_args, (size_t)b->ng * sizeof(sg_eval_args), cudaMemcpyHostToDevice),
        "upload eval args");
    if (ni > 0) BCU(cudaMemcpy(b->d_items, b->h_items, (size_t)ni * 2 * 4, cudaMemcpyHostToDevice), "upload items");
    for (g = 0; g <= b->ng; g++) b->eval_pt_off[g] = pt_off[g];
    b->eval_coords = coords;
    b->eval_out = out;
    for (k = 0; k <= SG_MAX_DIMS; k++) {
        b->eval_ppt_d[k] = ppt_of(b, k);
        b->eval_blk_d[k] = blk_of(b, k);
    }
    b->eval_sort = b->sort;
    return SG_OK;
}

static int make_fork_streams(sg_batch *b)
{
    int k;
    if (b->ev_fork) return SG_OK;
    BCU(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
    for (k = 1; k <= SG_MAX_DIMS; k++) {
        BCU(cudaStreamCreateWithFlags(&b->dst[k], cudaStreamNonBlocking), "cudaStreamCreate");
        BCU(cudaEventCreateWithFlags(&b->ev_d[k], cudaEventDisableTiming), "cudaEventCreate");
    }
    return SG_OK;
}

/* Repack, then one launch per dimension, each on its own stream forked from
 * and joined back to st (captured as parallel branches of the graph). */
static int eval_launches(sg_batch *b, cudaStream_t st)
{
    int k, e;
    if (b->sort && (e = sgk_batch_sort_points(b->eval_coords, b->d_sgrids, b->d_sitems, b->nsitems, b->sort_npts,
                                              b->sort_nbins, b->d_sscratch, b->d_sorted, b->d_perm, st)) !=
                       cudaSuccess)
        return bcuda((cudaError_t)e, "batch spatial ordering");
    if ((e = sgk_repack(b->d_alpha, b->d_blk, b->d_repack, b->nrepack, st)) != cudaSuccess)
        return bcuda((cudaError_t)e, "batch repack");
    BCU(cudaEventRecord(b->ev_fork, st), "cudaEventRecord");
    for (k = 1; k <= SG_MAX_DIMS; k++) {
        if (!b->items_count[k]) continue;
        BCU(cudaStreamWaitEvent(b->dst[k], b->ev_fork, 0), "cudaStreamWaitEvent");
        e = sgk_evaluate_batch(k, b->d_eval_args, b->d_items + 2 * (int64_t)b->items_first[k], b->items_count[k],
                               ppt_of(b, k), blk_of(b, k), b->dst[k]);
        if (e != cudaSuccess) return bcuda((cudaError_t)e, "batch evaluate");
        BCU(cudaEventRecord(b->ev_d[k], b->dst[k]), "cudaEventRecord");
        BCU(cudaStreamWaitEvent(st, b->ev_d[k], 0), "cudaStreamWaitEvent");
    }
    return SG_OK;
}

SG_API int sg_batch_evaluate_device(sg_batch *b, const int64_t *point_offsets, const float *coords, float *out,
                                    void *stream)
{
    int prev, r;
    cudaStream_t st = (cudaStream_t)stream;
    if (!b || !point_offsets || point_offsets[0] != 0) return bfail(SG_ERR_ARG, "sg_batch_evaluate_device: bad argument");
    if (!b->has_values) return bfail(SG_ERR_STATE, "sg_batch_evaluate: no values have been set");
    if (point_offsets[b->ng] > 0 && (!coords || !out)) return bfail(SG_ERR_ARG, "sg_batch_evaluate_device: NULL buffer");
    if (point_offsets[b->ng] >= ((int64_t)1 << 31)) return bfail(SG_ERR_RANGE, "sg_batch_evaluate: too many points");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    if ((r = make_fork_streams(b)) == SG_OK && (r = plan_eval(b, point_offsets, coords, out)) == SG_OK)
        r = b->use_graph ? run_graph(&b->eval_graph, &b->eval_graph_kernels, eval_launches, b, st) : eval_launches(b, st);
    if (r == SG_OK) b->eval_dirty = 0;
    leave(b, prev);
    return r;
}

SG_API int sg_batch_autotune(sg_batch *b, const int64_t *point_offsets, const float *coords, float *out, void *stream,
                             double *ms)
{
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0 = NULL, e1 = NULL;
    double t[2 * SG_EVAL_BLOCKINGS][SG_MAX_DIMS + 1];
    int prev, r, pi, k, q, rep, cfg;
    float el;
    if (!b || !point_offsets || point_offsets[0] != 0) return bfail(SG_ERR_ARG, "sg_batch_autotune: bad argument");
    if (!b->has_values || b->dev < 0) return bfail(SG_ERR_STATE, "sg_batch_autotune: no values have been set");
    if (point_offsets[b->ng] > 0 && (!coords || !out)) return bfail(SG_ERR_ARG, "sg_batch_autotune: NULL buffer");
    if ((r = enter(b, &prev)) != SG_OK) return r;
    for (cfg = 0; cfg < 2 * SG_EVAL_BLOCKINGS; cfg++)
        for (k = 0; k <= SG_MAX_DIMS; k++) t[cfg][k] = -1.0;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        r = bfail(SG_ERR_CUDA, "sg_batch_autotune: cudaEventCreate");
        goto done;
    }
    if ((r = make_fork_streams(b)) != SG_OK) goto done;
    /* every dimension's launch alone on st, at 1 and at 2 points per thread
     * (pi) under each blocking preset (cfg / 2) */
    for (cfg = 0; cfg < 2 * SG_EVAL_BLOCKINGS && r == SG_OK; cfg++) {
        pi = cfg % 2;
        for (k = 0; k <= SG_MAX_DIMS; k++) {
            b->ppt_d[k] = pi + 1;
            b->blk_d[k] = cfg / 2 + 1;
        }
        if ((r = plan_eval(b, point_offsets, coords, out)) != SG_OK) break;
        if (b->sort && sgk_batch_sort_points(coords, b->d_sgrids, b->d_sitems, b->nsitems, b->sort_npts, b->sort_nbins,
                                             b->d_sscratch, b->d_sorted, b->d_perm, st) != cudaSuccess) {
            r = bfail(SG_ERR_CUDA, "sg_batch_autotune: spatial ordering");
            break;
        }
        if (sgk_repack(b->d_alpha, b->d_blk, b->d_repack, b->nrepack, st) != cudaSuccess) {
            r = bfail(SG_ERR_CUDA, "sg_batch_autotune: repack");
            break;
        }
        for (k = 1; k <= SG_MAX_DIMS && r == SG_OK; k++) {
            if (!b->items_count[k]) continue;
            for (rep = 0; rep < 3; rep++) { /* first run warms */
                if (cudaEventRecord(e0, st) != cudaSuccess ||
                    sgk_evaluate_batch(k, b->d_eval_args, b->d_items + 2 * (int64_t)b->items_first[k],
                                       b->items_count[k], pi + 1, cfg / 2, st) != cudaSuccess ||
                    cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&el, e0, e1) != cudaSuccess) {
                    r = bfail(SG_ERR_CUDA, "sg_batch_autotune: timing d=%d", k);
                    break;
                }
                if (rep > 0 && (t[cfg][k] < 0.0 || el < t[cfg][k])) t[cfg][k] = el;
            }
        }
    }
    for (k = 0; k <= SG_MAX_DIMS; k++) {
        int best = -1;
        for (cfg = 0; r == SG_OK && cfg < 2 * SG_EVAL_BLOCKINGS; cfg++)
            if (t[cfg][k] >= 0.0 && (best < 0 || t[cfg][k] < t[best][k])) best = cfg;
        b->ppt_d[k] = best >= 0 ? best % 2 + 1 : 0;
        b->blk_d[k] = best >= 0 ? best / 2 + 1 : 0;
    }
    b->eval_dirty = 1;
    /* sweeps: per chain size class, the staged chain kernel or one warp per
     * chain (both bit-identical); the values are saved and restored */
    if (r == SG_OK && b->has_sweep_grids) {
        float *saved = NULL;
        const size_t vb = (size_t)b->doff[b->ng] * 4;
        int c, kern;
        if (b->precision == SG_HIER_FP64 && !b->d_work &&
            (r = balloc(b, (void **)&b->d_work, b->doff[b->ng] * 8, "batch FP64 working values")) != SG_OK)
            goto done;
        if (cudaMalloc((void **)&saved, vb) != cudaSuccess) {
            cudaGetLastError();
            r = bfail(SG_ERR_NOMEM, "sg_batch_autotune: no device memory to save the values");
            goto done;
        }
        if (cudaMemcpyAsync(saved, b->d_alpha, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            r = bfail(SG_ERR_CUDA, "sg_batch_autotune: save");
        for (c = 0; c < SG_SWEEP_CLASSES && r == SG_OK; c++) {
            double best = -1.0;
            int best_k = 0, any = 0;
            for (q = 0; q < b->ngroups; q++)
                for (k = 0; k < SG_MAX_DIMS; k++) any |= sweep_table(b, q, k, c)->nchains > 0;
            if (!any) continue;
            for (kern = 1; kern <= 3 && r == SG_OK; kern += 2) {
                b->hier_kernel[c] = kern;
                for (rep = 0; rep < 3 && r == SG_OK; rep++) {
                    if (cudaMemcpyAsync(b->d_alpha, saved, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
                        cudaEventRecord(e0, st) != cudaSuccess) {
                        r = bfail(SG_ERR_CUDA, "sg_batch_autotune: sweep timing");
                        break;
                    }
                    if ((r = hier_launches(b, st)) != SG_OK) break;
                    if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                        cudaEventElapsedTime(&el, e0, e1) != cudaSuccess) {
                        r = bfail(SG_ERR_CUDA, "sg_batch_autotune: sweep timing");
                        break;
                    }
                    if (rep > 0 && (best < 0.0 || el < best)) best = el, best_k = kern;
                }
            }
            b->hier_kernel[c] = best_k;
        }
        if (cudaMemcpyAsync(b->d_alpha, saved, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            if (r == SG_OK) r = bfail(SG_ERR_CUDA, "sg_batch_autotune: restore");
        }
        cudaFree(saved);
        if (b->hier_graph) {
            cudaGraphExecDestroy(b->hier_graph);
            b->hier_graph = NULL;
        }
    }
    if (ms)
        for (cfg = 0; cfg < 2 * SG_EVAL_BLOCKINGS; cfg++)
            for (k = 0; k <= SG_MAX_DIMS; k++) ms[cfg * (SG_MAX_DIMS + 1) + k] = t[cfg][k];
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    leave(b, prev);
    return r;
}

SG_API int sg_batch_set_option(sg_batch *b, int option, int64_t value)
{
    if (!b) return bfail(SG_ERR_ARG, "sg_batch_set_option: NULL batch");
    switch (option) {
    case SG_OPT_HIER_PRECISION:
        if (value != SG_HIER_FP32 && value != SG_HIER_FP64) return bfail(SG_ERR_ARG, "bad precision");
        if (b->precision != (int)value && b->hier_graph) {
            cudaGraphExecDestroy(b->hier_graph);
            b->hier_graph = NULL;
        }
        b->precision = (int)value;
        return SG_OK;
    case SG_OPT_EVAL_PPT:
        if (value < 0 || value > 2) return bfail(SG_ERR_ARG, "SG_OPT_EVAL_PPT is 0, 1 or 2");
        b->ppt = value == 0 ? 2 : (int)value;
        memset(b->ppt_d, 0, sizeof(b->ppt_d)); /* an explicit setting replaces tuned ones */
        return SG_OK;
    case SG_OPT_EVAL_BLOCKING:
        if (value < 0 || value > SG_EVAL_BLOCKINGS)
            return bfail(SG_ERR_ARG, "SG_OPT_EVAL_BLOCKING is 0 .. %d", SG_EVAL_BLOCKINGS);
        b->blocking = (int)value;
        memset(b->blk_d, 0, sizeof(b->blk_d));
        return SG_OK;
    case SG_OPT_USE_GRAPH:
        if (value != 0 && value != 1) return bfail(SG_ERR_ARG, "SG_OPT_USE_GRAPH is 0 or 1");
        b->use_graph = (int)value;
        return SG_OK;
    case SG_OPT_EVAL_SORT:
        if (value != 0 && value != 1) return bfail(SG_ERR_ARG, "SG_OPT_EVAL_SORT is 0 or 1");
        b->sort = (int)value;
        return SG_OK;
    case SG_OPT_HIER_KERNEL: {
        int c;
        if (value < 0 || value > 3) return bfail(SG_ERR_ARG, "SG_OPT_HIER_KERNEL is 0, 1, 2 or 3");
        for (c = 0; c < SG_SWEEP_CLASSES; c++) b->hier_kernel[c] = (int)value;
        if (b->hier_graph) {
            cudaGraphExecDestroy(b->hier_graph);
            b->hier_graph = NULL;
        }
        return SG_OK;
    }
    case SG_OPT_SWEEP_GROUP:
        /* the sweep tables are built by the first device call */
        if (value < 0 || value >= ((int64_t)1 << 32)) return bfail(SG_ERR_ARG, "SG_OPT_SWEEP_GROUP is 0 .. 2^32-1");
        if (b->dev >= 0 && value != b->sweep_group)
            return bfail(SG_ERR_STATE, "SG_OPT_SWEEP_GROUP must be set before the batch's first device call");
        b->sweep_group = value;
        return SG_OK;
    default:
        return bfail(SG_ERR_ARG, "option %d does not apply to batches", option);
    }
}

SG_API int sg_batch_device_bytes(const sg_batch *b, int64_t *bytes)
{
    if (!b || !bytes) return bfail(SG_ERR_ARG, "sg_batch_device_bytes: NULL argument");
    *bytes = b->dev_bytes;
    return SG_OK;
}
