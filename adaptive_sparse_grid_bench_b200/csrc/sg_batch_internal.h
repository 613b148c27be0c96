/* Internal state of a grid batch (sgrid_batch.c). */
#ifndef SG_BATCH_INTERNAL_H
#define SG_BATCH_INTERNAL_H

#include <cuda_runtime_api.h>
#include <stdarg.h>
#include <stdint.h>

#include "sg_kernels.h"
#include "sg_layout.h"

#define SG_BATCH_CLASSES 4 /* size classes of the shared-memory hierarchization */
#define SG_SWEEP_CLASSES 3 /* chain size classes of the batched sweeps          */
#define SG_SWEEP_STREAMS 4 /* concurrent streams of grouped sweeps             */

struct sg_batch {
    int ng;
    sg_layout *L;        /* per grid                                              */
    int64_t *voff;       /* compact value offsets (caller's concatenation), ng+1   */
    int64_t *doff;       /* offsets in the device value buffer (32-aligned), ng+1  */
    int64_t *boff;       /* offsets in the block-layout buffer, ng+1               */
    int dev, has_values, eval_dirty;
    int precision, ppt, use_graph;
    int hier_kernel[SG_SWEEP_CLASSES]; /* per chain size class: 0/1 chains (where they fit), 2 gather */
    int64_t dev_bytes;
    float *d_alpha;      /* all grids, group-aligned layout                       */
    double *d_work;      /* FP64 sweep values (lazy)                              */
    float *d_blk;        /* all grids, block layout                               */
    int *d_err;
    sg_copy_seg *d_segs;  /* per-grid level groups: compact <-> device layout */
    int64_t nsegs;
    float *d_stage;       /* host-buffer transfers: compact values on the device (lazy) */
    /* shared-memory path */
    int n_smem;
    int cls_first[SG_BATCH_CLASSES], cls_count[SG_BATCH_CLASSES], cls_max_npad[SG_BATCH_CLASSES];
    sg_smem_grid *d_smem_grids;
    sg_chain *d_smem_chains;
    uint32_t *d_smem_seg;
    /* chain-sweep path */
    int has_sweep_grids;
    /* sweep groups: consecutive runs of sweep grids holding at most
     * sweep_group values (0: the whole batch is one group).  Grouped, all d
     * sweeps of a group run back to back on one of SG_SWEEP_STREAMS
     * streams, so the group's values stay in L2 between its sweeps.  Per
     * group, the chains of sweep k are sorted by size into SG_SWEEP_CLASSES
     * classes that launch with their own CTA size and shared-memory stages:
     * table (q, k, c) is sweepG[(q * SG_MAX_DIMS + k) * SG_SWEEP_CLASSES + c] */
    int64_t sweep_group;
    int ngroups;
    sg_sweep_tables *sweepG;
    sg_chain *d_chB[SG_MAX_DIMS];
    uint32_t *d_segB[SG_MAX_DIMS];
    /* evaluation */
    sg_repack *d_repack;
    int64_t nrepack;
    sg_eval_args *h_eval_args, *d_eval_args;
    int32_t *h_items, *d_items;
    int64_t items_cap;
    int items_first[SG_MAX_DIMS + 1], items_count[SG_MAX_DIMS + 1];
    int64_t *eval_pt_off;
    const float *eval_coords;
    float *eval_out;
    int sort;                        /* spatial ordering of each grid's points (default 1) */
    int eval_sort;                   /* the setting the current plan was built for */
    sg_bsort_grid *d_sgrids;         /* sort: per-grid geometry                  */
    int32_t *d_sitems;               /* sort: CTA items, 256 points each          */
    int nsitems;
    int64_t sort_npts, sort_nbins, sort_bytes;
    void *d_sscratch;                /* sort: keys, histogram, scan               */
    float *d_sorted;                 /* sorted coordinates                         */
    int32_t *d_perm;                 /* sorted position -> caller's local index    */
    int ppt_d[SG_MAX_DIMS + 1];      /* points per thread per dimension (0: ppt) */
    int eval_ppt_d[SG_MAX_DIMS + 1]; /* the setting the current plan was built for */
    int blocking;                    /* SG_OPT_EVAL_BLOCKING (0: auto = wide)       */
    int blk_d[SG_MAX_DIMS + 1];      /* tuned blocking per dimension (0: blocking) */
    int eval_blk_d[SG_MAX_DIMS + 1]; /* the setting the current plan was built for */
    int *order;                      /* grids by dimension, most subspaces first */
    /* the per-dimension launches of an evaluation fork onto their own
     * streams (joined back before the caller's stream continues) */
    cudaStream_t dst[SG_MAX_DIMS + 1];
    cudaEvent_t ev_fork, ev_d[SG_MAX_DIMS + 1];
    cudaGraphExec_t hier_graph, eval_graph;
    int64_t hier_graph_kernels, eval_graph_kernels; /* kernel launches captured in each graph */
};

/* Sets the calling thread's sg_last_error() text (sgrid.c). */
void sg_set_error(const char *fmt, va_list ap);

#endif
