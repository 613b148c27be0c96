/*
 * Serving loop (sg_server_* in include/sgrid.h).  Host code in C with one
 * dispatcher thread.
 *
 * Resident grids: a pool of hierarchized grids kept on the device under a
 * byte cap.  The server reserves the whole cap as one device range at
 * creation and sub-allocates every grid buffer from it (first fit over an
 * offset-sorted free list, neighbours merged on free), so admitting and
 * evicting grids makes no cudaMalloc/cudaFree call: a cudaFree waits for the
 * whole device, which would stall the batches in flight.
 * sg_server_add_grid admits a new grid (create, sample, hierarchize, build
 * the evaluation layout) after evicting least recently used grids that no
 * queued or running request needs; if that cannot free enough memory the
 * admission fails with SG_ERR_NOMEM.
 *
 * Continuous batching: callers submit evaluate requests of any size (up to
 * the batch capacity) against resident grids and get a ticket.  The
 * dispatcher takes every request queued at that moment (up to the capacity)
 * into one batch: one host->device copy of all their coordinates, one
 * batched evaluation launch per dimension present (the batched kernel treats
 * each request as a grid of its own), one device->host copy of the results.
 * The per-dimension launches of a batch run concurrently on streams of their
 * own (forked from and joined back to the slot's stream), so their tails
 * overlap; inside a launch the CTAs of the grids with the most subspaces
 * come first (longest first).  One point's sum over a grid's subspaces is
 * a serial chain of work for one thread; on grids with many subspaces it is
 * split into parts (block ranges of the evaluation walk, fixed per grid at
 * admission), evaluated by separate CTAs and added in part order by a
 * combine launch, and launches that still hold long chains use one point
 * per thread: this bounds the latency of a request on a large grid.
 * Batches alternate between two slots, so a batch is staged and copied
 * while the previous one computes; requests that arrive while a batch runs
 * go into the next one as soon as a slot frees up.  Staging (coordinates
 * into pinned memory) and delivery (results into the callers' buffers) run
 * outside the server lock.  A request's result depends only on its grid
 * and points (the kernel's arithmetic for a point does not depend on the
 * CTA shape), so it is the same alone and in any mix.
 */
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "sg_batch_internal.h"
#include "sg_grid_internal.h"
#include "sg_kernels.h"

#define SG_API __attribute__((visibility("default")))
#define SRV_SLOTS 5               /* slots 0-2: light lane, 3-4: heavy lane */
#define SRV_LIGHT_SLOTS 3
#define SRV_HEAVY_PAIRS ((int64_t)1 << 27) /* default SG_SRV_OPT_HEAVY_PAIRS */
#define SRV_MAX_REQS 8192 /* requests per batch */
#define SRV_CTA_THREADS 256
#define SRV_SPLIT_SUBSPACES 4096  /* grids (d >= 4) with this many subspaces get split sums */
#define SRV_PART_SUBSPACES 2048   /* about this many subspaces per part (at most 8 parts) */
#define SRV_LONG_CHAIN 2048       /* light launches with a part this long use 1 point per thread */
#define SRV_WHOLE_POINTS 8192     /* heavy requests with this many points are not split: their
                                     own points give the launch enough CTAs */
#define SRV_RING_BATCHES 4        /* the staging ring holds this many full batches */

#define ARENA_ALIGN 256

typedef struct arena_rng {
    int64_t off, size;
} arena_rng;

typedef struct sg_arena {
    char *base;
    int64_t size, used;
    pthread_mutex_t mu;
    arena_rng *fr; /* free ranges, sorted by offset, never adjacent */
    int64_t nfr, capfr;
    arena_rng *live; /* handed-out ranges, unordered */
    int64_t nlive, caplive;
} sg_arena;

static int rng_reserve(arena_rng **a, int64_t *cap, int64_t need)
{
    arena_rng *na;
    int64_t nc;
    if (need <= *cap) return 1;
    nc = *cap ? 2 * *cap : 256;
    while (nc < need) nc *= 2;
    na = (arena_rng *)realloc(*a, (size_t)nc * sizeof(arena_rng));
    if (!na) return 0;
    *a = na;
    *cap = nc;
    return 1;
}

static int arena_alloc(void *ctx, void **ptr, int64_t bytes)
{
    sg_arena *A = (sg_arena *)ctx;
    int64_t i, sz = (bytes + ARENA_ALIGN - 1) & ~(int64_t)(ARENA_ALIGN - 1);
    int r = SG_ERR_NOMEM;
    *ptr = NULL;
    pthread_mutex_lock(&A->mu);
    for (i = 0; i < A->nfr; i++) {
        arena_rng *f = &A->fr[i];
        if (f->size < sz) continue;
        if (!rng_reserve(&A->live, &A->caplive, A->nlive + 1)) break;
        A->live[A->nlive].off = f->off;
        A->live[A->nlive].size = sz;
        A->nlive++;
        *ptr = A->base + f->off;
        f->off += sz;
        f->size -= sz;
        if (f->size == 0) {
            memmove(&A->fr[i], &A->fr[i + 1], (size_t)(A->nfr - i - 1) * sizeof(arena_rng));
            A->nfr--;
        }
        A->used += sz;
        r = SG_OK;
        break;
    }
    pthread_mutex_unlock(&A->mu);
    return r;
}

static void arena_free(void *ctx, void *ptr)
{
    sg_arena *A = (sg_arena *)ctx;
    int64_t i, off, sz, lo, hi;
    if (!ptr) return;
    off = (char *)ptr - A->base;
    pthread_mutex_lock(&A->mu);
    for (i = 0; i < A->nlive && A->live[i].off != off; i++) {
    }
    if (i == A->nlive || !rng_reserve(&A->fr, &A->capfr, A->nfr + 1)) {
        /* not ours (or no host memory to track it): leave it allocated */
        pthread_mutex_unlock(&A->mu);
        return;
    }
    sz = A->live[i].size;
    A->live[i] = A->live[--A->nlive];
    A->used -= sz;
    /* first free range after off */
    lo = 0;
    hi = A->nfr;
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (A->fr[mid].off < off) lo = mid + 1;
        else hi = mid;
    }
    if (lo > 0 && A->fr[lo - 1].off + A->fr[lo - 1].size == off) {
        A->fr[lo - 1].size += sz;
        if (lo < A->nfr && off + sz == A->fr[lo].off) {
            A->fr[lo - 1].size += A->fr[lo].size;
            memmove(&A->fr[lo], &A->fr[lo + 1], (size_t)(A->nfr - lo - 1) * sizeof(arena_rng));
            A->nfr--;
        }
    } else if (lo < A->nfr && off + sz == A->fr[lo].off) {
        A->fr[lo].off = off;
        A->fr[lo].size += sz;
    } else {
        memmove(&A->fr[lo + 1], &A->fr[lo], (size_t)(A->nfr - lo) * sizeof(arena_rng));
        A->fr[lo].off = off;
        A->fr[lo].size = sz;
        A->nfr++;
    }
    pthread_mutex_unlock(&A->mu);
}

static int64_t arena_used(sg_arena *A)
{
    int64_t u;
    pthread_mutex_lock(&A->mu);
    u = A->used;
    pthread_mutex_unlock(&A->mu);
    return u;
}

typedef struct srv_grid {
    int64_t id;
    sg_grid *g;
    int64_t bytes;
    uint64_t last_used;
    int pins;  /* queued or running requests */
    int alive;
} srv_grid;

typedef struct srv_req {
    int64_t ticket;
    int gi; /* index in the grid table */
    int d;
    const float *coords;
    float *out;
    int64_t m;
    double t_submit, t_take, t_launch, t_gpu, t_done; /* host clock, ms */
    int state; /* 0 queued, 1 running, 2 done, 3 failed */
    int64_t S;  /* subspaces of the grid (set when batched) */
    int64_t ring_off; /* staged copy of the coordinates in the ring, -1: none */
    int lane;         /* 0 light, 1 heavy (point x subspace pairs >= heavy_pairs) */
    sg_grid *g; /* the grid (set when batched) */
    struct srv_req *next;
} srv_req;

typedef struct srv_slot {
    cudaStream_t st;
    cudaStream_t dst[SG_MAX_DIMS + 1]; /* per dimension: the batch's launches overlap */
    cudaEvent_t done, ev_in, ev_d[SG_MAX_DIMS + 1];
    int busy;
    float *h_coords, *h_out, *d_coords, *d_out;
    float *m_coords, *m_out; /* device addresses of h_coords / h_out (mapped pinned memory) */
    sg_eval_args *h_args, *d_args;
    int32_t *h_items, *d_items;   /* evaluation CTAs, grouped by dimension */
    int32_t *h_citems, *d_citems; /* combine CTAs of the split requests     */
    float *d_part;                /* parts of split sums                    */
    float *d_sorted;              /* heavy slots: Morton-ordered coordinates */
    int32_t *d_perm;              /* heavy slots: sorted position -> point  */
    void *d_sscratch;             /* heavy slots: sort scratch              */
    const float *sort_src[SRV_MAX_REQS]; /* heavy slots: each request's coordinates */
    srv_req *reqs[SRV_MAX_REQS];
    int64_t out_off[SRV_MAX_REQS], coord_off[SRV_MAX_REQS], part_off[SRV_MAX_REQS];
    int order[SRV_MAX_REQS];
    int nreq;
    double t_launch, t_gpu; /* launch_batch returned; completion seen */
    int zero_copy;          /* the server's setting when the batch was taken */
    int sort;               /* the batch's requests are Morton-ordered first */
    int lane;               /* the queue this slot takes its batches from */
} srv_slot;

struct sg_server {
    int dev;
    pthread_mutex_t mu;
    pthread_mutex_t plain_mu; /* serialises sg_server_evaluate_now: a grid handle serves one thread at a time */
    pthread_cond_t cv_work, cv_done;
    pthread_t thr;
    int running, thread_ok;
    srv_grid *grids;
    int ngrids, cap_grids;
    int64_t next_id, cap_bytes;
    sg_arena arena; /* the cap, reserved once; every grid buffer lives here */
    uint64_t clock;
    srv_req *head[2], *tail[2]; /* per lane */
    int64_t queued_points;
    srv_req **by_ticket;
    int64_t next_ticket, cap_tickets;
    int64_t max_points;
    int zero_copy; /* SG_SRV_OPT_ZERO_COPY */
    int64_t heavy_pairs; /* SG_SRV_OPT_HEAVY_PAIRS */
    int light_slots;     /* SG_SRV_OPT_LIGHT_SLOTS */
    int sort_heavy;      /* SG_SRV_OPT_SORT_HEAVY */
    /* staging ring (pinned, mapped): submit copies a request's coordinates
     * here in the caller's thread; allocations are freed in any order and
     * reclaimed from the oldest */
    char *ring, *ring_dev;
    int64_t ring_size, ring_head, ring_tail;
    int64_t *rq_off, *rq_size; /* live allocations in order (circular) */
    char *rq_freed;
    int64_t rq_first, rq_count, rq_cap;
    srv_slot slot[SRV_SLOTS];
    cudaStream_t admit_st;
    int64_t st_batches, st_requests, st_points, st_evictions, st_failed;
    int fatal; /* a CUDA error in the dispatcher: the server is unusable */
};

static int sfail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    sg_set_error(fmt, ap);
    va_end(ap);
    return code;
}

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* Reserves `bytes` (256-aligned) of the staging ring (lock held); returns
 * the offset or -1 when the ring is full. */
static int64_t ring_alloc(sg_server *s, int64_t bytes)
{
    int64_t off;
    bytes = (bytes + 255) & ~(int64_t)255;
    if (!s->ring || bytes > s->ring_size || s->rq_count == s->rq_cap) return -1;
    if (s->rq_count == 0) {
        s->ring_head = s->ring_tail = 0; /* empty */
        off = 0;
    } else if (s->ring_head > s->ring_tail) {
        /* live range [tail, head): free are [head, size) and [0, tail) */
        if (s->ring_size - s->ring_head >= bytes) off = s->ring_head;
        else if (s->ring_tail >= bytes) off = 0;
        else return -1;
    } else {
        /* wrapped: live [tail, size) and [0, head); free is [head, tail) */
        if (s->ring_tail - s->ring_head >= bytes) off = s->ring_head;
        else return -1;
    }
    {
        const int64_t q = (s->rq_first + s->rq_count) % s->rq_cap;
        s->rq_off[q] = off;
        s->rq_size[q] = bytes;
        s->rq_freed[q] = 0;
        s->rq_count++;
    }
    s->ring_head = off + bytes;
    return off;
}

/* Frees the allocation at `off` (lock held) and reclaims freed space from
 * the oldest allocation on. */
static void ring_free(sg_server *s, int64_t off)
{
    int64_t i;
    for (i = 0; i < s->rq_count; i++) {
        const int64_t q = (s->rq_first + i) % s->rq_cap;
        if (!s->rq_freed[q] && s->rq_off[q] == off) {
            s->rq_freed[q] = 1;
            break;
        }
    }
    while (s->rq_count > 0 && s->rq_freed[s->rq_first]) {
        s->rq_first = (s->rq_first + 1) % s->rq_cap;
        s->rq_count--;
    }
    if (s->rq_count > 0) s->ring_tail = s->rq_off[s->rq_first];
    else s->ring_head = s->ring_tail = 0;
}

/* Delivers a finished batch (lock held; the results were copied into the
 * callers' buffers beforehand, outside the lock). */
static void finish_slot(sg_server *s, srv_slot *sl, int ok)
{
    const double t = now_ms();
    int i;
    for (i = 0; i < sl->nreq; i++) {
        srv_req *r = sl->reqs[i];
        r->t_gpu = sl->t_gpu;
        r->t_launch = sl->t_launch;
        r->t_done = t;
        r->state = ok ? 2 : 3;
        if (r->ring_off >= 0) {
            ring_free(s, r->ring_off);
            r->ring_off = -1;
        }
        s->grids[r->gi].pins--;
        if (!ok) s->st_failed++;
    }
    sl->nreq = 0;
    sl->busy = 0;
    pthread_cond_broadcast(&s->cv_done);
}

/* A heavy request with many points is evaluated with whole sums (one CTA
 * per 512 points gives it enough parallelism): split sums would only add
 * the walk's range checks and the combine.  The choice depends on the
 * request alone, so its result is the same in any batch. */
static int whole_sums(const srv_req *r) { return r->lane == 1 && r->m >= SRV_WHOLE_POINTS; }

/* Moves queued requests into slot sl (lock held): pointers and offsets
 * only; returns their count. */
static int take_batch(sg_server *s, srv_slot *sl)
{
    int64_t pts = 0, coff = 0, poff = 0;
    sl->nreq = 0;
    const int ln = sl->lane;
    while (s->head[ln] && sl->nreq < SRV_MAX_REQS) {
        srv_req *r = s->head[ln];
        if (sl->nreq > 0 && pts + r->m > s->max_points) break;
        s->head[ln] = r->next;
        if (!s->head[ln]) s->tail[ln] = NULL;
        s->queued_points -= r->m;
        r->state = 1;
        r->t_take = now_ms();
        r->S = s->grids[r->gi].g->L.S;
        r->g = s->grids[r->gi].g; /* pinned: stays resident until delivered */
        sl->reqs[sl->nreq] = r;
        sl->out_off[sl->nreq] = pts;
        sl->coord_off[sl->nreq] = coff;
        sl->part_off[sl->nreq] = poff;
        if (r->g->nparts > 1 && !whole_sums(r)) poff += r->m * r->g->nparts;
        coff += r->m * r->d;
        pts += r->m;
        sl->nreq++;
    }
    return sl->nreq;
}

/* order[] of a dimension's requests: most subspaces first */
static void sort_by_subspaces(srv_slot *sl, int lo, int hi)
{
    int i, j;
    for (i = lo + 1; i < hi; i++) {
        const int v = sl->order[i];
        const int64_t key = sl->reqs[v]->S;
        for (j = i; j > lo && sl->reqs[sl->order[j - 1]]->S < key; j--) sl->order[j] = sl->order[j - 1];
        sl->order[j] = v;
    }
}

/* Stages the slot's coordinates and kernel arguments (no lock), copies in,
 * forks one launch per dimension onto its own stream, joins, copies out. */
static int launch_batch(sg_server *s, srv_slot *sl)
{
    int64_t coff = 0, pts = 0, ni = 0, nc = 0;
    int i, d, e, no = 0;
    int first[SG_MAX_DIMS + 1], count[SG_MAX_DIMS + 1], ppt[SG_MAX_DIMS + 1];
    const int zc = sl->zero_copy; /* fixed for the batch when it was taken */
    const int sort = sl->sort;    /* heavy lane: spatial ordering of each request's points */
    for (i = 0; i < sl->nreq; i++) {
        srv_req *r = sl->reqs[i];
        int64_t p;
        const float *dc;
        if (zc && r->ring_off >= 0) {
            dc = (const float *)(s->ring_dev + r->ring_off); /* staged at submit, read in place */
        } else {
            memcpy(sl->h_coords + sl->coord_off[i], r->coords, (size_t)(r->m * r->d) * sizeof(float));
            dc = (zc ? sl->m_coords : sl->d_coords) + sl->coord_off[i];
        }
        if (sort) {
            /* evaluated from the request's own Morton-ordered copy; the
             * kernels write each result through the permutation */
            sl->sort_src[i] = dc;
            dc = sl->d_sorted + sl->coord_off[i];
        }
        sg_grid_eval_args(r->g, dc, (zc ? sl->m_out : sl->d_out) + sl->out_off[i], r->m, &sl->h_args[i]);
        if (sort) sl->h_args[i].perm = sl->d_perm + sl->out_off[i];
        if (whole_sums(r)) {
            sl->h_args[i].nparts = 1;
            sl->h_args[i].part_out = NULL;
        }
        if (sl->h_args[i].nparts > 1) {
            sl->h_args[i].part_out = sl->d_part + sl->part_off[i];
            for (p = 0; p < r->m; p += SRV_CTA_THREADS) {
                sl->h_citems[2 * nc] = i;
                sl->h_citems[2 * nc + 1] = (int32_t)p;
                nc++;
            }
        }
        coff += r->m * r->d;
        pts += r->m;
    }
    for (d = 1; d <= SG_MAX_DIMS; d++) {
        const int lo = no;
        int64_t chain = 0, cta;
        first[d] = (int)ni;
        for (i = 0; i < sl->nreq; i++)
            if (sl->reqs[i]->d == d) {
                const int64_t c = sl->reqs[i]->S / sl->h_args[i].nparts;
                sl->order[no++] = i;
                if (c > chain) chain = c;
            }
        sort_by_subspaces(sl, lo, no);
        ppt[d] = (sl->lane == 0 && chain >= SRV_LONG_CHAIN) ? 1 : 2;
        cta = (int64_t)SRV_CTA_THREADS * ppt[d];
        for (i = lo; i < no; i++) {
            const int q = sl->order[i], np = sl->h_args[q].nparts;
            int64_t p;
            int k;
            for (p = 0; p < sl->reqs[q]->m; p += cta)
                for (k = 0; k < np; k++) {
                    sl->h_items[2 * ni] = q | (k << 29);
                    sl->h_items[2 * ni + 1] = (int32_t)p;
                    ni++;
                }
        }
        count[d] = (int)ni - first[d];
    }
    if ((!zc &&
         cudaMemcpyAsync(sl->d_coords, sl->h_coords, (size_t)coff * 4, cudaMemcpyHostToDevice, sl->st) != cudaSuccess) ||
        cudaMemcpyAsync(sl->d_args, sl->h_args, (size_t)sl->nreq * sizeof(sg_eval_args), cudaMemcpyHostToDevice,
                        sl->st) != cudaSuccess ||
        cudaMemcpyAsync(sl->d_items, sl->h_items, (size_t)ni * 8, cudaMemcpyHostToDevice, sl->st) != cudaSuccess ||
        (nc && cudaMemcpyAsync(sl->d_citems, sl->h_citems, (size_t)nc * 8, cudaMemcpyHostToDevice, sl->st) !=
                   cudaSuccess))
        return SG_ERR_CUDA;
    for (i = 0; sort && i < sl->nreq; i++) {
        const srv_req *r = sl->reqs[i];
        /* issued after the copy in, so copied coordinates are in place */
        if (sgk_sort_points(sl->sort_src[i], r->m, r->d, sl->d_sscratch, sl->d_sorted + sl->coord_off[i],
                            sl->d_perm + sl->out_off[i], sl->st) != cudaSuccess)
            return SG_ERR_CUDA;
    }
    if (cudaEventRecord(sl->ev_in, sl->st) != cudaSuccess) return SG_ERR_CUDA;
    for (d = 1; d <= SG_MAX_DIMS; d++) {
        if (!count[d]) continue;
        if (cudaStreamWaitEvent(sl->dst[d], sl->ev_in, 0) != cudaSuccess) return SG_ERR_CUDA;
        e = sgk_evaluate_batch(d, sl->d_args, sl->d_items + 2 * (int64_t)first[d], count[d], ppt[d], 0, sl->dst[d]);
        if (e != cudaSuccess || cudaEventRecord(sl->ev_d[d], sl->dst[d]) != cudaSuccess ||
            cudaStreamWaitEvent(sl->st, sl->ev_d[d], 0) != cudaSuccess)
            return SG_ERR_CUDA;
    }
    if (nc && sgk_combine_parts(sl->d_args, sl->d_citems, (int)nc, sl->st) != cudaSuccess) return SG_ERR_CUDA;
    if ((!zc &&
         cudaMemcpyAsync(sl->h_out, sl->d_out, (size_t)pts * 4, cudaMemcpyDeviceToHost, sl->st) != cudaSuccess) ||
        cudaEventRecord(sl->done, sl->st) != cudaSuccess)
        return SG_ERR_CUDA;
    return SG_OK;
}

/* Copies a finished slot's results into the callers' buffers (no lock:
 * the requests are not visible as done until finish_slot). */
static void deliver(srv_slot *sl)
{
    int i;
    for (i = 0; i < sl->nreq; i++) {
        srv_req *r = sl->reqs[i];
        memcpy(r->out, sl->h_out + sl->out_off[i], (size_t)r->m * sizeof(float));
    }
}

static void *dispatcher(void *arg)
{
    sg_server *s = (sg_server *)arg;
    cudaSetDevice(s->dev);
    pthread_mutex_lock(&s->mu);
    while (s->running) {
        int i, any_busy = 0, free_slot = -1;
        for (i = 0; i < SRV_SLOTS; i++) {
            srv_slot *sl = &s->slot[(s->st_batches + i) % SRV_SLOTS];
            if (sl->busy == 1) {
                cudaError_t q = cudaEventQuery(sl->done);
                if (q == cudaSuccess) {
                    sl->t_gpu = now_ms();
                    sl->busy = 2; /* delivering: not free, not polled */
                    pthread_mutex_unlock(&s->mu);
                    deliver(sl);
                    pthread_mutex_lock(&s->mu);
                    finish_slot(s, sl, 1);
                } else if (q != cudaErrorNotReady) {
                    finish_slot(s, sl, 0);
                    s->fatal = 1;
                }
            }
        }
        /* light lane first: its slots run at the higher stream priority */
        for (i = 0; i < SRV_SLOTS; i++) {
            if (s->slot[i].busy) any_busy = 1;
            else if (free_slot < 0 && s->head[s->slot[i].lane] && (s->slot[i].lane || i < s->light_slots))
                free_slot = i;
        }
        if (free_slot >= 0 && !s->fatal) {
            srv_slot *sl = &s->slot[free_slot];
            take_batch(s, sl);
            sl->zero_copy = s->zero_copy;
            sl->sort = sl->lane == 1 && s->sort_heavy && sl->d_sorted != NULL;
            sl->busy = 1;
            s->st_batches++;
            s->st_requests += sl->nreq;
            pthread_mutex_unlock(&s->mu);
            i = launch_batch(s, sl);
            sl->t_launch = now_ms();
            pthread_mutex_lock(&s->mu);
            if (i != SG_OK) {
                finish_slot(s, sl, 0);
                s->fatal = 1;
            }
            continue;
        }
        if (any_busy) {
            /* poll the running batches, wake early on new work */
            struct timespec ts;
            clock_gettime(CLOCK_REALTIME, &ts);
            ts.tv_nsec += 20000;
            if (ts.tv_nsec >= 1000000000L) {
                ts.tv_sec++;
                ts.tv_nsec -= 1000000000L;
            }
            pthread_cond_timedwait(&s->cv_work, &s->mu, &ts);
        } else {
            pthread_cond_wait(&s->cv_work, &s->mu);
        }
    }
    /* drain: wait for running batches, fail what is still queued */
    for (int i = 0; i < SRV_SLOTS; i++)
        if (s->slot[i].busy) {
            int ok;
            pthread_mutex_unlock(&s->mu);
            ok = cudaEventSynchronize(s->slot[i].done) == cudaSuccess;
            s->slot[i].t_gpu = now_ms();
            if (ok) deliver(&s->slot[i]);
            pthread_mutex_lock(&s->mu);
            finish_slot(s, &s->slot[i], ok);
        }
    for (int ln = 0; ln < 2; ln++) {
        while (s->head[ln]) {
            srv_req *r = s->head[ln];
            s->head[ln] = r->next;
            r->state = 3;
            s->grids[r->gi].pins--;
        }
        s->tail[ln] = NULL;
    }
    pthread_cond_broadcast(&s->cv_done);
    pthread_mutex_unlock(&s->mu);
    return NULL;
}

static void free_slots(sg_server *s)
{
    int i, d;
    for (i = 0; i < SRV_SLOTS; i++) {
        srv_slot *sl = &s->slot[i];
        if (sl->st) cudaStreamDestroy(sl->st);
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->ev_in) cudaEventDestroy(sl->ev_in);
        for (d = 0; d <= SG_MAX_DIMS; d++) {
            if (sl->dst[d]) cudaStreamDestroy(sl->dst[d]);
            if (sl->ev_d[d]) cudaEventDestroy(sl->ev_d[d]);
        }
        cudaFreeHost(sl->h_coords);
        cudaFreeHost(sl->h_out);
        cudaFreeHost(sl->h_args);
        cudaFreeHost(sl->h_items);
        cudaFreeHost(sl->h_citems);
        cudaFree(sl->d_citems);
        cudaFree(sl->d_part);
        cudaFree(sl->d_sorted);
        cudaFree(sl->d_perm);
        cudaFree(sl->d_sscratch);
        cudaFree(sl->d_coords);
        cudaFree(sl->d_out);
        cudaFree(sl->d_args);
        cudaFree(sl->d_items);
    }
}

SG_API int sg_server_create(int64_t hbm_cap_bytes, int64_t max_batch_points, sg_server **out)
{
    sg_server *s;
    int i, prio_low = 0, prio_high = 0;
    int64_t max_items;
    if (!out || hbm_cap_bytes <= 0 || max_batch_points < 1 || max_batch_points > ((int64_t)1 << 28))
        return sfail(SG_ERR_ARG, "sg_server_create: bad argument");
    *out = NULL;
    s = (sg_server *)calloc(1, sizeof(sg_server));
    if (!s) return sfail(SG_ERR_NOMEM, "sg_server_create: out of host memory");
    if (cudaGetDevice(&s->dev) != cudaSuccess || sgk_eval_setup() != cudaSuccess) {
        free(s);
        return sfail(SG_ERR_CUDA, "sg_server_create: no CUDA device");
    }
    s->cap_bytes = hbm_cap_bytes;
    s->max_points = max_batch_points;
    s->zero_copy = 1;
    s->heavy_pairs = SRV_HEAVY_PAIRS;
    s->light_slots = SRV_LIGHT_SLOTS;
    s->sort_heavy = 1;
    max_items = ((max_batch_points + SRV_CTA_THREADS - 1) / SRV_CTA_THREADS + SRV_MAX_REQS) * SG_EVAL_MAX_PARTS;
    pthread_mutex_init(&s->mu, NULL);
    pthread_mutex_init(&s->plain_mu, NULL);
    pthread_cond_init(&s->cv_work, NULL);
    pthread_cond_init(&s->cv_done, NULL);
    /* batches run at the highest stream priority and admissions at the
     * lowest, so a long hierarchization of a new grid yields SMs to the
     * evaluation batches as its CTAs retire */
    if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) prio_low = prio_high = 0;
    for (i = 0; i < SRV_SLOTS; i++) {
        srv_slot *sl = &s->slot[i];
        const size_t cb = (size_t)max_batch_points * SG_MAX_DIMS * 4, ob = (size_t)max_batch_points * 4;
        int ok = 1, d;
        /* light batches at the highest priority, heavy ones one step below
         * (still above admissions): as CTAs retire, light work takes SMs
         * before the remaining CTAs of a heavy batch */
        const int prio = i < SRV_LIGHT_SLOTS ? prio_high : (prio_high < prio_low ? prio_high + 1 : prio_high);
        sl->lane = i < SRV_LIGHT_SLOTS ? 0 : 1;
        for (d = 1; d <= SG_MAX_DIMS && ok; d++)
            ok = cudaStreamCreateWithPriority(&sl->dst[d], cudaStreamNonBlocking, prio) == cudaSuccess &&
                 cudaEventCreateWithFlags(&sl->ev_d[d], cudaEventDisableTiming) == cudaSuccess;
        if (!ok || cudaStreamCreateWithPriority(&sl->st, cudaStreamNonBlocking, prio) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl->ev_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_coords, cb) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_out, ob) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_args, SRV_MAX_REQS * sizeof(sg_eval_args)) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_items, (size_t)max_items * 8) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_citems, (size_t)max_items * 8) != cudaSuccess ||
            cudaMalloc((void **)&sl->d_citems, (size_t)max_items * 8) != cudaSuccess ||
            cudaMalloc((void **)&sl->d_part, ob * SG_EVAL_MAX_PARTS) != cudaSuccess ||
            cudaMalloc((void **)&sl->d_coords, cb) != cudaSuccess || cudaMalloc((void **)&sl->d_out, ob) != cudaSuccess ||
            cudaMalloc((void **)&sl->d_args, SRV_MAX_REQS * sizeof(sg_eval_args)) != cudaSuccess ||
            cudaMalloc((void **)&sl->d_items, (size_t)max_items * 8) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&sl->m_coords, sl->h_coords, 0) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&sl->m_out, sl->h_out, 0) != cudaSuccess ||
            (sl->lane == 1 &&
             (cudaMalloc((void **)&sl->d_sorted, cb) != cudaSuccess ||
              cudaMalloc((void **)&sl->d_perm, ob) != cudaSuccess ||
              cudaMalloc(&sl->d_sscratch, (size_t)sgk_sort_scratch_bytes(max_batch_points, SG_MAX_DIMS)) !=
                  cudaSuccess))) {
            cudaGetLastError();
            free_slots(s);
            free(s);
            return sfail(SG_ERR_NOMEM, "sg_server_create: cannot allocate batch buffers for %lld points",
                         (long long)max_batch_points);
        }
    }
    if (cudaStreamCreateWithPriority(&s->admit_st, cudaStreamNonBlocking, prio_low) != cudaSuccess) {
        free_slots(s);
        free(s);
        return sfail(SG_ERR_CUDA, "sg_server_create: stream");
    }
    /* staging ring for zero-copy batches: room for SRV_RING_BATCHES full
     * batches of 20-dimensional points (optional: without it, zero-copy
     * batches stage in the dispatcher as the copying ones do) */
    s->ring_size = SRV_RING_BATCHES * max_batch_points * SG_MAX_DIMS * (int64_t)sizeof(float);
    s->rq_cap = SRV_RING_BATCHES * SRV_MAX_REQS;
    s->rq_off = (int64_t *)malloc((size_t)s->rq_cap * sizeof(int64_t));
    s->rq_size = (int64_t *)malloc((size_t)s->rq_cap * sizeof(int64_t));
    s->rq_freed = (char *)malloc((size_t)s->rq_cap);
    if (!s->rq_off || !s->rq_size || !s->rq_freed || cudaMallocHost((void **)&s->ring, (size_t)s->ring_size) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&s->ring_dev, s->ring, 0) != cudaSuccess) {
        cudaGetLastError();
        if (s->ring) cudaFreeHost(s->ring);
        s->ring = s->ring_dev = NULL;
        s->ring_size = 0;
    }
    pthread_mutex_init(&s->arena.mu, NULL);
    s->arena.size = hbm_cap_bytes & ~(int64_t)(ARENA_ALIGN - 1);
    if (s->arena.size < ARENA_ALIGN || cudaMalloc((void **)&s->arena.base, (size_t)s->arena.size) != cudaSuccess ||
        !rng_reserve(&s->arena.fr, &s->arena.capfr, 1)) {
        cudaGetLastError();
        cudaStreamDestroy(s->admit_st);
        free_slots(s);
        free(s->arena.fr);
        free(s);
        return sfail(SG_ERR_NOMEM, "sg_server_create: cannot reserve %lld device bytes for resident grids",
                     (long long)hbm_cap_bytes);
    }
    s->arena.fr[0].off = 0;
    s->arena.fr[0].size = s->arena.size;
    s->arena.nfr = 1;
    s->running = 1;
    if (pthread_create(&s->thr, NULL, dispatcher, s) != 0) {
        cudaStreamDestroy(s->admit_st);
        free_slots(s);
        cudaFree(s->arena.base);
        free(s->arena.fr);
        free(s);
        return sfail(SG_ERR_STATE, "sg_server_create: cannot start the dispatcher thread");
    }
    s->thread_ok = 1;
    *out = s;
    return SG_OK;
}

SG_API int sg_server_destroy(sg_server *s)
{
    int i;
    int64_t t;
    if (!s) return SG_OK;
    pthread_mutex_lock(&s->mu);
    s->running = 0;
    pthread_cond_broadcast(&s->cv_work);
    pthread_mutex_unlock(&s->mu);
    if (s->thread_ok) pthread_join(s->thr, NULL);
    for (i = 0; i < s->ngrids; i++)
        if (s->grids[i].alive) sg_destroy(s->grids[i].g);
    for (t = 0; t < s->next_ticket; t++) free(s->by_ticket[t]);
    free(s->by_ticket);
    free(s->grids);
    cudaStreamDestroy(s->admit_st);
    free_slots(s);
    if (s->ring) cudaFreeHost(s->ring);
    free(s->rq_off);
    free(s->rq_size);
    free(s->rq_freed);
    cudaFree(s->arena.base);
    free(s->arena.fr);
    free(s->arena.live);
    pthread_mutex_destroy(&s->arena.mu);
    pthread_cond_destroy(&s->cv_work);
    pthread_cond_destroy(&s->cv_done);
    pthread_mutex_destroy(&s->mu);
    pthread_mutex_destroy(&s->plain_mu);
    free(s);
    return SG_OK;
}

/* device bytes a grid will take once resident (values, block layout and
 * tables), from its host layout */
static int64_t grid_bytes_estimate(const sg_layout *L)
{
    return L->Npad * 4 + L->Nblk * 4 + L->S * (int64_t)(sizeof(sg_repack) + 12 * L->d) + (1 << 16);
}

/* Evicts the least recently used grid that no request needs (lock held);
 * returns 0 if every resident grid is pinned. */
static int evict_one(sg_server *s)
{
    int i, victim = -1;
    for (i = 0; i < s->ngrids; i++) {
        const srv_grid *e = &s->grids[i];
        if (e->alive && e->pins == 0 && (victim < 0 || e->last_used < s->grids[victim].last_used)) victim = i;
    }
    if (victim < 0) return 0;
    sg_destroy(s->grids[victim].g); /* returns its ranges to the arena: no driver call */
    s->grids[victim].g = NULL;
    s->grids[victim].alive = 0;
    s->st_evictions++;
    return 1;
}

/* Creates, samples and hierarchizes a grid in the arena and builds its
 * evaluation layout, all on the admission stream. */
static int build_grid(sg_server *s, int d, int n, const int *limits, int fn, const double *params, int num_params,
                      sg_grid **out)
{
    sg_grid *g = NULL;
    int r = sg_create_with_allocator(d, n, limits, arena_alloc, arena_free, &s->arena, &g);
    if (r == SG_OK) r = sg_sample_function(g, fn, params, num_params, s->admit_st);
    if (r == SG_OK) r = sg_hierarchize_async(g, s->admit_st);
    if (r == SG_OK) r = sg_grid_prepare_eval(g, s->admit_st);
    if (r == SG_OK && d >= 4 && g->L.S >= SRV_SPLIT_SUBSPACES) {
        const int64_t np = g->L.S / SRV_PART_SUBSPACES;
        r = sg_grid_set_parts(g, np > SG_EVAL_MAX_PARTS ? SG_EVAL_MAX_PARTS : (int)np, s->admit_st);
    }
    if (r == SG_OK) r = sg_sync(g, s->admit_st);
    if (r != SG_OK) {
        if (g) {
            cudaStreamSynchronize(s->admit_st); /* nothing of g may still run when its ranges are reused */
            sg_destroy(g);
        }
        return r;
    }
    *out = g;
    return SG_OK;
}

SG_API int sg_server_add_grid(sg_server *s, int d, int n, const int *limits, int fn, const double *params,
                              int num_params, int64_t *grid_id)
{
    sg_grid *g = NULL;
    sg_layout L;
    int64_t est, bytes = 0;
    int r, slot;
    if (!s || !grid_id) return sfail(SG_ERR_ARG, "sg_server_add_grid: NULL argument");
    if ((r = sg_layout_init(&L, d, n, limits)) != SG_OK) return sfail(r, "sg_server_add_grid: bad grid shape");
    est = grid_bytes_estimate(&L);
    if (est > s->arena.size)
        return sfail(SG_ERR_NOMEM, "sg_server_add_grid: %lld bytes exceed the cap %lld", (long long)est,
                     (long long)s->arena.size);
    pthread_mutex_lock(&s->mu);
    while (arena_used(&s->arena) + est > s->arena.size)
        if (!evict_one(s)) break;
    pthread_mutex_unlock(&s->mu);
    for (;;) {
        int evicted;
        r = build_grid(s, d, n, limits, fn, params, num_params, &g);
        if (r != SG_ERR_NOMEM) break;
        /* the free ranges were too fragmented (or another admission took
         * them): evict one more grid and try again */
        pthread_mutex_lock(&s->mu);
        evicted = evict_one(s);
        pthread_mutex_unlock(&s->mu);
        if (!evicted)
            return sfail(SG_ERR_NOMEM, "sg_server_add_grid: %lld bytes do not fit under the cap (%lld used of %lld)",
                         (long long)est, (long long)arena_used(&s->arena), (long long)s->arena.size);
    }
    if (r != SG_OK) return r;
    sg_device_bytes(g, &bytes);

    pthread_mutex_lock(&s->mu);
    if (s->ngrids == s->cap_grids) {
        int nc = s->cap_grids ? 2 * s->cap_grids : 64;
        srv_grid *ng = (srv_grid *)realloc(s->grids, (size_t)nc * sizeof(srv_grid));
        if (!ng) {
            pthread_mutex_unlock(&s->mu);
            sg_destroy(g);
            return sfail(SG_ERR_NOMEM, "sg_server_add_grid: out of host memory");
        }
        s->grids = ng;
        s->cap_grids = nc;
    }
    slot = s->ngrids++;
    s->grids[slot].id = s->next_id++;
    s->grids[slot].g = g;
    s->grids[slot].bytes = bytes;
    s->grids[slot].last_used = ++s->clock;
    s->grids[slot].pins = 0;
    s->grids[slot].alive = 1;
    *grid_id = s->grids[slot].id;
    pthread_mutex_unlock(&s->mu);
    return SG_OK;
}

static int find_grid(const sg_server *s, int64_t id)
{
    /* ids are handed out in table order */
    if (id < 0 || id >= s->ngrids || s->grids[id].id != id) return -1;
    return (int)id;
}

SG_API int sg_server_submit(sg_server *s, int64_t grid_id, const float *coord_mat, int64_t num_evals, float *out,
                            int64_t *ticket)
{
    srv_req *r;
    int gi;
    if (!s || !ticket || num_evals < 1 || !coord_mat || !out) return sfail(SG_ERR_ARG, "sg_server_submit: bad argument");
    if (num_evals > s->max_points)
        return sfail(SG_ERR_RANGE, "sg_server_submit: %lld points exceed the batch capacity %lld", (long long)num_evals,
                     (long long)s->max_points);
    r = (srv_req *)calloc(1, sizeof(srv_req));
    if (!r) return sfail(SG_ERR_NOMEM, "sg_server_submit: out of host memory");
    pthread_mutex_lock(&s->mu);
    gi = find_grid(s, grid_id);
    if (gi < 0 || !s->grids[gi].alive || s->fatal) {
        pthread_mutex_unlock(&s->mu);
        free(r);
        return sfail(s->fatal ? SG_ERR_CUDA : SG_ERR_ARG, "sg_server_submit: grid %lld is not resident",
                     (long long)grid_id);
    }
    if (s->next_ticket == s->cap_tickets) {
        int64_t nc = s->cap_tickets ? 2 * s->cap_tickets : 4096;
        srv_req **nb = (srv_req **)realloc(s->by_ticket, (size_t)nc * sizeof(srv_req *));
        if (!nb) {
            pthread_mutex_unlock(&s->mu);
            free(r);
            return sfail(SG_ERR_NOMEM, "sg_server_submit: out of host memory");
        }
        s->by_ticket = nb;
        s->cap_tickets = nc;
    }
    r->ticket = s->next_ticket++;
    s->by_ticket[r->ticket] = r;
    r->gi = gi;
    r->d = s->grids[gi].g->L.d;
    r->coords = coord_mat;
    r->out = out;
    r->m = num_evals;
    r->t_submit = now_ms();
    s->grids[gi].pins++;
    s->grids[gi].last_used = ++s->clock;
    r->ring_off = s->zero_copy ? ring_alloc(s, num_evals * r->d * (int64_t)sizeof(float)) : -1;
    if (r->ring_off >= 0) {
        /* stage the coordinates in the caller's thread, outside the lock:
         * the request is not queued yet, so nothing else reads the range */
        pthread_mutex_unlock(&s->mu);
        memcpy(s->ring + r->ring_off, coord_mat, (size_t)(num_evals * r->d) * sizeof(float));
        pthread_mutex_lock(&s->mu);
    }
    r->lane = (double)num_evals * (double)s->grids[gi].g->L.S >= (double)s->heavy_pairs ? 1 : 0;
    if (s->tail[r->lane]) s->tail[r->lane]->next = r;
    else s->head[r->lane] = r;
    s->tail[r->lane] = r;
    s->queued_points += num_evals;
    s->st_points += num_evals;
    *ticket = r->ticket;
    pthread_cond_signal(&s->cv_work);
    pthread_mutex_unlock(&s->mu);
    return SG_OK;
}

SG_API int sg_server_wait(sg_server *s, int64_t ticket, double *latency_ms)
{
    double ms[5];
    int r = sg_server_wait_detail(s, ticket, ms);
    if (latency_ms) *latency_ms = ms[4];
    return r;
}

SG_API int sg_server_wait_detail(sg_server *s, int64_t ticket, double *ms)
{
    srv_req *r;
    int st;
    if (!s) return sfail(SG_ERR_ARG, "sg_server_wait: NULL server");
    pthread_mutex_lock(&s->mu);
    if (ticket < 0 || ticket >= s->next_ticket || !(r = s->by_ticket[ticket])) {
        pthread_mutex_unlock(&s->mu);
        return sfail(SG_ERR_ARG, "sg_server_wait: unknown or already collected ticket %lld", (long long)ticket);
    }
    while (r->state < 2) pthread_cond_wait(&s->cv_done, &s->mu);
    st = r->state;
    if (ms) {
        ms[0] = r->t_take - r->t_submit;
        ms[1] = r->t_launch - r->t_submit;
        ms[2] = r->t_gpu - r->t_submit;
        ms[3] = (double)r->m * (double)r->S;
        ms[4] = r->t_done - r->t_submit;
    }
    s->by_ticket[ticket] = NULL;
    pthread_mutex_unlock(&s->mu);
    free(r);
    return st == 2 ? SG_OK : sfail(SG_ERR_CUDA, "sg_server_wait: the request failed");
}

SG_API int sg_server_set_option(sg_server *s, int option, int64_t value)
{
    if (!s) return sfail(SG_ERR_ARG, "sg_server_set_option: NULL server");
    switch (option) {
    case SG_SRV_OPT_ZERO_COPY:
        if (value != 0 && value != 1) return sfail(SG_ERR_ARG, "SG_SRV_OPT_ZERO_COPY is 0 or 1");
        pthread_mutex_lock(&s->mu);
        s->zero_copy = (int)value;
        pthread_mutex_unlock(&s->mu);
        return SG_OK;
    case SG_SRV_OPT_LIGHT_SLOTS:
        if (value < 1 || value > SRV_LIGHT_SLOTS) return sfail(SG_ERR_ARG, "SG_SRV_OPT_LIGHT_SLOTS is 1 .. %d", SRV_LIGHT_SLOTS);
        pthread_mutex_lock(&s->mu);
        s->light_slots = (int)value;
        pthread_mutex_unlock(&s->mu);
        return SG_OK;
    case SG_SRV_OPT_SORT_HEAVY:
        if (value != 0 && value != 1) return sfail(SG_ERR_ARG, "SG_SRV_OPT_SORT_HEAVY is 0 or 1");
        pthread_mutex_lock(&s->mu);
        s->sort_heavy = (int)value;
        pthread_mutex_unlock(&s->mu);
        return SG_OK;
    case SG_SRV_OPT_HEAVY_PAIRS:
        if (value < 1) return sfail(SG_ERR_ARG, "SG_SRV_OPT_HEAVY_PAIRS is >= 1");
        pthread_mutex_lock(&s->mu);
        s->heavy_pairs = value;
        pthread_mutex_unlock(&s->mu);
        return SG_OK;
    default:
        return sfail(SG_ERR_ARG, "sg_server_set_option: unknown option %d", option);
    }
}

SG_API int sg_server_stats(sg_server *s, int64_t *stats)
{
    int i;
    int64_t resident = 0;
    if (!s || !stats) return sfail(SG_ERR_ARG, "sg_server_stats: NULL argument");
    pthread_mutex_lock(&s->mu);
    for (i = 0; i < s->ngrids; i++) resident += s->grids[i].alive;
    stats[0] = s->st_batches;
    stats[1] = s->st_requests;
    stats[2] = s->st_points;
    stats[3] = s->st_evictions;
    stats[4] = resident;
    stats[5] = arena_used(&s->arena);
    stats[6] = s->st_failed;
    pthread_mutex_unlock(&s->mu);
    return SG_OK;
}

SG_API int sg_server_evaluate_now(sg_server *s, int64_t grid_id, const float *coord_mat, int64_t num_evals, float *out)
{
    /* the plain arrangement, for comparison: this one request alone through
     * the single-grid host-buffer call */
    int gi, r;
    sg_grid *g;
    if (!s) return sfail(SG_ERR_ARG, "sg_server_evaluate_now: NULL server");
    pthread_mutex_lock(&s->mu);
    gi = find_grid(s, grid_id);
    if (gi < 0 || !s->grids[gi].alive) {
        pthread_mutex_unlock(&s->mu);
        return sfail(SG_ERR_ARG, "sg_server_evaluate_now: grid %lld is not resident", (long long)grid_id);
    }
    g = s->grids[gi].g;
    s->grids[gi].pins++;
    s->grids[gi].last_used = ++s->clock;
    pthread_mutex_unlock(&s->mu);
    pthread_mutex_lock(&s->plain_mu);
    r = sg_evaluate(g, coord_mat, out, num_evals);
    pthread_mutex_unlock(&s->plain_mu);
    pthread_mutex_lock(&s->mu);
    s->grids[gi].pins--;
    pthread_mutex_unlock(&s->mu);
    return r;
}
