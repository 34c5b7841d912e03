/*
 * ag_runtime.cu -- device context, graph upload and work planning, the
 * CUDA-graph iteration loop and the status-returning entry points.
 *
 * Replaces the reference's accelerator runtime for this path
 * (02_capi_graph/src/capi_utils/capienv.c: mapGraphCSRToWED :832-874,
 * setupAFUGraphCSR :329-372, startAFU/startCU/waitAFU :375-638,
 * releaseAFU :765-782).  Where the reference crosses the host/accelerator
 * boundary twice per iteration (startCU + waitAFU, pageRank.c:1041-1046),
 * a solve here is one cudaGraphLaunch: init kernel -> WHILE(condition){pull
 * pass} -> normalise, with the condition set on the device by the pass that
 * converged or reached the iteration cap.  Host waits are bounded
 * (AG_WAIT_TIMEOUT_S), after the pattern of the reference's watchdog
 * (accelerator_verification.c:177-320), and return AG_ERR_TIMEOUT instead of
 * exiting.
 */
#include <cuda_runtime.h>
#include <omp.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <vector>

#include "ag_device.h"
#include "ag_internal.h"

/* ------------------------------------------------------------ context */
struct AgContext
{
    int ready;
    int device;
    int num_sms;
    cudaStream_t stream;
};

static AgContext g_ctx = {0, -1, 0, nullptr};

#define AG_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return cudaGetLastError(), ag_set_error(AG_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                __FILE__, __LINE__);                                           \
    } while (0)

static ag_status_t ctx_ensure(int want_device)
{
    if (g_ctx.ready && (want_device < 0 || want_device == g_ctx.device)) {
        /* a call from another host thread: make the library's device the
         * current one there too */
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != g_ctx.device)
            AG_CUDA(cudaSetDevice(g_ctx.device));
        return AG_OK;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return ag_set_error(AG_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    int dev = want_device;
    if (dev < 0)
        AG_CUDA(cudaGetDevice(&dev));
    if (dev >= n)
        return ag_set_error(AG_ERR_INVALID_ARG, "device %d out of range (%d devices)", dev, n);
    AG_CUDA(cudaSetDevice(dev));
    if (g_ctx.ready && g_ctx.stream) {
        cudaStreamDestroy(g_ctx.stream);
        g_ctx.stream = nullptr;
    }
    AG_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
    AG_CUDA(cudaDeviceGetAttribute(&g_ctx.num_sms, cudaDevAttrMultiProcessorCount, dev));
    /* keep freed stream-ordered allocations in this process's pool so that
     * repeated uploads reuse them */
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    g_ctx.device = dev;
    g_ctx.ready = 1;
    return AG_OK;
}

extern "C" ag_status_t ag_init(int device)
{
    ag_clear_error();
    return ctx_ensure(device);
}

extern "C" void *ag_stream(void)
{
    if (ctx_ensure(-1) != AG_OK)
        return nullptr;
    return (void *)g_ctx.stream;
}

/* launch on a caller-owned stream from now on (NULL: back to the library's
 * own stream); the caller keeps the stream alive while the library uses it */
static cudaStream_t g_own_stream = nullptr;
extern "C" ag_status_t ag_set_stream(void *stream)
{
    ag_status_t st = ctx_ensure(-1);
    if (st != AG_OK)
        return st;
    AG_CUDA(cudaStreamSynchronize(g_ctx.stream));
    if (!g_own_stream)
        g_own_stream = g_ctx.stream;
    g_ctx.stream = stream ? (cudaStream_t)stream : g_own_stream;
    return AG_OK;
}

extern "C" int ag_num_sms(void)
{
    if (ctx_ensure(-1) != AG_OK)
        return 0;
    return g_ctx.num_sms;
}

extern "C" const char *ag_version(void) { return "accelgraph-b200 0.1 sm_100a"; }

static double wait_limit_s(double timeout_s)
{
    if (timeout_s > 0)
        return timeout_s;
    const char *env = getenv("AG_WAIT_TIMEOUT_S");
    if (env) {
        double v = atof(env);
        if (v > 0)
            return v;
    }
    return 600.0;
}

/* bounded wait: poll the stream until it drains or the deadline passes */
static ag_status_t stream_wait(cudaStream_t s, double timeout_s)
{
    const double limit = wait_limit_s(timeout_s);
    const double t0 = ag_wall_seconds();
    unsigned spins = 0;
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess)
            return AG_OK;
        if (e != cudaErrorNotReady)
            return ag_set_error(AG_ERR_CUDA, "stream failed: %s", cudaGetErrorString(e));
        if (ag_wall_seconds() - t0 > limit)
            return ag_set_error(AG_ERR_TIMEOUT, "device work did not finish within %.1f s", limit);
        if (++spins > 64) {
            struct timespec ts = {0, 20000};
            nanosleep(&ts, nullptr);
        }
    }
}

extern "C" ag_status_t ag_synchronize(double timeout_s)
{
    ag_status_t st = ctx_ensure(-1);
    if (st != AG_OK)
        return st;
    return stream_wait(g_ctx.stream, timeout_s);
}

extern "C" void *ag_rt_host_alloc(size_t bytes, int pinned, int *got_pinned)
{
    *got_pinned = 0;
    if (pinned && ctx_ensure(-1) == AG_OK) {
        void *p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) == cudaSuccess) {
            *got_pinned = 1;
            return p;
        }
        cudaGetLastError();
    }
    return malloc(bytes);
}

/* frees either kind: a graph whose page-locked allocations ran out part way
 * holds both, so the kind is asked per pointer, `pinned` being a hint */
extern "C" void ag_rt_host_free(void *ptr, int pinned)
{
    if (!ptr)
        return;
    bool page_locked = false;
    if (g_ctx.ready) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) == cudaSuccess)
            page_locked = at.type == cudaMemoryTypeHost;
        else
            cudaGetLastError();
    } else {
        page_locked = pinned != 0;
    }
    if (page_locked)
        cudaFreeHost(ptr);
    else
        free(ptr);
}

/* ------------------------------------------------ device-to-host copies */
#define AG_STAGE_CHUNK ((size_t)4 << 20)

static struct
{
    unsigned char *buf; /* two page-locked chunks */
    cudaEvent_t ev[2];
    int state;          /* 0: not set up, 1: ready, -1: unavailable */
} g_stage = {nullptr, {nullptr, nullptr}, 0};

static ag_status_t event_wait(cudaEvent_t ev, double timeout_s)
{
    const double limit = wait_limit_s(timeout_s);
    const double t0 = ag_wall_seconds();
    unsigned spins = 0;
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess)
            return AG_OK;
        if (e != cudaErrorNotReady)
            return ag_set_error(AG_ERR_CUDA, "device copy failed: %s", cudaGetErrorString(e));
        if (ag_wall_seconds() - t0 > limit)
            return ag_set_error(AG_ERR_TIMEOUT, "device copy did not finish within %.1f s", limit);
        if (++spins > 64) {
            struct timespec ts = {0, 5000};
            nanosleep(&ts, nullptr);
        }
    }
}

/* host memcpy split over up to 16 OpenMP threads (one thread copies about
 * 10 GB/s; the device link moves about 50 GB/s) */
static void par_memcpy(void *dst, const void *src, size_t n)
{
    const int nt = std::min(16, omp_get_max_threads());
    if (n < ((size_t)1 << 20) || nt <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t piece = ((n + (size_t)nt - 1) / (size_t)nt + 4095) & ~(size_t)4095;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int t = 0; t < nt; ++t) {
        const size_t a = (size_t)t * piece;
        if (a < n)
            memcpy((unsigned char *)dst + a, (const unsigned char *)src + a, std::min(piece, n - a));
    }
}

/* Copy `bytes` of device memory to host memory `dst` on the library stream
 * and wait for it (bounded).  A page-locked destination is copied directly;
 * a pageable one goes through two page-locked chunks, so that the device
 * copy of one chunk overlaps the host copy of the other. */
static ag_status_t copy_to_host(void *dst, const void *src, size_t bytes)
{
    cudaStream_t s = g_ctx.stream;
    if (!bytes)
        return AG_OK;
    cudaPointerAttributes at;
    bool pinned = false;
    if (cudaPointerGetAttributes(&at, dst) == cudaSuccess)
        pinned = at.type == cudaMemoryTypeHost;
    else
        cudaGetLastError();
    if (!pinned && bytes >= ((size_t)1 << 20) && g_stage.state == 0) {
        g_stage.state = -1;
        void *p = nullptr;
        if (cudaHostAlloc(&p, 2 * AG_STAGE_CHUNK, cudaHostAllocDefault) == cudaSuccess) {
            if (cudaEventCreateWithFlags(&g_stage.ev[0], cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&g_stage.ev[1], cudaEventDisableTiming) == cudaSuccess) {
                g_stage.buf = (unsigned char *)p;
                g_stage.state = 1;
            } else {
                cudaFreeHost(p);
            }
        }
        cudaGetLastError();
    }
    if (pinned || bytes < ((size_t)1 << 20) || g_stage.state != 1) {
        AG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        return stream_wait(s, 0);
    }
    unsigned char *d = (unsigned char *)dst;
    const unsigned char *sp = (const unsigned char *)src;
    const size_t nch = (bytes + AG_STAGE_CHUNK - 1) / AG_STAGE_CHUNK;
    auto len = [&](size_t k) { return std::min(AG_STAGE_CHUNK, bytes - k * AG_STAGE_CHUNK); };
    auto issue = [&](size_t k) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(g_stage.buf + (k & 1) * AG_STAGE_CHUNK, sp + k * AG_STAGE_CHUNK, len(k),
                                        cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaEventRecord(g_stage.ev[k & 1], s) : e;
    };
    AG_CUDA(issue(0));
    for (size_t k = 0; k < nch; ++k) {
        /* chunk k + 1 reuses the buffer chunk k - 1 was copied out of */
        if (k + 1 < nch)
            AG_CUDA(issue(k + 1));
        ag_status_t st = event_wait(g_stage.ev[k & 1], 0);
        if (st != AG_OK)
            return st;
        par_memcpy(d + k * AG_STAGE_CHUNK, g_stage.buf + (k & 1) * AG_STAGE_CHUNK, len(k));
    }
    return AG_OK;
}

/* ------------------------------------------------------- graph handle */
/* the integer pulls, AG_PREC_FIXED64 .. AG_PREC_QUANT8: contribution width in
 * bytes and whether the form is quantised */
#define AG_NUM_INT_FORMS (AG_PREC_QUANT8 - AG_PREC_FIXED64 + 1)

static int is_int_prec(int prec) { return prec >= AG_PREC_FIXED64 && prec <= AG_PREC_QUANT8; }

static int int_bytes(int prec)
{
    switch (prec) {
    case AG_PREC_FIXED32: case AG_PREC_QUANT32: return 4;
    case AG_PREC_FIXED16: case AG_PREC_QUANT16: return 2;
    case AG_PREC_FIXED8: case AG_PREC_QUANT8: return 1;
    default: return 8;
    }
}

static int int_quant(int prec) { return prec >= AG_PREC_QUANT32 && prec <= AG_PREC_QUANT8; }

struct AgExec
{
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaGraphNode_t init_node;
    cudaGraphConditionalHandle cond;
    AgPullParams params;
    unsigned grid;
};

struct ag_graph_s
{
    uint32_t N, E, E4;
    uint32_t *row_off, *ids, *outdeg;
    float *w;
    uint32_t *perm, *inv;   /* relabelling (NULL with AG_UPLOAD_KEEP_ORDER)  */
    float *out;             /* normalised ranks, caller order                */
    float *xbuf, *ybuf;     /* SpMV vectors in device order                  */
    uint32_t hot_n;         /* entries of the shared-memory hot table        */
    uint32_t warm_n;        /* ids below this may allocate L1 lines          */
    ag_tile_config tiles;   /* work-list and cache shape in use              */
    uint32_t hot_allowed;   /* 0 when uploaded with AG_UPLOAD_NO_SMEM_CACHE  */
    uint32_t c_base;        /* partitioned solve: this rank's slice offset    */
    uint32_t norm_n;        /* partitioned solve: global vertex count         */
    std::vector<uint32_t> *gstart_host;
    /* union of independent graphs (ag_multigraph_upload) */
    uint32_t ngraphs;
    uint32_t *gstart;       /* device, ngraphs + 1                           */
    uint32_t *g_u32;        /* device: active, done, passes, conv (4 x ngraphs) */
    double *g_f64;          /* device: err, err_last (2 x ngraphs)           */
    uint4 *tasks_fast, *tasks_exact;
    uint32_t ntasks_fast, ntasks_exact;
    uint32_t nparts;
    uint32_t num_hub_rows, max_in_degree;
    float *rank;
    float *c32[2];
    uint16_t *c16[2];
    float *hub_part;
    uint32_t *hub_cnt;
    float *hub_vals; /* EXACT order: staged values of hub rows */
    uint32_t *hub_pred; /* EXACT order: chunk starting binades of the last pass */
    uint32_t *hub_t;    /* EXACT order: per-round integer step totals */
    AgControl *ctl;
    float *init_buf;
    uint32_t *flag;
    AgExec exe[3][2];
    int have_exe[3][2];
    /* data-driven mode: its launch graphs (FAST, EXACT) */
    AgExec exe_dd[2];
    /* integer pulls (fixed point and quantised): contribution buffers (the
     * narrow forms use the first N * W/8 bytes), hub partials (capacity in
     * chunks), the quantised forms' binary32 contributions and min/max key
     * slots, and one launch graph per form (both orders give the same bits) */
    uint64_t *c64[2];
    uint64_t *hub_part64;
    uint32_t hub64_cap;
    float *cqf;
    uint32_t *qmm;
    AgExec exe_int[AG_NUM_INT_FORMS];
    int have_exe_int[AG_NUM_INT_FORMS];
    /* push and residual forms: forward edge list sorted by source, vertex
     * vectors, residuals, deltas, the two worklists, one launch graph per form */
    uint32_t *fwd_src, *fwd_dst;
    float *pa, *pb, *res, *delta;
    uint8_t *wl;
    AgExec exe_push[AG_NUM_PUSH_FORMS];
    int have_exe_push[AG_NUM_PUSH_FORMS];
    int have_exe_dd[2];
    cudaEvent_t ev0, ev1;
    int launched;
    int last_prec, last_exact;
    uint64_t device_bytes;
};

static void *dev_alloc(ag_graph_s *g, size_t bytes, ag_status_t *st)
{
    void *p = nullptr;
    if (*st != AG_OK)
        return nullptr;
    if (bytes == 0)
        bytes = 16;
    cudaError_t e = cudaMallocAsync(&p, bytes, g_ctx.stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *st = ag_set_error(AG_ERR_OOM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return nullptr;
    }
    g->device_bytes += bytes;
    return p;
}

static void dev_free(void *p)
{
    if (p)
        cudaFreeAsync(p, g_ctx.stream);
}

static void free_exec(AgExec *x)
{
    if (x->exec)
        cudaGraphExecDestroy(x->exec);
    if (x->graph)
        cudaGraphDestroy(x->graph);
    x->exec = nullptr;
    x->graph = nullptr;
}

/* forget every cached launch graph (they carry buffer pointers and tiles) */
static void drop_execs(ag_graph_s *g)
{
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 2; ++b)
            if (g->have_exe[a][b]) {
                free_exec(&g->exe[a][b]);
                g->have_exe[a][b] = 0;
            }
    for (int b = 0; b < 2; ++b)
        if (g->have_exe_dd[b]) {
            free_exec(&g->exe_dd[b]);
            g->have_exe_dd[b] = 0;
        }
    for (int b = 0; b < AG_NUM_INT_FORMS; ++b)
        if (g->have_exe_int[b]) {
            free_exec(&g->exe_int[b]);
            g->have_exe_int[b] = 0;
        }
    for (int b = 0; b < AG_NUM_PUSH_FORMS; ++b)
        if (g->have_exe_push[b]) {
            free_exec(&g->exe_push[b]);
            g->have_exe_push[b] = 0;
        }
}

extern "C" ag_status_t ag_graph_release(ag_graph_t g)
{
    if (!g)
        return AG_OK;
    if (g_ctx.ready)
        stream_wait(g_ctx.stream, 0);
    drop_execs(g);
    dev_free(g->c64[0]);
    dev_free(g->c64[1]);
    dev_free(g->hub_part64);
    dev_free(g->cqf);
    dev_free(g->qmm);
    dev_free(g->fwd_src);
    dev_free(g->fwd_dst);
    dev_free(g->pa);
    dev_free(g->pb);
    dev_free(g->res);
    dev_free(g->delta);
    dev_free(g->wl);
    dev_free(g->row_off);
    dev_free(g->ids);
    dev_free(g->perm);
    dev_free(g->inv);
    dev_free(g->gstart);
    dev_free(g->g_u32);
    dev_free(g->g_f64);
    delete g->gstart_host;
    dev_free(g->out);
    dev_free(g->xbuf);
    dev_free(g->ybuf);
    dev_free(g->outdeg);
    dev_free(g->w);
    dev_free(g->tasks_fast);
    dev_free(g->tasks_exact);
    dev_free(g->rank);
    dev_free(g->c32[0]);
    dev_free(g->c32[1]);
    dev_free(g->c16[0]);
    dev_free(g->c16[1]);
    dev_free(g->hub_part);
    dev_free(g->hub_cnt);
    dev_free(g->hub_vals);
    dev_free(g->hub_pred);
    dev_free(g->hub_t);
    dev_free(g->ctl);
    dev_free(g->init_buf);
    dev_free(g->flag);
    if (g->ev0)
        cudaEventDestroy(g->ev0);
    if (g->ev1)
        cudaEventDestroy(g->ev1);
    if (g_ctx.ready)
        cudaStreamSynchronize(g_ctx.stream);
    delete g;
    return AG_OK;
}

/* Work lists of the fused pull kernel (one item per warp), planned on the
 * device from the device row offsets (ag_plan.cu).  Rows longer than `cap`
 * in-edges run on their own warp, rows longer than `whub` are split into
 * whub-edge chunks (in EXACT order the chunks stage their values and the last
 * one sums the row in stream order).  Other
 * rows are packed into items of <= AG_WROWS consecutive rows holding <= cap
 * in-edges.  Heavy items come first so that they start early.  On success the
 * lists replace the graph's current ones. */
static ag_status_t plan_device(ag_graph_s *g, uint32_t cap, uint32_t whub)
{
    const uint32_t N = g->N;
    if (N > AG_ROW_MASK)
        return ag_set_error(AG_ERR_INVALID_GRAPH, "%u vertices exceed the 2^30 row limit", N);
    if (((uint64_t)g->max_in_degree + whub - 1) / whub >= (1u << (32 - AG_SLOT_BITS)))
        return ag_set_error(AG_ERR_UNSUPPORTED, "a row of %u in-edges exceeds the hub split limits",
                            g->max_in_degree);
    cudaStream_t s = g_ctx.stream;
    AgPlanState ps;
    uint32_t tot[4] = {0, 0, 0, 0};
    cudaError_t e = ag_plan_count(g->row_off, N, cap, whub, g->gstart, g->ngraphs, &ps, tot, s);
    ag_status_t st = AG_OK;
    if (e != cudaSuccess) {
        cudaGetLastError();
        ag_plan_release(&ps, s);
        return ag_set_error(AG_ERR_CUDA, "work-list planning failed: %s", cudaGetErrorString(e));
    }
    st = stream_wait(s, 0);
    if (st != AG_OK) {
        ag_plan_release(&ps, s);
        return st;
    }
    if (tot[0] > AG_SLOT_MASK) {
        ag_plan_release(&ps, s);
        return ag_set_error(AG_ERR_UNSUPPORTED, "%u hub chunks exceed the hub split limits", tot[0]);
    }
    const uint32_t nf = tot[0] + tot[1] + tot[2], ne = nf;
    uint4 *tdf = (uint4 *)dev_alloc(g, (size_t)nf * sizeof(uint4), &st);
    uint4 *tde = (uint4 *)dev_alloc(g, (size_t)ne * sizeof(uint4), &st);
    float *hp = (float *)dev_alloc(g, (size_t)tot[0] * 4 + 16, &st);
    /* hub arrival counters, then the EXACT order's donor table */
    const size_t hc_bytes = ((size_t)tot[0] + 4 + AG_STEAL_WORDS) * 4;
    uint32_t *hc = (uint32_t *)dev_alloc(g, hc_bytes, &st);
    /* EXACT order stages a hub row's gathered values here (chunk slot x
     * chunk size + offset in the row) before summing them in stream order */
    float *hv = (float *)dev_alloc(g, (size_t)tot[0] * whub * 4 + 16, &st);
    /* and keeps each chunk's starting binade and per-round integer step
     * totals (the predictions start unknown) */
    uint32_t *hpr = (uint32_t *)dev_alloc(g, (size_t)tot[0] * 4 + 16, &st);
    uint32_t *ht = (uint32_t *)dev_alloc(g, (size_t)tot[0] * AG_XWORDS * 4 + 16, &st);
    if (st == AG_OK) {
        e = ag_plan_write(&ps, tot, tdf, tde, s);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(hc, 0, hc_bytes, s);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(hpr, 0, (size_t)tot[0] * 4 + 16, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = ag_set_error(AG_ERR_CUDA, "work-list planning failed: %s", cudaGetErrorString(e));
        }
    }
    ag_plan_release(&ps, s);
    if (st != AG_OK) {
        dev_free(tdf);
        dev_free(tde);
        dev_free(hp);
        dev_free(hc);
        dev_free(hv);
        dev_free(hpr);
        dev_free(ht);
        return st;
    }
    dev_free(g->tasks_fast);
    dev_free(g->tasks_exact);
    dev_free(g->hub_part);
    dev_free(g->hub_cnt);
    dev_free(g->hub_vals);
    dev_free(g->hub_pred);
    dev_free(g->hub_t);
    g->tasks_fast = tdf;
    g->tasks_exact = tde;
    g->hub_part = hp;
    g->hub_cnt = hc;
    g->hub_vals = hv;
    g->hub_pred = hpr;
    g->hub_t = ht;
    g->ntasks_fast = nf;
    g->ntasks_exact = ne;
    g->nparts = tot[0];
    g->num_hub_rows = tot[3];
    return AG_OK;
}

static ag_status_t upload_impl(const struct GraphCSR *graph, uint32_t flags, const uint32_t *gstart_host,
                               uint32_t ngraphs, uint32_t gather_n, ag_graph_t *out, const AgDevCSR *dev = nullptr);

extern "C" ag_status_t ag_graph_upload(const struct GraphCSR *graph, uint32_t flags, ag_graph_t *out)
{
    return upload_impl(graph, flags, nullptr, 0, 0, out);
}

/* The upload's copy stream (one per device): the in-edge copies of a host
 * graph run on it while the library stream lays out the relabelled rows and
 * plans the work lists from the degrees.  ev[0] orders it after the
 * library stream's allocations, ev[1] the library stream after its copies. */
static struct
{
    int device;
    cudaStream_t stream;
    cudaEvent_t ev[2];
} g_copy = {-1, nullptr, {nullptr, nullptr}};

static ag_status_t copy_stream_ensure(void)
{
    if (g_copy.stream && g_copy.device == g_ctx.device)
        return AG_OK;
    g_copy.stream = nullptr; /* a stream of another device is left to it */
    AG_CUDA(cudaStreamCreateWithFlags(&g_copy.stream, cudaStreamNonBlocking));
    AG_CUDA(cudaEventCreateWithFlags(&g_copy.ev[0], cudaEventDisableTiming));
    AG_CUDA(cudaEventCreateWithFlags(&g_copy.ev[1], cudaEventDisableTiming));
    g_copy.device = g_ctx.device;
    return AG_OK;
}

/* gather_n: length of the vector the in-edges index (0: num_vertices).
 * dev: the graph's CSR already in device memory (built by ag_graph_build);
 * `graph` is then unused, and the device arrays are copied, not checked. */
static ag_status_t upload_impl(const struct GraphCSR *graph, uint32_t flags, const uint32_t *gstart_host,
                               uint32_t ngraphs, uint32_t gather_n, ag_graph_t *out, const AgDevCSR *dev)
{
    ag_clear_error();
    if ((!graph && !dev) || !out)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_upload: NULL argument");
    *out = nullptr;
    ag_status_t st = ctx_ensure(-1);
    if (st != AG_OK)
        return st;
    const uint32_t N = dev ? dev->N : graph->num_vertices, E = dev ? dev->E : graph->num_edges;
    const struct Vertex *iv = dev ? nullptr : graph->inverse_vertices;
    const struct Vertex *fv = dev ? nullptr : graph->vertices;
    const struct EdgeList *iel = dev ? nullptr : graph->inverse_sorted_edges_array;
    if (!dev && N > 0 && (!iv || !iv->out_degree || !iv->edges_idx || !fv || !fv->out_degree))
        return ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_upload: missing vertex arrays");
    if (!dev && E > 0 && (!iel || !iel->edges_array_dest))
        return ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_upload: missing inverse edge array");
    if (E >= 0xFFFFFFF0u)
        return ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_upload: too many edges");
    if (dev)
        flags |= AG_UPLOAD_TRUSTED; /* the builder checked every endpoint */
    const bool want_w = (flags & AG_UPLOAD_WEIGHTS) && (dev ? dev->inv_w != nullptr : iel && iel->edges_array_weight);

    ag_graph_s *g = new ag_graph_s();
    memset((void *)g, 0, sizeof(*g));
    g->N = N;
    g->E = E;
    g->E4 = ((E + 3u) & ~3u) + 4u;

    cudaStream_t s = g_ctx.stream;
    const bool relabel = !(flags & AG_UPLOAD_KEEP_ORDER) && N > 0;
    /* the caller's layout first ("old"); relabelled copies replace it */
    uint32_t *off_old = (uint32_t *)dev_alloc(g, (size_t)(N + 1) * 4, &st);
    uint32_t *ids_old = (uint32_t *)dev_alloc(g, (size_t)g->E4 * 4, &st);
    uint32_t *outdeg_old = (uint32_t *)dev_alloc(g, (size_t)N * 4 + 16, &st);
    float *w_old = want_w ? (float *)dev_alloc(g, (size_t)g->E4 * 4, &st) : nullptr;
    g->rank = (float *)dev_alloc(g, (size_t)N * 4 + 16, &st);
    g->out = (float *)dev_alloc(g, (size_t)N * 4 + 16, &st);
    g->c32[0] = (float *)dev_alloc(g, (size_t)N * 4 + 16, &st);
    g->c32[1] = (float *)dev_alloc(g, (size_t)N * 4 + 16, &st);
    g->ctl = (AgControl *)dev_alloc(g, sizeof(AgControl), &st);
    g->flag = (uint32_t *)dev_alloc(g, 16, &st);
    if (relabel) {
        g->perm = (uint32_t *)dev_alloc(g, (size_t)N * 4 + 16, &st);
        g->inv = (uint32_t *)dev_alloc(g, (size_t)N * 4 + 16, &st);
        g->row_off = (uint32_t *)dev_alloc(g, (size_t)(N + 1) * 4, &st);
        g->ids = (uint32_t *)dev_alloc(g, (size_t)g->E4 * 4, &st);
        g->outdeg = (uint32_t *)dev_alloc(g, (size_t)N * 4 + 16, &st);
        if (want_w)
            g->w = (float *)dev_alloc(g, (size_t)g->E4 * 4, &st);
    } else {
        g->row_off = off_old;
        g->ids = ids_old;
        g->outdeg = outdeg_old;
        g->w = w_old;
    }
    /* in-edges of a host graph travel on the copy stream */
    if (st == AG_OK && !dev)
        st = copy_stream_ensure();
    if (st != AG_OK) {
        if (relabel) {
            dev_free(off_old);
            dev_free(ids_old);
            dev_free(outdeg_old);
            dev_free(w_old);
        }
        ag_graph_release(g);
        return st;
    }
    cudaStream_t cs = dev ? s : g_copy.stream;
    /* every exit before the join waits for the copy stream first: neither the
     * caller's arrays nor the device buffers it writes may go while it runs */
    auto join_copies = [&]() {
        if (cs != s)
            cudaStreamSynchronize(cs);
    };
#define UP(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            cudaGetLastError();                                                                  \
            join_copies();                                                                       \
            st = ag_set_error(AG_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
            if (relabel) {                                                                       \
                dev_free(off_old);                                                               \
                dev_free(ids_old);                                                               \
                dev_free(outdeg_old);                                                            \
                dev_free(w_old);                                                                 \
            }                                                                                    \
            ag_graph_release(g);                                                                 \
            return st;                                                                           \
        }                                                                                        \
    } while (0)
#define UPFAIL(status)                                                                           \
    do {                                                                                         \
        join_copies();                                                                           \
        st = (status);                                                                           \
        if (relabel) {                                                                           \
            dev_free(off_old);                                                                   \
            dev_free(ids_old);                                                                   \
            dev_free(outdeg_old);                                                                \
            dev_free(w_old);                                                                     \
        }                                                                                        \
        ag_graph_release(g);                                                                     \
        return st;                                                                               \
    } while (0)
    if (dev) {
        g->max_in_degree = dev->max_in_degree;
        UP(cudaMemcpyAsync(off_old, dev->inv_idx, (size_t)(N + 1) * 4, cudaMemcpyDeviceToDevice, s));
        UP(cudaMemsetAsync(ids_old + E, 0, (size_t)(g->E4 - E) * 4, s));
        if (E)
            UP(cudaMemcpyAsync(ids_old, dev->inv_dst, (size_t)E * 4, cudaMemcpyDeviceToDevice, s));
        if (want_w) {
            if (E)
                UP(cudaMemcpyAsync(w_old, dev->inv_w, (size_t)E * 4, cudaMemcpyDeviceToDevice, s));
            UP(cudaMemsetAsync(w_old + E, 0, (size_t)(g->E4 - E) * 4, s));
        }
        if (N)
            UP(cudaMemcpyAsync(outdeg_old, dev->out_deg, (size_t)N * 4, cudaMemcpyDeviceToDevice, s));
    } else {
        /* The bulk copies start first, assuming the usual layout of contiguous
         * rows; the host checks the rows while they run.  A layout that is not
         * contiguous is repacked and copied again (ordered after the first copy
         * on the same stream).  Every error path below waits for the stream
         * before the caller's arrays can be freed (ag_graph_release does). */
        const bool guess_contiguous = N == 0 || iv->edges_idx[0] == 0;
        /* the copy stream starts after the library stream's allocations */
        UP(cudaEventRecord(g_copy.ev[0], s));
        UP(cudaStreamWaitEvent(cs, g_copy.ev[0], 0));
        if (guess_contiguous) {
            if (E)
                UP(cudaMemcpyAsync(ids_old, iel->edges_array_dest, (size_t)E * 4, cudaMemcpyHostToDevice, cs));
            if (want_w && E)
                UP(cudaMemcpyAsync(w_old, iel->edges_array_weight, (size_t)E * 4, cudaMemcpyHostToDevice, cs));
        }
        if (N)
            UP(cudaMemcpyAsync(outdeg_old, fv->out_degree, (size_t)N * 4, cudaMemcpyHostToDevice, s));
        /* host view of the inverse rows: contiguous rows are uploaded as they
         * are; any other layout (gaps, overlap, reordering) is repacked */
        bool contiguous = true;
        uint64_t total = 0;
        uint32_t maxd = 0;
        for (uint32_t v = 0; v < N; ++v) {
            const uint32_t d = iv->out_degree[v];
            if (iv->edges_idx[v] != total)
                contiguous = false;
            if ((uint64_t)iv->edges_idx[v] + d > E)
                UPFAIL(ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_upload: row %u [%u, +%u) exceeds %u edges", v,
                                    iv->edges_idx[v], d, E));
            total += d;
            if (d > maxd)
                maxd = d;
        }
        if (total != E)
            UPFAIL(ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_upload: in-degrees sum to %llu, expected %u edges",
                                (unsigned long long)total, E));
        g->max_in_degree = maxd;
        /* row starts: the caller's own array when its rows are contiguous (its
         * N entries plus E), else a packed copy */
        std::vector<uint32_t> off;
        if (!contiguous) {
            off.resize((size_t)N + 1);
            uint32_t o = 0;
            for (uint32_t v = 0; v < N; ++v) {
                off[v] = o;
                o += iv->out_degree[v];
            }
            off[N] = E;
        }

        if (contiguous) {
            if (N)
                UP(cudaMemcpyAsync(off_old, iv->edges_idx, (size_t)N * 4, cudaMemcpyHostToDevice, s));
            UP(ag_set_u32(off_old + N, E, s));
        } else {
            UP(cudaMemcpyAsync(off_old, off.data(), (size_t)(N + 1) * 4, cudaMemcpyHostToDevice, s));
        }
        UP(cudaMemsetAsync(ids_old + E, 0, (size_t)(g->E4 - E) * 4, cs));
        if (contiguous) {
            if (!guess_contiguous && E)
                UP(cudaMemcpyAsync(ids_old, iel->edges_array_dest, (size_t)E * 4, cudaMemcpyHostToDevice, cs));
            if (!guess_contiguous && want_w && E)
                UP(cudaMemcpyAsync(w_old, iel->edges_array_weight, (size_t)E * 4, cudaMemcpyHostToDevice, cs));
        } else {
            std::vector<uint32_t> packed(E);
            std::vector<float> packw(want_w ? E : 0);
            for (uint32_t v = 0; v < N; ++v) {
                const uint32_t d = iv->out_degree[v], b = iv->edges_idx[v];
                memcpy(packed.data() + off[v], iel->edges_array_dest + b, (size_t)d * 4);
                if (want_w)
                    memcpy(packw.data() + off[v], iel->edges_array_weight + b, (size_t)d * 4);
            }
            if (E)
                UP(cudaMemcpyAsync(ids_old, packed.data(), (size_t)E * 4, cudaMemcpyHostToDevice, cs));
            if (want_w && E)
                UP(cudaMemcpyAsync(w_old, packw.data(), (size_t)E * 4, cudaMemcpyHostToDevice, cs));
            UP(cudaStreamSynchronize(cs)); /* the packed copies are stack-owned */
        }
        if (want_w)
            UP(cudaMemsetAsync(w_old + E, 0, (size_t)(g->E4 - E) * 4, cs));
        UP(cudaEventRecord(g_copy.ev[1], cs));
    }
    UP(cudaMemsetAsync(g->ctl, 0, sizeof(AgControl), s));
    UP(cudaMemsetAsync(g->flag, 0, 4, s));
    UP(cudaMemsetAsync(g->flag + 1, 0xFF, 4, s));

    /* While the in-edges travel: the relabelled layout, the tunables and the
     * work lists need only the degrees. */
    if (relabel) {
        UP(cudaMemsetAsync(g->ids + E, 0, (size_t)(g->E4 - E) * 4, s));
        if (want_w)
            UP(cudaMemsetAsync(g->w + E, 0, (size_t)(g->E4 - E) * 4, s));
        UP(ag_relabel_layout(off_old, outdeg_old, N, g->perm, g->inv, g->row_off, g->outdeg, s));
    }
    {
        /* tunables (the defaults were measured best on R-MAT s20/s22):
         * AG_HOT_ENTRIES -- shared-memory table entries (<= AG_HOT_MAX)
         * AG_WARM_ENTRIES -- ids below this may allocate L1 lines */
        uint32_t hot = AG_HOT_CAP, warm = AG_WARM_DEFAULT;
        const char *eh = getenv("AG_HOT_ENTRIES");
        const char *ew = getenv("AG_WARM_ENTRIES");
        if (eh)
            hot = (uint32_t)strtoul(eh, nullptr, 10);
        if (ew)
            warm = (uint32_t)strtoul(ew, nullptr, 10);
        hot = std::min<uint32_t>(hot, AG_HOT_MAX);
        g->hot_allowed = (flags & AG_UPLOAD_NO_SMEM_CACHE) ? 0u : 1u;
        g->hot_n = g->hot_allowed ? std::min<uint32_t>(N & ~63u, hot & ~63u) : 0u;
        g->warm_n = std::max<uint32_t>(warm, g->hot_n);
        g->tiles.task_edges = AG_WCAP;
        g->tiles.hub_chunk = AG_WHUB;
        g->tiles.hot_entries = g->hot_n;
        g->tiles.warm_entries = g->warm_n;
    }
    if (ngraphs) {
        g->ngraphs = ngraphs;
        g->gstart_host = new std::vector<uint32_t>(gstart_host, gstart_host + ngraphs + 1);
        g->gstart = (uint32_t *)dev_alloc(g, (size_t)(ngraphs + 1) * 4, &st);
        g->g_u32 = (uint32_t *)dev_alloc(g, (size_t)ngraphs * 4 * 4, &st);
        g->g_f64 = (double *)dev_alloc(g, (size_t)ngraphs * 2 * 8, &st);
        if (st != AG_OK)
            UPFAIL(st);
        UP(cudaMemcpyAsync(g->gstart, gstart_host, (size_t)(ngraphs + 1) * 4, cudaMemcpyHostToDevice, s));
    }
    st = plan_device(g, g->tiles.task_edges, g->tiles.hub_chunk);
    if (st != AG_OK)
        UPFAIL(st);

    /* the in-edges have arrived */
    if (cs != s)
        UP(cudaStreamWaitEvent(s, g_copy.ev[1], 0));
    /* every in-edge must name a vertex < N before anything reads through it */
    if (!(flags & AG_UPLOAD_TRUSTED)) {
        uint32_t hflag[2] = {0, 0};
        UP(ag_validate_ids(ids_old, E, gather_n ? gather_n : N, g->flag, s));
        UP(cudaMemcpyAsync(hflag, g->flag, 8, cudaMemcpyDeviceToHost, s));
        UP(cudaStreamSynchronize(s));
        if (hflag[0]) {
            st = ag_set_error(AG_ERR_INVALID_GRAPH, "in-edge %u names a vertex >= %u", hflag[1],
                              gather_n ? gather_n : N);
            if (relabel) {
                dev_free(off_old);
                dev_free(ids_old);
                dev_free(outdeg_old);
                dev_free(w_old);
            }
            ag_graph_release(g);
            return st;
        }
    }
    if (relabel) {
        UP(ag_relabel_rows(g->perm, g->inv, off_old, g->row_off, ids_old, g->ids, w_old, g->w, N, E, s));
        dev_free(off_old);
        dev_free(ids_old);
        dev_free(outdeg_old);
        dev_free(w_old);
        g->device_bytes -= (uint64_t)(N + 1) * 4 + (uint64_t)g->E4 * 4 * (want_w ? 2 : 1) + (uint64_t)N * 4 + 16;
        off_old = ids_old = outdeg_old = nullptr;
        w_old = nullptr;
    }
    UP(cudaEventCreate(&g->ev0));
    UP(cudaEventCreate(&g->ev1));
    /* the host-side vectors die at return: wait for the copies */
    st = stream_wait(s, 0);
    if (st != AG_OK) {
        ag_graph_release(g);
        return st;
    }
#undef UP
#undef UPFAIL
    *out = g;
    return AG_OK;
}

static size_t pull_smem(const ag_graph_s *g);
static ag_status_t pull_kernel_prepare(const void *kern, size_t smem);

extern "C" ag_status_t ag_graph_get_info(ag_graph_t g, ag_graph_info *info)
{
    if (!g || !info)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_get_info: NULL argument");
    memset(info, 0, sizeof(*info));
    info->num_vertices = g->N;
    info->num_edges = g->E;
    info->num_tasks = g->ntasks_fast;
    info->num_hub_rows = g->num_hub_rows;
    info->max_in_degree = g->max_in_degree;
    info->device_bytes = g->device_bytes;
    int nb = 0;
    if (pull_kernel_prepare(ag_pull_kernel_ptr(AG_MODE_PR, 0, 0), pull_smem(g)) == AG_OK &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ag_pull_kernel_ptr(AG_MODE_PR, 0, 0), AG_BLK,
                                                      pull_smem(g)) == cudaSuccess)
        info->grid = (uint32_t)std::min<uint64_t>((uint64_t)nb * g_ctx.num_sms,
                                                  std::max<uint64_t>(1, ((uint64_t)g->ntasks_fast + AG_WARPS - 1) / AG_WARPS));
    return AG_OK;
}

/* persistent grid: every SM filled to its occupancy, never more CTAs than
 * work items */
static size_t pull_smem(const ag_graph_s *g) { return (size_t)AG_STAGE_BYTES + (size_t)g->hot_n * 4; }

/* the pull kernels take up to AG_SMEM_MAX bytes of shared memory */
static ag_status_t pull_kernel_prepare(const void *kern, size_t smem = 0)
{
    AG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 AG_SMEM_MAX - AG_SMEM_STATIC));
    if (smem) {
        /* carve out only the shared memory the CTAs need: the rest of the
         * SM's unified 256 KB is L1 for the warm gathers */
        const size_t per_sm = (smem + AG_SMEM_STATIC + 1024) * AG_CTAS_PER_SM;
        int pct = (int)((per_sm * 100 + 233471) / 233472);
        if (pct > 100)
            pct = 100;
        AG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    }
    return AG_OK;
}

static unsigned pull_grid(const void *kern, uint32_t ntasks, size_t smem)
{
    int nb = 0;
    if (pull_kernel_prepare(kern, smem) != AG_OK ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, AG_BLK, smem) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    uint64_t g = (uint64_t)nb * (uint64_t)g_ctx.num_sms;
    const uint64_t need = ((uint64_t)ntasks + AG_WARPS - 1) / AG_WARPS;
    if (g > need)
        g = need;
    if (g < 1)
        g = 1;
    return (unsigned)g;
}

static ag_status_t ensure_buffers(ag_graph_s *g, int prec)
{
    ag_status_t st = AG_OK;
    if (prec != 0 && !g->c16[0]) {
        g->c16[0] = (uint16_t *)dev_alloc(g, (size_t)g->N * 2 + 16, &st);
        g->c16[1] = (uint16_t *)dev_alloc(g, (size_t)g->N * 2 + 16, &st);
    }
    return st;
}

/* polls of the hot-table copy's mbarrier before a pull kernel reports the wait
 * as run out: AG_MBAR_SPINS (0 allowed: the first wait runs out at once, the
 * kernel flags it and then waits, bounded, for the copies) or 2^20 */
static uint32_t mbar_spins(void)
{
    const char *env = getenv("AG_MBAR_SPINS");
    if (env && *env) {
        char *end = nullptr;
        const unsigned long v = strtoul(env, &end, 10);
        if (end && *end == 0 && v <= 0xFFFFFFFFul)
            return (uint32_t)v;
    }
    return 1u << 20;
}

static AgPullParams base_params(ag_graph_s *g, int exact)
{
    AgPullParams p;
    memset(&p, 0, sizeof(p));
    p.mbar_spins = mbar_spins();
    p.row_off = g->row_off;
    p.ids = g->ids;
    p.w = g->w;
    p.outdeg = g->outdeg;
    p.tasks = exact ? g->tasks_exact : g->tasks_fast;
    p.ntasks = exact ? g->ntasks_exact : g->ntasks_fast;
    p.N = g->N;
    p.rank = g->rank;
    p.c32_0 = g->c32[0];
    p.c32_1 = g->c32[1];
    p.c16_0 = g->c16[0];
    p.c16_1 = g->c16[1];
    p.hub_part = g->hub_part;
    p.hub_cnt = g->hub_cnt;
    p.hub_vals = g->hub_vals;
    p.hub_pred = g->hub_pred;
    p.hub_t = g->hub_t;
    p.steal = g->hub_cnt + g->nparts + 4;
    p.ctl = g->ctl;
    p.init_ranks = g->init_buf;
    p.perm = g->perm;
    p.inv = g->inv;
    p.out = g->out;
    p.hot_n = g->hot_n;
    p.c_base = g->c_base;
    p.norm_n = g->norm_n;
    p.hot_n16 = std::min<uint32_t>(2 * g->hot_n, g->N & ~63u);
    p.warm_n = g->warm_n;
    p.whub = g->tiles.hub_chunk;
    p.ngraphs = g->ngraphs;
    p.gstart = g->gstart;
    if (g->ngraphs) {
        p.g_active = g->g_u32;
        p.g_done = g->g_u32 + g->ngraphs;
        p.g_passes = g->g_u32 + 2 * g->ngraphs;
        p.g_conv = g->g_u32 + 3 * g->ngraphs;
        p.g_err = g->g_f64;
        p.g_err_last = g->g_f64 + g->ngraphs;
    }
    p.c64_0 = g->c64[0];
    p.c64_1 = g->c64[1];
    p.hub_part64 = g->hub_part64;
    p.cqf = g->cqf;
    p.qmm = g->qmm;
    p.fwd_src = g->fwd_src;
    p.fwd_dst = g->fwd_dst;
    p.E = g->E;
    p.pa = g->pa;
    p.pb = g->pb;
    p.res = g->res;
    p.delta = g->delta;
    p.wl = g->wl;
    p.base = 1.0f - Damp; /* pageRank.c:57-58: base_pr = 1.0f - damp */
    p.damp = Damp;
    return p;
}

static int pull_mode(const ag_graph_s *g, int dd)
{
    return dd ? AG_MODE_DD : (g->ngraphs ? AG_MODE_MULTI : AG_MODE_PR);
}

/* the solve's kernels: pull, init and (quantised forms) quantise */
static const void *solve_pull_kernel(const ag_graph_s *g, int prec, int exact, int dd)
{
    return is_int_prec(prec) ? ag_int_kernel_ptr(int_bytes(prec), int_quant(prec), 0)
                             : ag_pull_kernel_ptr(pull_mode(g, dd), prec, exact);
}

static size_t solve_smem(const ag_graph_s *g, int prec)
{
    return is_int_prec(prec) ? ag_fixed_smem_bytes(int_bytes(prec)) : pull_smem(g);
}

static dim3 elem_grid(const ag_graph_s *g)
{
    return dim3((unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)g->N + AG_SBLK - 1) / AG_SBLK, (uint64_t)g_ctx.num_sms * 8)));
}

/* the quantiser: one wave of CTAs (each thread issues several groups' loads
 * at once) */
static dim3 quant_grid(const ag_graph_s *g)
{
    const uint64_t groups = ((uint64_t)g->N + 3) / 4;
    return dim3((unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((groups + AG_SBLK - 1) / AG_SBLK, (uint64_t)g_ctx.num_sms * 8)));
}

/* prec: AG_PREC_* (the integer forms take both orders through one graph) */
static AgExec *exec_slot(ag_graph_s *g, int prec, int exact, int dd)
{
    return is_int_prec(prec) ? &g->exe_int[prec - AG_PREC_FIXED64] : dd ? &g->exe_dd[exact] : &g->exe[prec][exact];
}

static ag_status_t build_exec(ag_graph_s *g, int prec, int exact, int dd = 0)
{
    const int ip = is_int_prec(prec), quant = ip && int_quant(prec);
    AgExec *x = exec_slot(g, prec, exact, dd);
    memset(x, 0, sizeof(*x));
    AG_CUDA(cudaGraphCreate(&x->graph, 0));
    AG_CUDA(cudaGraphConditionalHandleCreate(&x->cond, x->graph, 1, cudaGraphCondAssignDefault));
    x->params = base_params(g, exact);
    x->params.cond = x->cond;
    x->params.use_cond = 1;
    const void *kpull = solve_pull_kernel(g, prec, exact, dd);
    const size_t smem = solve_smem(g, prec);
    x->grid = pull_grid(kpull, x->params.ntasks, smem);

    /* quantised forms: both min/max slots cleared before the init kernel
     * folds the first contributions into slot 0 */
    cudaGraphNode_t pre[2];
    int npre = 0;
    if (quant) {
        cudaMemsetParams ms = {};
        ms.dst = g->qmm;
        ms.elementSize = 4;
        ms.width = 2;
        ms.height = 1;
        ms.pitch = 0;
        ms.value = 0xFFFFFFFFu;
        AG_CUDA(cudaGraphAddMemsetNode(&pre[npre++], x->graph, nullptr, 0, &ms));
        ms.dst = g->qmm + 2;
        ms.value = 0u;
        AG_CUDA(cudaGraphAddMemsetNode(&pre[npre++], x->graph, nullptr, 0, &ms));
    }

    AgRunConfig run;
    memset(&run, 0, sizeof(run));
    void *init_args[2] = {&x->params, &run};
    cudaKernelNodeParams kp = {};
    kp.func = (void *)(ip ? ag_int_init_kernel_ptr(int_bytes(prec), quant) : ag_init_kernel_ptr(prec));
    kp.gridDim = elem_grid(g);
    kp.blockDim = dim3(AG_SBLK);
    kp.kernelParams = init_args;
    AG_CUDA(cudaGraphAddKernelNode(&x->init_node, x->graph, npre ? pre : nullptr, (size_t)npre, &kp));

    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = x->cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    AG_CUDA(cudaGraphAddNode(&wnode, x->graph, &x->init_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    void *pull_args[1] = {&x->params};
    /* quantised forms: each iteration first quantises the contributions */
    cudaGraphNode_t qnode;
    if (quant) {
        cudaKernelNodeParams kq = {};
        kq.func = (void *)ag_quant_kernel_ptr(int_bytes(prec));
        kq.gridDim = quant_grid(g);
        kq.blockDim = dim3(AG_SBLK);
        kq.kernelParams = pull_args;
        AG_CUDA(cudaGraphAddKernelNode(&qnode, body, nullptr, 0, &kq));
    }
    cudaKernelNodeParams kb = {};
    kb.func = (void *)kpull;
    kb.gridDim = dim3(x->grid);
    kb.blockDim = dim3(AG_BLK);
    kb.sharedMemBytes = (unsigned)smem;
    kb.kernelParams = pull_args;
    cudaGraphNode_t pnode;
    AG_CUDA(cudaGraphAddKernelNode(&pnode, body, quant ? &qnode : nullptr, quant ? 1 : 0, &kb));

    void *norm_args[1] = {&x->params};
    cudaKernelNodeParams kn = {};
    kn.func = (void *)ag_normalize_kernel_ptr();
    kn.gridDim = kp.gridDim;
    kn.blockDim = dim3(AG_SBLK);
    kn.kernelParams = norm_args;
    cudaGraphNode_t nnode;
    AG_CUDA(cudaGraphAddKernelNode(&nnode, x->graph, &wnode, 1, &kn));

    AG_CUDA(cudaGraphInstantiate(&x->exec, x->graph, 0));
    if (ip)
        g->have_exe_int[prec - AG_PREC_FIXED64] = 1;
    else if (dd)
        g->have_exe_dd[exact] = 1;
    else
        g->have_exe[prec][exact] = 1;
    return AG_OK;
}

static int have_exec(const ag_graph_s *g, int prec, int exact, int dd)
{
    return is_int_prec(prec) ? g->have_exe_int[prec - AG_PREC_FIXED64]
           : dd              ? g->have_exe_dd[exact]
                             : g->have_exe[prec][exact];
}

/* integer pull buffers, made on first use; the hub partials follow the
 * work list's chunk count (a new tile shape may need more) */
static ag_status_t ensure_fixed(ag_graph_s *g, int quant = 0)
{
    ag_status_t st = AG_OK;
    if (quant && !g->cqf) {
        g->cqf = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        g->qmm = (uint32_t *)dev_alloc(g, 16, &st);
        if (st != AG_OK)
            return st;
        drop_execs(g);
    }
    if (!g->c64[0]) {
        g->c64[0] = (uint64_t *)dev_alloc(g, (size_t)g->N * 8 + 16, &st);
        g->c64[1] = (uint64_t *)dev_alloc(g, (size_t)g->N * 8 + 16, &st);
        if (st != AG_OK)
            return st;
        drop_execs(g);
    }
    if (!g->hub_part64 || g->hub64_cap < g->nparts) {
        dev_free(g->hub_part64);
        g->hub_part64 = (uint64_t *)dev_alloc(g, (size_t)g->nparts * 8 + 16, &st);
        if (st != AG_OK) {
            g->hub_part64 = nullptr;
            g->hub64_cap = 0;
            return st;
        }
        g->hub64_cap = g->nparts;
        drop_execs(g);
    }
    return AG_OK;
}

/* push and residual forms: the forward edge list (built once from the
 * device inverse CSR) and the vectors each form needs, made on first use */
static ag_status_t ensure_push(ag_graph_s *g, int kind)
{
    ag_status_t st = AG_OK;
    if (kind == AG_PUSH_FLOAT || kind == AG_PUSH_FIXED || kind == AG_PUSH_QUANT) {
        /* 64-bit next sums (and the quantised form's min/max slots) */
        st = ensure_fixed(g, kind == AG_PUSH_QUANT);
        if (st != AG_OK)
            return st;
    }
    if (!g->fwd_src) {
        g->fwd_src = (uint32_t *)dev_alloc(g, (size_t)g->E * 4 + 16, &st);
        g->fwd_dst = (uint32_t *)dev_alloc(g, (size_t)g->E * 4 + 16, &st);
        if (st != AG_OK)
            return st;
        AG_CUDA(ag_forward_build(g->row_off, g->ids, g->N, g->E, g->fwd_src, g->fwd_dst, g_ctx.stream));
        drop_execs(g);
    }
    if (!g->pa) {
        g->pa = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        g->pb = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        if (st != AG_OK)
            return st;
        drop_execs(g);
    }
    if ((kind == AG_PUSH_DD || kind == AG_PUSH_PULLPUSH) && !g->res) {
        g->res = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        g->delta = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        g->wl = (uint8_t *)dev_alloc(g, (size_t)g->N * 2 + 16, &st);
        if (st != AG_OK)
            return st;
        drop_execs(g);
    }
    return AG_OK;
}

/* parameters of an SpMV launch inside a push-family solve: y = pb, the unit
 * row sums of x = pa (EXACT: stream order) */
static AgPullParams push_spmv_params(ag_graph_s *g, int exact)
{
    AgPullParams q = base_params(g, exact);
    q.x = g->pa;
    q.rank = g->pb;
    q.wmode = AG_SPMV_W_UNIT;
    q.honor_stop = 1;
    return q;
}

static size_t push_spmv_smem(const AgPullParams &q) { return (size_t)AG_STAGE_BYTES + (size_t)q.hot_n * 4; }

/* launch shape of the push scatter: a persistent grid at the kernel's
 * occupancy, with its shared-memory table */
struct PushScatterShape
{
    dim3 grid, block;
    size_t smem;
};

static ag_status_t push_scatter_shape(int kind, PushScatterShape *sh)
{
    unsigned threads = 0;
    size_t smem = 0;
    ag_push_scatter_shape(&threads, &smem);
    /* the push scatter (stage 1) or the residual forms' edge phase (stage 2) */
    const bool residual = kind == AG_PUSH_DD || kind == AG_PUSH_PULLPUSH;
    const void *k = ag_push_kernel_ptr(kind, residual ? 2 : 1);
    AG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, (int)threads, smem) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    sh->grid = dim3((unsigned)(nb * g_ctx.num_sms));
    sh->block = dim3(threads);
    sh->smem = smem;
    return AG_OK;
}

/* The push form's graph: [qmm clears] init, WHILE { [quantiser] scatter,
 * update }, normalise; the residual forms: seed, stream-order SpMV (first
 * residuals), init, WHILE { [SpMV of the contributions] vertex phase, edge
 * phase }, normalise. */
static ag_status_t build_exec_push(ag_graph_s *g, int kind)
{
    AgExec *x = &g->exe_push[kind];
    memset(x, 0, sizeof(*x));
    AG_CUDA(cudaGraphCreate(&x->graph, 0));
    AG_CUDA(cudaGraphConditionalHandleCreate(&x->cond, x->graph, 1, cudaGraphCondAssignDefault));
    x->params = base_params(g, 0);
    x->params.cond = x->cond;
    x->params.use_cond = 1;
    const bool residual = kind == AG_PUSH_DD || kind == AG_PUSH_PULLPUSH;
    const dim3 eg = elem_grid(g), blk(AG_SBLK);
    void *pargs[1] = {&x->params};

    cudaGraphNode_t prev[2];
    int nprev = 0;
    if (kind == AG_PUSH_QUANT) {
        cudaMemsetParams ms = {};
        ms.dst = g->qmm;
        ms.elementSize = 4;
        ms.width = 2;
        ms.height = 1;
        ms.value = 0xFFFFFFFFu;
        AG_CUDA(cudaGraphAddMemsetNode(&prev[nprev++], x->graph, nullptr, 0, &ms));
        ms.dst = g->qmm + 2;
        ms.value = 0u;
        AG_CUDA(cudaGraphAddMemsetNode(&prev[nprev++], x->graph, nullptr, 0, &ms));
    }
    AgPullParams seed_spmv = push_spmv_params(g, 1), loop_spmv = push_spmv_params(g, 0);
    seed_spmv.honor_stop = 0;
    if (residual) {
        cudaKernelNodeParams ks = {};
        ks.func = (void *)ag_push_kernel_ptr(kind, 3);
        ks.gridDim = eg;
        ks.blockDim = blk;
        ks.kernelParams = pargs;
        cudaGraphNode_t nseed, nspmv;
        AG_CUDA(cudaGraphAddKernelNode(&nseed, x->graph, nullptr, 0, &ks));
        void *sargs[1] = {&seed_spmv};
        const void *ksp = ag_pull_kernel_ptr(AG_MODE_SPMV, 0, 1);
        const size_t ssm = push_spmv_smem(seed_spmv);
        if (seed_spmv.ntasks) {
            cudaKernelNodeParams kv = {};
            kv.func = (void *)ksp;
            kv.gridDim = dim3(pull_grid(ksp, seed_spmv.ntasks, ssm));
            kv.blockDim = dim3(AG_BLK);
            kv.sharedMemBytes = (unsigned)ssm;
            kv.kernelParams = sargs;
            AG_CUDA(cudaGraphAddKernelNode(&nspmv, x->graph, &nseed, 1, &kv));
            prev[nprev++] = nspmv;
        } else {
            prev[nprev++] = nseed;
        }
    }
    AgRunConfig run;
    memset(&run, 0, sizeof(run));
    void *init_args[2] = {&x->params, &run};
    cudaKernelNodeParams kp = {};
    kp.func = (void *)ag_push_kernel_ptr(kind, 0);
    kp.gridDim = eg;
    kp.blockDim = blk;
    kp.kernelParams = init_args;
    AG_CUDA(cudaGraphAddKernelNode(&x->init_node, x->graph, nprev ? prev : nullptr, (size_t)nprev, &kp));

    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = x->cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    AG_CUDA(cudaGraphAddNode(&wnode, x->graph, &x->init_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    cudaGraphNode_t last = nullptr;
    auto add = [&](const void *func, dim3 grid, dim3 block, size_t smem, void **args) -> cudaError_t {
        cudaKernelNodeParams kn = {};
        kn.func = (void *)func;
        kn.gridDim = grid;
        kn.blockDim = block;
        kn.sharedMemBytes = (unsigned)smem;
        kn.kernelParams = args;
        cudaGraphNode_t n;
        cudaError_t e = cudaGraphAddKernelNode(&n, body, last ? &last : nullptr, last ? 1 : 0, &kn);
        if (e == cudaSuccess)
            last = n;
        return e;
    };
    void *largs[1] = {&loop_spmv};
    if (kind == AG_PUSH_QUANT)
        AG_CUDA(add(ag_push_kernel_ptr(kind, 3), eg, blk, 0, pargs));
    if (kind == AG_PUSH_PULLPUSH && loop_spmv.ntasks) {
        const void *ksp = ag_pull_kernel_ptr(AG_MODE_SPMV, 0, 0);
        const size_t lsm = push_spmv_smem(loop_spmv);
        AG_CUDA(add(ksp, dim3(pull_grid(ksp, loop_spmv.ntasks, lsm)), dim3(AG_BLK), lsm, largs));
    }
    PushScatterShape sh;
    ag_status_t sst = push_scatter_shape(kind, &sh);
    if (sst != AG_OK)
        return sst;
    if (residual) {
        AG_CUDA(add(ag_push_kernel_ptr(kind, 1), eg, blk, 0, pargs));
        AG_CUDA(add(ag_push_kernel_ptr(kind, 2), sh.grid, sh.block, sh.smem, pargs));
    } else {
        AG_CUDA(add(ag_push_kernel_ptr(kind, 1), sh.grid, sh.block, sh.smem, pargs));
        AG_CUDA(add(ag_push_kernel_ptr(kind, 2), eg, blk, 0, pargs));
    }

    void *norm_args[1] = {&x->params};
    cudaKernelNodeParams kn = {};
    kn.func = (void *)ag_normalize_kernel_ptr();
    kn.gridDim = eg;
    kn.blockDim = blk;
    kn.kernelParams = norm_args;
    cudaGraphNode_t nnode;
    AG_CUDA(cudaGraphAddKernelNode(&nnode, x->graph, &wnode, 1, &kn));
    AG_CUDA(cudaGraphInstantiate(&x->exec, x->graph, 0));
    g->have_exe_push[kind] = 1;
    return AG_OK;
}

/* the same kernels as separate launches (profiling form; passes after the
 * loop stops return at once) */
static ag_status_t push_stream_launch(ag_graph_s *g, int kind, const AgRunConfig &run)
{
    cudaStream_t s = g_ctx.stream;
    AgPullParams sp = base_params(g, 0);
    sp.use_cond = 0;
    const bool residual = kind == AG_PUSH_DD || kind == AG_PUSH_PULLPUSH;
    const dim3 eg = elem_grid(g), blk(AG_SBLK);
    void *pa[1] = {&sp};
    AgRunConfig r = run;
    void *ia[2] = {&sp, &r};
    AgPullParams seed_spmv = push_spmv_params(g, 1), loop_spmv = push_spmv_params(g, 0);
    seed_spmv.honor_stop = 0;
    void *sa[1] = {&seed_spmv}, *la[1] = {&loop_spmv};
    const void *kse = ag_pull_kernel_ptr(AG_MODE_SPMV, 0, 1), *ksl = ag_pull_kernel_ptr(AG_MODE_SPMV, 0, 0);
    PushScatterShape sh;
    ag_status_t sst = push_scatter_shape(kind, &sh);
    if (sst != AG_OK)
        return sst;
    if (kind == AG_PUSH_QUANT) {
        AG_CUDA(cudaMemsetAsync(g->qmm, 0xFF, 8, s));
        AG_CUDA(cudaMemsetAsync(g->qmm + 2, 0, 8, s));
    }
    if (residual) {
        AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 3), eg, blk, pa, 0, s));
        if (seed_spmv.ntasks)
            AG_CUDA(cudaLaunchKernel(kse, dim3(pull_grid(kse, seed_spmv.ntasks, push_spmv_smem(seed_spmv))),
                                     dim3(AG_BLK), sa, push_spmv_smem(seed_spmv), s));
    }
    AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 0), eg, blk, ia, 0, s));
    for (uint32_t i = 0; i < run.max_iter; ++i) {
        if (kind == AG_PUSH_QUANT)
            AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 3), eg, blk, pa, 0, s));
        if (kind == AG_PUSH_PULLPUSH && loop_spmv.ntasks)
            AG_CUDA(cudaLaunchKernel(ksl, dim3(pull_grid(ksl, loop_spmv.ntasks, push_spmv_smem(loop_spmv))),
                                     dim3(AG_BLK), la, push_spmv_smem(loop_spmv), s));
        if (residual) {
            AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 1), eg, blk, pa, 0, s));
            AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 2), sh.grid, sh.block, pa, sh.smem, s));
        } else {
            AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 1), sh.grid, sh.block, pa, sh.smem, s));
            AG_CUDA(cudaLaunchKernel(ag_push_kernel_ptr(kind, 2), eg, blk, pa, 0, s));
        }
    }
    AG_CUDA(cudaLaunchKernel(ag_normalize_kernel_ptr(), eg, blk, pa, 0, s));
    return AG_OK;
}

/* push-direction and residual solves (ag_pr_opts.direction != AG_DIR_PULL) */
static ag_status_t push_launch(ag_graph_s *g, const ag_pr_opts &o, uint32_t max_iterations, double epsilon)
{
    int kind;
    if (o.direction == AG_DIR_PULL_PUSH)
        kind = AG_PUSH_PULLPUSH;
    else if (o.data_driven)
        kind = AG_PUSH_DD;
    else if (o.precision == AG_PREC_FP32)
        kind = AG_PUSH_FLOAT;
    else if (o.precision == AG_PREC_FIXED64)
        kind = AG_PUSH_FIXED;
    else if (o.precision == AG_PREC_QUANT32)
        kind = AG_PUSH_QUANT;
    else
        return ag_set_error(AG_ERR_UNSUPPORTED, "the push runs in FP32, 64-bit fixed point or 32-bit quantised");
    if ((kind == AG_PUSH_DD || kind == AG_PUSH_PULLPUSH) && o.precision != AG_PREC_FP32)
        return ag_set_error(AG_ERR_UNSUPPORTED, "the data-driven push and pull-push run in FP32");
    if (g->ngraphs || g->norm_n || g->c_base)
        return ag_set_error(AG_ERR_UNSUPPORTED, "the push forms run on a whole graph");
    ag_status_t st = ensure_push(g, kind);
    if (st != AG_OK)
        return st;
    if (o.init_ranks && !g->init_buf) {
        g->init_buf = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        if (st != AG_OK)
            return st;
        drop_execs(g);
    }
    if (!g->have_exe_push[kind]) {
        st = build_exec_push(g, kind);
        if (st != AG_OK)
            return st;
    }
    AgExec *x = &g->exe_push[kind];
    cudaStream_t s = g_ctx.stream;
    if (o.init_ranks && g->N)
        AG_CUDA(cudaMemcpyAsync(g->init_buf, o.init_ranks, (size_t)g->N * 4,
                                o.init_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    AgRunConfig run;
    memset(&run, 0, sizeof(run));
    run.max_iter = std::min<uint32_t>(max_iterations, AG_MAX_HISTORY);
    run.use_init = o.init_ranks ? 1u : 0u;
    run.eps = epsilon;
    run.switch_residual = 1e-4;
    void *init_args[2] = {&x->params, &run};
    cudaKernelNodeParams kp;
    AG_CUDA(cudaGraphKernelNodeGetParams(x->init_node, &kp));
    kp.kernelParams = init_args;
    AG_CUDA(cudaGraphExecKernelNodeSetParams(x->exec, x->init_node, &kp));
    AG_CUDA(cudaEventRecord(g->ev0, s));
    const char *mode = getenv("AG_LAUNCH_MODE");
    if (mode && strcmp(mode, "stream") == 0) {
        st = push_stream_launch(g, kind, run);
        if (st != AG_OK)
            return st;
    } else {
        AG_CUDA(cudaGraphLaunch(x->exec, s));
    }
    AG_CUDA(cudaEventRecord(g->ev1, s));
    g->launched = 1;
    g->last_prec = o.precision;
    g->last_exact = 0;
    return AG_OK;
}

extern "C" void ag_pr_opts_init(ag_pr_opts *o)
{
    if (!o)
        return;
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(*o);
    o->precision = AG_PREC_FP32;
    /* the reference's stream-order sums unless the caller asks for FAST */
    o->order = AG_ORDER_EXACT;
    o->switch_residual = 1e-4;
}

/* a row-partitioned upload names other ranks' rows by padded global id and
 * writes its contributions at its slice of a full-length vector: only the
 * ag_partition_* entries run on it */
static ag_status_t whole_graph(const ag_graph_s *g, const char *what)
{
    if (g->norm_n)
        return ag_set_error(AG_ERR_UNSUPPORTED, "%s: a row-partitioned graph runs through ag_partition_step", what);
    return AG_OK;
}

extern "C" ag_status_t ag_pagerank_launch(ag_graph_t g, uint32_t max_iterations, double epsilon,
                                          const ag_pr_opts *opts)
{
    ag_clear_error();
    if (!g)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_pagerank_launch: NULL graph");
    if (whole_graph(g, "ag_pagerank_launch") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    ag_pr_opts o;
    ag_pr_opts_init(&o);
    if (opts)
        memcpy(&o, opts, std::min<size_t>(sizeof(o), opts->struct_size ? opts->struct_size : sizeof(o)));
    if (o.precision < 0 || o.precision > AG_PREC_QUANT8)
        return ag_set_error(AG_ERR_INVALID_ARG, "unknown precision %d", o.precision);
    if (o.direction < AG_DIR_PULL || o.direction > AG_DIR_PULL_PUSH)
        return ag_set_error(AG_ERR_INVALID_ARG, "unknown direction %d", o.direction);
    if (o.direction != AG_DIR_PULL)
        return push_launch(g, o, max_iterations, epsilon);
    if (g->ngraphs && (o.precision != AG_PREC_FP32 || o.init_ranks || o.data_driven))
        return ag_set_error(AG_ERR_UNSUPPORTED, "a graph union runs the FP32 form without a warm start");
    const int dd = o.data_driven ? 1 : 0;
    if (dd && (o.precision != AG_PREC_FP32 || g->norm_n || g->c_base))
        return ag_set_error(AG_ERR_UNSUPPORTED, "the data-driven pull runs in FP32 on a whole graph");
    const int ip = is_int_prec(o.precision);
    if (ip && (g->norm_n || g->c_base))
        return ag_set_error(AG_ERR_UNSUPPORTED, "the fixed-point and quantised pulls run on a whole graph");
    const int prec = o.precision, exact = o.order == AG_ORDER_EXACT ? 1 : 0;
    const int quant = ip && int_quant(prec);
    ag_status_t st = ip ? ensure_fixed(g, quant) : ensure_buffers(g, prec);
    if (st != AG_OK)
        return st;
    if (o.init_ranks && !g->init_buf) {
        g->init_buf = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        if (st != AG_OK)
            return st;
        /* rebuild cached graphs: their parameters carry the warm-start pointer */
        drop_execs(g);
    }
    if (!have_exec(g, prec, exact, dd)) {
        st = build_exec(g, prec, exact, dd);
        if (st != AG_OK)
            return st;
    }
    AgExec *x = exec_slot(g, prec, exact, dd);
    cudaStream_t s = g_ctx.stream;
    if (o.init_ranks && g->N)
        AG_CUDA(cudaMemcpyAsync(g->init_buf, o.init_ranks, (size_t)g->N * 4,
                                o.init_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    AgRunConfig run;
    memset(&run, 0, sizeof(run));
    run.max_iter = std::min<uint32_t>(max_iterations, AG_MAX_HISTORY);
    run.use_init = o.init_ranks ? 1u : 0u;
    run.eps = epsilon;
    run.switch_residual = o.switch_residual > 0 ? o.switch_residual : 1e-4;
    void *init_args[2] = {&x->params, &run};
    cudaKernelNodeParams kp;
    AG_CUDA(cudaGraphKernelNodeGetParams(x->init_node, &kp));
    kp.kernelParams = init_args;
    AG_CUDA(cudaGraphExecKernelNodeSetParams(x->exec, x->init_node, &kp));
    AG_CUDA(cudaEventRecord(g->ev0, s));
    const char *mode = getenv("AG_LAUNCH_MODE");
    if (mode && strcmp(mode, "stream") == 0) {
        /* profiling form: the same kernels as separate launches (a profiler
         * sees every pass); passes after convergence return at once */
        AgPullParams sp = x->params;
        sp.use_cond = 0;
        cudaKernelNodeParams ki;
        AG_CUDA(cudaGraphKernelNodeGetParams(x->init_node, &ki));
        void *ia[2] = {&sp, &run};
        if (quant) {
            AG_CUDA(cudaMemsetAsync(g->qmm, 0xFF, 8, s));
            AG_CUDA(cudaMemsetAsync(g->qmm + 2, 0, 8, s));
        }
        AG_CUDA(cudaLaunchKernel(ki.func, ki.gridDim, ki.blockDim, ia, 0, s));
        void *pa[1] = {&sp};
        const void *kpull = solve_pull_kernel(g, prec, exact, dd);
        const size_t smem = solve_smem(g, prec);
        for (uint32_t i = 0; i < run.max_iter; ++i) {
            if (quant)
                AG_CUDA(cudaLaunchKernel(ag_quant_kernel_ptr(int_bytes(prec)), quant_grid(g), dim3(AG_SBLK), pa, 0, s));
            AG_CUDA(cudaLaunchKernel(kpull, dim3(x->grid), dim3(AG_BLK), pa, smem, s));
        }
        AG_CUDA(cudaLaunchKernel(ag_normalize_kernel_ptr(), ki.gridDim, ki.blockDim, pa, 0, s));
    } else {
        AG_CUDA(cudaGraphLaunch(x->exec, s));
    }
    AG_CUDA(cudaEventRecord(g->ev1, s));
    g->launched = 1;
    g->last_prec = prec;
    g->last_exact = exact;
    return AG_OK;
}

extern "C" ag_status_t ag_pagerank_fetch(ag_graph_t g, float *ranks, ag_pr_result *res, uint32_t *hist_active,
                                         double *hist_error, double *hist_seconds, uint32_t history_len)
{
    if (!g)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_pagerank_fetch: NULL graph");
    if (!g->launched)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_pagerank_fetch: nothing launched on this graph");
    cudaStream_t s = g_ctx.stream;
    ag_status_t st = stream_wait(s, 0);
    if (st != AG_OK)
        return st;
    AgControl *hc = (AgControl *)malloc(sizeof(AgControl));
    if (!hc)
        return ag_set_error(AG_ERR_OOM, "host allocation failed");
    cudaError_t e = cudaMemcpy(hc, g->ctl, sizeof(AgControl), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        free(hc);
        return ag_set_error(AG_ERR_CUDA, "control readback failed: %s", cudaGetErrorString(e));
    }
    if (ranks && g->N) {
        st = copy_to_host(ranks, g->out, (size_t)g->N * 4);
        if (st != AG_OK) {
            free(hc);
            return st;
        }
    }
    const uint32_t passes = hc->iter;
    if (res) {
        memset(res, 0, sizeof(*res));
        res->passes = passes;
        res->converged = hc->converged;
        res->iterations = hc->converged ? (passes ? passes - 1 : 0) : passes;
        res->active_last = passes ? hc->hist_active[std::min<uint32_t>(passes, AG_MAX_HISTORY) - 1] : 0;
        res->error_total = passes ? hc->hist_err[std::min<uint32_t>(passes, AG_MAX_HISTORY) - 1] : 0.0;
        res->rank_sum = hc->rank_sum;
        res->switch_pass = hc->switch_pass;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) == cudaSuccess)
            res->device_ms = ms;
    }
    const uint32_t n = std::min<uint32_t>(std::min<uint32_t>(passes, history_len), AG_MAX_HISTORY);
    for (uint32_t i = 0; i < n; ++i) {
        if (hist_active)
            hist_active[i] = hc->hist_active[i];
        if (hist_error)
            hist_error[i] = hc->hist_err[i];
        if (hist_seconds) {
            const unsigned long long prev = i ? hc->hist_t[i - 1] : hc->t0;
            hist_seconds[i] = (double)(hc->hist_t[i] - prev) * 1e-9;
        }
    }
    const uint32_t fault = hc->fault;
    free(hc);
    if (fault)
        return ag_set_error(AG_ERR_DEVICE_WAIT, "a pull kernel's bounded wait for its hot-table copy ran out "
                            "(the copies completed before the kernel went on; results are filled in)");
    return AG_OK;
}

extern "C" const float *ag_pagerank_device_ranks(ag_graph_t g) { return g ? g->out : nullptr; }

/* ------------------------------------------------------------------ SpMV */
extern "C" ag_status_t ag_spmv_pull_device(ag_graph_t g, const float *x, float *y, uint32_t mode)
{
    ag_clear_error();
    if (!g || (g->N && (!x || !y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_pull_device: NULL argument");
    if (whole_graph(g, "ag_spmv_pull_device") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    if (g->N == 0)
        return AG_OK;
    cudaStream_t s = g_ctx.stream;
    ag_status_t st = AG_OK;
    if (g->perm && !g->xbuf) {
        g->xbuf = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        g->ybuf = (float *)dev_alloc(g, (size_t)g->N * 4 + 16, &st);
        if (st != AG_OK)
            return st;
    }
    const int exact = (mode & AG_SPMV_EXACT) ? 1 : 0;
    AgPullParams p = base_params(g, exact);
    /* caller order in and out; the product runs in device order */
    if (g->perm)
        AG_CUDA(ag_permute_in(g->perm, x, g->xbuf, g->N, s));
    p.x = g->perm ? g->xbuf : x;
    p.rank = g->perm ? g->ybuf : y;
    /* the hot table needs a 16-byte aligned vector */
    if (((uintptr_t)p.x & 15u) != 0)
        p.hot_n = 0;
    p.wmode = (mode & AG_SPMV_UNIT) ? AG_SPMV_W_UNIT : (g->w ? AG_SPMV_W_GRAPH : AG_SPMV_W_CONST);
    const void *k = ag_pull_kernel_ptr(AG_MODE_SPMV, 0, exact);
    const size_t smem = (size_t)AG_STAGE_BYTES + (size_t)p.hot_n * 4;
    const unsigned grid = pull_grid(k, p.ntasks, smem);
    void *args[1] = {&p};
    AG_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(AG_BLK), args, smem, s));
    if (g->perm)
        AG_CUDA(ag_permute_out(g->inv, g->ybuf, y, g->N, s));
    return AG_OK;
}

extern "C" ag_status_t ag_spmv_pull(ag_graph_t g, const float *x, float *y, uint32_t mode)
{
    ag_clear_error();
    if (!g || (g->N && (!x || !y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_pull: NULL argument");
    if (whole_graph(g, "ag_spmv_pull") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    if (g->N == 0)
        return AG_OK;
    ag_status_t st = AG_OK;
    float *dx = nullptr, *dy = nullptr;
    cudaStream_t s = g_ctx.stream;
    AG_CUDA(cudaMallocAsync((void **)&dx, (size_t)g->N * 4, s));
    AG_CUDA(cudaMallocAsync((void **)&dy, (size_t)g->N * 4, s));
    AG_CUDA(cudaMemcpyAsync(dx, x, (size_t)g->N * 4, cudaMemcpyHostToDevice, s));
    st = ag_spmv_pull_device(g, dx, dy, mode);
    if (st == AG_OK)
        st = copy_to_host(y, dy, (size_t)g->N * 4);
    cudaFreeAsync(dx, s);
    cudaFreeAsync(dy, s);
    ag_status_t w = stream_wait(s, 0);
    return st != AG_OK ? st : w;
}

/* -------------------------------------------------------- FP64 oracle */
extern "C" ag_status_t ag_pagerank_f64(ag_graph_t g, uint32_t max_iterations, double tol, double *ranks,
                                       uint32_t *passes)
{
    ag_clear_error();
    if (!g || !ranks)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_pagerank_f64: NULL argument");
    if (whole_graph(g, "ag_pagerank_f64") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    cudaStream_t s = g_ctx.stream;
    double *r = nullptr, *r2 = nullptr, *c = nullptr, *md = nullptr;
    const size_t nb = (size_t)g->N * 8 + 16;
    AG_CUDA(cudaMallocAsync((void **)&r, nb, s));
    AG_CUDA(cudaMallocAsync((void **)&r2, nb, s));
    AG_CUDA(cudaMallocAsync((void **)&c, nb, s));
    AG_CUDA(cudaMallocAsync((void **)&md, 16, s));
    uint32_t it = 0;
    cudaError_t e = ag_pr_f64_run(g->row_off, g->ids, g->outdeg, g->N, max_iterations, tol, r, r2, c, md, &it, s);
    if (e == cudaSuccess && g->N)
        e = cudaMemcpyAsync(ranks, r, (size_t)g->N * 8, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(r, s);
    cudaFreeAsync(r2, s);
    cudaFreeAsync(c, s);
    cudaFreeAsync(md, s);
    ag_status_t w = stream_wait(s, 0);
    if (e != cudaSuccess)
        return ag_set_error(AG_ERR_CUDA, "FP64 oracle failed: %s", cudaGetErrorString(e));
    if (w != AG_OK)
        return w;
    if (g->inv) {
        std::vector<uint32_t> inv(g->N);
        std::vector<double> dev_order(ranks, ranks + g->N);
        AG_CUDA(cudaMemcpy(inv.data(), g->inv, (size_t)g->N * 4, cudaMemcpyDeviceToHost));
        for (uint32_t v = 0; v < g->N; ++v)
            ranks[v] = dev_order[inv[v]];
    }
    for (uint32_t v = 0; v < g->N; ++v)
        ranks[v] /= (double)g->N;
    if (passes)
        *passes = it;
    return AG_OK;
}

extern "C" ag_status_t ag_spmv_run_host(ag_graph_t g, const float *x, float *y, uint32_t iterations, uint32_t mode,
                                        double *iter_seconds)
{
    if (!g || (g->N && (!x || !y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_run_host: NULL argument");
    if (whole_graph(g, "ag_spmv_run_host") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    if (g->N == 0)
        return AG_OK;
    cudaStream_t s = g_ctx.stream;
    float *dx = nullptr, *dy = nullptr;
    std::vector<cudaEvent_t> ev(iterations + 1);
    ag_status_t st = AG_OK;
    AG_CUDA(cudaMallocAsync((void **)&dx, (size_t)g->N * 4, s));
    AG_CUDA(cudaMallocAsync((void **)&dy, (size_t)g->N * 4, s));
    AG_CUDA(cudaMemcpyAsync(dx, x, (size_t)g->N * 4, cudaMemcpyHostToDevice, s));
    AG_CUDA(cudaMemsetAsync(dy, 0, (size_t)g->N * 4, s));
    for (uint32_t i = 0; i <= iterations; ++i)
        AG_CUDA(cudaEventCreate(&ev[i]));
    AG_CUDA(cudaEventRecord(ev[0], s));
    for (uint32_t i = 0; i < iterations && st == AG_OK; ++i) {
        st = ag_spmv_pull_device(g, dx, dy, mode);
        if (st == AG_OK)
            AG_CUDA(cudaEventRecord(ev[i + 1], s));
    }
    if (st == AG_OK) {
        cudaError_t e = cudaMemcpyAsync(y, dy, (size_t)g->N * 4, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess)
            st = ag_set_error(AG_ERR_CUDA, "y readback failed: %s", cudaGetErrorString(e));
    }
    ag_status_t w = stream_wait(s, 0);
    if (st == AG_OK && w == AG_OK && iter_seconds) {
        for (uint32_t i = 0; i < iterations; ++i) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
            iter_seconds[i] = ms * 1e-3;
        }
    }
    for (uint32_t i = 0; i <= iterations; ++i)
        cudaEventDestroy(ev[i]);
    cudaFreeAsync(dx, s);
    cudaFreeAsync(dy, s);
    return st != AG_OK ? st : w;
}


extern "C" ag_status_t ag_rt_graph_view(ag_graph_t g, AgGraphView *v)
{
    if (!g || !v)
        return ag_set_error(AG_ERR_INVALID_ARG, "NULL graph");
    if (g->norm_n)
        return ag_set_error(AG_ERR_UNSUPPORTED, "a row-partitioned graph names other ranks' rows by global id; this "
                            "entry needs a whole graph");
    v->row_off = g->row_off;
    v->ids = g->ids;
    v->outdeg = g->outdeg;
    v->perm = g->perm;
    v->inv = g->inv;
    v->N = g->N;
    v->E = g->E;
    v->stream = g_ctx.stream;
    v->tasks = g->tasks_fast;
    v->ntasks = g->ntasks_fast;
    v->hub_slots = g->nparts;
    return AG_OK;
}

/* ------------------------------------------------- union of graphs */
extern "C" ag_status_t ag_multigraph_upload(const struct GraphCSR *const *graphs, uint32_t count, uint32_t flags,
                                            ag_graph_t *out)
{
    ag_clear_error();
    if (!graphs || !out || count == 0)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_multigraph_upload: need at least one graph");
    uint64_t N = 0, E = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (!graphs[i])
            return ag_set_error(AG_ERR_INVALID_ARG, "ag_multigraph_upload: graph %u is NULL", i);
        N += graphs[i]->num_vertices;
        E += graphs[i]->num_edges;
    }
    if (N > AG_ROW_MASK || E >= 0xFFFFFFF0ull)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_multigraph_upload: union of %llu vertices, %llu edges too large",
                            (unsigned long long)N, (unsigned long long)E);
    /* block-diagonal union: graph i's vertices follow graph i-1's */
    std::vector<uint32_t> gstart(count + 1), indeg(N), idx(N), outdeg(N), nb(E);
    uint64_t vb = 0, ebase = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const struct GraphCSR *gi = graphs[i];
        const uint32_t n = gi->num_vertices;
        gstart[i] = (uint32_t)vb;
        uint64_t pos = ebase;
        for (uint32_t v = 0; v < n; ++v) {
            const uint32_t d = gi->inverse_vertices->out_degree[v], b = gi->inverse_vertices->edges_idx[v];
            if ((uint64_t)b + d > gi->num_edges)
                return ag_set_error(AG_ERR_INVALID_GRAPH, "graph %u row %u exceeds its edges", i, v);
            indeg[vb + v] = d;
            idx[vb + v] = (uint32_t)pos;
            outdeg[vb + v] = gi->vertices->out_degree[v];
            for (uint32_t j = 0; j < d; ++j) {
                const uint32_t u = gi->inverse_sorted_edges_array->edges_array_dest[b + j];
                if (u >= n)
                    return ag_set_error(AG_ERR_INVALID_GRAPH, "graph %u: in-edge names vertex %u >= %u", i, u, n);
                nb[pos + j] = (uint32_t)(vb + u);
            }
            pos += d;
        }
        vb += n;
        ebase = pos;
    }
    gstart[count] = (uint32_t)vb;
    struct Vertex fv = {outdeg.data(), indeg.data(), nullptr};
    struct Vertex iv = {indeg.data(), outdeg.data(), idx.data()};
    struct EdgeList iel;
    memset(&iel, 0, sizeof(iel));
    iel.num_edges = (uint32_t)E;
    iel.num_vertices = (uint32_t)N;
    iel.edges_array_dest = nb.data();
    struct GraphCSR u;
    memset(&u, 0, sizeof(u));
    u.num_vertices = (uint32_t)N;
    u.num_edges = (uint32_t)E;
    u.vertices = &fv;
    u.inverse_vertices = &iv;
    u.inverse_sorted_edges_array = &iel;
    /* vertices stay grouped by graph; the union is L2-resident at the sizes
     * it is meant for, so no shared-memory table */
    return upload_impl(&u, flags | AG_UPLOAD_KEEP_ORDER | AG_UPLOAD_NO_SMEM_CACHE, gstart.data(), count, 0, out);
}

extern "C" ag_status_t ag_multigraph_fetch(ag_graph_t g, float *ranks, uint32_t *iterations, uint32_t *passes,
                                           uint32_t *converged, double *error_total, double *device_ms)
{
    if (!g || !g->ngraphs)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_multigraph_fetch: not a graph union");
    ag_pr_result res;
    ag_status_t st = ag_pagerank_fetch(g, ranks, &res, nullptr, nullptr, nullptr, 0);
    if (st != AG_OK)
        return st;
    const uint32_t n = g->ngraphs;
    std::vector<uint32_t> h(4 * (size_t)n);
    std::vector<double> hd(2 * (size_t)n);
    AG_CUDA(cudaMemcpy(h.data(), g->g_u32, h.size() * 4, cudaMemcpyDeviceToHost));
    AG_CUDA(cudaMemcpy(hd.data(), g->g_f64, hd.size() * 8, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t np = h[2 * (size_t)n + i], cv = h[3 * (size_t)n + i];
        if (passes)
            passes[i] = np;
        if (converged)
            converged[i] = cv;
        if (iterations)
            iterations[i] = cv ? (np ? np - 1 : 0) : np; /* reference semantics per graph */
        if (error_total)
            error_total[i] = hd[(size_t)n + i];
    }
    if (device_ms)
        *device_ms = res.device_ms;
    return AG_OK;
}

/* ------------------------------------------------------------ tiles */
extern "C" ag_status_t ag_graph_get_tiles(ag_graph_t g, ag_tile_config *cfg)
{
    if (!g || !cfg)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_get_tiles: NULL argument");
    *cfg = g->tiles;
    return AG_OK;
}

extern "C" ag_status_t ag_graph_get_tasks(ag_graph_t g, int exact, uint32_t *items, uint32_t capacity,
                                         uint32_t *count)
{
    ag_clear_error();
    if (!g || !count || (capacity && !items))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_get_tasks: NULL argument");
    const uint32_t n = exact ? g->ntasks_exact : g->ntasks_fast;
    *count = n;
    const uint32_t k = std::min(n, capacity);
    if (k) {
        ag_status_t st = stream_wait(g_ctx.stream, 0);
        if (st != AG_OK)
            return st;
        AG_CUDA(cudaMemcpy(items, exact ? g->tasks_exact : g->tasks_fast, (size_t)k * sizeof(uint4),
                           cudaMemcpyDeviceToHost));
    }
    return AG_OK;
}

/* re-plan the work lists for a new tile shape; cached launch graphs are
 * rebuilt on the next launch */
extern "C" ag_status_t ag_graph_set_tiles(ag_graph_t g, const ag_tile_config *cfg)
{
    ag_clear_error();
    if (!g || !cfg)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_set_tiles: NULL argument");
    /* hub_chunk is a multiple of 32: an EXACT-order hub row's staging slots
     * then start on 16-byte boundaries and hold whole 16-byte groups */
    if (cfg->task_edges < 32 || cfg->task_edges > AG_WCAP || cfg->hub_chunk < cfg->task_edges ||
        cfg->hub_chunk > (1u << 20) || cfg->hub_chunk % 32u != 0)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_set_tiles: task_edges in [32, %u], hub_chunk a multiple "
                            "of 32 in [task_edges, 2^20]", AG_WCAP);
    cudaStream_t s = g_ctx.stream;
    ag_status_t st = stream_wait(s, 0);
    if (st != AG_OK)
        return st;
    const uint32_t N = g->N;
    st = plan_device(g, cfg->task_edges, cfg->hub_chunk);
    if (st != AG_OK)
        return st;
    g->tiles = *cfg;
    g->hot_n = g->hot_allowed ? std::min<uint32_t>(std::min<uint32_t>(cfg->hot_entries, AG_HOT_MAX), N) & ~63u : 0u;
    g->warm_n = std::max<uint32_t>(cfg->warm_entries, g->hot_n);
    g->tiles.hot_entries = g->hot_n;
    g->tiles.warm_entries = g->warm_n;
    drop_execs(g);
    return stream_wait(s, 0);
}

/* Time each candidate tile shape on this graph (FP32, FAST order, a fixed
 * number of passes that never stop early) and keep the fastest.  Candidates:
 * item caps {128, 256}, hub chunks {1024, 2048, 4096}, and, when the
 * shared-memory table is allowed, table sizes {0, 8K, 16K, 24K} entries.
 * With AG_TUNE_CACHE naming a file, results are read from and appended to it
 * (one line per graph shape: N E max-in-degree device cap chunk hot warm us). */
extern "C" ag_status_t ag_autotune(ag_graph_t g, uint32_t passes, ag_tile_config *best, double *best_pass_us)
{
    ag_clear_error();
    if (!g)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_autotune: NULL graph");
    if (whole_graph(g, "ag_autotune") != AG_OK)
        return AG_ERR_UNSUPPORTED;
    if (passes == 0)
        passes = 8;
    char dev_name[256] = "unknown";
    {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, g_ctx.device) == cudaSuccess) {
            snprintf(dev_name, sizeof(dev_name), "%s", prop.name);
            for (char *c = dev_name; *c; ++c)
                if (*c == ' ')
                    *c = '_';
        }
    }
    const char *cache = getenv("AG_TUNE_CACHE");
    if (cache) {
        FILE *f = fopen(cache, "r");
        if (f) {
            unsigned n, e, md, cap, chunk, hot, warm;
            double us;
            char dn[256];
            while (fscanf(f, "%u %u %u %255s %u %u %u %u %lf", &n, &e, &md, dn, &cap, &chunk, &hot, &warm, &us) == 9) {
                if (n == g->N && e == g->E && md == g->max_in_degree && strcmp(dn, dev_name) == 0) {
                    ag_tile_config c = {cap, chunk, hot, warm};
                    fclose(f);
                    ag_status_t st = ag_graph_set_tiles(g, &c);
                    if (st == AG_OK) {
                        if (best)
                            *best = g->tiles;
                        if (best_pass_us)
                            *best_pass_us = us;
                    }
                    return st;
                }
            }
            fclose(f);
        }
    }
    std::vector<ag_tile_config> cands;
    const uint32_t caps[2] = {128, 256};
    const uint32_t chunks[3] = {1024, 2048, 4096};
    const uint32_t hots[4] = {0, 8192, 16384, 24576};
    const int nh = g->hot_allowed ? 4 : 1;
    for (uint32_t c : caps)
        for (uint32_t h : chunks)
            for (int k = 0; k < nh; ++k)
                cands.push_back({c, h, hots[k], std::max<uint32_t>(65536u, hots[k])});
    ag_tile_config bestc = g->tiles;
    double bestus = 1e300;
    ag_pr_opts o;
    ag_pr_opts_init(&o);
    o.quiet = 1;
    for (const ag_tile_config &c : cands) {
        ag_status_t st = ag_graph_set_tiles(g, &c);
        if (st != AG_OK)
            return st;
        ag_pr_result r;
        double us = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            st = ag_pagerank_launch(g, passes, 0.0, &o);
            if (st == AG_OK)
                st = ag_pagerank_fetch(g, nullptr, &r, nullptr, nullptr, nullptr, 0);
            if (st != AG_OK)
                return st;
            if (rep == 1 && r.passes)
                us = r.device_ms * 1e3 / r.passes;
        }
        if (us < bestus) {
            bestus = us;
            bestc = g->tiles;
        }
    }
    ag_status_t st = ag_graph_set_tiles(g, &bestc);
    if (st != AG_OK)
        return st;
    if (cache) {
        FILE *f = fopen(cache, "a");
        if (f) {
            fprintf(f, "%u %u %u %s %u %u %u %u %.3f\n", g->N, g->E, g->max_in_degree, dev_name, bestc.task_edges,
                    bestc.hub_chunk, bestc.hot_entries, bestc.warm_entries, bestus);
            fclose(f);
        }
    }
    if (best)
        *best = g->tiles;
    if (best_pass_us)
        *best_pass_us = bestus;
    return AG_OK;
}

/* --------------------------------------------- row-partitioned solves */
extern "C" ag_status_t ag_graph_upload_rows(const struct GraphCSR *graph, const uint32_t *bounds, uint32_t nranks,
                                            uint32_t rank, uint32_t slice, uint32_t flags, ag_graph_t *out)
{
    ag_clear_error();
    if (!graph || !bounds || !out || nranks == 0 || rank >= nranks)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_upload_rows: bad argument");
    const uint32_t N = graph->num_vertices;
    if (bounds[0] != 0 || bounds[nranks] != N)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_upload_rows: bounds must run from 0 to num_vertices");
    for (uint32_t r = 0; r < nranks; ++r)
        if (bounds[r] > bounds[r + 1] || bounds[r + 1] - bounds[r] > slice)
            return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_upload_rows: range %u exceeds the slice %u", r, slice);
    if ((uint64_t)slice * nranks > AG_ROW_MASK)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_graph_upload_rows: padded vector too long");
    const uint32_t rb = bounds[rank], re = bounds[rank + 1], n = re - rb;
    const struct Vertex *iv = graph->inverse_vertices;
    const struct EdgeList *iel = graph->inverse_sorted_edges_array;
    /* padded id of vertex u: owner rank's slice start + offset in the range */
    std::vector<uint32_t> owner_base(N);
    for (uint32_t r = 0; r < nranks; ++r)
        for (uint32_t u = bounds[r]; u < bounds[r + 1]; ++u)
            owner_base[u] = r * slice + (u - bounds[r]);
    uint64_t e = 0;
    for (uint32_t v = rb; v < re; ++v)
        e += iv->out_degree[v];
    if (e >= 0xFFFFFFF0ull)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_graph_upload_rows: too many edges in one range");
    std::vector<uint32_t> indeg(n), idx(n), outdeg(n), nb(e);
    uint64_t pos = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t v = rb + i, d = iv->out_degree[v], b = iv->edges_idx[v];
        if ((uint64_t)b + d > graph->num_edges)
            return ag_set_error(AG_ERR_INVALID_GRAPH, "row %u exceeds the edge array", v);
        indeg[i] = d;
        idx[i] = (uint32_t)pos;
        outdeg[i] = graph->vertices->out_degree[v];
        for (uint32_t j = 0; j < d; ++j) {
            const uint32_t u = iel->edges_array_dest[b + j];
            if (u >= N)
                return ag_set_error(AG_ERR_INVALID_GRAPH, "in-edge names vertex %u >= %u", u, N);
            nb[pos + j] = owner_base[u];
        }
        pos += d;
    }
    struct Vertex fv = {outdeg.data(), indeg.data(), nullptr};
    struct Vertex lv = {indeg.data(), outdeg.data(), idx.data()};
    struct EdgeList lel;
    memset(&lel, 0, sizeof(lel));
    lel.num_edges = (uint32_t)e;
    lel.num_vertices = n;
    lel.edges_array_dest = nb.data();
    struct GraphCSR lg;
    memset(&lg, 0, sizeof(lg));
    lg.num_vertices = n;
    lg.num_edges = (uint32_t)e;
    lg.vertices = &fv;
    lg.inverse_vertices = &lv;
    lg.inverse_sorted_edges_array = &lel;
    ag_graph_t g = nullptr;
    ag_status_t st = upload_impl(&lg, flags | AG_UPLOAD_KEEP_ORDER | AG_UPLOAD_NO_SMEM_CACHE, nullptr, 0,
                                 slice * nranks, &g);
    if (st != AG_OK)
        return st;
    g->c_base = rank * slice;
    g->norm_n = N;
    *out = g;
    return AG_OK;
}

/* first contributions of this rank's rows into its slice of c_full
 * (ranks start at base_pr) */
extern "C" ag_status_t ag_partition_init(ag_graph_t g, float *c_full)
{
    ag_clear_error();
    if (!g || !c_full || !g->norm_n)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_init: not a row partition");
    AgPullParams p = base_params(g, 0);
    p.c32_0 = c_full;
    AgRunConfig run;
    memset(&run, 0, sizeof(run));
    run.max_iter = AG_MAX_HISTORY;
    run.eps = 0.0;
    void *args[2] = {&p, &run};
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)g->N + AG_SBLK - 1) / AG_SBLK, (uint64_t)g_ctx.num_sms * 8));
    AG_CUDA(cudaLaunchKernel(ag_init_kernel_ptr(0), dim3(grid), dim3(AG_SBLK), args, 0, g_ctx.stream));
    return AG_OK;
}

__global__ void ag_partition_setup_kernel(AgControl *c, double eps)
{
    c->iter = 0;
    c->max_iter = AG_MAX_HISTORY;
    c->active_acc = 0;
    c->done_ctas = 0;
    c->err_acc = 0.0;
    c->eps = eps;
    c->stop = 0;
    c->mode_read = 0;
    c->mode_write = 0;
}

__global__ void ag_partition_stats_kernel(const AgControl *c, double *stats)
{
    stats[0] = (double)c->hist_active[0];
    stats[1] = c->last_err_sum;
}

/* one pull pass over this rank's rows: gathers from c_in_full (all ranks'
 * slices), writes this rank's slice of c_out_full; stats_dev[0] = active
 * rows, stats_dev[1] = sum of |r' - r| (device doubles, for the caller's
 * all-reduce).  Enqueued on ag_stream() without waiting. */
extern "C" ag_status_t ag_partition_pass(ag_graph_t g, const float *c_in_full, float *c_out_full, double epsilon,
                                         double *stats_dev)
{
    ag_clear_error();
    if (!g || !c_in_full || !c_out_full || !stats_dev || !g->norm_n)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_pass: not a row partition / NULL argument");
    cudaStream_t s = g_ctx.stream;
    ag_partition_setup_kernel<<<1, 1, 0, s>>>(g->ctl, epsilon);
    AG_CUDA(cudaGetLastError());
    if (g->N) {
        AgPullParams p = base_params(g, 0);
        p.c32_0 = const_cast<float *>(c_in_full);
        p.c32_1 = c_out_full;
        p.use_cond = 0;
        const void *k = ag_pull_kernel_ptr(AG_MODE_PR, 0, 0);
        const unsigned grid = pull_grid(k, p.ntasks, pull_smem(g));
        void *args[1] = {&p};
        AG_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(AG_BLK), args, pull_smem(g), s));
    }
    ag_partition_stats_kernel<<<1, 1, 0, s>>>(g->ctl, stats_dev);
    AG_CUDA(cudaGetLastError());
    return AG_OK;
}

/* the pass of a solve driven by a device stop flag: state[0] != 0 makes the
 * pull kernel return at once and the statistics zero */
__global__ void ag_partition_step_setup_kernel(AgControl *c, double eps, const uint32_t *state)
{
    c->iter = 0;
    c->max_iter = AG_MAX_HISTORY;
    c->active_acc = 0;
    c->done_ctas = 0;
    c->err_acc = 0.0;
    c->eps = eps;
    c->stop = state[0] ? 1u : 0u;
    c->mode_read = 0;
    c->mode_write = 0;
    c->hist_active[0] = 0;
    c->last_err_sum = 0.0;
}

__global__ void ag_partition_close_kernel(const double *stats, uint32_t *state, double *err)
{
    if (state[0])
        return;
    state[1] += 1;
    *err = stats[1];
    if (stats[0] == 0.0) {
        state[0] = 1;
        state[2] = 1;
    }
}

extern "C" ag_status_t ag_partition_step(ag_graph_t g, const float *c_in_full, float *c_out_full, double epsilon,
                                         int32_t order, double *stats_dev, const uint32_t *state_dev)
{
    ag_clear_error();
    if (!g || !c_in_full || !c_out_full || !stats_dev || !state_dev || !g->norm_n)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_step: not a row partition / NULL argument");
    if (order != AG_ORDER_FAST && order != AG_ORDER_EXACT)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_step: order %d", order);
    cudaStream_t s = g_ctx.stream;
    ag_partition_step_setup_kernel<<<1, 1, 0, s>>>(g->ctl, epsilon, state_dev);
    AG_CUDA(cudaGetLastError());
    if (g->N) {
        const int exact = order == AG_ORDER_EXACT;
        AgPullParams p = base_params(g, exact);
        p.c32_0 = const_cast<float *>(c_in_full);
        p.c32_1 = c_out_full;
        p.use_cond = 0;
        const void *k = ag_pull_kernel_ptr(AG_MODE_PR, 0, exact);
        const unsigned grid = pull_grid(k, p.ntasks, pull_smem(g));
        void *args[1] = {&p};
        AG_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(AG_BLK), args, pull_smem(g), s));
    }
    ag_partition_stats_kernel<<<1, 1, 0, s>>>(g->ctl, stats_dev);
    AG_CUDA(cudaGetLastError());
    return AG_OK;
}

extern "C" ag_status_t ag_partition_close(const double *stats_dev, uint32_t *state_dev, double *err_dev)
{
    ag_clear_error();
    if (!stats_dev || !state_dev || !err_dev)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_close: NULL argument");
    ag_status_t st = ctx_ensure(-1);
    if (st != AG_OK)
        return st;
    ag_partition_close_kernel<<<1, 1, 0, g_ctx.stream>>>(stats_dev, state_dev, err_dev);
    AG_CUDA(cudaGetLastError());
    return AG_OK;
}

/* this rank's ranks divided by the global vertex count (host array) */
extern "C" ag_status_t ag_partition_fetch(ag_graph_t g, float *ranks_local)
{
    ag_clear_error();
    if (!g || !g->norm_n)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_partition_fetch: not a row partition");
    if (g->N == 0)
        return AG_OK;
    AgPullParams p = base_params(g, 0);
    AG_CUDA(cudaMemsetAsync(&g->ctl->rank_sum, 0, sizeof(double), g_ctx.stream));
    void *args[1] = {&p};
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)g->N + AG_SBLK - 1) / AG_SBLK, (uint64_t)g_ctx.num_sms * 8));
    AG_CUDA(cudaLaunchKernel(ag_normalize_kernel_ptr(), dim3(grid), dim3(AG_SBLK), args, 0, g_ctx.stream));
    ag_status_t st = stream_wait(g_ctx.stream, 0);
    if (st != AG_OK)
        return st;
    if (ranks_local)
        AG_CUDA(cudaMemcpy(ranks_local, g->out, (size_t)g->N * 4, cudaMemcpyDeviceToHost));
    return AG_OK;
}

/* ------------------------------------------------ device graph build */
/* device copy of an input array: device memory is used in place, host
 * memory (pageable or page-locked) is copied on the library stream */
static ag_status_t stage_in(const void *p, size_t bytes, const void **dev, void **owned)
{
    *dev = nullptr;
    *owned = nullptr;
    if (!p)
        return AG_OK;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess &&
        (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged)) {
        *dev = p;
        return AG_OK;
    }
    cudaGetLastError();
    void *d = nullptr;
    AG_CUDA(cudaMallocAsync(&d, bytes ? bytes : 16, g_ctx.stream));
    if (bytes) {
        cudaError_t e = cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, g_ctx.stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaFreeAsync(d, g_ctx.stream);
            return ag_set_error(AG_ERR_CUDA, "edge list copy failed: %s", cudaGetErrorString(e));
        }
    }
    *dev = d;
    *owned = d;
    return AG_OK;
}

static ag_status_t build_device_csr(uint32_t N, uint64_t m, const uint32_t *src, const uint32_t *dst,
                                    const float *w, uint32_t flags, AgDevCSR *csr)
{
    memset(csr, 0, sizeof(*csr));
    if (m > 0 && (!src || !dst))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_build: NULL edge arrays");
    const bool sym = (flags & AG_BUILD_SYMMETRIC) != 0;
    if ((sym ? 2 * m : m) >= (1ull << 31))
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_graph_build: %llu edges exceed the 2^31 device build limit",
                            (unsigned long long)(sym ? 2 * m : m));
    if (N > AG_ROW_MASK)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_graph_build: %u vertices exceed the 2^30 row limit", N);
    ag_status_t st = ctx_ensure(-1);
    if (st != AG_OK)
        return st;
    cudaStream_t s = g_ctx.stream;
    const void *ds = nullptr, *dd = nullptr, *dw = nullptr;
    void *os = nullptr, *od = nullptr, *ow = nullptr;
    st = stage_in(src, (size_t)m * 4, &ds, &os);
    if (st == AG_OK)
        st = stage_in(dst, (size_t)m * 4, &dd, &od);
    if (st == AG_OK && w)
        st = stage_in(w, (size_t)m * 4, &dw, &ow);
    void *sym_buf = nullptr;
    if (st == AG_OK && sym) {
        /* every edge followed, after the input list, by its reverse */
        const size_t b = (size_t)m * 4;
        cudaError_t e = cudaMallocAsync(&sym_buf, 6 * b + 16, s);
        unsigned char *q = (unsigned char *)sym_buf;
        if (e == cudaSuccess && b) {
            cudaMemcpyAsync(q, ds, b, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(q + b, dd, b, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(q + 2 * b, dd, b, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(q + 3 * b, ds, b, cudaMemcpyDeviceToDevice, s);
            if (dw) {
                cudaMemcpyAsync(q + 4 * b, dw, b, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(q + 5 * b, dw, b, cudaMemcpyDeviceToDevice, s);
            }
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = ag_set_error(AG_ERR_CUDA, "ag_graph_build: reverse edges: %s", cudaGetErrorString(e));
        } else {
            ds = q;
            dd = q + 2 * b;
            if (dw)
                dw = q + 4 * b;
            m *= 2;
        }
    }
    if (st == AG_OK) {
        uint32_t bad = UINT32_MAX;
        cudaError_t e = ag_csr_build_device(N, (uint32_t)m, (const uint32_t *)ds, (const uint32_t *)dd,
                                            (const float *)dw, flags & ~AG_BUILD_SYMMETRIC, csr, &bad, s);
        if (sym && bad != UINT32_MAX)
            bad = bad % (uint32_t)(m / 2); /* report the input edge */
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (bad != UINT32_MAX)
                st = ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_build: edge %u has an endpoint outside %u vertices",
                                  bad, N);
            else
                st = ag_set_error(AG_ERR_CUDA, "ag_graph_build: device build failed: %s", cudaGetErrorString(e));
        }
    }
    if (os)
        cudaFreeAsync(os, s);
    if (od)
        cudaFreeAsync(od, s);
    if (ow)
        cudaFreeAsync(ow, s);
    if (sym_buf)
        cudaFreeAsync(sym_buf, s);
    return st;
}

extern "C" struct GraphCSR *ag_graph_build_csr(uint32_t num_vertices, uint64_t num_edges, const uint32_t *src,
                                              const uint32_t *dst, const float *weight, uint32_t flags)
{
    ag_clear_error();
    AgDevCSR c;
    if (build_device_csr(num_vertices, num_edges, src, dst, weight, flags, &c) != AG_OK)
        return nullptr;
    const uint32_t N = c.N, E = c.E;
    struct GraphCSR *g = ag_host_graph_new(N, E, weight != nullptr, (flags & AG_BUILD_PINNED) ? 1 : 0);
    ag_status_t st = g ? AG_OK : ag_set_error(AG_ERR_OOM, "ag_graph_build_csr: host allocation failed");
    struct
    {
        void *h;
        const void *d;
        size_t bytes;
    } cp[] = {{g ? g->vertices->out_degree : nullptr, c.out_deg, (size_t)N * 4},
              {g ? g->vertices->in_degree : nullptr, c.in_deg, (size_t)N * 4},
              {g ? g->vertices->edges_idx : nullptr, c.fwd_idx, ((size_t)N + 1) * 4},
              {g ? g->inverse_vertices->edges_idx : nullptr, c.inv_idx, ((size_t)N + 1) * 4},
              {g ? g->sorted_edges_array->edges_array_src : nullptr, c.fwd_src, (size_t)E * 4},
              {g ? g->sorted_edges_array->edges_array_dest : nullptr, c.fwd_dst, (size_t)E * 4},
              {g ? g->inverse_sorted_edges_array->edges_array_src : nullptr, c.inv_src, (size_t)E * 4},
              {g ? g->inverse_sorted_edges_array->edges_array_dest : nullptr, c.inv_dst, (size_t)E * 4},
              {g ? g->sorted_edges_array->edges_array_weight : nullptr, c.fwd_w, (size_t)E * 4},
              {g ? g->inverse_sorted_edges_array->edges_array_weight : nullptr, c.inv_w, (size_t)E * 4}};
    for (auto &x : cp)
        if (st == AG_OK && x.h && x.d)
            st = copy_to_host(x.h, x.d, x.bytes);
    const float max_w = c.max_w;
    ag_csr_free_device(&c, g_ctx.stream);
    if (st != AG_OK) {
        ag_graph_free(g);
        return nullptr;
    }
    g->max_weight = g->sorted_edges_array->max_weight = g->inverse_sorted_edges_array->max_weight = max_w;
    return g;
}

extern "C" ag_status_t ag_graph_build(uint32_t num_vertices, uint64_t num_edges, const uint32_t *src,
                                      const uint32_t *dst, const float *weight, uint32_t build_flags,
                                      uint32_t upload_flags, ag_graph_t *out)
{
    ag_clear_error();
    if (!out)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_build: NULL output");
    *out = nullptr;
    AgDevCSR c;
    ag_status_t st = build_device_csr(num_vertices, num_edges, src, dst, weight, build_flags, &c);
    if (st != AG_OK)
        return st;
    st = upload_impl(nullptr, upload_flags, nullptr, 0, 0, out, &c);
    ag_csr_free_device(&c, g_ctx.stream);
    ag_status_t w = stream_wait(g_ctx.stream, 0);
    return st != AG_OK ? st : w;
}

/* ------------------------------------------------ integer gathers */
extern "C" ag_status_t ag_gather_uint(ag_graph_t g, const void *x, uint32_t elem_bytes, uint64_t *y)
{
    ag_clear_error();
    if (!g || (g->N && (!x || !y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_gather_uint: NULL argument");
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_gather_uint: element size %u is not 1, 2, 4 or 8", elem_bytes);
    if (g->norm_n || g->c_base)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_gather_uint: a row partition indexes a vector it does not hold");
    if (g->N == 0)
        return AG_OK;
    ag_status_t st = ensure_fixed(g);
    if (st != AG_OK)
        return st;
    cudaStream_t s = g_ctx.stream;
    const size_t xbytes = (size_t)g->N * elem_bytes, ybytes = (size_t)g->N * 8;
    /* two 64-bit vectors, the second 256-byte aligned; the kernel's 16-byte
     * table copy may read up to 15 bytes past x */
    const size_t off = (ybytes + 255) & ~(size_t)255;
    uint8_t *buf = nullptr;
    AG_CUDA(cudaMallocAsync((void **)&buf, off + ybytes + 16, s));
    uint64_t *ya = (uint64_t *)buf, *yb = (uint64_t *)(buf + off);
    /* x lands in ya (caller order), is permuted into yb (device order); the
     * sums go to ya, then back to caller order in yb */
    cudaError_t e = cudaMemcpyAsync(ya, x, xbytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = ag_permute_uint_in(g->perm, ya, yb, g->N, (int)elem_bytes, s);
    if (e == cudaSuccess) {
        AgPullParams p = base_params(g, 0);
        p.x64 = yb;
        p.y64 = ya;
        const void *k = ag_int_kernel_ptr((int)elem_bytes, 0, 1);
        const size_t smem = ag_fixed_smem_bytes((int)elem_bytes);
        const unsigned grid = pull_grid(k, p.ntasks, smem);
        void *args[1] = {&p};
        if (p.ntasks)
            e = cudaLaunchKernel(k, dim3(grid), dim3(AG_BLK), args, smem, s);
        else
            e = cudaMemsetAsync(ya, 0, ybytes, s);
    }
    if (e == cudaSuccess)
        e = ag_permute_u64_out(g->inv, ya, yb, g->N, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        st = ag_set_error(AG_ERR_CUDA, "ag_gather_uint: %s", cudaGetErrorString(e));
    }
    if (st == AG_OK)
        st = copy_to_host(y, yb, ybytes);
    cudaFreeAsync(buf, s);
    ag_status_t w = stream_wait(s, 0);
    return st != AG_OK ? st : w;
}

extern "C" ag_status_t ag_gather_u64(ag_graph_t g, const uint64_t *x, uint64_t *y)
{
    return ag_gather_uint(g, x, 8, y);
}
