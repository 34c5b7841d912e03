/*
 * ag_capi.c -- the reference's algorithm entry points for the CSR data
 * structure, backed by the B200 kernels.
 *
 * Mirrors 02_capi_graph/src/algorithms/capi/pageRank.c (newPageRankStatsGraphCSR
 * :50-78, freePageRankStats :170-180, pageRankGraphCSR :874-939,
 * pageRankPullGraphCSR :942-1109) and SPMV.c (newSPMVStatsGraphCSR :51-73,
 * freeSPMVStats :145-158, SPMVGraphCSR :594-621, SPMVPullGraphCSR :622-751):
 * same stats objects, same iteration and convergence semantics, same stdout
 * tables.  The per-iteration table is printed after the device-resident loop
 * finishes, from the per-pass record the device keeps.  The legacy symbols
 * print one diagnostic line and exit on a device failure, as the reference's
 * accelerator calls do (capienv.c:113-131); the *_ex forms return the status.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ag_internal.h"

static int env_quiet(void)
{
    const char *q = getenv("AG_QUIET");
    return q && q[0] && q[0] != '0';
}

static void fail_exit(const char *phase, ag_status_t st)
{
    fprintf(stderr, "Accelerator verification failed: phase=%s reason=%s detail=%s\n", phase, ag_status_string(st),
            ag_last_error());
    exit(EXIT_FAILURE);
}

static int env_keep(void)
{
    const char *k = getenv("AG_KEEP_GRAPH");
    return k && k[0] && k[0] != '0';
}

/* The CSR entry points run one at a time: callers in several host threads
 * are serialised here, as one context per process with one stream expects
 * (the reference is not re-entrant either, capienv.c:35-36).  The kept
 * uploads below are only touched under this lock. */
static pthread_mutex_t g_csr_lock = PTHREAD_MUTEX_INITIALIZER;

/* ------------------------------------------------ uploads kept between calls */
/* A caller that solves on one unchanged GraphCSR several times pays the
 * upload once when it asks for it.  An entry matches on the GraphCSR
 * address, its vertex and edge counts, the addresses of every array the
 * upload reads and the upload flags.  The table is only read and written
 * under g_csr_lock. */
#define AG_KEEP_SLOTS 8

typedef struct keep_slot
{
    const struct GraphCSR *graph;
    uint32_t num_vertices, num_edges, flags;
    const void *arrays[5];
    ag_graph_t g;
    uint64_t used;
} keep_slot;

static keep_slot g_keep[AG_KEEP_SLOTS];
static uint64_t g_keep_tick;

static void keep_key(const struct GraphCSR *graph, const void *a[5])
{
    const struct Vertex *iv = graph->inverse_vertices, *fv = graph->vertices;
    const struct EdgeList *iel = graph->inverse_sorted_edges_array;
    a[0] = iv ? (const void *)iv->edges_idx : NULL;
    a[1] = iv ? (const void *)iv->out_degree : NULL;
    a[2] = fv ? (const void *)fv->out_degree : NULL;
    a[3] = iel ? (const void *)iel->edges_array_dest : NULL;
    a[4] = iel ? (const void *)iel->edges_array_weight : NULL;
}

/* the device graph of `graph` uploaded with `flags`: with `keep`, a kept
 * one that matches or a new upload that is then kept (*kept = 1: the caller
 * does not release it); without, a new upload the caller releases */
static ag_status_t upload_graph(const struct GraphCSR *graph, uint32_t flags, int keep, ag_graph_t *out, int *kept)
{
    const void *a[5];
    int i, victim = -1;
    ag_status_t st;
    keep_slot *s;

    *kept = 0;
    if (!keep)
        return ag_graph_upload(graph, flags, out);
    keep_key(graph, a);
    for (i = 0; i < AG_KEEP_SLOTS; i++) {
        s = &g_keep[i];
        if (s->g && s->graph == graph && s->num_vertices == graph->num_vertices &&
            s->num_edges == graph->num_edges && s->flags == flags && !memcmp(s->arrays, a, sizeof(a))) {
            s->used = ++g_keep_tick;
            *out = s->g;
            *kept = 1;
            return AG_OK;
        }
    }
    /* an empty slot, else the least recently used */
    for (i = 0; i < AG_KEEP_SLOTS; i++)
        if (!g_keep[i].g || victim < 0 || (g_keep[victim].g && g_keep[i].used < g_keep[victim].used))
            victim = i;
    st = ag_graph_upload(graph, flags, out);
    if (st != AG_OK)
        return st;
    s = &g_keep[victim];
    if (s->g)
        ag_graph_release(s->g);
    s->graph = graph;
    s->num_vertices = graph->num_vertices;
    s->num_edges = graph->num_edges;
    s->flags = flags;
    memcpy(s->arrays, a, sizeof(a));
    s->g = *out;
    s->used = ++g_keep_tick;
    *kept = 1;
    return AG_OK;
}

/* release a device graph after a call: a kept one stays unless the call
 * failed, when it is forgotten (its state after a failure is not reused) */
static void finish_graph(ag_graph_t g, int kept, int failed)
{
    int i;
    if (!g)
        return;
    if (kept && !failed)
        return;
    for (i = 0; i < AG_KEEP_SLOTS; i++)
        if (g_keep[i].g == g)
            memset(&g_keep[i], 0, sizeof(g_keep[i]));
    ag_graph_release(g);
}

ag_status_t ag_graph_forget(const struct GraphCSR *graph)
{
    int i;
    ag_clear_error();
    pthread_mutex_lock(&g_csr_lock);
    for (i = 0; i < AG_KEEP_SLOTS; i++) {
        if (g_keep[i].g && (!graph || g_keep[i].graph == graph)) {
            ag_graph_release(g_keep[i].g);
            memset(&g_keep[i], 0, sizeof(g_keep[i]));
        }
    }
    pthread_mutex_unlock(&g_csr_lock);
    return AG_OK;
}

/* ------------------------------------------------------------ PageRank */
struct PageRankStats *newPageRankStatsGraphCSR(struct GraphCSR *graph)
{
    uint32_t v, n = graph ? graph->num_vertices : 0;
    struct PageRankStats *stats = (struct PageRankStats *)calloc(1, sizeof(struct PageRankStats));
    if (!stats)
        return NULL;
    stats->damp = Damp;
    stats->base_pr = (1.0f - stats->damp);
    stats->iterations = 0;
    stats->num_vertices = n;
    stats->time_total = 0.0;
    stats->error_total = 0.0;
    stats->realRanks = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    stats->pageRanks = (float *)malloc((n ? n : 1) * sizeof(float));
    if (!stats->realRanks || !stats->pageRanks) {
        free(stats->realRanks);
        free(stats->pageRanks);
        free(stats);
        return NULL;
    }
    /* first touch of the two arrays spread over the host threads, as the
     * reference does (pageRank.c:68-73) */
#pragma omp parallel for schedule(static)
    for (v = 0; v < n; v++) {
        stats->pageRanks[v] = stats->base_pr;
        stats->realRanks[v] = v;
    }
    return stats;
}

void freePageRankStats(struct PageRankStats *stats)
{
    if (stats) {
        free(stats->realRanks);
        free(stats->pageRanks);
        free(stats);
    }
}

static ag_status_t pagerank_pull_locked(const struct Arguments *arguments, const struct GraphCSR *graph,
                                        const ag_pr_opts *opts, struct PageRankStats **out);

ag_status_t ag_pagerank_pull_ex(const struct Arguments *arguments, const struct GraphCSR *graph,
                                const ag_pr_opts *opts, struct PageRankStats **out)
{
    ag_status_t st;
    pthread_mutex_lock(&g_csr_lock);
    st = pagerank_pull_locked(arguments, graph, opts, out);
    pthread_mutex_unlock(&g_csr_lock);
    return st;
}

static ag_status_t pagerank_pull_locked(const struct Arguments *arguments, const struct GraphCSR *graph,
                                        const ag_pr_opts *opts, struct PageRankStats **out)
{
    ag_pr_opts o;
    ag_pr_result res;
    ag_graph_t g = NULL;
    int kept = 0;
    ag_status_t st;
    struct PageRankStats *stats = NULL;
    uint32_t *h_active = NULL;
    double *h_err = NULL, *h_sec = NULL;
    uint32_t cap, i;
    int quiet;
    double t0 = ag_wall_seconds();

    ag_clear_error();
    if (!arguments || !graph || !out)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_pagerank_pull_ex: NULL argument");
    *out = NULL;
    ag_pr_opts_init(&o);
    if (opts)
        memcpy(&o, opts, opts->struct_size && opts->struct_size < sizeof(o) ? opts->struct_size : sizeof(o));
    quiet = o.quiet || env_quiet();

    if (!quiet) {
        printf(" -----------------------------------------------------\n");
        printf("| %-51s | \n", "               ---->>> B200 <<<----");
        printf(" -----------------------------------------------------\n");
        if (o.direction == AG_DIR_PULL_PUSH)
            printf("| %-51s | \n", "Starting Page Rank Pull-Push DD (tolerance/epsilon)");
        else if (o.direction == AG_DIR_PUSH && o.data_driven)
            printf("| %-51s | \n", "Starting Page Rank Push DD (tolerance/epsilon)");
        else if (o.direction == AG_DIR_PUSH && o.precision == AG_PREC_QUANT32)
            printf("| %-30s %-19s| \n", "Starting Page Rank Push Quant_32", "(tolerance/epsilon)");
        else if (o.direction == AG_DIR_PUSH)
            printf("| %-51s | \n", o.precision == AG_PREC_FIXED64 ? "Starting Page Rank Push FP (tolerance/epsilon)"
                                                                 : "Starting Page Rank Push (tolerance/epsilon)");
        else if (o.precision >= AG_PREC_QUANT32 && o.precision <= AG_PREC_QUANT8)
            /* the quantised forms' title layout (pageRank.c:2155) */
            printf("| %-30s %-19s| \n",
                   o.precision == AG_PREC_QUANT32   ? "Starting Page Rank Pull Quant_32"
                   : o.precision == AG_PREC_QUANT16 ? "Starting Page Rank Pull Quant_16"
                                                    : "Starting Page Rank Pull Quant_8",
                   "(tolerance/epsilon)");
        else
            printf("| %-51s | \n", o.data_driven                     ? "Starting Page Rank Pull DD (tolerance/epsilon)"
                                    : o.precision == AG_PREC_FIXED64 ? "Starting Page Rank Pull FP_64 (tolerance/epsilon)"
                                    : o.precision == AG_PREC_FIXED32 ? "Starting Page Rank Pull FP_32 (tolerance/epsilon)"
                                    : o.precision == AG_PREC_FIXED16 ? "Starting Page Rank Pull FP_16 (tolerance/epsilon)"
                                    : o.precision == AG_PREC_FIXED8  ? "Starting Page Rank Pull FP_8 (tolerance/epsilon)"
                                                                     : "Starting Page Rank Pull (tolerance/epsilon)");
        printf(" -----------------------------------------------------\n");
        printf("| %-51.13lf | \n", arguments->epsilon);
        printf(" -----------------------------------------------------\n");
        printf("| %-10s | %-8s | %-15s | %-9s | \n", "Iteration", "Active", "Error", "Time (S)");
        printf(" -----------------------------------------------------\n");
        if (o.data_driven || o.direction == AG_DIR_PULL_PUSH)
            /* every vertex starts on the worklist (pageRank.c:2857-2868, 3019-3033, 3182-3196) */
            printf("| %-10s | %-8u | %-15.13lf | %-9f | \n", "Init", graph->num_vertices, 0.0, 0.0);
    }

    st = upload_graph(graph, 0, o.keep_graph || env_keep(), &g, &kept);
    if (st != AG_OK)
        goto fail;
    st = ag_pagerank_launch(g, arguments->iterations, arguments->epsilon, &o);
    if (st != AG_OK)
        goto fail;
    /* the host allocates and first-touches the stats object while the
     * device solves */
    stats = newPageRankStatsGraphCSR((struct GraphCSR *)graph);
    if (!stats) {
        st = ag_set_error(AG_ERR_OOM, "stats allocation failed");
        goto fail;
    }
    cap = arguments->iterations ? arguments->iterations : 1;
    h_active = (uint32_t *)calloc(cap, sizeof(uint32_t));
    h_err = (double *)calloc(cap, sizeof(double));
    h_sec = (double *)calloc(cap, sizeof(double));
    if (!h_active || !h_err || !h_sec) {
        st = ag_set_error(AG_ERR_OOM, "history allocation failed");
        goto fail;
    }
    st = ag_pagerank_fetch(g, stats->pageRanks, &res, h_active, h_err, h_sec, cap);
    if (st != AG_OK)
        goto fail;
    finish_graph(g, kept, 0);
    g = NULL;

    stats->iterations = res.iterations;
    stats->error_total = res.error_total;
    stats->activeVertices = res.active_last;
    stats->time_total = ag_wall_seconds() - t0;

    if (!quiet) {
        for (i = 0; i < res.passes && i < cap; i++)
            printf("| %-10u | %-8u | %-15.13lf | %-9f | \n", i, h_active[i], h_err[i], h_sec[i]);
        printf(" -----------------------------------------------------\n");
        printf("| %-10s | %-8s | %-15s | %-9s | \n", "Iterations", "PR Sum", "Error", "Time (S)");
        printf(" -----------------------------------------------------\n");
        printf("| %-10u | %-8lf | %-15.13lf | %-9f | \n", stats->iterations, res.rank_sum, stats->error_total,
               stats->time_total);
        printf(" -----------------------------------------------------\n");
        fflush(stdout);
    }
    free(h_active);
    free(h_err);
    free(h_sec);
    *out = stats;
    return AG_OK;

fail:
    finish_graph(g, kept, 1);
    free(h_active);
    free(h_err);
    free(h_sec);
    freePageRankStats(stats);
    return st;
}

struct PageRankStats *pageRankPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    struct PageRankStats *stats = NULL;
    ag_status_t st = ag_pagerank_pull_ex(arguments, graph, NULL, &stats);
    if (st != AG_OK)
        fail_exit("pagerank-pull", st);
    return stats;
}

/* one form of the reference's dispatcher on the GPU: the pull entry with the
 * form's precision, direction and worklist options; on failure the
 * reference's failure line and exit, with the form's phase name */
static struct PageRankStats *run_form(struct Arguments *arguments, struct GraphCSR *graph, int32_t precision,
                                      int32_t direction, int32_t data_driven, const char *phase)
{
    struct PageRankStats *stats = NULL;
    ag_pr_opts o;
    ag_status_t st;
    ag_pr_opts_init(&o);
    o.precision = precision;
    o.direction = direction;
    o.data_driven = data_driven;
    st = ag_pagerank_pull_ex(arguments, graph, &o, &stats);
    if (st != AG_OK)
        fail_exit(phase, st);
    return stats;
}

/* the reference's per-form entry points (pageRank.h:71-86); each runs the
 * form that pageRankGraphCSR selects for its pushpull code */
struct PageRankStats *pageRankPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FP32, AG_DIR_PUSH, 0, "pagerank-push");
}

struct PageRankStats *pageRankPullFixedPoint64BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FIXED64, AG_DIR_PULL, 0, "pagerank-pull-fp64");
}

struct PageRankStats *pageRankPullFixedPoint32BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FIXED32, AG_DIR_PULL, 0, "pagerank-pull-fp32");
}

struct PageRankStats *pageRankPullFixedPoint16BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FIXED16, AG_DIR_PULL, 0, "pagerank-pull-fp16");
}

struct PageRankStats *pageRankPullFixedPoint8BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FIXED8, AG_DIR_PULL, 0, "pagerank-pull-fp8");
}

struct PageRankStats *pageRankPushFixedPointGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FIXED64, AG_DIR_PUSH, 0, "pagerank-push-fp64");
}

struct PageRankStats *pageRankPullQuant32BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_QUANT32, AG_DIR_PULL, 0, "pagerank-pull-quant32");
}

struct PageRankStats *pageRankPullQuant16BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_QUANT16, AG_DIR_PULL, 0, "pagerank-pull-quant16");
}

struct PageRankStats *pageRankPullQuant8BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_QUANT8, AG_DIR_PULL, 0, "pagerank-pull-quant8");
}

struct PageRankStats *pageRankPushQuantGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_QUANT32, AG_DIR_PUSH, 0, "pagerank-push-quant32");
}

struct PageRankStats *pageRankDataDrivenPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FP32, AG_DIR_PULL, 1, "pagerank-pull-dd");
}

struct PageRankStats *pageRankDataDrivenPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FP32, AG_DIR_PUSH, 1, "pagerank-push-dd");
}

struct PageRankStats *pageRankDataDrivenPullPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    return run_form(arguments, graph, AG_PREC_FP32, AG_DIR_PULL_PUSH, 1, "pagerank-pull-push-dd");
}

/* dispatch on arguments->pushpull as pageRank.c:874-939 does: 0 the pull,
 * 1 the push, 2, 9, 10, 11 the 64/32/16/8-bit fixed-point pulls, 3 the
 * fixed-point push, 4, 12, 13 the 32/16/8-bit quantised pulls, 5 the
 * quantised push, 6 the data-driven pull, 7 the data-driven push, 8 the
 * data-driven pull-push; other codes run the pull, as the reference's default
 * case does, with a note on stderr */
struct PageRankStats *pageRankGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    static struct PageRankStats *(*const forms[14])(struct Arguments *, struct GraphCSR *) = {
        pageRankPullGraphCSR,
        pageRankPushGraphCSR,
        pageRankPullFixedPoint64BitGraphCSR,
        pageRankPushFixedPointGraphCSR,
        pageRankPullQuant32BitGraphCSR,
        pageRankPushQuantGraphCSR,
        pageRankDataDrivenPullGraphCSR,
        pageRankDataDrivenPushGraphCSR,
        pageRankDataDrivenPullPushGraphCSR,
        pageRankPullFixedPoint32BitGraphCSR,
        pageRankPullFixedPoint16BitGraphCSR,
        pageRankPullFixedPoint8BitGraphCSR,
        pageRankPullQuant16BitGraphCSR,
        pageRankPullQuant8BitGraphCSR,
    };
    if (arguments && arguments->pushpull < 14)
        return forms[arguments->pushpull](arguments, graph);
    if (arguments)
        fprintf(stderr, "pageRankGraphCSR: pushpull=%u runs the FP32 pull on the GPU\n", arguments->pushpull);
    return pageRankPullGraphCSR(arguments, graph);
}

/* ---------------------------------------------------------------- SpMV */
struct SPMVStats *newSPMVStatsGraphCSR(struct GraphCSR *graph)
{
    uint32_t n = graph ? graph->num_vertices : 0;
    struct SPMVStats *stats = (struct SPMVStats *)calloc(1, sizeof(struct SPMVStats));
    if (!stats)
        return NULL;
    stats->iterations = 0;
    stats->num_vertices = n;
    stats->time_total = 0.0;
    stats->vector_output = (float *)calloc(n ? n : 1, sizeof(float));
    stats->vector_input = (float *)calloc(n ? n : 1, sizeof(float));
    if (!stats->vector_output || !stats->vector_input) {
        free(stats->vector_output);
        free(stats->vector_input);
        free(stats);
        return NULL;
    }
    return stats;
}

void freeSPMVStats(struct SPMVStats *stats)
{
    if (stats) {
        free(stats->vector_output);
        free(stats->vector_input);
        free(stats);
    }
}

static ag_status_t spmv_pull_locked(const struct Arguments *arguments, const struct GraphCSR *graph, int quiet,
                                    struct SPMVStats **out);

ag_status_t ag_spmv_pull_ex(const struct Arguments *arguments, const struct GraphCSR *graph, int quiet,
                            struct SPMVStats **out)
{
    ag_status_t st;
    pthread_mutex_lock(&g_csr_lock);
    st = spmv_pull_locked(arguments, graph, quiet, out);
    pthread_mutex_unlock(&g_csr_lock);
    return st;
}

static ag_status_t spmv_pull_locked(const struct Arguments *arguments, const struct GraphCSR *graph, int quiet,
                                    struct SPMVStats **out)
{
    ag_graph_t g = NULL;
    int kept = 0;
    ag_status_t st;
    struct SPMVStats *stats;
    double *sec = NULL;
    double sum = 0.0;
    uint32_t v, i, iters;
    double t0;

    ag_clear_error();
    if (!arguments || !graph || !out)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_pull_ex: NULL argument");
    *out = NULL;
    quiet = quiet || env_quiet();
    stats = newSPMVStatsGraphCSR((struct GraphCSR *)graph);
    if (!stats)
        return ag_set_error(AG_ERR_OOM, "stats allocation failed");
    iters = arguments->iterations;

    st = upload_graph(graph, AG_UPLOAD_WEIGHTS, env_keep(), &g, &kept);
    if (st != AG_OK)
        goto fail;
    if (!quiet) {
        printf(" -----------------------------------------------------\n");
        printf("| %-51s | \n", "Starting SPMV-PULL");
        printf(" -----------------------------------------------------\n");
        printf("| %-21s | %-27s | \n", "Iteration", "Time (S)");
        printf(" -----------------------------------------------------\n");
    }
    /* input vector of the reference benchmark (SPMV.c:694-701) */
    for (v = 0; v < graph->num_vertices; v++) {
        if (graph->vertices->out_degree[v])
            stats->vector_input[v] = (1.0f / graph->vertices->out_degree[v]);
        else
            stats->vector_input[v] = 0.001f;
    }
    t0 = ag_wall_seconds();
    sec = (double *)calloc(iters ? iters : 1, sizeof(double));
    if (!sec) {
        st = ag_set_error(AG_ERR_OOM, "allocation failed");
        goto fail;
    }
    /* rows summed in stream order: the reference's sequential binary32 sums
     * (cu_sum_kernel_control.sv), bit for bit */
    st = ag_spmv_run_host(g, stats->vector_input, stats->vector_output, iters, AG_SPMV_GRAPH_WEIGHTS | AG_SPMV_EXACT,
                          sec);
    if (st != AG_OK)
        goto fail;
    stats->iterations = iters;
    if (!quiet)
        for (i = 0; i < iters; i++)
            printf("| %-21u | %-27f | \n", i, sec[i]);
    for (v = 0; v < graph->num_vertices; v++)
        sum += ((int)(stats->vector_output[v] * 100 + .5) / 100.0);
    stats->time_total = ag_wall_seconds() - t0;
    if (!quiet) {
        printf(" -----------------------------------------------------\n");
        printf("| %-15s | %-15s | %-15s | \n", "Iterations", "Sum", "Time (S)");
        printf(" -----------------------------------------------------\n");
        printf("| %-15u | %-15lf | %-15f | \n", stats->iterations, sum, stats->time_total);
        printf(" -----------------------------------------------------\n");
        fflush(stdout);
    }
    finish_graph(g, kept, 0);
    free(sec);
    *out = stats;
    return AG_OK;

fail:
    finish_graph(g, kept, 1);
    free(sec);
    freeSPMVStats(stats);
    return st;
}

struct SPMVStats *SPMVPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    struct SPMVStats *stats = NULL;
    ag_status_t st = ag_spmv_pull_ex(arguments, graph, 0, &stats);
    if (st != AG_OK)
        fail_exit("spmv-pull", st);
    return stats;
}

struct SPMVStats *SPMVGraphCSR(struct Arguments *arguments, struct GraphCSR *graph)
{
    if (arguments && arguments->pushpull != 0)
        fprintf(stderr, "SPMVGraphCSR: pushpull=%u runs the FP32 pull on the GPU\n", arguments->pushpull);
    return SPMVPullGraphCSR(arguments, graph);
}
