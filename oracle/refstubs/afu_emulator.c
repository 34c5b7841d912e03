/*
 * afu_emulator.c -- CPU stand-in for the reference's accelerator runtime
 * (TEST INFRASTRUCTURE ONLY).
 *
 * The reference's pull calls (pageRank.c:942-1109, SPMV.c:622-751) hand the
 * per-vertex gather to an FPGA through the calls declared in
 * 02_capi_graph/include/capi_utils/capienv.h.  This file supplies those calls
 * so that the reference's own host code can run here unmodified:
 *   - mapGraphCSRToWED fills the work-element descriptor from a GraphCSR as
 *     capienv.c:832-874 does (WEIGHTED = 0, DIRECTED = 1: the inverse arrays,
 *     no weight pointers);
 *   - waitAFU performs one gather over the WED's inverse CSR: for every
 *     vertex v with in-edges, auxiliary2[v] = sum over its in-edges j, in
 *     stream order, of auxiliary1[src_j] (PageRank CU) or w_j * auxiliary1[src_j]
 *     (SpMV CU, binary32 multiply then add), the accumulator starting from the
 *     first value, or the exact modulo-2^64 integer sum of 64-bit
 *     contributions (fixed-point PageRank CU, pagerank_kernel_tb.sv:13-16), or
 *     the same sum of 32-, 16- or 8-bit contributions zero-extended into
 *     64 bits (the narrow fixed-point and quantised pulls; the testbench's
 *     Quantized context reads 4 bytes into the 8-byte accumulator,
 *     pagerank_kernel_tb.sv:17-19); for the push CU (pageRank.c:1111-1272)
 *     the scatter next[u] += c[v] along each forward edge, one source after
 *     the other in vertex order;
 *     vertices without in-edges are not written.  These are the
 *     compute units' semantics (cu_sum_kernel_control.sv, golden models
 *     pagerank_kernel_tb.sv:303-314, spmv_kernel_tb.sv:304,359).  With no
 *     weight array (WEIGHTED = 0) the SpMV weight is the reference's
 *     unweighted constant 0.0001f (SPMV.c:1206);
 *   - the other runtime calls only check their arguments.
 * It is compiled with -ffp-contract=off so that every product is rounded
 * before it is added.  It also supplies OpenGraph's timer, my_malloc and
 * the two worklist helpers of the data-driven variant (clear a byte list,
 * swap two list pointers).  The gather runs over
 * vertices with OpenMP, schedule(dynamic, 1024), as the reference's CPU
 * gathers do (pageRank.c:2898-2907).
 */
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "graphConfig.h"
#include "capienv.h"
#include "timer.h"
#include "worklist.h"

/* 0: PageRank CU, 1: SpMV CU, 2: 64-bit fixed-point PageRank CU,
 * 3, 4, 5: 32-, 16-, 8-bit contributions into 64-bit sums, 6: PageRank push
 * CU (binary32 adds along the forward edges, one source after the other) */
static int g_emu_kernel = 0;
static struct WEDGraphCSR *g_emu_wed = NULL;
static uint64_t g_emu_runs = 0;

void refemu_set_kernel(int kind) { g_emu_kernel = (kind >= 1 && kind <= 6) ? kind : 0; }
uint64_t refemu_gathers(void) { return g_emu_runs; }

void Start(struct Timer *timer) { clock_gettime(CLOCK_MONOTONIC, &timer->start_time); }
void Stop(struct Timer *timer) { clock_gettime(CLOCK_MONOTONIC, &timer->end_time); }
double Seconds(struct Timer *timer)
{
    return (double)(timer->end_time.tv_sec - timer->start_time.tv_sec) +
           (double)(timer->end_time.tv_nsec - timer->start_time.tv_nsec) * 1e-9;
}

void resetWorkList(uint8_t *workList, uint32_t size) { memset(workList, 0, size); }

void swapWorkLists(uint8_t **workList1, uint8_t **workList2)
{
    uint8_t *t = *workList1;
    *workList1 = *workList2;
    *workList2 = t;
}

void *my_malloc(size_t size)
{
    void *p = malloc(size ? size : 1);
    if (!p) {
        fprintf(stderr, "my_malloc: %zu bytes failed\n", size);
        exit(EXIT_FAILURE);
    }
    return p;
}

struct WEDGraphCSR *mapGraphCSRToWED(struct GraphCSR *graph)
{
    struct WEDGraphCSR *wed = (struct WEDGraphCSR *)my_malloc(sizeof(struct WEDGraphCSR));
    memset(wed, 0, sizeof(*wed));
    wed->num_edges = graph->num_edges;
    wed->num_vertices = graph->num_vertices;
    wed->max_weight = 0;
    wed->vertex_out_degree = graph->vertices->out_degree;
    wed->vertex_in_degree = graph->vertices->in_degree;
    wed->vertex_edges_idx = graph->vertices->edges_idx;
    if (graph->sorted_edges_array) {
        wed->edges_array_src = graph->sorted_edges_array->edges_array_src;
        wed->edges_array_dest = graph->sorted_edges_array->edges_array_dest;
    }
    wed->inverse_vertex_out_degree = graph->inverse_vertices->out_degree;
    wed->inverse_vertex_in_degree = graph->inverse_vertices->in_degree;
    wed->inverse_vertex_edges_idx = graph->inverse_vertices->edges_idx;
    wed->inverse_edges_array_src = graph->inverse_sorted_edges_array->edges_array_src;
    wed->inverse_edges_array_dest = graph->inverse_sorted_edges_array->edges_array_dest;
    wed->inverse_edges_array_weight = 0;
    wed->auxiliary0 = 0;
    return wed;
}

int setupAFUGraphCSR(struct cxl_afu_h **afu, struct WEDGraphCSR *wedGraphCSR)
{
    if (!afu || !wedGraphCSR) {
        fprintf(stderr, "setupAFUGraphCSR: NULL argument\n");
        exit(EXIT_FAILURE);
    }
    *afu = (struct cxl_afu_h *)wedGraphCSR; /* any non-NULL handle */
    g_emu_wed = wedGraphCSR;
    return 0;
}

void startAFU(struct cxl_afu_h **afu, struct AFUStatus *afu_status)
{
    (void)afu;
    afu_status->afu_status = 1;
}

void startCU(struct cxl_afu_h **afu, struct AFUStatus *afu_status)
{
    (void)afu;
    if (!afu_status->cu_config) {
        fprintf(stderr, "CU configuration must be non-zero\n");
        exit(EXIT_FAILURE);
    }
    afu_status->cu_status = 1;
}

void waitAFU(struct cxl_afu_h **afu, struct AFUStatus *afu_status)
{
    (void)afu;
    const struct WEDGraphCSR *w = g_emu_wed;
    const uint32_t n = w->num_vertices;
    const uint32_t *deg = (const uint32_t *)w->inverse_vertex_out_degree;
    const uint32_t *idx = (const uint32_t *)w->inverse_vertex_edges_idx;
    const uint32_t *src = (const uint32_t *)w->inverse_edges_array_dest;
    const float *wt = (const float *)w->inverse_edges_array_weight;
    const float *x = (const float *)w->auxiliary1;
    float *y = (float *)w->auxiliary2;
    const int spmv = g_emu_kernel == 1;
    int64_t v;
    if (g_emu_kernel == 6) {
        /* push CU: next[u] += c[v] along every forward edge, sources in order */
        const uint32_t *fdeg = (const uint32_t *)w->vertex_out_degree;
        const uint32_t *fidx = (const uint32_t *)w->vertex_edges_idx;
        const uint32_t *fdst = (const uint32_t *)w->edges_array_dest;
        for (v = 0; v < (int64_t)n; ++v)
            for (uint32_t j = fidx[v]; j < fidx[v] + fdeg[v]; ++j)
                y[fdst[j]] = y[fdst[j]] + x[v];
        afu_status->cu_return_done = n;
        afu_status->cu_status = 0;
        ++g_emu_runs;
        return;
    }
    if (g_emu_kernel >= 2) {
        /* integer CU: 64-, 32-, 16- or 8-bit contributions, exact integer sum
         * modulo 2^64 (pagerank_kernel_tb.sv:13-19) */
        const int kind = g_emu_kernel;
        const void *xi = w->auxiliary1;
        uint64_t *y64 = (uint64_t *)w->auxiliary2;
#pragma omp parallel for schedule(dynamic, 1024)
        for (v = 0; v < (int64_t)n; ++v) {
            const uint32_t d = deg[v], b = idx[v];
            uint64_t s = 0;
            if (!d)
                continue;
            for (uint32_t j = 0; j < d; ++j) {
                const uint32_t u = src[b + j];
                s += kind == 2   ? ((const uint64_t *)xi)[u]
                     : kind == 3 ? ((const uint32_t *)xi)[u]
                     : kind == 4 ? ((const uint16_t *)xi)[u]
                                 : ((const uint8_t *)xi)[u];
            }
            y64[v] = s;
        }
        afu_status->cu_return_done = n;
        afu_status->cu_status = 0;
        ++g_emu_runs;
        return;
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (v = 0; v < (int64_t)n; ++v) {
        const uint32_t d = deg[v], b = idx[v];
        if (!d)
            continue;
        float s;
        if (spmv) {
            s = (wt ? wt[b] : 0.0001f) * x[src[b]];
            for (uint32_t j = 1; j < d; ++j)
                s = s + (wt ? wt[b + j] : 0.0001f) * x[src[b + j]];
        } else {
            s = x[src[b]];
            for (uint32_t j = 1; j < d; ++j)
                s = s + x[src[b + j]];
        }
        y[v] = s;
    }
    afu_status->cu_return_done = n;
    afu_status->cu_status = 0;
    ++g_emu_runs;
}

void releaseAFU(struct cxl_afu_h **afu)
{
    if (afu)
        *afu = NULL;
    g_emu_wed = NULL;
}
