/*
 * ag_oracle.c -- CPU oracle of the pull PageRank / SpMV hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and only
 * as the checker or the timed CPU baseline; the product library never links
 * or calls it.
 *
 * The reference's OpenMP pull PageRank lives in the OpenGraph submodule,
 * which is empty in the reference checkout, so this is a restatement of the
 * loops that are present in the reference sources:
 *   host steps   02_capi_graph/src/algorithms/capi/pageRank.c:942-1109
 *                (init 50-78, contribution loop 1026-1033, update/residual
 *                loop 1055-1069, stop test 1073-1074, normalise 1079-1085)
 *   CPU gather   pageRank.c:2890-2907 (inverse CSR: degree =
 *                inverse_vertices->out_degree[v], u = edges_array_dest[j],
 *                nodeIncomingPR += riDividedOnDiClause[u], from 0.0f) and
 *                pageRank.c:3419-3439 (schedule(dynamic, 1024))
 *   SpMV pull    02_capi_graph/src/algorithms/capi/SPMV.c:622-751 (input
 *                vector 694-701, checksum 726-730) with the per-edge product
 *                of SPMV.c:1200-1224 (weight * x[src]; 0.0001f unweighted)
 * compiled with the reference's flags (-O3 -Wall -m64 -fopenmp,
 * 02_capi_graph/Makefile:250), which on x86-64 keeps every binary32 multiply
 * and add separate (no FMA contraction).
 * The gather arithmetic (sequential binary32 in stream order) is pinned by the
 * RTL testbench goldens (pagerank_kernel_tb.sv:303-314, spmv_kernel_tb.sv:
 * 349-359) through tests/golden/rtl_fixtures.json.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define ORACLE_DAMP 0.85f

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* y[v] = sum over v's inverse row of x[u], binary32 from 0.0f in stream order */
void oracle_gather(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                   const float *x, float *y, int threads)
{
    uint32_t v;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (v = 0; v < n; v++) {
        float s = 0.0f;
        uint32_t j, b = in_idx[v], d = in_deg[v];
        for (j = b; j < b + d; j++)
            s += x[in_nb[j]];
        y[v] = s;
    }
}

/* y[v] = sum of (w_j * x[u_j]) -- one binary32 multiply, then a binary32 add
 * in stream order; w == NULL uses the reference's unweighted 0.0001f */
void oracle_spmv_pull(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                      const float *w, const float *x, float *y, int threads)
{
    uint32_t v;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (v = 0; v < n; v++) {
        float s = 0.0f;
        uint32_t j, b = in_idx[v], d = in_deg[v];
        for (j = b; j < b + d; j++) {
            float wj = w ? w[j] : 0.0001f;
            float prod = wj * x[in_nb[j]];
            s += prod;
        }
        y[v] = s;
    }
}

/* SPMV.c:694-701 input vector and SPMV.c:726-730 checksum */
void oracle_spmv_input(uint32_t n, const uint32_t *out_deg, float *x)
{
    uint32_t v;
    for (v = 0; v < n; v++)
        x[v] = out_deg[v] ? (1.0f / out_deg[v]) : 0.001f;
}

double oracle_spmv_checksum(uint32_t n, const float *y)
{
    double sum = 0.0;
    uint32_t v;
    for (v = 0; v < n; v++)
        sum += ((int)(y[v] * 100 + .5) / 100.0);
    return sum;
}

/* pageRankPullGraphCSR restated.  ranks_out receives the normalised ranks.
 * init (n floats, may be NULL) replaces base_pr as the starting ranks.
 * hist_active / hist_err / hist_sec (may be NULL, >= iterations entries)
 * receive the per-pass record.  Returns stats->iterations semantics in
 * *iterations_out, the last pass's error_total in *error_total, the FP64
 * rank sum in *rank_sum and the number of passes executed (return value). */
uint32_t oracle_pagerank_pull(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                              const uint32_t *out_deg, uint32_t iterations, double epsilon, const float *init,
                              float *ranks_out, uint32_t *iterations_out, double *error_total_out,
                              double *rank_sum_out, uint32_t *hist_active, double *hist_err, double *hist_sec,
                              int threads)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    float *pageRanks = ranks_out;
    float *pageRanksNext = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    float *riDividedOnDiClause = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v;

    for (v = 0; v < n; v++) {
        pageRanks[v] = init ? init[v] : base_pr;
        pageRanksNext[v] = 0.0f;
    }
    for (it = 0; it < iterations; it++) {
        double t0 = now_s();
        error_total = 0;
        activeVertices = 0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++) {
            if (out_deg[v])
                riDividedOnDiClause[v] = pageRanks[v] / out_deg[v];
            else
                riDividedOnDiClause[v] = 0.0f;
        }
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
        for (v = 0; v < n; v++) {
            uint32_t j, b = in_idx[v], d = in_deg[v];
            float nodeIncomingPR = 0.0f;
            for (j = b; j < b + d; j++)
                nodeIncomingPR += riDividedOnDiClause[in_nb[j]];
            pageRanksNext[v] = nodeIncomingPR;
        }
#pragma omp parallel for reduction(+ : error_total, activeVertices) num_threads(nt)
        for (v = 0; v < n; v++) {
            float prevPageRank = pageRanks[v];
            float nextPageRank = base_pr + (damp * pageRanksNext[v]);
            pageRanks[v] = nextPageRank;
            pageRanksNext[v] = 0.0f;
            double error = fabs(nextPageRank - prevPageRank);
            error_total += (error / n);
            if (error >= epsilon)
                activeVertices++;
        }
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (hist_err)
            hist_err[it] = error_total;
        if (hist_sec)
            hist_sec[it] = now_s() - t0;
        if (activeVertices == 0)
            break;
    }
    {
        double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) num_threads(nt)
        for (v = 0; v < n; v++) {
            pageRanks[v] = pageRanks[v] / n;
            sum += pageRanks[v];
        }
        if (rank_sum_out)
            *rank_sum_out = sum;
    }
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(pageRanksNext);
    free(riDividedOnDiClause);
    return passes;
}

/* Fixed-point conversions of the 64-bit pull (OpenGraph's fixedPoint.h is
 * absent from the reference checkout; restated as 32 fractional bits, the
 * conversion to fixed point truncating toward zero). */
#define ORACLE_FIXED64_ONE 4294967296.0
static inline uint64_t oracle_d2fixed64(double x) { return (uint64_t)(int64_t)(x * ORACLE_FIXED64_ONE); }
static inline double oracle_fixed64_2d(uint64_t x) { return (double)(int64_t)x / ORACLE_FIXED64_ONE; }

/* fixed-point gather: y[v] = sum of x[u] over v's in-edges, modulo 2^64,
 * for every vertex with in-edges (pagerank_kernel_tb.sv:13-16, 303-314) */
void oracle_gather_u64(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                       const uint64_t *x, uint64_t *y, int threads)
{
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    uint32_t v;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
    for (v = 0; v < n; v++) {
        uint64_t s = 0;
        uint32_t j;
        if (!in_deg[v])
            continue;
        for (j = in_idx[v]; j < in_idx[v] + in_deg[v]; j++)
            s += x[in_nb[j]];
        y[v] = s;
    }
}

/* 64-bit fixed-point pull, pageRank.c:1276-1453 (pushpull 2): contributions
 * DoubleToFixed64(r / out_degree) (binary32 division), the accelerator's
 * integer sums, and the update base + damp * Fixed64ToDouble(sum) evaluated in
 * binary64 and stored in binary32; residual, stop test and normalisation as
 * in the plain pull. */
uint32_t oracle_pagerank_fixed64(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                                 const uint32_t *out_deg, uint32_t iterations, double epsilon, float *ranks_out,
                                 uint32_t *iterations_out, double *error_total_out, uint32_t *hist_active,
                                 int threads)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    float *pageRanks = ranks_out;
    uint64_t *next = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    uint64_t *contrib = (uint64_t *)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v;
    for (v = 0; v < n; v++)
        pageRanks[v] = base_pr;
    for (it = 0; it < iterations; it++) {
        error_total = 0;
        activeVertices = 0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++) {
            if (out_deg[v])
                contrib[v] = oracle_d2fixed64(pageRanks[v] / out_deg[v]);
            else
                contrib[v] = 0;
        }
        oracle_gather_u64(n, in_idx, in_deg, in_nb, contrib, next, nt);
#pragma omp parallel for reduction(+ : error_total, activeVertices) num_threads(nt)
        for (v = 0; v < n; v++) {
            float prevPageRank = pageRanks[v];
            float nextPageRank = base_pr + (damp * oracle_fixed64_2d(next[v]));
            pageRanks[v] = nextPageRank;
            next[v] = 0;
            double error = fabs(nextPageRank - prevPageRank);
            error_total += (error / n);
            if (error >= epsilon)
                activeVertices++;
        }
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (activeVertices == 0)
            break;
    }
#pragma omp parallel for num_threads(nt)
    for (v = 0; v < n; v++)
        pageRanks[v] = pageRanks[v] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(next);
    free(contrib);
    return passes;
}

/* Integer gather of W-bit elements (elem_bytes 1, 2, 4 or 8), each
 * zero-extended into a 64-bit sum modulo 2^64: the FixedPoint and Quantized
 * compute units' contract (pagerank_kernel_tb.sv:13-19; 4-byte reads zero
 * extended into the 8-byte accumulator in the Quantized context).  Rows
 * without in-edges are not written. */
void oracle_gather_uint(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                        const void *x, uint32_t elem_bytes, uint64_t *y, int threads)
{
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    uint32_t v;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
    for (v = 0; v < n; v++) {
        uint64_t s = 0;
        uint32_t j;
        if (!in_deg[v])
            continue;
        for (j = in_idx[v]; j < in_idx[v] + in_deg[v]; j++) {
            const uint32_t u = in_nb[j];
            switch (elem_bytes) {
            case 1: s += ((const uint8_t *)x)[u]; break;
            case 2: s += ((const uint16_t *)x)[u]; break;
            case 4: s += ((const uint32_t *)x)[u]; break;
            default: s += ((const uint64_t *)x)[u]; break;
            }
        }
        y[v] = s;
    }
}

/* Narrow fixed point (OpenGraph's FloatToFixed32/16/8 and Fixed32/16/8ToFloat
 * are absent from the reference checkout): W-bit values with W/2 fractional
 * bits.  Q16.16 for 32 bits is the format the reference's fixed-point SpMV
 * compute unit assumes of its 32-bit operands (products shifted right by
 * SCALEF = 16, cu_SPMV/CSR/PULL/FixedPoint/pkg/globals_cu_pkg.sv:37,
 * cu_sum_kernel_control.sv:164); Q8.8 and Q4.4 follow it.  To fixed point:
 * the binary32 product x * 2^(W/2) (exact) truncated toward zero, kept modulo
 * 2^W.  Back: the 64-bit sum rounded once to binary32, scaled by 2^-(W/2). */
static inline uint64_t oracle_f2fixed(float x, int W)
{
    const uint64_t mask = W >= 64 ? ~0ull : ((1ull << W) - 1);
    return (uint64_t)(int64_t)(x * (float)(1u << (W / 2))) & mask;
}

static inline float oracle_fixed2f(uint64_t s, int W) { return (float)s / (float)(1u << (W / 2)); }

/* Affine quantisation (OpenGraph's quantization.h is absent; restated from
 * the published uniform affine scheme, Jacob et al., CVPR 2018, with the
 * zero point the reference forces to 0, pageRank.c:2225-2226):
 * scale = (max - min) / (2^W - 1) in binary32, q = round-half-even(x / scale)
 * clamped to [0, 2^W - 1]; a zero scale quantises everything to 0. */
static void oracle_minmax(const float *x, uint32_t n, float *mn, float *mx)
{
    uint32_t v;
    float a = n ? x[0] : 0.0f, b = n ? x[0] : 0.0f;
    for (v = 1; v < n; v++) {
        if (x[v] < a)
            a = x[v];
        if (x[v] > b)
            b = x[v];
    }
    *mn = a;
    *mx = b;
}

static inline float oracle_quant_scale(float mn, float mx, int W)
{
    return (mx - mn) / (float)((1ull << W) - 1);
}

static inline uint64_t oracle_quantize(float x, float scale, int W)
{
    const uint64_t top = (1ull << W) - 1;
    float q;
    if (!(scale > 0.0f))
        return 0;
    q = rintf(x / scale);
    if (!(q > 0.0f))
        return 0;
    if (q >= (float)top)
        return top;
    return (uint64_t)q;
}

static void oracle_store_uint(void *a, uint32_t v, uint64_t x, int W)
{
    switch (W) {
    case 8: ((uint8_t *)a)[v] = (uint8_t)x; break;
    case 16: ((uint16_t *)a)[v] = (uint16_t)x; break;
    default: ((uint32_t *)a)[v] = (uint32_t)x; break;
    }
}

/* Narrow integer pulls (W = 32, 16, 8):
 *   quant = 0: fixed point, pageRank.c:1455-1991 (pushpull 9, 10, 11):
 *     c[v] = FloatToFixedW(r[v] / out_degree[v]) (0 without out-edges),
 *     r' = base + damp * FixedWToFloat(sum) in binary32;
 *   quant = 1: quantised, pageRank.c:2119-2677 (pushpull 4, 12, 13):
 *     f[v] = r[v] / out_degree[v] (0.0f without out-edges), min and max of f
 *     over all vertices, scale from them, c[v] = quantize(f[v]),
 *     r' = base + damp * (scale * (float)sum) in binary32.
 * The W-bit contributions are gathered into 64-bit sums; residual, stop test
 * and normalisation as in the plain pull. */
uint32_t oracle_pagerank_narrow(int quant, int W, uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg,
                                const uint32_t *in_nb, const uint32_t *out_deg, uint32_t iterations, double epsilon,
                                float *ranks_out, uint32_t *iterations_out, double *error_total_out,
                                uint32_t *hist_active, int threads)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    float *pageRanks = ranks_out;
    uint64_t *next = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    float *f = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    void *c = malloc((size_t)(n ? n : 1) * (size_t)(W / 8));
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v;
    for (v = 0; v < n; v++)
        pageRanks[v] = base_pr;
    for (it = 0; it < iterations; it++) {
        float scale = 0.0f;
        error_total = 0;
        activeVertices = 0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++)
            f[v] = out_deg[v] ? pageRanks[v] / out_deg[v] : 0.0f;
        if (quant) {
            float mn, mx;
            oracle_minmax(f, n, &mn, &mx);
            scale = oracle_quant_scale(mn, mx, W);
        }
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++)
            oracle_store_uint(c, v, quant ? oracle_quantize(f[v], scale, W) : (out_deg[v] ? oracle_f2fixed(f[v], W) : 0),
                              W);
        oracle_gather_uint(n, in_idx, in_deg, in_nb, c, (uint32_t)(W / 8), next, nt);
#pragma omp parallel for reduction(+ : error_total, activeVertices) num_threads(nt)
        for (v = 0; v < n; v++) {
            float prevPageRank = pageRanks[v];
            float nextPageRank = quant ? base_pr + damp * (scale * (float)next[v])
                                       : base_pr + (damp * oracle_fixed2f(next[v], W));
            pageRanks[v] = nextPageRank;
            next[v] = 0;
            double error = fabs(nextPageRank - prevPageRank);
            error_total += (error / n);
            if (error >= epsilon)
                activeVertices++;
        }
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (activeVertices == 0)
            break;
    }
#pragma omp parallel for num_threads(nt)
    for (v = 0; v < n; v++)
        pageRanks[v] = pageRanks[v] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(next);
    free(f);
    free(c);
    return passes;
}

/* Data-driven (worklist) pull, pageRank.c:2810-2969: every vertex starts
 * active; in each iteration the contributions of all vertices are formed
 * from the current ranks, every active vertex v gathers its in-edges in
 * stream order (accumulator starting at 0.0f) and computes
 * new = base + damp * sum; the residual |new - old| (binary32 subtract,
 * binary64 compare) is added to error_total for every active vertex; only
 * when it reaches epsilon is the rank replaced and every out-neighbour of v
 * (forward CSR) put on the next worklist.  Stops when no vertex changed
 * (iterations = that iteration's index) or at the cap; ranks / n at the end. */
uint32_t oracle_pagerank_dd(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                            const uint32_t *out_idx, const uint32_t *out_deg, const uint32_t *out_nb,
                            uint32_t iterations, double epsilon, float *ranks_out, uint32_t *iterations_out,
                            double *error_total_out, uint32_t *hist_active, int threads)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    float *pageRanks = ranks_out;
    float *riDividedOnDiClause = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    uint8_t *wl_curr = (uint8_t *)calloc(n ? n : 1, 1);
    uint8_t *wl_next = (uint8_t *)calloc(n ? n : 1, 1);
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v;

    for (v = 0; v < n; v++) {
        pageRanks[v] = base_pr;
        wl_curr[v] = 1;
    }
    for (it = 0; it < iterations; it++) {
        uint8_t *t;
        error_total = 0;
        activeVertices = 0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++) {
            if (out_deg[v])
                riDividedOnDiClause[v] = pageRanks[v] / out_deg[v];
            else
                riDividedOnDiClause[v] = 0.0f;
        }
#pragma omp parallel for reduction(+ : error_total, activeVertices) schedule(dynamic, 1024) num_threads(nt)
        for (v = 0; v < n; v++) {
            if (wl_curr[v]) {
                uint32_t j, b = in_idx[v], d = in_deg[v];
                float nodeIncomingPR = 0.0f;
                for (j = b; j < b + d; j++)
                    nodeIncomingPR += riDividedOnDiClause[in_nb[j]];
                float oldPageRank = pageRanks[v];
                float newPageRank = base_pr + (damp * nodeIncomingPR);
                double error = fabs(newPageRank - oldPageRank);
                error_total += error / n;
                if (error >= epsilon) {
                    pageRanks[v] = newPageRank;
                    for (j = out_idx[v]; j < out_idx[v] + out_deg[v]; j++) {
#pragma omp atomic write
                        wl_next[out_nb[j]] = 1;
                    }
                    activeVertices++;
                }
            }
        }
        t = wl_curr;
        wl_curr = wl_next;
        wl_next = t;
        memset(wl_next, 0, n);
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (activeVertices == 0)
            break;
    }
#pragma omp parallel for num_threads(nt)
    for (v = 0; v < n; v++)
        pageRanks[v] = pageRanks[v] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(riDividedOnDiClause);
    free(wl_curr);
    free(wl_next);
    return passes;
}

/* Push forms (pageRankGraphCSR pushpull 1, 3, 5): the host steps of the pull
 * with the gather turned around: every vertex v adds its contribution into
 * next[u] along each of its forward edges.  The reference runs these with
 * OpenMP (pushpull 3, 5: unsynchronised or atomic adds from many threads) or
 * on the FPGA's push unit (pushpull 1), so their add order is not fixed; this
 * restatement is their single-thread instance: sources in vertex order, each
 * source's out-edges in forward-row order, every next[u] starting from 0.
 *   kind 0: pushpull 1, pageRank.c:1111-1272: binary32 c = r / out_degree,
 *           binary32 adds, r' = base + damp * next;
 *   kind 1: pushpull 3, pageRank.c:1992-2118: c = DoubleToFixed64(r / od),
 *           64-bit integer adds, r' = base + damp * Fixed64ToDouble(next) in
 *           binary64, stored binary32;
 *   kind 2: pushpull 5, pageRank.c:2678-2809: binary32 c, min/max, 32-bit
 *           quantisation with the pass's scale and zero point (OpenGraph's
 *           GetZeroPoint is absent; its value is restated as 0, the zero
 *           point the quantised pulls use), binary32 adds of
 *           scale * (q - zero), r' = base + damp * next.
 * Residual, stop test and normalisation as in the pull. */
uint32_t oracle_pagerank_push(int kind, uint32_t n, const uint32_t *out_idx, const uint32_t *out_deg,
                              const uint32_t *out_nb, uint32_t iterations, double epsilon, float *ranks_out,
                              uint32_t *iterations_out, double *error_total_out, uint32_t *hist_active)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    float *pageRanks = ranks_out;
    float *next = (float *)calloc(n ? n : 1, sizeof(float));
    uint64_t *next64 = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    float *c = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    uint64_t *c64 = (uint64_t *)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    uint32_t *q = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v, j;
    for (v = 0; v < n; v++)
        pageRanks[v] = base_pr;
    for (it = 0; it < iterations; it++) {
        float scale = 0.0f;
        const uint32_t zero = 0;
        error_total = 0;
        activeVertices = 0;
        for (v = 0; v < n; v++) {
            c[v] = out_deg[v] ? pageRanks[v] / out_deg[v] : 0.0f;
            if (kind == 1)
                c64[v] = out_deg[v] ? oracle_d2fixed64(pageRanks[v] / out_deg[v]) : 0;
        }
        if (kind == 2) {
            float mn, mx;
            oracle_minmax(c, n, &mn, &mx);
            scale = oracle_quant_scale(mn, mx, 32);
            for (v = 0; v < n; v++)
                q[v] = (uint32_t)oracle_quantize(c[v], scale, 32) + zero;
        }
        for (v = 0; v < n; v++)
            for (j = out_idx[v]; j < out_idx[v] + out_deg[v]; j++) {
                const uint32_t u = out_nb[j];
                if (kind == 1)
                    next64[u] += c64[v];
                else if (kind == 2)
                    next[u] += scale * (q[v] - zero);
                else
                    next[u] += c[v];
            }
        for (v = 0; v < n; v++) {
            float prevPageRank = pageRanks[v];
            float nextPageRank = kind == 1 ? base_pr + (damp * oracle_fixed64_2d(next64[v]))
                                           : base_pr + (damp * next[v]);
            pageRanks[v] = nextPageRank;
            next[v] = 0;
            next64[v] = 0;
            double error = fabs(nextPageRank - prevPageRank);
            error_total += (error / n);
            if (error >= epsilon)
                activeVertices++;
        }
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (activeVertices == 0)
            break;
    }
    for (v = 0; v < n; v++)
        pageRanks[v] = pageRanks[v] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(next);
    free(next64);
    free(c);
    free(c64);
    free(q);
    return passes;
}

/* Residual forms with a worklist (pushpull 7, 8), single-thread instance
 * (vertices in order).  Both start from r = base and the residual
 * res[v] = ((1 - damp) * damp) * (sum over v's in-edges u with out-edges of
 * 1.0f / out_degree[u], in stream order), every vertex on the worklist.  Per
 * iteration each vertex v on the worklist:
 *   pull_push = 0 (data-driven push, pageRank.c:2971-3127):
 *     r'[v] = res[v] + r[v];
 *   pull_push = 1 (data-driven pull-push, pageRank.c:3128-3325):
 *     r'[v] = base + damp * (sum over v's in-edges of r[u] / out_degree[u],
 *     stream order, reading ranks already updated in this iteration);
 *   then error_total += |r'[v] / n - r[v] / n| (binary32, summed in binary64),
 *   delta = damp * (res[v] / out_degree[v]), and for each out-edge u:
 *   prev = res[u]; res[u] += delta; if |prev + delta| >= epsilon and
 *   prev <= epsilon, the iteration counts one activation and puts u on the
 *   next worklist (the pull-push form adds delta to res[u] a second time
 *   there, as the reference does); finally res[v] = 0.
 * Stops after an iteration without activations (iterations = its index) or at
 * the cap; ranks / n at the end.  hist_active: activations per iteration. */
uint32_t oracle_pagerank_residual(int pull_push, uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg,
                                  const uint32_t *in_nb, const uint32_t *out_idx, const uint32_t *out_deg,
                                  const uint32_t *out_nb, uint32_t iterations, double epsilon, float *ranks_out,
                                  uint32_t *iterations_out, double *error_total_out, uint32_t *hist_active)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    float *pageRanks = ranks_out;
    float *res = (float *)calloc(n ? n : 1, sizeof(float));
    uint8_t *wl_curr = (uint8_t *)calloc(n ? n : 1, 1);
    uint8_t *wl_next = (uint8_t *)calloc(n ? n : 1, 1);
    double error_total = 0.0;
    uint32_t activeVertices = 0, it, passes = 0, v, j;
    for (v = 0; v < n; v++) {
        pageRanks[v] = base_pr;
        res[v] = 0.0f;
        wl_curr[v] = 1;
        for (j = in_idx[v]; j < in_idx[v] + in_deg[v]; j++)
            if (out_deg[in_nb[j]])
                res[v] += 1.0f / out_deg[in_nb[j]];
        res[v] = (1.0f - damp) * damp * res[v];
    }
    for (it = 0; it < iterations; it++) {
        uint8_t *t;
        error_total = 0;
        activeVertices = 0;
        for (v = 0; v < n; v++) {
            if (!wl_curr[v])
                continue;
            float oldPageRank = pageRanks[v];
            float newPageRank;
            if (pull_push) {
                float nodeIncomingPR = 0.0f;
                for (j = in_idx[v]; j < in_idx[v] + in_deg[v]; j++)
                    nodeIncomingPR += pageRanks[in_nb[j]] / out_deg[in_nb[j]];
                newPageRank = base_pr + (damp * nodeIncomingPR);
            } else {
                newPageRank = res[v] + pageRanks[v];
            }
            error_total += fabs(newPageRank / n - oldPageRank / n);
            pageRanks[v] = newPageRank;
            float delta = damp * (res[v] / out_deg[v]);
            for (j = out_idx[v]; j < out_idx[v] + out_deg[v]; j++) {
                const uint32_t u = out_nb[j];
                float prevResidual = res[u];
                res[u] += delta;
                if ((fabs(prevResidual + delta) >= epsilon) && (prevResidual <= epsilon)) {
                    activeVertices++;
                    if (pull_push)
                        res[u] += delta;
                    wl_next[u] = 1;
                }
            }
            res[v] = 0.0f;
        }
        t = wl_curr;
        wl_curr = wl_next;
        wl_next = t;
        memset(wl_next, 0, n);
        passes++;
        if (hist_active)
            hist_active[it] = activeVertices;
        if (activeVertices == 0)
            break;
    }
    for (v = 0; v < n; v++)
        pageRanks[v] = pageRanks[v] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    if (error_total_out)
        *error_total_out = error_total;
    free(res);
    free(wl_curr);
    free(wl_next);
    return passes;
}

/* FP64 fixpoint with the reference's constants ((double)0.85f and
 * (double)(1.0f - 0.85f)): every operation in binary64, iterated until
 * max |r' - r| <= tol or max_iter passes.  ranks_out receives r / n. */
uint32_t oracle_pagerank_f64(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                             const uint32_t *out_deg, uint32_t max_iter, double tol, double *ranks_out,
                             int threads)
{
    const double damp = (double)0.85f, base = (double)(1.0f - 0.85f);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    double *r = ranks_out;
    double *c = (double *)malloc((size_t)(n ? n : 1) * sizeof(double));
    double *rn = (double *)malloc((size_t)(n ? n : 1) * sizeof(double));
    uint32_t it, v;
    for (v = 0; v < n; v++)
        r[v] = base;
    for (it = 0; it < max_iter; it++) {
        double md = 0.0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++)
            c[v] = out_deg[v] ? r[v] / (double)out_deg[v] : 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(max : md) num_threads(nt)
        for (v = 0; v < n; v++) {
            double s = 0.0;
            uint32_t j, b = in_idx[v], d = in_deg[v];
            for (j = b; j < b + d; j++)
                s += c[in_nb[j]];
            rn[v] = base + damp * s;
            double dd = fabs(rn[v] - r[v]);
            if (dd > md)
                md = dd;
        }
        memcpy(r, rn, (size_t)n * sizeof(double));
        if (md <= tol) {
            it++;
            break;
        }
    }
    for (v = 0; v < n; v++)
        r[v] /= (double)n;
    free(c);
    free(rn);
    return it;
}

/* Batched personalized PageRank restated column by column: column i is the
 * pull loop above with the teleport mass (1.0f - 0.85f) * n on sources[i]
 * (zero elsewhere); a pass is active while any (vertex, column) pair changes
 * by >= epsilon.  ranks_out receives n x k values r / n (row-major). */
uint32_t oracle_ppr(uint32_t n, const uint32_t *in_idx, const uint32_t *in_deg, const uint32_t *in_nb,
                    const uint32_t *out_deg, uint32_t k, const uint32_t *sources, uint32_t iterations, double epsilon,
                    float *ranks_out, uint32_t *iterations_out, int threads)
{
    const float damp = ORACLE_DAMP;
    const float base_src = (1.0f - damp) * (float)n;
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    float *r = ranks_out;
    float *c = (float *)malloc((size_t)(n ? n : 1) * k * sizeof(float));
    uint32_t it, passes = 0, v;
    for (v = 0; v < n; v++)
        for (uint32_t i = 0; i < k; i++)
            r[(size_t)v * k + i] = (v == sources[i]) ? base_src : 0.0f;
    for (it = 0; it < iterations; it++) {
        unsigned long long active = 0;
#pragma omp parallel for num_threads(nt)
        for (v = 0; v < n; v++)
            for (uint32_t i = 0; i < k; i++)
                c[(size_t)v * k + i] = out_deg[v] ? r[(size_t)v * k + i] / out_deg[v] : 0.0f;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : active) num_threads(nt)
        for (v = 0; v < n; v++) {
            for (uint32_t i = 0; i < k; i++) {
                float s = 0.0f;
                for (uint32_t j = in_idx[v]; j < in_idx[v] + in_deg[v]; j++)
                    s += c[(size_t)in_nb[j] * k + i];
                float prev = r[(size_t)v * k + i];
                float next = ((v == sources[i]) ? base_src : 0.0f) + damp * s;
                r[(size_t)v * k + i] = next;
                if (fabs(next - prev) >= epsilon)
                    active++;
            }
        }
        passes++;
        if (active == 0)
            break;
    }
    for (size_t t = 0; t < (size_t)n * k; t++)
        r[t] = r[t] / n;
    if (iterations_out)
        *iterations_out = it < iterations ? it : iterations;
    free(c);
    return passes;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* ----------------------------------------------------------------------
 * Seeded R-MAT graph as an inverse CSR, for the CPU legs that must not load
 * the product library.  Graph500-style quadrant recursion: edge e draws one
 * 32-bit uniform per level, 64-bit draw k of stream e covering levels 2k and
 * 2k+1 (low half first), where draw k of stream e under `seed` is the
 * SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014) of
 * mix(seed + G) + (64 e + k + 1) G, G = 0x9E3779B97F4A7C15, mix(z) the two
 * xor-shift-multiply rounds of that finaliser.  A level's draw u picks the
 * quadrant: u < a 2^32 top-left, < (a+b) 2^32 top-right (destination bit),
 * < (a+b+c) 2^32 bottom-left (source bit), else bottom-right.
 * Self loops and duplicate edges are dropped (the reference's -k), and each
 * inverse row lists its sources in ascending order.  Returns the edge count;
 * in_nb must hold edge_factor * 2^scale entries. */
static inline uint64_t oracle_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* parallel LSD radix sort of 64-bit keys, 8 bits per pass, `bits` low bits
 * significant; tmp holds n keys */
static void oracle_radix64(uint64_t *a, uint64_t *tmp, uint64_t n, int bits)
{
    const int T = omp_get_max_threads();
    uint64_t *cnt = (uint64_t *)malloc((size_t)T * 256 * sizeof(uint64_t));
    for (int shift = 0; shift < bits; shift += 8) {
        memset(cnt, 0, (size_t)T * 256 * sizeof(uint64_t));
#pragma omp parallel num_threads(T)
        {
            const int t = omp_get_thread_num();
            const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
            uint64_t *c = cnt + (size_t)t * 256;
            for (uint64_t i = lo; i < hi; ++i)
                c[(a[i] >> shift) & 255u]++;
#pragma omp barrier
#pragma omp single
            {
                uint64_t base = 0;
                for (int d = 0; d < 256; ++d)
                    for (int u = 0; u < T; ++u) {
                        const uint64_t x = cnt[(size_t)u * 256 + d];
                        cnt[(size_t)u * 256 + d] = base;
                        base += x;
                    }
            }
            for (uint64_t i = lo; i < hi; ++i)
                tmp[c[(a[i] >> shift) & 255u]++] = a[i];
        }
        uint64_t *s = a;
        a = tmp;
        tmp = s;
    }
    /* an odd number of passes leaves the result in the scratch array */
    if (((bits + 7) / 8) & 1)
        memcpy(tmp, a, n * sizeof(uint64_t));
    free(cnt);
}

uint64_t oracle_rmat_inverse(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                             uint32_t *in_idx, uint32_t *in_deg, uint32_t *in_nb, uint32_t *out_deg)
{
    const uint64_t G = 0x9E3779B97F4A7C15ull;
    const uint64_t N = 1ull << scale, m = (uint64_t)edge_factor * N;
    const uint32_t ta = (uint32_t)fmin(4294967295.0, floor(a * 4294967296.0));
    const uint32_t tb = (uint32_t)fmin(4294967295.0, floor((a + b) * 4294967296.0));
    const uint32_t tc = (uint32_t)fmin(4294967295.0, floor((a + b + c) * 4294967296.0));
    const uint64_t base = oracle_mix64(seed + G);
    uint64_t *key = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    uint64_t *tmp = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    if (!key || !tmp) {
        free(key);
        free(tmp);
        return ~0ull;
    }
    /* key = destination * N + source: sorting it orders the inverse rows */
#pragma omp parallel for schedule(static)
    for (uint64_t e = 0; e < m; ++e) {
        uint64_t s = 0, d = 0, r = 0;
        for (uint32_t l = 0; l < scale; ++l) {
            if ((l & 1u) == 0)
                r = oracle_mix64(base + (e * 64ull + (l >> 1) + 1ull) * G);
            const uint32_t u = (l & 1u) ? (uint32_t)(r >> 32) : (uint32_t)r;
            const uint64_t sb = u >= tb, db = (u >= ta && u < tb) || u >= tc;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        key[e] = (d << scale) | s;
    }
    oracle_radix64(key, tmp, m, 2 * (int)scale);
    free(tmp);
    memset(in_deg, 0, N * sizeof(uint32_t));
    memset(out_deg, 0, N * sizeof(uint32_t));
    uint64_t E = 0;
    for (uint64_t i = 0; i < m; ++i) {
        const uint64_t k = key[i];
        const uint32_t d = (uint32_t)(k >> scale), s = (uint32_t)(k & (N - 1));
        if (s == d || (i > 0 && key[i - 1] == k))
            continue;
        in_nb[E++] = s;
        in_deg[d]++;
        out_deg[s]++;
    }
    free(key);
    uint64_t off = 0;
    for (uint64_t v = 0; v < N; ++v) {
        in_idx[v] = (uint32_t)off;
        off += in_deg[v];
    }
    in_idx[N] = (uint32_t)off;
    return E;
}

/* One pull pass of a row partition (the multi-GPU solve's per-rank step):
 * rows [rb, re) of the inverse CSR, with the contribution of vertex u at
 * pos[u] of the rank-padded vectors c_in_full / c_out_full.  Each row is summed
 * in stream order as in oracle_pagerank_pull (binary32 from 0.0f), then the
 * update of pageRank.c:1055-1069 (binary32 multiply and add, |r' - r| in
 * binary32 compared in binary64) and the next contribution written at pos[v].
 * rank_local[v - rb] holds the rows' un-normalised ranks.  stats[0] = rows
 * that moved by at least eps, stats[1] = sum of |r' - r|. */
void oracle_partition_pass(uint32_t rb, uint32_t re, const uint32_t *in_idx, const uint32_t *in_deg,
                           const uint32_t *in_nb, const uint32_t *out_deg, const uint32_t *pos,
                           const float *c_in_full, float *c_out_full, float *rank_local, double eps, double *stats)
{
    const float damp = ORACLE_DAMP;
    const float base_pr = (1.0f - damp);
    double err_sum = 0.0;
    uint32_t active = 0;
    for (uint32_t v = rb; v < re; ++v) {
        float s = 0.0f;
        for (uint32_t j = in_idx[v]; j < in_idx[v] + in_deg[v]; ++j)
            s += c_in_full[pos[in_nb[j]]];
        const float next = base_pr + (damp * s);
        const double err = fabs(next - rank_local[v - rb]);
        err_sum += err;
        if (err >= eps)
            active++;
        rank_local[v - rb] = next;
        c_out_full[pos[v]] = out_deg[v] ? next / (float)out_deg[v] : 0.0f;
    }
    stats[0] = (double)active;
    stats[1] = err_sum;
}
