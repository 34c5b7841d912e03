/*
 * graph_host.c -- host graph substrate: edge lists to forward and inverse CSR,
 * seeded generators and the binary edge-list reader.
 *
 * The reference obtains struct GraphCSR from OpenGraph
 * (generateGraphDataStructure, 02_capi_graph/src/main/accel-graph.c:345), a
 * submodule that is empty in the reference checkout.  This file restates the
 * behaviour the reference relies on:
 *   - `-k` removes self loops and duplicate edges and forces sort = 1
 *     (accel-graph.c:142-145,336-337): rows ordered by neighbour id;
 *   - the inverse CSR lists, for every vertex v, the sources u of its
 *     in-edges; inverse_vertices->out_degree is the in-degree
 *     (pageRank.c:2898-2907);
 *   - binary edge lists hold uint32 (src, dst) pairs, 8 bytes per edge
 *     (04_test_graphs/TEST/graphbrew/graph.bin: 152 bytes, 19 edges).
 * Sorting is a parallel LSD radix sort (stable), so unsorted builds keep the
 * input order of each row's edges.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <math.h>
#include <omp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "ag_internal.h"
#include "ag_rng.h"

/* ------------------------------------------------------------ errors */
static __thread char ag_errbuf[512];

ag_status_t ag_set_error(ag_status_t status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ag_errbuf, sizeof(ag_errbuf), fmt, ap);
    va_end(ap);
    return status;
}

void ag_clear_error(void) { ag_errbuf[0] = '\0'; }

const char *ag_last_error(void) { return ag_errbuf; }

const char *ag_status_string(ag_status_t s)
{
    switch (s) {
    case AG_OK: return "ok";
    case AG_ERR_INVALID_ARG: return "invalid argument";
    case AG_ERR_INVALID_GRAPH: return "invalid graph";
    case AG_ERR_CUDA: return "CUDA error";
    case AG_ERR_OOM: return "out of memory";
    case AG_ERR_TIMEOUT: return "timeout";
    case AG_ERR_NO_DEVICE: return "no CUDA device";
    case AG_ERR_UNSUPPORTED: return "unsupported";
    case AG_ERR_DEVICE_WAIT: return "device wait ran out";
    default: return "unknown status";
    }
}

double ag_wall_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------- owned graphs */
#define AG_GRAPH_MAGIC 0x41474352u /* "AGCR" */

typedef struct ag_host_graph
{
    struct GraphCSR g;       /* first member: GraphCSR* casts back to this */
    struct Vertex v, iv;
    struct EdgeList el, iel;
    uint32_t magic;
    int pinned;
} ag_host_graph;

static void *halloc(size_t bytes, int want_pinned, int *pinned_flag)
{
    int got = 0;
    void *p;
    if (bytes == 0)
        bytes = 16;
    p = ag_rt_host_alloc(bytes, want_pinned, &got);
    if (p && !got)
        *pinned_flag = 0;
    return p;
}

static void hfree(void *p, int pinned)
{
    if (p)
        ag_rt_host_free(p, pinned);
}

void ag_graph_free(struct GraphCSR *graph)
{
    ag_host_graph *h = (ag_host_graph *)graph;
    if (!graph)
        return;
    if (h->magic != AG_GRAPH_MAGIC) {
        fprintf(stderr, "ag_graph_free: graph was not built by this library; not freed\n");
        return;
    }
    hfree(h->v.out_degree, h->pinned);
    hfree(h->v.in_degree, h->pinned);
    hfree(h->v.edges_idx, h->pinned);
    hfree(h->iv.edges_idx, h->pinned);
    hfree(h->el.edges_array_src, h->pinned);
    hfree(h->el.edges_array_dest, h->pinned);
    hfree(h->el.edges_array_weight, h->pinned);
    hfree(h->iel.edges_array_src, h->pinned);
    hfree(h->iel.edges_array_dest, h->pinned);
    hfree(h->iel.edges_array_weight, h->pinned);
    h->magic = 0;
    free(h);
}

/* an empty host graph with every array of the builder's layout allocated:
 * row starts of N + 1 entries, inverse degrees aliasing the forward ones */
struct GraphCSR *ag_host_graph_new(uint32_t N, uint32_t E, int weighted, int pinned)
{
    ag_host_graph *h = (ag_host_graph *)calloc(1, sizeof(*h));
    if (!h)
        return NULL;
    h->magic = AG_GRAPH_MAGIC;
    h->pinned = pinned;
    h->g.num_vertices = N;
    h->g.num_edges = E;
    h->g.avg_degree = N ? E / N : 0;
    h->g.vertices = &h->v;
    h->g.inverse_vertices = &h->iv;
    h->g.sorted_edges_array = &h->el;
    h->g.inverse_sorted_edges_array = &h->iel;
    h->el.num_edges = h->iel.num_edges = E;
    h->el.num_vertices = h->iel.num_vertices = N;
    h->el.avg_degree = h->iel.avg_degree = h->g.avg_degree;
    h->v.out_degree = (uint32_t *)halloc((size_t)N * 4, pinned, &h->pinned);
    h->v.in_degree = (uint32_t *)halloc((size_t)N * 4, pinned, &h->pinned);
    h->v.edges_idx = (uint32_t *)halloc((size_t)N * 4 + 4, pinned, &h->pinned);
    h->iv.edges_idx = (uint32_t *)halloc((size_t)N * 4 + 4, pinned, &h->pinned);
    h->el.edges_array_src = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->el.edges_array_dest = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->iel.edges_array_src = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->iel.edges_array_dest = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    if (weighted) {
        h->el.edges_array_weight = (float *)halloc((size_t)E * 4, pinned, &h->pinned);
        h->iel.edges_array_weight = (float *)halloc((size_t)E * 4, pinned, &h->pinned);
    }
    h->iv.out_degree = h->v.in_degree;
    h->iv.in_degree = h->v.out_degree;
    if (!h->v.out_degree || !h->v.in_degree || !h->v.edges_idx || !h->iv.edges_idx || !h->el.edges_array_src ||
        !h->el.edges_array_dest || !h->iel.edges_array_src || !h->iel.edges_array_dest ||
        (weighted && (!h->el.edges_array_weight || !h->iel.edges_array_weight))) {
        ag_graph_free(&h->g);
        return NULL;
    }
    return &h->g;
}

/* ------------------------------------------------------- radix sort */
static int bits_for(uint64_t max_value)
{
    int b = 1;
    while (b < 64 && (max_value >> b) != 0)
        b++;
    return b;
}

/* Stable LSD radix sort of keys (low key_bits bits) with optional uint32
 * payload.  Returns 0 on success, -1 on allocation failure. */
static int radix_sort_u64(uint64_t *keys, uint32_t *vals, uint64_t n, int key_bits)
{
    enum { DIG = 11, NB = 1 << DIG };
    uint64_t *k_src = keys, *k_dst;
    uint32_t *v_src = vals, *v_dst = NULL;
    int max_t = omp_get_max_threads();
    size_t *hist;
    int passes = 0;

    if (n < 2)
        return 0;
    k_dst = (uint64_t *)malloc(n * sizeof(uint64_t));
    if (vals)
        v_dst = (uint32_t *)malloc(n * sizeof(uint32_t));
    hist = (size_t *)malloc((size_t)max_t * NB * sizeof(size_t));
    if (!k_dst || (vals && !v_dst) || !hist) {
        free(k_dst);
        free(v_dst);
        free(hist);
        return -1;
    }

    for (int shift = 0; shift < key_bits; shift += DIG) {
#pragma omp parallel num_threads(max_t)
        {
            int t = omp_get_thread_num();
            int T = omp_get_num_threads();
            uint64_t lo = n * (uint64_t)t / (uint64_t)T;
            uint64_t hi = n * (uint64_t)(t + 1) / (uint64_t)T;
            size_t *h = hist + (size_t)t * NB;
            memset(h, 0, NB * sizeof(size_t));
            for (uint64_t i = lo; i < hi; i++)
                h[(k_src[i] >> shift) & (NB - 1)]++;
#pragma omp barrier
#pragma omp single
            {
                size_t sum = 0;
                for (int d = 0; d < NB; d++)
                    for (int tt = 0; tt < T; tt++) {
                        size_t c = hist[(size_t)tt * NB + d];
                        hist[(size_t)tt * NB + d] = sum;
                        sum += c;
                    }
            }
            for (uint64_t i = lo; i < hi; i++) {
                size_t pos = h[(k_src[i] >> shift) & (NB - 1)]++;
                k_dst[pos] = k_src[i];
                if (v_src)
                    v_dst[pos] = v_src[i];
            }
        }
        { uint64_t *tk = k_src; k_src = k_dst; k_dst = tk; }
        { uint32_t *tv = v_src; v_src = v_dst; v_dst = tv; }
        passes++;
    }
    if (passes & 1) {
        /* result is in the scratch buffers: copy back */
        memcpy(keys, k_src, n * sizeof(uint64_t));
        if (vals)
            memcpy(vals, v_src, n * sizeof(uint32_t));
        free(k_src);
        free(v_src);
    } else {
        free(k_dst);
        free(v_dst);
    }
    free(hist);
    return 0;
}

/* row starts of a list sorted by row id: idx[v] = first i with row(i) >= v */
static void row_starts(const uint32_t *row, uint64_t n, uint32_t num_vertices, uint32_t *idx)
{
    if (n == 0) {
        for (uint32_t v = 0; v < num_vertices; v++)
            idx[v] = 0;
        return;
    }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) {
        int64_t prev = (i == 0) ? -1 : (int64_t)row[i - 1];
        for (int64_t v = prev + 1; v <= (int64_t)row[i]; v++)
            idx[v] = (uint32_t)i;
    }
    for (uint64_t v = (uint64_t)row[n - 1] + 1; v < num_vertices; v++)
        idx[v] = (uint32_t)n;
}

/* ----------------------------------------------------------- CSR build */
struct GraphCSR *ag_graph_from_edges(uint32_t num_vertices, uint64_t num_edges,
                                     const uint32_t *src, const uint32_t *dst,
                                     const float *weight, uint32_t flags)
{
    ag_host_graph *h;
    uint64_t *keys = NULL;
    uint32_t *perm = NULL;
    uint64_t m, E;
    int nb, sorted = (flags & (AG_BUILD_SORT | AG_BUILD_DEDUPE)) != 0;
    int dedupe = (flags & AG_BUILD_DEDUPE) != 0;
    int pinned = (flags & AG_BUILD_PINNED) != 0;
    int weighted = weight != NULL;
    uint32_t N = num_vertices;

    ag_clear_error();
    if (num_edges > 0 && (!src || !dst)) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_from_edges: NULL edge arrays");
        return NULL;
    }
    if (num_edges >= 0xFFFFFFF0ull) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_from_edges: %llu edges exceed the uint32 edge index",
                     (unsigned long long)num_edges);
        return NULL;
    }
    for (uint64_t i = 0; i < num_edges; i++) {
        if (src[i] >= N || dst[i] >= N) {
            ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_from_edges: edge %llu (%u -> %u) outside %u vertices",
                         (unsigned long long)i, src[i], dst[i], N);
            return NULL;
        }
    }

    if (flags & AG_BUILD_SYMMETRIC) {
        /* every edge followed, after the input list, by its reverse */
        struct GraphCSR *sg = NULL;
        uint64_t m2 = 2 * num_edges;
        uint32_t *s2, *d2;
        float *w2 = NULL;
        if (m2 >= 0xFFFFFFF0ull) {
            ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_from_edges: %llu edges with their reverses exceed the "
                         "uint32 edge index", (unsigned long long)num_edges);
            return NULL;
        }
        s2 = (uint32_t *)malloc((m2 ? m2 : 1) * 4);
        d2 = (uint32_t *)malloc((m2 ? m2 : 1) * 4);
        if (weighted)
            w2 = (float *)malloc((m2 ? m2 : 1) * 4);
        if (s2 && d2 && (!weighted || w2)) {
            if (num_edges) {
                memcpy(s2, src, num_edges * 4);
                memcpy(s2 + num_edges, dst, num_edges * 4);
                memcpy(d2, dst, num_edges * 4);
                memcpy(d2 + num_edges, src, num_edges * 4);
                if (weighted) {
                    memcpy(w2, weight, num_edges * 4);
                    memcpy(w2 + num_edges, weight, num_edges * 4);
                }
            }
            sg = ag_graph_from_edges(N, m2, s2, d2, w2, flags & ~AG_BUILD_SYMMETRIC);
        } else {
            ag_set_error(AG_ERR_OOM, "ag_graph_from_edges: host allocation failed");
        }
        free(s2);
        free(d2);
        free(w2);
        return sg;
    }

    h = (ag_host_graph *)calloc(1, sizeof(*h));
    if (!h) {
        ag_set_error(AG_ERR_OOM, "ag_graph_from_edges: host allocation failed");
        return NULL;
    }
    h->magic = AG_GRAPH_MAGIC;
    h->pinned = pinned;

    nb = bits_for(N > 0 ? (uint64_t)(N - 1) : 0);
    m = num_edges;
    keys = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    if (!sorted || weighted)
        perm = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!keys || ((!sorted || weighted) && !perm))
        goto oom;

    /* forward order */
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m; i++) {
        keys[i] = sorted ? (((uint64_t)src[i] << nb) | dst[i]) : (uint64_t)src[i];
        if (perm)
            perm[i] = (uint32_t)i;
    }
    if (radix_sort_u64(keys, perm, m, sorted ? 2 * nb : nb) != 0)
        goto oom;

    /* dedupe + self-loop removal on the sorted keys (keeps first occurrence) */
    if (dedupe && m > 0) {
        uint64_t w = 0;
        uint64_t mask = (1ull << nb) - 1;
        for (uint64_t i = 0; i < m; i++) {
            uint64_t k = keys[i];
            uint32_t s = (uint32_t)(k >> nb), d = (uint32_t)(k & mask);
            if (s == d)
                continue;
            if (w > 0 && keys[w - 1] == k)
                continue;
            keys[w] = k;
            if (perm)
                perm[w] = perm[i];
            w++;
        }
        m = w;
    }
    E = m;

    h->g.num_vertices = N;
    h->g.num_edges = (uint32_t)E;
    h->g.avg_degree = N ? (uint32_t)(E / N) : 0;
    h->g.vertices = &h->v;
    h->g.inverse_vertices = &h->iv;
    h->g.sorted_edges_array = &h->el;
    h->g.inverse_sorted_edges_array = &h->iel;
    h->el.num_edges = h->iel.num_edges = (uint32_t)E;
    h->el.num_vertices = h->iel.num_vertices = N;
    h->el.avg_degree = h->iel.avg_degree = h->g.avg_degree;

    h->v.out_degree = (uint32_t *)halloc((size_t)N * 4, pinned, &h->pinned);
    h->v.in_degree = (uint32_t *)halloc((size_t)N * 4, pinned, &h->pinned);
    h->v.edges_idx = (uint32_t *)halloc((size_t)N * 4 + 4, pinned, &h->pinned);
    h->iv.edges_idx = (uint32_t *)halloc((size_t)N * 4 + 4, pinned, &h->pinned);
    h->el.edges_array_src = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->el.edges_array_dest = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->iel.edges_array_src = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    h->iel.edges_array_dest = (uint32_t *)halloc((size_t)E * 4, pinned, &h->pinned);
    if (!h->v.out_degree || !h->v.in_degree || !h->v.edges_idx || !h->iv.edges_idx ||
        !h->el.edges_array_src || !h->el.edges_array_dest || !h->iel.edges_array_src ||
        !h->iel.edges_array_dest)
        goto oom;
    if (weighted) {
        h->el.edges_array_weight = (float *)halloc((size_t)E * 4, pinned, &h->pinned);
        h->iel.edges_array_weight = (float *)halloc((size_t)E * 4, pinned, &h->pinned);
        if (!h->el.edges_array_weight || !h->iel.edges_array_weight)
            goto oom;
    }
    /* the inverse graph's degree arrays are the forward ones, swapped */
    h->iv.out_degree = h->v.in_degree;
    h->iv.in_degree = h->v.out_degree;

    {
        uint64_t mask = (1ull << nb) - 1;
        float maxw = 0.0f;
#pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < E; i++) {
            uint32_t s, d;
            if (sorted) {
                s = (uint32_t)(keys[i] >> nb);
                d = (uint32_t)(keys[i] & mask);
            } else {
                s = (uint32_t)keys[i];
                d = dst[perm[i]];
            }
            h->el.edges_array_src[i] = s;
            h->el.edges_array_dest[i] = d;
            if (weighted)
                h->el.edges_array_weight[i] = weight[perm[i]];
        }
        if (weighted) {
            for (uint64_t i = 0; i < E; i++)
                if (h->el.edges_array_weight[i] > maxw)
                    maxw = h->el.edges_array_weight[i];
        }
        h->g.max_weight = h->el.max_weight = h->iel.max_weight = maxw;
    }
    row_starts(h->el.edges_array_src, E, N, h->v.edges_idx);
    h->v.edges_idx[N] = (uint32_t)E; /* sentinel beyond the struct contract */
#pragma omp parallel for schedule(static)
    for (uint64_t v = 0; v < N; v++)
        h->v.out_degree[v] = ((v + 1 < N) ? h->v.edges_idx[v + 1] : (uint32_t)E) - h->v.edges_idx[v];

    /* inverse: stable sort of the forward order by destination.  With sorted
     * forward rows this orders every inverse row by source id. */
    if (!perm && E > 0) {
        perm = (uint32_t *)malloc(E * sizeof(uint32_t));
        if (!perm)
            goto oom;
    }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < E; i++) {
        keys[i] = (uint64_t)h->el.edges_array_dest[i];
        perm[i] = (uint32_t)i;
    }
    if (radix_sort_u64(keys, perm, E, nb) != 0)
        goto oom;
#pragma omp parallel for schedule(static)
    for (uint64_t j = 0; j < E; j++) {
        uint32_t f = perm[j];
        h->iel.edges_array_src[j] = (uint32_t)keys[j];
        h->iel.edges_array_dest[j] = h->el.edges_array_src[f];
        if (weighted)
            h->iel.edges_array_weight[j] = h->el.edges_array_weight[f];
    }
    row_starts(h->iel.edges_array_src, E, N, h->iv.edges_idx);
    h->iv.edges_idx[N] = (uint32_t)E;
#pragma omp parallel for schedule(static)
    for (uint64_t v = 0; v < N; v++)
        h->v.in_degree[v] = ((v + 1 < N) ? h->iv.edges_idx[v + 1] : (uint32_t)E) - h->iv.edges_idx[v];

    free(keys);
    free(perm);
    return &h->g;

oom:
    free(keys);
    free(perm);
    ag_graph_free(&h->g);
    ag_set_error(AG_ERR_OOM, "ag_graph_from_edges: host allocation failed (%llu edges)",
                 (unsigned long long)num_edges);
    return NULL;
}

/* --------------------------------------------------------- generators */
static struct GraphCSR *finish_generated(uint32_t N, uint64_t m, uint32_t *src, uint32_t *dst,
                                         uint64_t seed, uint32_t flags)
{
    struct GraphCSR *g;
    float *w = NULL;
    if (flags & AG_BUILD_WEIGHTS) {
        /* weights are attached per generated edge, so they follow an edge
         * through sorting; duplicates keep their first occurrence */
        w = (float *)malloc((m ? m : 1) * sizeof(float));
        if (!w) {
            ag_set_error(AG_ERR_OOM, "generator: weight allocation failed");
            return NULL;
        }
#pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < m; i++)
            w[i] = ag_u01(ag_draw64(seed + 1, i, 0));
    }
    g = ag_graph_from_edges(N, m, src, dst, w, flags & ~AG_BUILD_WEIGHTS);
    free(w);
    return g;
}

struct GraphCSR *ag_graph_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                               uint64_t seed, uint32_t flags)
{
    uint64_t N, m;
    uint32_t *src, *dst;
    uint32_t ta, tab, tabc;
    struct GraphCSR *g;

    ag_clear_error();
    if (scale == 0 || scale > 31 || edge_factor == 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_rmat: bad parameters (scale %u, ef %u)", scale, edge_factor);
        return NULL;
    }
    N = 1ull << scale;
    m = (uint64_t)edge_factor * N;
    if (m >= 0xFFFFFFF0ull) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_rmat: too many edges");
        return NULL;
    }
    ta = (uint32_t)fmin(4294967295.0, floor(a * 4294967296.0));
    tab = (uint32_t)fmin(4294967295.0, floor((a + b) * 4294967296.0));
    tabc = (uint32_t)fmin(4294967295.0, floor((a + b + c) * 4294967296.0));
    src = (uint32_t *)malloc(m * sizeof(uint32_t));
    dst = (uint32_t *)malloc(m * sizeof(uint32_t));
    if (!src || !dst) {
        free(src);
        free(dst);
        ag_set_error(AG_ERR_OOM, "ag_graph_rmat: allocation failed");
        return NULL;
    }
#pragma omp parallel for schedule(static)
    for (uint64_t e = 0; e < m; e++) {
        uint32_t s = 0, d = 0;
        uint64_t bits = 0;
        for (uint32_t l = 0; l < scale; l++) {
            uint32_t u;
            if ((l & 1) == 0)
                bits = ag_draw64(seed, e, l >> 1);
            u = (l & 1) ? (uint32_t)(bits >> 32) : (uint32_t)bits;
            s <<= 1;
            d <<= 1;
            if (u < ta) {
            } else if (u < tab) {
                d |= 1;
            } else if (u < tabc) {
                s |= 1;
            } else {
                s |= 1;
                d |= 1;
            }
        }
        src[e] = s;
        dst[e] = d;
    }
    g = finish_generated((uint32_t)N, m, src, dst, seed, flags);
    free(src);
    free(dst);
    return g;
}

struct GraphCSR *ag_graph_er(uint32_t num_vertices, uint32_t avg_degree, uint64_t seed, uint32_t flags)
{
    uint64_t m = (uint64_t)num_vertices * avg_degree;
    uint32_t *src, *dst;
    struct GraphCSR *g;
    ag_clear_error();
    if (num_vertices == 0 || m >= 0xFFFFFFF0ull) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_er: bad parameters");
        return NULL;
    }
    src = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    dst = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!src || !dst) {
        free(src);
        free(dst);
        ag_set_error(AG_ERR_OOM, "ag_graph_er: allocation failed");
        return NULL;
    }
#pragma omp parallel for schedule(static)
    for (uint64_t e = 0; e < m; e++) {
        uint64_t bits = ag_draw64(seed, e, 0);
        src[e] = (uint32_t)(((bits & 0xFFFFFFFFull) * num_vertices) >> 32);
        dst[e] = (uint32_t)(((bits >> 32) * num_vertices) >> 32);
    }
    g = finish_generated(num_vertices, m, src, dst, seed, flags);
    free(src);
    free(dst);
    return g;
}

struct GraphCSR *ag_graph_read_edge_file(const char *path, int weighted, uint32_t flags)
{
    FILE *f;
    long size;
    size_t rec = weighted ? 12 : 8;
    uint64_t m;
    uint32_t *src = NULL, *dst = NULL, maxid = 0;
    float *w = NULL;
    unsigned char *buf = NULL;
    struct GraphCSR *g = NULL;

    ag_clear_error();
    if (!path) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read_edge_file: NULL path");
        return NULL;
    }
    f = fopen(path, "rb");
    if (!f) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read_edge_file: cannot open %s: %s", path, strerror(errno));
        return NULL;
    }
    fseek(f, 0, SEEK_END);
    size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 0 || (size_t)size % rec != 0) {
        fclose(f);
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read_edge_file: %s size %ld is not a multiple of %zu",
                     path, size, rec);
        return NULL;
    }
    m = (uint64_t)size / rec;
    buf = (unsigned char *)malloc(size ? (size_t)size : 1);
    src = (uint32_t *)malloc((m ? m : 1) * 4);
    dst = (uint32_t *)malloc((m ? m : 1) * 4);
    if (weighted)
        w = (float *)malloc((m ? m : 1) * 4);
    if (!buf || !src || !dst || (weighted && !w)) {
        ag_set_error(AG_ERR_OOM, "ag_graph_read_edge_file: allocation failed");
        goto done;
    }
    if (size && fread(buf, 1, (size_t)size, f) != (size_t)size) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read_edge_file: short read on %s", path);
        goto done;
    }
    for (uint64_t i = 0; i < m; i++) {
        memcpy(&src[i], buf + i * rec, 4);
        memcpy(&dst[i], buf + i * rec + 4, 4);
        if (weighted)
            memcpy(&w[i], buf + i * rec + 8, 4);
        if (src[i] > maxid)
            maxid = src[i];
        if (dst[i] > maxid)
            maxid = dst[i];
    }
    g = ag_graph_from_edges(m ? maxid + 1 : 0, m, src, dst, w, flags);
done:
    fclose(f);
    free(buf);
    free(src);
    free(dst);
    free(w);
    return g;
}

void ag_fill_uniform(float *out, uint64_t n, uint64_t seed)
{
    if (!out)
        return;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++)
        out[i] = ag_u01(ag_draw64(seed, i, 0));
}

/* ---------------------------------------------------------- graph files */
/* text edge list: "src dst [weight]" per line, blanks between fields */
static struct GraphCSR *read_text_edges(const char *path, int weighted, uint32_t flags)
{
    FILE *f = fopen(path, "r");
    char line[512];
    uint64_t m = 0, cap = 1u << 16, lineno = 0;
    uint32_t *src = NULL, *dst = NULL, maxid = 0;
    float *w = NULL;
    struct GraphCSR *g = NULL;
    if (!f) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: cannot open %s: %s", path, strerror(errno));
        return NULL;
    }
    src = (uint32_t *)malloc(cap * 4);
    dst = (uint32_t *)malloc(cap * 4);
    w = weighted ? (float *)malloc(cap * 4) : NULL;
    if (!src || !dst || (weighted && !w))
        goto oom;
    while (fgets(line, sizeof(line), f)) {
        char *p = line, *end;
        unsigned long long a, b;
        ++lineno;
        if (!strchr(line, '\n') && !feof(f)) {
            ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: %s:%llu: line too long", path,
                         (unsigned long long)lineno);
            goto fail;
        }
        while (*p == ' ' || *p == '\t' || *p == '\r')
            ++p;
        if (*p == '\n' || *p == '\0' || *p == '#' || *p == '%')
            continue;
        errno = 0;
        a = strtoull(p, &end, 10);
        if (end == p || errno)
            goto bad;
        p = end;
        b = strtoull(p, &end, 10);
        if (end == p || errno)
            goto bad;
        p = end;
        if (a > 0xFFFFFFFEull || b > 0xFFFFFFFEull)
            goto bad;
        if (m == cap) {
            uint32_t *ns, *nd;
            float *nw = NULL;
            cap *= 2;
            ns = (uint32_t *)realloc(src, cap * 4);
            if (ns)
                src = ns;
            nd = (uint32_t *)realloc(dst, cap * 4);
            if (nd)
                dst = nd;
            if (weighted) {
                nw = (float *)realloc(w, cap * 4);
                if (nw)
                    w = nw;
            }
            if (!ns || !nd || (weighted && !nw))
                goto oom;
        }
        if (weighted) {
            float x = strtof(p, &end);
            if (end == p)
                goto bad;
            w[m] = x;
            p = end;
        }
        while (*p == ' ' || *p == '\t' || *p == '\r')
            ++p;
        if (*p != '\n' && *p != '\0')
            goto bad;
        src[m] = (uint32_t)a;
        dst[m] = (uint32_t)b;
        if (src[m] > maxid)
            maxid = src[m];
        if (dst[m] > maxid)
            maxid = dst[m];
        ++m;
        if (m >= 0xFFFFFFF0ull) {
            ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: %s: too many edges", path);
            goto fail;
        }
    }
    g = ag_graph_from_edges(m ? maxid + 1 : 0, m, src, dst, w, flags);
    goto fail; /* common exit */
bad:
    ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: %s:%llu: expected \"src dst%s\"", path,
                 (unsigned long long)lineno, weighted ? " weight" : "");
    goto fail;
oom:
    ag_set_error(AG_ERR_OOM, "ag_graph_read: allocation failed");
fail:
    fclose(f);
    free(src);
    free(dst);
    free(w);
    return g;
}

/* serialised CSR: header, then every array of the graph, little endian */
static const char csr_magic[8] = {'A', 'G', 'C', 'S', 'R', '1', 0, 0};

struct csr_header
{
    char magic[8];
    uint32_t num_vertices, num_edges, weighted, avg_degree;
    float max_weight;
    uint32_t reserved[3];
};

static int write_all(FILE *f, const void *p, size_t bytes)
{
    return bytes == 0 || fwrite(p, 1, bytes, f) == bytes;
}

static int read_all(FILE *f, void *p, size_t bytes)
{
    return bytes == 0 || fread(p, 1, bytes, f) == bytes;
}

static struct GraphCSR *read_csr(const char *path, uint32_t flags)
{
    FILE *f = fopen(path, "rb");
    struct csr_header hd;
    struct GraphCSR *g;
    long size;
    uint64_t N, E, need;
    int ok;
    if (!f) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: cannot open %s: %s", path, strerror(errno));
        return NULL;
    }
    if (!read_all(f, &hd, sizeof(hd)) || memcmp(hd.magic, csr_magic, sizeof(csr_magic)) != 0 || hd.weighted > 1) {
        fclose(f);
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: %s is not a serialised CSR", path);
        return NULL;
    }
    N = hd.num_vertices;
    E = hd.num_edges;
    need = sizeof(hd) + 4 * (2 * N + 2 * (N + 1) + 4 * E + (hd.weighted ? 2 * E : 0));
    fseek(f, 0, SEEK_END);
    size = ftell(f);
    fseek(f, (long)sizeof(hd), SEEK_SET);
    if (size < 0 || (uint64_t)size != need) {
        fclose(f);
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: %s holds %ld bytes, its header needs %llu", path, size,
                     (unsigned long long)need);
        return NULL;
    }
    g = ag_host_graph_new((uint32_t)N, (uint32_t)E, (int)hd.weighted, (flags & AG_BUILD_PINNED) ? 1 : 0);
    if (!g) {
        fclose(f);
        ag_set_error(AG_ERR_OOM, "ag_graph_read: allocation failed");
        return NULL;
    }
    ok = read_all(f, g->vertices->out_degree, N * 4) && read_all(f, g->vertices->in_degree, N * 4) &&
         read_all(f, g->vertices->edges_idx, (N + 1) * 4) && read_all(f, g->inverse_vertices->edges_idx, (N + 1) * 4) &&
         read_all(f, g->sorted_edges_array->edges_array_src, E * 4) &&
         read_all(f, g->sorted_edges_array->edges_array_dest, E * 4) &&
         read_all(f, g->inverse_sorted_edges_array->edges_array_src, E * 4) &&
         read_all(f, g->inverse_sorted_edges_array->edges_array_dest, E * 4);
    if (ok && hd.weighted)
        ok = read_all(f, g->sorted_edges_array->edges_array_weight, E * 4) &&
             read_all(f, g->inverse_sorted_edges_array->edges_array_weight, E * 4);
    fclose(f);
    if (!ok) {
        ag_graph_free(g);
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: short read on %s", path);
        return NULL;
    }
    g->avg_degree = g->sorted_edges_array->avg_degree = g->inverse_sorted_edges_array->avg_degree = hd.avg_degree;
    g->max_weight = g->sorted_edges_array->max_weight = g->inverse_sorted_edges_array->max_weight = hd.max_weight;
    return g;
}

struct GraphCSR *ag_graph_read(const char *path, int format, int weighted, uint32_t flags)
{
    ag_clear_error();
    if (!path) {
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: NULL path");
        return NULL;
    }
    switch (format) {
    case AG_FILE_TEXT:
        return read_text_edges(path, weighted, flags);
    case AG_FILE_BINARY:
        return ag_graph_read_edge_file(path, weighted, flags);
    case AG_FILE_CSR:
        return read_csr(path, flags);
    default:
        ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_read: unknown format %d", format);
        return NULL;
    }
}

ag_status_t ag_graph_write(const struct GraphCSR *graph, const char *path, int format)
{
    FILE *f;
    const struct EdgeList *el, *iel;
    uint64_t N, E;
    int ok = 1, weighted;
    ag_clear_error();
    if (!graph || !path)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_write: NULL argument");
    if (format < AG_FILE_TEXT || format > AG_FILE_CSR)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_write: unknown format %d", format);
    N = graph->num_vertices;
    E = graph->num_edges;
    el = graph->sorted_edges_array;
    iel = graph->inverse_sorted_edges_array;
    if ((E && (!el || !el->edges_array_src || !el->edges_array_dest)) || !graph->vertices ||
        (format == AG_FILE_CSR && (!iel || !graph->inverse_vertices || !graph->vertices->edges_idx ||
                                   !graph->inverse_vertices->edges_idx || !graph->vertices->out_degree ||
                                   !graph->vertices->in_degree || (E && (!iel->edges_array_src ||
                                                                         !iel->edges_array_dest)))))
        return ag_set_error(AG_ERR_INVALID_GRAPH, "ag_graph_write: the graph lacks arrays this format needs");
    weighted = el && el->edges_array_weight && (format != AG_FILE_CSR || (iel && iel->edges_array_weight));
    f = fopen(path, format == AG_FILE_TEXT ? "w" : "wb");
    if (!f)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_write: cannot open %s: %s", path, strerror(errno));
    if (format == AG_FILE_TEXT) {
        for (uint64_t i = 0; i < E && ok; i++) {
            if (weighted)
                ok = fprintf(f, "%u %u %.9g\n", el->edges_array_src[i], el->edges_array_dest[i],
                             (double)el->edges_array_weight[i]) > 0;
            else
                ok = fprintf(f, "%u %u\n", el->edges_array_src[i], el->edges_array_dest[i]) > 0;
        }
    } else if (format == AG_FILE_BINARY) {
        for (uint64_t i = 0; i < E && ok; i++) {
            ok = write_all(f, &el->edges_array_src[i], 4) && write_all(f, &el->edges_array_dest[i], 4);
            if (ok && weighted)
                ok = write_all(f, &el->edges_array_weight[i], 4);
        }
    } else {
        /* the first N + 1 row starts: the builder keeps a closing entry; a
         * graph without one gets E written in its place */
        struct csr_header hd;
        uint32_t e32 = (uint32_t)E;
        memset(&hd, 0, sizeof(hd));
        memcpy(hd.magic, csr_magic, sizeof(csr_magic));
        hd.num_vertices = (uint32_t)N;
        hd.num_edges = (uint32_t)E;
        hd.weighted = (uint32_t)weighted;
        hd.avg_degree = graph->avg_degree;
        hd.max_weight = graph->max_weight;
        ok = write_all(f, &hd, sizeof(hd)) && write_all(f, graph->vertices->out_degree, N * 4) &&
             write_all(f, graph->vertices->in_degree, N * 4) && write_all(f, graph->vertices->edges_idx, N * 4) &&
             write_all(f, &e32, 4) && write_all(f, graph->inverse_vertices->edges_idx, N * 4) &&
             write_all(f, &e32, 4) && write_all(f, el->edges_array_src, E * 4) &&
             write_all(f, el->edges_array_dest, E * 4) && write_all(f, iel->edges_array_src, E * 4) &&
             write_all(f, iel->edges_array_dest, E * 4);
        if (ok && weighted)
            ok = write_all(f, el->edges_array_weight, E * 4) && write_all(f, iel->edges_array_weight, E * 4);
    }
    if (fclose(f) != 0)
        ok = 0;
    return ok ? AG_OK : ag_set_error(AG_ERR_INVALID_ARG, "ag_graph_write: write to %s failed", path);
}
