/*
 * graphCSR.h -- the graph container the algorithm entry points read.
 *
 * The reference's struct GraphCSR / struct Vertex / struct EdgeList live in the
 * OpenGraph submodule, which is empty in the reference checkout.  This header
 * restates them from their uses in the reference sources:
 *   02_capi_graph/src/capi_utils/capienv.c:837-868   (WED mapping: every array
 *                                                    the accelerator reads)
 *   02_capi_graph/src/algorithms/capi/pageRank.c:968-969,1029-1030
 *   02_capi_graph/src/algorithms/capi/SPMV.c:641-645
 *   02_capi_graph/src/tests/test_betweenness_root.c:10-19 (num_vertices,
 *                                                    avg_degree, vertices)
 *
 * Semantics (DIRECTED = 1):
 *   vertices->out_degree[v]   forward out-degree of v
 *   vertices->in_degree[v]    in-degree of v
 *   vertices->edges_idx[v]    first index of v's forward row
 *   sorted_edges_array        forward edges, rows grouped by source
 *   inverse_vertices->out_degree[v]  in-degree of v (row length of the
 *                                    inverse CSR, pageRank.c:2901)
 *   inverse_vertices->in_degree[v]   forward out-degree of v
 *   inverse_vertices->edges_idx[v]   first index of v's inverse row
 *   inverse_sorted_edges_array->edges_array_dest[j]  source u of the j-th
 *                                    in-edge (the gather index, pageRank.c:2904)
 *   inverse_sorted_edges_array->edges_array_src[j]   the row owner v
 *   inverse_sorted_edges_array->edges_array_weight[j] weight of that in-edge
 * All ids, degrees and offsets are uint32 (the accelerator's 4-byte vertex and
 * edge words, cu_PageRank/.../pkg/globals_cu_pkg.sv:45,51).
 */
#ifndef GRAPHCSR_H
#define GRAPHCSR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct Vertex
{
    uint32_t *out_degree;
    uint32_t *in_degree;
    uint32_t *edges_idx;
};

struct EdgeList
{
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t avg_degree;
    float max_weight;
    uint32_t *edges_array_src;
    uint32_t *edges_array_dest;
    float *edges_array_weight;     /* NULL when the graph is unweighted */
    uint32_t *label_array;         /* optional relabelling, may be NULL */
    uint32_t *inverse_label_array; /* optional relabelling, may be NULL */
};

struct GraphCSR
{
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t avg_degree;
    float max_weight;
    struct Vertex *vertices;
    struct Vertex *inverse_vertices;
    struct EdgeList *sorted_edges_array;
    struct EdgeList *inverse_sorted_edges_array;
};

#ifdef __cplusplus
}
#endif

#endif /* GRAPHCSR_H */
