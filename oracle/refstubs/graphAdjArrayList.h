/* stand-in for OpenGraph's graphAdjArrayList.h (declared so that the
 * adjacency-array variants compile; never constructed here) */
#ifndef REFSTUB_GRAPHADJARRAYLIST_H
#define REFSTUB_GRAPHADJARRAYLIST_H
#include <stdint.h>
#include "graphCSR.h"
struct AdjArrayList
{
    uint32_t out_degree;
    uint32_t in_degree;
    struct EdgeList *outNodes;
    struct EdgeList *inNodes;
};
struct GraphAdjArrayList
{
    uint32_t num_edges;
    uint32_t num_vertices;
    float max_weight;
    struct AdjArrayList *vertices;
    struct Grid *grid;
    struct EdgeList *sorted_edges_array;
    struct EdgeList *inverse_sorted_edges_array;
    struct Vertex *inverse_vertices;
};
#endif
