/* stand-in for OpenGraph's graphGrid.h (declared so that the grid variants
 * compile; never constructed here) */
#ifndef REFSTUB_GRAPHGRID_H
#define REFSTUB_GRAPHGRID_H
#include <stdint.h>
#include "graphCSR.h"
struct Partition
{
    uint32_t num_edges;
    uint32_t num_vertices;
    struct EdgeList *edgeList;
};
struct Grid
{
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t num_partitions;
    struct Partition *partitions;
    uint32_t *activePartitions;
    uint32_t *out_degree;
    uint32_t *in_degree;
};
struct GraphGrid
{
    uint32_t num_edges;
    uint32_t num_vertices;
    float max_weight;
    struct Grid *grid;
    struct EdgeList *sorted_edges_array;
    struct EdgeList *inverse_sorted_edges_array;
    struct Vertex *vertices;
    struct Vertex *inverse_vertices;
};
#endif
