/* stand-in for OpenGraph's graphAdjLinkedList.h (declared so that the
 * linked-list variants compile; never constructed here) */
#ifndef REFSTUB_GRAPHADJLINKEDLIST_H
#define REFSTUB_GRAPHADJLINKEDLIST_H
#include <stdint.h>
#include "graphCSR.h"
struct AdjLinkedListNode
{
    uint32_t dest;
    float weight;
    struct AdjLinkedListNode *next;
    uint32_t *edges_array_dest;
};
struct AdjLinkedList
{
    uint32_t out_degree;
    uint32_t in_degree;
    struct AdjLinkedListNode *outNodes;
    struct AdjLinkedListNode *inNodes;
};
struct GraphAdjLinkedList
{
    uint32_t num_edges;
    uint32_t num_vertices;
    float max_weight;
    struct AdjLinkedList *vertices;
    struct Grid *grid;
    struct EdgeList *sorted_edges_array;
    struct EdgeList *inverse_sorted_edges_array;
    struct Vertex *inverse_vertices;
};
#endif
