/*
 * SPMV.h -- sparse matrix-vector product entry points of the B200 library.
 *
 * Replaces 02_capi_graph/include/algorithms/capi/SPMV.h:19-35,51-52 for the CSR
 * data structure.  SPMVPullGraphCSR computes, for every vertex v with at least
 * one in-edge, y[v] = sum over the inverse row of (w_j * x[u_j]) with one
 * binary32 multiply per edge followed by an in-order binary32 add
 * (cu_SPMV/CSR/PULL/FloatPoint/cu/cu_sum_kernel_control.sv:345-368); vertices
 * without in-edges keep y[v] = 0.  The input vector is x[v] = 1/out_degree[v],
 * or 0.001f for a vertex without out-edges (SPMV.c:694-701).  Weights come
 * from inverse_sorted_edges_array->edges_array_weight; a graph without weights
 * uses the reference's unweighted constant 0.0001f (SPMV.c:1206).
 * Each iteration recomputes y from the same x, as the accelerator does.
 */
#ifndef SPMV_H
#define SPMV_H

#include <stdint.h>

#include "graphConfig.h"
#include "graphCSR.h"

#ifdef __cplusplus
extern "C" {
#endif

struct SPMVStats
{
    uint32_t iterations;
    struct Arguments *arguments;
    uint32_t num_vertices;
    float *vector_output;
    float *vector_input;
    double time_total;
};

/* SPMV.c:51-73 */
struct SPMVStats *newSPMVStatsGraphCSR(struct GraphCSR *graph);
/* SPMV.c:145-158 */
void freeSPMVStats(struct SPMVStats *stats);

/* SPMV.c:594-621 -- dispatch on arguments->pushpull; every selector runs the
 * pull product on the GPU */
struct SPMVStats *SPMVGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* SPMV.c:622-751 */
struct SPMVStats *SPMVPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);

#ifdef __cplusplus
}
#endif

#endif /* SPMV_H */
