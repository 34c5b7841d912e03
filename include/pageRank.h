/*
 * pageRank.h -- PageRank entry points of the B200 library.
 *
 * Replaces 02_capi_graph/include/algorithms/capi/pageRank.h:13-37,69-70 for the
 * CSR data structure.  Same symbol names, argument meaning and ownership:
 * the caller owns `arguments` and `graph` (read only); the callee returns a
 * heap-allocated stats object that the caller releases with
 * freePageRankStats().  pageRanks[] holds the ranks divided by num_vertices
 * (pageRank.c:1079-1085); iterations is the 0-based index of the pass that
 * converged, or arguments->iterations when the cap was reached
 * (pageRank.c:1021,1073-1074); error_total is the last pass's mean absolute
 * change (pageRank.c:1062).
 *
 * Errors follow the reference convention for these legacy symbols: a device
 * failure prints one diagnostic line and exits the process
 * (capienv.c:113-131).  The ag_* entries in accelgraph_b200.h return a status
 * code instead.
 */
#ifndef PAGERANK_H
#define PAGERANK_H

#include <stdint.h>

#include "graphConfig.h"
#include "graphCSR.h"

#ifdef __cplusplus
extern "C" {
#endif

#define Damp 0.85f

struct PageRankStats
{
    float damp;
    float base_pr;
    uint32_t iterations;
    uint32_t num_vertices;
    uint32_t activeVertices;
    uint32_t *realRanks;
    float *pageRanks;
    double time_total;
    double error_total;
};

/* pageRank.c:50-78 -- ranks start at base_pr = 1.0f - Damp, realRanks[v] = v */
struct PageRankStats *newPageRankStatsGraphCSR(struct GraphCSR *graph);
/* pageRank.c:170-180 */
void freePageRankStats(struct PageRankStats *stats);

/* pageRank.c:874-939 -- dispatch on arguments->pushpull.  The B200 library
 * implements the pull direction: 0 (FP32), and the precision forms of the
 * pull kernel selected through ag_pagerank_pull_ex().  Any other selector
 * runs the FP32 pull, which is also the reference's default case. */
struct PageRankStats *pageRankGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:942-1109 -- topology-driven pull over the inverse CSR */
struct PageRankStats *pageRankPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);

#ifdef __cplusplus
}
#endif

#endif /* PAGERANK_H */
