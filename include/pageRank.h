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

/* pageRank.c:874-939 -- dispatch on arguments->pushpull to the forms below:
 * 0 pull, 1 push, 2 / 9 / 10 / 11 64 / 32 / 16 / 8-bit fixed-point pull,
 * 3 fixed-point push, 4 / 12 / 13 32 / 16 / 8-bit quantised pull, 5 quantised
 * push, 6 data-driven pull, 7 data-driven push, 8 data-driven pull-push.  Any
 * other selector runs the FP32 pull, the reference's default case, with a note
 * on stderr. */
struct PageRankStats *pageRankGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:942-1109 -- topology-driven pull over the inverse CSR */
struct PageRankStats *pageRankPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);

/* The reference's per-form entry points (pageRank.h:71-86), each with the
 * semantics of the pageRank.c function named: */
/* pageRank.c:1111-1272 -- push, binary32 contributions */
struct PageRankStats *pageRankPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:1276-1453 -- pull, 64-bit fixed-point contributions */
struct PageRankStats *pageRankPullFixedPoint64BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:1455-1633 -- pull, 32-bit fixed-point contributions */
struct PageRankStats *pageRankPullFixedPoint32BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:1635-1811 -- pull, 16-bit fixed-point contributions */
struct PageRankStats *pageRankPullFixedPoint16BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:1813-1990 -- pull, 8-bit fixed-point contributions */
struct PageRankStats *pageRankPullFixedPoint8BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:1992-2117 -- push, 64-bit fixed-point contributions */
struct PageRankStats *pageRankPushFixedPointGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2119-2303 -- pull, 32-bit quantised contributions */
struct PageRankStats *pageRankPullQuant32BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2305-2489 -- pull, 16-bit quantised contributions */
struct PageRankStats *pageRankPullQuant16BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2491-2676 -- pull, 8-bit quantised contributions */
struct PageRankStats *pageRankPullQuant8BitGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2678-2808 -- push, 32-bit quantised contributions */
struct PageRankStats *pageRankPushQuantGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2810-2969 -- data-driven (worklist) pull */
struct PageRankStats *pageRankDataDrivenPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:2971-3126 -- data-driven push (residuals) */
struct PageRankStats *pageRankDataDrivenPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.c:3128-3325 -- data-driven pull-push (residuals) */
struct PageRankStats *pageRankDataDrivenPullPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);

#ifdef __cplusplus
}
#endif

#endif /* PAGERANK_H */
