/*
 * graphConfig.h -- run configuration passed to every algorithm entry point.
 *
 * Replaces: 02_capi_graph/include/config/graphConfig.h:7-52 (struct Arguments,
 * WEIGHTED, DIRECTED).  Field names, order and types follow that header so a
 * caller written against the reference compiles unchanged.  The reference
 * pulls `mt19937state` from OpenGraph's mt19937.h, which is not part of the
 * reference checkout; this header defines a state of the classic MT19937 shape
 * (624 words + index) in its place.  Binary layout compatibility with an
 * OpenGraph build is therefore not claimed, only source compatibility.
 *
 * Fields read by the B200 path (everything else is carried, never read):
 *   iterations      -- iteration cap (reference default 20, accel-graph.c:295)
 *   epsilon         -- per-vertex convergence threshold (default 1e-4, :297)
 *   pushpull        -- direction/precision selector (0 = pull FP32)
 *   ker_numThreads  -- reference CU count; on the GPU an optional SM cap
 *                      (0 or negative = all SMs)
 *   verbosity       -- 0 prints the reference's tables; see AG_QUIET in
 *                      accelgraph_b200.h for silencing them
 */
#ifndef GRAPHCONFIG_H
#define GRAPHCONFIG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Compile-time graph semantics of the reference build (graphConfig.h:7-8). */
#ifndef WEIGHTED
#define WEIGHTED 0
#endif
#ifndef DIRECTED
#define DIRECTED 1
#endif

#ifndef AG_MT19937_STATE_DEFINED
#define AG_MT19937_STATE_DEFINED
typedef struct mt19937state
{
    uint32_t mt[624];
    int32_t mti;
} mt19937state;
#endif

struct Arguments
{
    int wflag;
    int xflag;
    int sflag;
    int Sflag;
    int dflag;
    uint32_t binSize;
    uint32_t verbosity;
    uint32_t iterations;
    uint32_t trials;
    double epsilon;
    int source;
    uint32_t algorithm;
    uint32_t datastructure;
    uint32_t pushpull;
    uint32_t sort;
    uint32_t lmode;
    uint32_t lmode_l2;
    uint32_t lmode_l3;
    uint32_t mmode;
    uint32_t symmetric;
    uint32_t weighted;
    uint32_t delta;
    int pre_numThreads;
    int algo_numThreads;
    int ker_numThreads;
    char *fnameb;
    char *fnamel;
    uint32_t fnameb_format;
    uint32_t convert_format;
    mt19937state mt19937var;
    uint32_t cache_size;

    /* CAPI integration (carried for source compatibility; unused on the GPU) */
    uint64_t afu_config;
    uint64_t afu_config_2;
    uint64_t cu_config;
    uint64_t cu_config_2;
    uint64_t cu_config_3;
    uint64_t cu_config_4;
};

#ifdef __cplusplus
}
#endif

#endif /* GRAPHCONFIG_H */
