/*
 * ag_internal.h -- declarations shared by the host C sources and the CUDA
 * runtime of libaccelgraph_b200.so.  Not part of the public ABI.
 */
#ifndef AG_INTERNAL_H
#define AG_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "accelgraph_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* formatted detail for ag_last_error(); returns `status` for chaining */
ag_status_t ag_set_error(ag_status_t status, const char *fmt, ...);
void ag_clear_error(void);

/* host allocation used for graph arrays: page-locked when `pinned` is
 * requested and a device is usable, plain malloc otherwise.  *got_pinned
 * tells the matching free which allocator was used. */
void *ag_rt_host_alloc(size_t bytes, int pinned, int *got_pinned);
void ag_rt_host_free(void *ptr, int pinned);

/* an empty host graph of the builder's layout (all arrays allocated, page-
 * locked when requested); NULL on allocation failure */
struct GraphCSR *ag_host_graph_new(uint32_t N, uint32_t E, int weighted, int pinned);

/* wall clock in seconds (CLOCK_MONOTONIC) */
double ag_wall_seconds(void);

/* SpMV iterations on host vectors: x is copied once, every iteration
 * recomputes y on the device (timed per iteration with events), y is copied
 * back at the end.  iter_seconds (may be NULL) receives one entry per
 * iteration. */
ag_status_t ag_spmv_run_host(ag_graph_t g, const float *x, float *y, uint32_t iterations, uint32_t mode,
                             double *iter_seconds);

#ifdef __cplusplus
}
#endif

#endif /* AG_INTERNAL_H */
