/*
 * accelgraph_b200.h -- extended C ABI of the B200 pull PageRank / SpMV library.
 *
 * The reference-compatible symbols (pageRankPullGraphCSR, SPMVPullGraphCSR,
 * ...) are declared in pageRank.h and SPMV.h.  This header adds:
 *   - status-returning entry points that never exit the process
 *     (the reference's legacy calls exit on a device failure,
 *     02_capi_graph/src/capi_utils/capienv.c:113-131);
 *   - a device-resident graph handle, so repeated runs skip the upload that
 *     the reference's coherent CAPI memory never needed (capienv.c:832-874
 *     maps the same arrays into the accelerator's address space);
 *   - the host graph substrate the reference takes from OpenGraph (edge-list
 *     to CSR / inverse CSR, seeded RMAT and Erdos-Renyi generators, the 8-byte
 *     binary edge-list reader) -- OpenGraph is absent from the reference
 *     checkout, so these restate its documented behaviour (-k: drop self loops
 *     and duplicates and sort, accel-graph.c:142-145,336-337).
 * All pointers are plain host or device pointers; no library types from any
 * framework appear in the signatures.  The CSR entry points (pageRank.h,
 * SPMV.h, ag_pagerank_pull_ex, ag_spmv_pull_ex, ag_graph_forget) serialise
 * callers from several host threads behind one lock; the handle API below is
 * called from one host thread at a time (the reference is not re-entrant
 * either, capienv.c:35-36).
 */
#ifndef ACCELGRAPH_B200_H
#define ACCELGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#include "graphConfig.h"
#include "graphCSR.h"
#include "pageRank.h"
#include "SPMV.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef int32_t ag_status_t;
#define AG_OK                  0
#define AG_ERR_INVALID_ARG    -1  /* bad argument (NULL, size out of range)      */
#define AG_ERR_INVALID_GRAPH  -2  /* malformed CSR found by the host or device    */
#define AG_ERR_CUDA           -3  /* a CUDA call failed; see ag_last_error()      */
#define AG_ERR_OOM            -4  /* host or device allocation failed             */
#define AG_ERR_TIMEOUT        -5  /* a bounded host wait ran out                  */
#define AG_ERR_NO_DEVICE      -6  /* no usable CUDA device                        */
#define AG_ERR_UNSUPPORTED    -7  /* option not available for this input          */
#define AG_ERR_DEVICE_WAIT    -8  /* a bounded wait inside a kernel ran out (the
                                     solve still finished; its results are
                                     returned, but the device was not answering
                                     in time)                                     */

const char *ag_status_string(ag_status_t status);
/* Detail of the most recent failure of this thread's last call ("" if none). */
const char *ag_last_error(void);
/* Library version string, e.g. "accelgraph-b200 0.1 sm_100a". */
const char *ag_version(void);

/* ------------------------------------------------------------ device set-up */
/* Select the CUDA device for this process's library context.  Optional: the
 * first call that needs a device uses the current device.  */
ag_status_t ag_init(int device);
/* The cudaStream_t (as void*) every launch of this library goes to. */
void *ag_stream(void);
/* Make every later launch of this library go to the caller's stream (NULL:
 * back to the library's own); waits for work already queued.  The library's
 * own stream is non-blocking: it does not wait for work on the legacy
 * default stream, whose handle is also NULL, so a caller that orders its
 * own work against the library's passes a stream it created. */
ag_status_t ag_set_stream(void *stream);
/* Wait for the library stream, polling with a deadline (seconds; <=0 means
 * the AG_WAIT_TIMEOUT_S environment variable, default 600).  Returns
 * AG_ERR_TIMEOUT when the deadline passes with work still queued. */
ag_status_t ag_synchronize(double timeout_s);
/* Number of streaming multiprocessors of the library's device (0 if none). */
int ag_num_sms(void);

/* ------------------------------------------------- host graph substrate */
#define AG_BUILD_DEDUPE   1u  /* drop self loops and duplicate edges; implies SORT */
#define AG_BUILD_SORT     2u  /* rows ordered by neighbour id (radix sort)       */
#define AG_BUILD_PINNED   4u  /* page-locked host arrays (faster uploads)        */
#define AG_BUILD_WEIGHTS  8u  /* generators: attach weights uniform in [0,1)     */
#define AG_BUILD_SYMMETRIC 16u /* add the reverse of every edge (reference -s),
                                  appended after the input edges             */

/* Build forward and inverse CSR from an edge list (src[i] -> dst[i]).
 * Without SORT, rows keep the input order of their edges (stable counting
 * sort by source, then a stable one by destination for the inverse).
 * weight may be NULL.  Returns NULL on failure (see ag_last_error()). */
struct GraphCSR *ag_graph_from_edges(uint32_t num_vertices, uint64_t num_edges,
                                     const uint32_t *src, const uint32_t *dst,
                                     const float *weight, uint32_t flags);
/* Seeded R-MAT (Graph500 quadrant recursion, no noise, no relabelling):
 * 2^scale vertices, edge_factor * 2^scale generated edges, quadrant
 * probabilities a, b, c (d = 1-a-b-c).  Weights, when requested, are
 * uniform in [0,1) drawn per forward edge from seed + 1. */
struct GraphCSR *ag_graph_rmat(uint32_t scale, uint32_t edge_factor,
                               double a, double b, double c,
                               uint64_t seed, uint32_t flags);
/* Seeded directed Erdos-Renyi: num_vertices * avg_degree edges with
 * independent uniform endpoints. */
struct GraphCSR *ag_graph_er(uint32_t num_vertices, uint32_t avg_degree,
                             uint64_t seed, uint32_t flags);
/* The same CSR as ag_graph_from_edges (bit for bit, same flags), built on
 * the GPU by device radix sorts and copied back to a host graph (free it
 * with ag_graph_free).  src, dst and weight may be host (pageable or
 * page-locked) or device arrays; num_edges < 2^31, num_vertices <= 2^30.
 * Replaces OpenGraph's CSR construction, which the reference calls from
 * 02_capi_graph/src/main/accel-graph.c:345 (generateGraphDataStructure). */
struct GraphCSR *ag_graph_build_csr(uint32_t num_vertices, uint64_t num_edges,
                                    const uint32_t *src, const uint32_t *dst,
                                    const float *weight, uint32_t flags);
struct ag_graph_s;
/* Edge list straight to a device graph (ag_graph_t): the CSR is built on the
 * GPU as ag_graph_build_csr builds it and stays there; upload_flags as for
 * ag_graph_upload.  No host CSR is made. */
ag_status_t ag_graph_build(uint32_t num_vertices, uint64_t num_edges, const uint32_t *src,
                           const uint32_t *dst, const float *weight, uint32_t build_flags,
                           uint32_t upload_flags, struct ag_graph_s **out);
/* Binary edge list: 8 bytes per edge (uint32 src, uint32 dst), or 12 bytes
 * (..., float weight) when weighted != 0.  num_vertices = max id + 1. */
struct GraphCSR *ag_graph_read_edge_file(const char *path, int weighted, uint32_t flags);

/* Graph files, in the reference's -z / -c format codes
 * (02_capi_graph/src/main/accel-graph.c:50-53,114-117):
 *   AG_FILE_TEXT      text edge list: one edge per line, "src dst" or
 *                     "src dst weight", any blanks between fields; empty lines
 *                     and lines starting with '#' or '%' are skipped
 *   AG_FILE_BINARY    binary edge list (ag_graph_read_edge_file's format)
 *   AG_FILE_CSR       serialised CSR written by ag_graph_write: every array of
 *                     the GraphCSR, so a read skips the build (this library's
 *                     own layout; OpenGraph's is not part of the reference)
 * Edge-list reads build with `flags` (num_vertices = largest id + 1); a CSR
 * read ignores them (only AG_BUILD_PINNED applies). */
#define AG_FILE_TEXT   0
#define AG_FILE_BINARY 1
#define AG_FILE_CSR    2
struct GraphCSR *ag_graph_read(const char *path, int format, int weighted, uint32_t flags);
/* Write a graph in one of the formats above (edge lists hold the forward
 * edges in CSR order, with weights when the graph has them). */
ag_status_t ag_graph_write(const struct GraphCSR *graph, const char *path, int format);
/* Free a graph returned by one of the builders above. */
void ag_graph_free(struct GraphCSR *graph);
/* n values uniform in [0,1) from the library's counter-based generator. */
void ag_fill_uniform(float *out, uint64_t n, uint64_t seed);

/* ------------------------------------------------- device-resident graph */
typedef struct ag_graph_s *ag_graph_t;

#define AG_UPLOAD_WEIGHTS  1u  /* also upload inverse edge weights (SpMV)    */
#define AG_UPLOAD_VALIDATE 2u  /* kept for clarity: the check is the default  */
#define AG_UPLOAD_TRUSTED  4u  /* skip the device check that every in-edge
                                  names a vertex < num_vertices (the caller
                                  guarantees it); without this flag a bad id
                                  makes the upload fail with
                                  AG_ERR_INVALID_GRAPH before any kernel
                                  reads through it                          */
#define AG_UPLOAD_KEEP_ORDER 8u  /* keep the caller's vertex order on the
                                    device (default: relabel by descending
                                    out-degree so the most-gathered
                                    contributions are contiguous)           */
#define AG_UPLOAD_NO_SMEM_CACHE 16u /* serve every gather from global memory
                                    (default: the most-gathered values are
                                    copied into shared memory each pass)    */

typedef struct ag_graph_info
{
    uint32_t num_vertices;
    uint32_t num_edges;
    uint32_t num_tasks;      /* work items of the fused pull kernel           */
    uint32_t num_hub_rows;   /* rows split across several CTAs                */
    uint32_t grid;           /* persistent CTAs per launch                    */
    uint32_t max_in_degree;
    uint64_t device_bytes;   /* device memory held by the handle              */
} ag_graph_info;

/* Work-list and cache shape of a device graph (see ag_autotune). */
typedef struct ag_tile_config
{
    uint32_t task_edges;   /* in-edges per warp item of consecutive rows (32..256) */
    uint32_t hub_chunk;    /* in-edges per warp for rows split across warps        */
    uint32_t hot_entries;  /* contributions kept in shared memory per pass          */
    uint32_t warm_entries; /* contributions below this id may take L1 lines        */
} ag_tile_config;

/* Copy the inverse CSR (and forward out-degrees) of `graph` to the device
 * and plan the kernel work list.  The handle stays valid until released;
 * the host graph may be freed after the call returns. */
ag_status_t ag_graph_upload(const struct GraphCSR *graph, uint32_t flags, ag_graph_t *out);
ag_status_t ag_graph_release(ag_graph_t g);
/* Device copies kept between calls.  With ag_pr_opts.keep_graph (or the
 * environment variable AG_KEEP_GRAPH=1, which also covers the reference entry
 * points of pageRank.h and SPMV.h), the CSR entry points keep the upload of
 * a GraphCSR (copy, relabelling, work-list plan) in a table of 8 entries,
 * least recently used first out, and a later call reuses it when the
 * GraphCSR address, its vertex and edge counts, the addresses of the arrays
 * the upload reads and the upload flags all match.  A caller that changes
 * the arrays in place, or frees the GraphCSR, calls ag_graph_forget(graph)
 * first; NULL forgets every kept graph.  A failed solve forgets its graph. */
ag_status_t ag_graph_forget(const struct GraphCSR *graph);
ag_status_t ag_graph_get_info(ag_graph_t g, ag_graph_info *info);
ag_status_t ag_graph_get_tiles(ag_graph_t g, ag_tile_config *cfg);
/* Copy a work list of the pull kernel (exact = 0: FAST order, 1: EXACT
 * order) into `items` as 4 words per item (kind << 30 | first row, end row
 * or hub slot, first in-edge, end in-edge), in device row numbering;
 * *count receives the list's length.  At most `capacity` items are copied
 * (items may be NULL with capacity 0 to ask for the length). */
ag_status_t ag_graph_get_tasks(ag_graph_t g, int exact, uint32_t *items, uint32_t capacity, uint32_t *count);
/* Re-plan the work list for another tile shape (results are unchanged in
 * EXACT order; FAST-order sums of rows split differently may differ in the
 * last bits). */
ag_status_t ag_graph_set_tiles(ag_graph_t g, const ag_tile_config *cfg);
/* Autotuner: time each candidate tile shape for `passes` pull passes on this
 * graph and keep the fastest; *best and *best_pass_us (may be NULL) receive
 * it.  AG_TUNE_CACHE names an optional cache file of earlier results. */
ag_status_t ag_autotune(ag_graph_t g, uint32_t passes, ag_tile_config *best, double *best_pass_us);

/* --------------------------------------------------------------- PageRank */
#define AG_PREC_FP32 0   /* contributions stored in binary32 (reference)     */
#define AG_PREC_BF16 1   /* contributions stored in bfloat16, FP32 accumulate */
#define AG_PREC_FP16 2   /* contributions stored in binary16, FP32 accumulate */
#define AG_PREC_FIXED64 3 /* the reference's 64-bit fixed-point pull (pushpull
                             2, pageRank.c:1276-1453): contributions converted
                             to fixed point with 32 fractional bits
                             (truncating), rows summed as integers modulo
                             2^64, the update formed in binary64; both orders
                             give the same bits */
/* The reference's narrow integer pulls (pageRank.c:1455-1991 fixed point,
 * :2119-2677 quantised; dispatched by pageRankGraphCSR on pushpull 9, 10, 11,
 * 4, 12, 13).  Contributions are stored in W bits, rows summed as integers
 * zero-extended into 64 bits, the update formed in binary32; both orders give
 * the same bits.  Fixed point: W/2 fractional bits (Q16.16, Q8.8, Q4.4),
 * conversion truncating.  Quantised: per pass, scale = (max - min) / (2^W - 1)
 * over all contributions, q = round-half-even(c / scale) clamped to
 * [0, 2^W - 1], r' = base + damp * (scale * sum). */
#define AG_PREC_FIXED32 4
#define AG_PREC_FIXED16 5
#define AG_PREC_FIXED8  6
#define AG_PREC_QUANT32 7
#define AG_PREC_QUANT16 8
#define AG_PREC_QUANT8  9

/* Direction of a solve.  The push and residual forms (pageRank.c:1111-1272,
 * 1992-2118, 2678-2809, 2971-3325) add along forward edges with atomic adds,
 * as the reference's threads do.  The 64-bit fixed-point push is exact and
 * equals the fixed-point pull; the binary32 pushes sum in binary64 (rounded
 * once to binary32), so they differ from a sequential binary32 sum in the
 * last bits; the residual forms' worklists depend on the interleaving. */
#define AG_DIR_PULL      0
#define AG_DIR_PUSH      1
#define AG_DIR_PULL_PUSH 2

#define AG_ORDER_FAST  0 /* rows of <= 32 in-edges summed in stream order,
                            longer rows by a fixed lane-strided tree: ranks
                            within 1e-5 relative L1 of the reference's, the
                            stopping pass not guaranteed equal               */
#define AG_ORDER_EXACT 1 /* every row summed in stream order: bit-identical
                            to a sequential binary32 loop, so ranks, active
                            counts and iterations are the reference's.  The
                            default of ag_pr_opts_init and of the reference
                            entry points (pageRank.h)                         */

typedef struct ag_pr_opts
{
    uint32_t struct_size;      /* sizeof(ag_pr_opts)                          */
    int32_t precision;         /* AG_PREC_*                                   */
    int32_t order;             /* AG_ORDER_*                                  */
    int32_t quiet;             /* nonzero: print no tables                    */
    double switch_residual;    /* low-precision forms switch to FP32 storage
                                  once a pass's error_total falls below this
                                  (<= 0: 1e-4), or when the residual stops
                                  falling                                     */
    const float *init_ranks;   /* warm start: num_vertices un-normalised ranks
                                  in caller order; NULL = base_pr everywhere  */
    int32_t init_on_device;    /* nonzero: init_ranks is a device pointer     */
    int32_t data_driven;       /* nonzero: data-driven (worklist) pull, the
                                  reference's pushpull 6 (pageRank.c:2810-2969):
                                  only vertices on the worklist are recomputed,
                                  a rank is replaced only when it moves by at
                                  least epsilon, which activates its
                                  out-neighbours; FP32, one graph              */
    int32_t direction;         /* AG_DIR_*: AG_DIR_PUSH runs the push forms
                                  (pushpull 1, 3, 5 with precision FP32,
                                  FIXED64, QUANT32; with data_driven the
                                  data-driven push, pushpull 7), AG_DIR_PULL_PUSH
                                  the data-driven pull-push (pushpull 8)      */
    int32_t keep_graph;        /* nonzero: ag_pagerank_pull_ex keeps the
                                  device copy of `graph` after the call and a
                                  later call on the same GraphCSR reuses it
                                  (see ag_graph_forget); 0: upload per call,
                                  as the reference maps the arrays per call  */
} ag_pr_opts;

typedef struct ag_pr_result
{
    uint32_t iterations;       /* reference semantics (see pageRank.h)        */
    uint32_t passes;           /* pull passes executed                        */
    uint32_t converged;        /* 1 if a pass had no active vertex            */
    uint32_t active_last;      /* active vertices of the last pass            */
    uint32_t switch_pass;      /* first pass that read FP32 contributions
                                  (low-precision forms; 0 for FP32)           */
    uint32_t reserved;
    double error_total;        /* last pass's mean |r' - r|                   */
    double rank_sum;           /* sum of normalised ranks (FP64)              */
    double device_ms;          /* device time of the solve                    */
} ag_pr_result;

/* Defaults: FP32, EXACT order (the reference's results bit for bit), no warm
 * start, pull, topology-driven, tables printed, switch_residual 1e-4. */
void ag_pr_opts_init(ag_pr_opts *opts);

/* Fixed-point gather on a device graph: y[v] = sum of x[u] over v's in-edges,
 * as 64-bit integers modulo 2^64 (0 for a vertex without in-edges), x and y in
 * caller vertex order, host memory.  The arithmetic of the reference's
 * FixedPoint compute unit (cu_PageRank/CSR/PULL/FixedPoint; testbench contract
 * pagerank_kernel_tb.sv:13-16). */
ag_status_t ag_gather_u64(struct ag_graph_s *g, const uint64_t *x, uint64_t *y);
/* Integer gather of 8-, 16-, 32- or 64-bit elements (elem_bytes 1, 2, 4, 8):
 * y[v] = sum of x[u] over v's in-edges, each element zero-extended, as 64-bit
 * integers modulo 2^64 (0 without in-edges); x and y in caller vertex order,
 * host memory.  The Quantized compute unit's arithmetic for 4-byte elements
 * (cu_PageRank/CSR/PULL/Quantized; testbench contract
 * pagerank_kernel_tb.sv:17-19). */
ag_status_t ag_gather_uint(struct ag_graph_s *g, const void *x, uint32_t elem_bytes, uint64_t *y);

/* Status-returning form of pageRankPullGraphCSR with the precision, order and
 * warm-start options.  *out receives a stats object owned by the caller. */
ag_status_t ag_pagerank_pull_ex(const struct Arguments *arguments, const struct GraphCSR *graph,
                                const ag_pr_opts *opts, struct PageRankStats **out);

/* Device-resident solve: enqueue init, the iteration loop (one CUDA graph with
 * an on-device convergence test) and normalisation on ag_stream().  Returns
 * without waiting.  Results stay in the handle until the next launch. */
ag_status_t ag_pagerank_launch(ag_graph_t g, uint32_t max_iterations, double epsilon,
                               const ag_pr_opts *opts);
/* Wait for the last launch and copy its results.  ranks: host array of
 * num_vertices normalised ranks, or NULL.  history arrays (host, may be NULL)
 * receive per-pass active counts, error totals and device seconds for up to
 * history_len passes. */
ag_status_t ag_pagerank_fetch(ag_graph_t g, float *ranks, ag_pr_result *result,
                              uint32_t *hist_active, double *hist_error,
                              double *hist_seconds, uint32_t history_len);
/* Device pointer to the normalised ranks of the last launch (valid until the
 * next launch on the handle). */
const float *ag_pagerank_device_ranks(ag_graph_t g);

/* FP64 oracle on the GPU: every operation in binary64 (contribution,
 * gather, update), iterated until max |r' - r| <= tol or max_iterations.
 * ranks (host, num_vertices) receives normalised FP64 ranks. */
ag_status_t ag_pagerank_f64(ag_graph_t g, uint32_t max_iterations, double tol,
                            double *ranks, uint32_t *passes);

/* --------------------------------------------- many independent graphs */
/* Upload `count` graphs as one block-diagonal union (vertex ids of graph i
 * follow those of graph i-1).  ag_pagerank_launch on the handle then solves
 * every graph in the same CUDA-graph launch: one pass covers all graphs still
 * running, each graph stops on its own convergence test or at the iteration
 * cap, and its items are skipped afterwards; ag_pagerank_fetch's ranks are
 * each graph's ranks normalised by its own vertex count, concatenated. */
ag_status_t ag_multigraph_upload(const struct GraphCSR *const *graphs, uint32_t count, uint32_t flags,
                                 ag_graph_t *out);
/* Per-graph results of the last launch on a union (arrays of `count`
 * entries, each may be NULL): iterations (reference semantics), passes,
 * converged flags, last-pass error totals; device_ms for the whole launch. */
ag_status_t ag_multigraph_fetch(ag_graph_t g, float *ranks, uint32_t *iterations, uint32_t *passes,
                                uint32_t *converged, double *error_total, double *device_ms);

/* ------------------------------------------------- row-partitioned solves */
/* One GPU's share of a PageRank solve over several GPUs: the caller's rows
 * are cut into nranks contiguous ranges bounds[r] .. bounds[r+1] (bounds has
 * nranks + 1 entries, from 0 to num_vertices; every range at most `slice`
 * rows), and vertex u of range r is addressed as r * slice + (u - bounds[r])
 * in the contribution vector of nranks * slice floats that every rank holds
 * in full.  Each pass reads that vector and writes this rank's slice of the
 * next one; the caller all-gathers the slices (e.g. NCCL) and all-reduces the
 * pass statistics between passes.  Row sums are those of a one-GPU solve. */
ag_status_t ag_graph_upload_rows(const struct GraphCSR *graph, const uint32_t *bounds, uint32_t nranks,
                                 uint32_t rank, uint32_t slice, uint32_t flags, ag_graph_t *out);
/* ranks start at base_pr; writes this rank's first contributions into its
 * slice of c_full (device) */
ag_status_t ag_partition_init(ag_graph_t g, float *c_full);
/* one pass (FAST order); stats_dev (device, 2 doubles) receives this rank's
 * active count and sum of |r' - r| */
ag_status_t ag_partition_pass(ag_graph_t g, const float *c_in_full, float *c_out_full, double epsilon,
                              double *stats_dev);
/* A solve whose loop needs no host round trip per pass.  state_dev (device,
 * 3 uint32: stop, passes, converged; zeroed by the caller before the solve)
 * is shared by the two calls:
 *  - ag_partition_step: one pass in `order` (AG_ORDER_*), the same as
 *    ag_partition_pass, except that once state_dev[0] is set the pass does
 *    nothing and stats_dev is {0, 0};
 *  - ag_partition_close, after the caller's all-reduce of stats_dev: counts
 *    the pass, keeps its error sum in err_dev (device double) and sets the stop
 *    flag when no vertex of any rank was active.
 * All ranks issue the same calls and collectives every pass; the host reads
 * state_dev when it wants to know whether to stop (every few passes). */
ag_status_t ag_partition_step(ag_graph_t g, const float *c_in_full, float *c_out_full, double epsilon,
                              int32_t order, double *stats_dev, const uint32_t *state_dev);
ag_status_t ag_partition_close(const double *stats_dev, uint32_t *state_dev, double *err_dev);
/* this rank's ranks / num_vertices (host array of bounds[r+1] - bounds[r]) */
ag_status_t ag_partition_fetch(ag_graph_t g, float *ranks_local);

/* ------------------------------------------------- batched personalized PR */
/* Personalized PageRank of k <= 64 source vertices (caller ids) solved
 * together: one pass is one sparse x dense (N x 64) product.  Column i
 * teleports to sources[i] with mass (1 - 0.85) * N (the reference's
 * un-normalised scale, so epsilon keeps its meaning); the loop stops when no
 * (vertex, column) pair changes by >= epsilon, or after max_iterations.
 * ranks (host, may be NULL) receives num_vertices x k binary32 values r / N,
 * row-major in caller vertex order.  result->error_total is the mean
 * |r' - r| over all pairs of the last pass. */
ag_status_t ag_ppr_spmm(ag_graph_t g, const uint32_t *sources, uint32_t k, uint32_t max_iterations,
                        double epsilon, float *ranks, ag_pr_result *result);

/* ------------------------------------------------------- learned warm start */
/* A small MLP (8 -> 64 -> 64 -> 1, ReLU; bfloat16 weights, binary32
 * accumulation) that predicts log(un-normalised rank) from per-vertex degree
 * features, trained and run by this library's own kernels.  Its predictions
 * only choose the starting ranks: the solve still iterates to the same
 * epsilon, and uniform starting ranks remain the default. */
typedef struct ag_mlp_s *ag_mlp_t;
/* number of binary32 parameters: W1[64][8] b1[64] W2[64][64] b2[64] w3[64] b3 */
uint32_t ag_mlp_num_params(void);
ag_status_t ag_mlp_create(uint64_t seed, ag_mlp_t *out);
ag_status_t ag_mlp_release(ag_mlp_t m);
ag_status_t ag_mlp_set_params(ag_mlp_t m, const float *params);   /* host array */
ag_status_t ag_mlp_get_params(ag_mlp_t m, float *params);          /* host array */
/* Device array of num_vertices x 8 features in caller vertex order:
 * log1p of in-degree, out-degree, sum of in-neighbours' in-degrees, sum of
 * their out-degrees, min and max of their out-degrees, sum of their
 * 1/out-degree, max of their in-degrees. */
ag_status_t ag_features(ag_graph_t g, float *features);
/* Y[i] = MLP(X[i]) for n samples; X (n x 8) and Y (n) are device arrays.
 * The training forward pass: binary32 activations with the bfloat16 weights. */
ag_status_t ag_mlp_forward(ag_mlp_t m, const float *X, uint32_t n, float *Y);
/* The same prediction on the tensor cores (mma.sync bfloat16 operands,
 * binary32 accumulation; each feature and activation split into a bfloat16
 * head and tail): what the warm start uses.  Within about 1e-4 of
 * ag_mlp_forward in log-rank. */
ag_status_t ag_mlp_predict(ag_mlp_t m, const float *X, uint32_t n, float *Y);
/* Gradient of the mean squared error of MLP(X) against T (device arrays)
 * with respect to the parameters (host array of ag_mlp_num_params()
 * values, may be NULL) and the loss (may be NULL). */
ag_status_t ag_mlp_gradients(ag_mlp_t m, const float *X, const float *T, uint32_t n, float *grad, float *loss);
/* Adam on mini-batches of `batch` consecutive samples for `epochs` epochs
 * (the caller shuffles); *final_loss receives the last batch's loss. */
ag_status_t ag_mlp_train(ag_mlp_t m, const float *X, const float *T, uint32_t n, uint32_t epochs, uint32_t batch,
                         float lr, float *final_loss);
/* Predicted starting ranks for ag_pr_opts.init_ranks (host array of
 * num_vertices, caller order; never below 1 - damp). */
ag_status_t ag_mlp_warm_start(ag_graph_t g, ag_mlp_t m, float *init_ranks);
/* The same into a device array, enqueued on ag_stream() without waiting:
 * pass it on with ag_pr_opts.init_on_device = 1. */
ag_status_t ag_mlp_warm_start_device(ag_graph_t g, ag_mlp_t m, float *init_ranks_device);

/* ------------------------------------------------------------------- SpMV */
#define AG_SPMV_GRAPH_WEIGHTS 0u /* w = uploaded inverse weights (0.0001f if none) */
#define AG_SPMV_UNIT          1u /* pure gather: y[v] = sum x[u]                   */
#define AG_SPMV_EXACT         2u /* every row summed in stream order (bit-identical
                                    to a sequential binary32 loop)                */

/* y = A x over the inverse CSR on ag_stream(); x and y are device pointers of
 * num_vertices floats.  Rows without in-edges get y[v] = 0. */
ag_status_t ag_spmv_pull_device(ag_graph_t g, const float *x, float *y, uint32_t mode);
/* Host-pointer form: uploads x, runs, copies y back and waits. */
ag_status_t ag_spmv_pull(ag_graph_t g, const float *x, float *y, uint32_t mode);
/* SpMV pull that allocates nothing, for callers that may not allocate device
 * memory once running (a host framework that owns all device memory, or a
 * latency-critical path that cannot afford cudaMalloc's device-wide
 * synchronisation).  No counterpart in the reference: it has no device
 * memory of its own to manage.
 * Inputs and outputs are caller-owned DEVICE pointers: row_off[num_vertices+1]
 * (inverse-CSR row starts), ids[num_edges] (in-neighbours), w[num_edges] (or
 * NULL: the reference's unweighted 0.0001f), x and y[num_vertices]; mode is
 * AG_SPMV_GRAPH_WEIGHTS or AG_SPMV_UNIT (any other bit, AG_SPMV_EXACT
 * included, is rejected with AG_ERR_INVALID_ARG); stream is a cudaStream_t
 * (NULL: the legacy default stream).  The work is enqueued on that stream and
 * the call returns without waiting.
 * Limit: its only scratch is a fixed 256 KB device array listing the rows of
 * more than 4096 in-edges (at most 65536 of them), so num_edges must be at
 * most 2^28; larger inputs are rejected with AG_ERR_UNSUPPORTED.  Every GPU
 * that loads the library holds that array until the process exits.  The
 * first call on a device looks up the array's device address, so make it
 * before any stream capture; the address is kept for the process, so a call
 * after cudaDeviceReset is not supported.  All calls share the array: calls
 * whose work overlaps on the GPU race, so issue them on one stream. */
ag_status_t ag_spmv_pull_noalloc(uint32_t num_vertices, uint32_t num_edges, const uint32_t *row_off,
                                 const uint32_t *ids, const float *w, const float *x, float *y,
                                 uint32_t mode, void *stream);

/* Status-returning form of SPMVPullGraphCSR. */
ag_status_t ag_spmv_pull_ex(const struct Arguments *arguments, const struct GraphCSR *graph,
                            int quiet, struct SPMVStats **out);

#ifdef __cplusplus
}
#endif

#endif /* ACCELGRAPH_B200_H */
