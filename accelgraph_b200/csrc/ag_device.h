/*
 * ag_device.h -- device-side data layout shared by the CUDA sources.
 *
 * Layout of a graph in HBM (one ag_graph_s handle):
 *   row_off[N+1]   uint32  inverse-CSR row starts (contiguous rows)
 *   ids[E4]        uint32  in-neighbour ids, E rounded up to a multiple of 4
 *                          plus 4 zero words, 256-byte aligned, read as uint4
 *   w[E4]          float   inverse edge weights (SpMV only, same padding)
 *   outdeg[N]      uint32  forward out-degree (contribution divisor)
 *   tasks[T]       uint4   work list of the fused pull kernel
 *   rank[N]        float   un-normalised ranks, updated in place
 *   c32[2][N]      float   contribution ping-pong buffers
 *   c16[2][N]      16-bit  low-precision contribution buffers (precision form)
 *   hub_part[H]    float   per-chunk partial sums of split rows
 *   hub_cnt[H]     uint32  arrival counters of split rows, then 4 spare words
 *                          and the EXACT order's donor table (AG_STEAL_WORDS)
 *   hub_vals[H*C]  float   EXACT order: hub rows' gathered values (C = chunk)
 *   hub_pred[H]    uint32  EXACT order: each chunk's starting binade, last pass
 *   hub_t[H*64]    uint32  EXACT order: per-round integer step totals
 *   ctl            AgControl  iteration state read and written on the device
 */
#ifndef AG_DEVICE_H
#define AG_DEVICE_H

#include <cuda_runtime.h>
#include <stdint.h>

/* SMs of the library's device (ag_runtime.cu) */
extern "C" int ag_num_sms(void);

/* grid cap of a grid-stride kernel: `per_sm` CTAs on every SM of the device */
static inline unsigned ag_sm_grid(unsigned per_sm)
{
    const int n = ag_num_sms();
    return (unsigned)(n > 0 ? n : 1) * per_sm;
}

/* ---------------------------------------------------------- tiling */
#ifndef AG_BLK
#define AG_BLK 1024       /* threads per CTA of the pull kernel              */
#endif
#ifndef AG_CTAS_PER_SM
#define AG_CTAS_PER_SM 1  /* pull CTAs resident per SM; each holds its own
                             copy of the hot table                          */
#endif
#define AG_WARPS (AG_BLK / 32)
#define AG_SBLK 256       /* threads per CTA of the element-wise kernels     */
#ifndef AG_WCAP
#define AG_WCAP 256       /* in-edges staged in shared memory per warp task  */
#endif
#define AG_WROWS 32       /* rows per warp task (one per lane)              */
#define AG_TSEQ 32        /* FAST order: rows up to this length summed by
                             one lane in stream order                       */
#ifndef AG_WHUB
#define AG_WHUB 2048      /* rows longer than this are split into chunks of
                             AG_WHUB in-edges on separate warps (EXACT
                             order: the chunks stage their values and the
                             last one sums the row in stream order)         */
#endif
#if AG_WHUB % 32 != 0
#error "AG_WHUB must be a multiple of 32 (EXACT-order hub rows are read in 16-byte groups)"
#endif
#ifndef AG_STEAL_MIN
#define AG_STEAL_MIN 4096  /* EXACT order: the warp that composes a hub row of
                              at least this many in-edges gives the rest of
                              its work list away to warps that run out of
                              work (measured best of 2049 .. 32768 at R-MAT
                              s22 and s24, with AG_STEAL_CAP 4096)          */
#endif
#ifndef AG_STEAL_CAP
#define AG_STEAL_CAP 4096 /* donors per pass: above the number of rows of
                             AG_STEAL_MIN in-edges or more at R-MAT s24,
                             whose composers all give their lists away    */
#endif
#define AG_XWORDS 64      /* EXACT order: words per hub chunk of integer step
                             totals (two per 256-value round, the last word
                             the chunk's data-driven sign tag)              */
#define AG_XROUNDS 31     /* rounds of a chunk with step totals              */
#define AG_XNOT 0x80000000u /* a round's total that does not apply          */
#define AG_XFELL 0x100u   /* hub_pred: the chunk had a round summed one value
                             after another in the pass before              */
#ifndef AG_STEAL_PROBES
#define AG_STEAL_PROBES 8 /* donor entries a warp out of work tries          */
#endif
#define AG_STEAL_WORDS (2 + 2 * AG_STEAL_CAP)
#define AG_STAGE_BYTES (AG_WARPS * AG_WCAP * 4)
#if AG_CTAS_PER_SM == 1
#define AG_SMEM_MAX 232448 /* shared memory per CTA: the 227 KB maximum     */
#else
#define AG_SMEM_MAX (233472 / AG_CTAS_PER_SM - 1024)
#endif
#define AG_SMEM_STATIC 1024 /* static shared memory of the pull kernel (upper bound) */
#ifndef AG_HOT_CAP
#define AG_HOT_CAP 16384  /* default hot-table entries: a 64 KB table leaves
                             about 150 KB of the SM's unified L1/shared
                             memory to L1, which keeps the next tier of warm
                             contributions (measured best on R-MAT s20, s22) */
#endif
#ifndef AG_WARM_DEFAULT
#define AG_WARM_DEFAULT 65536 /* ids below this may allocate L1 lines      */
#endif
#define AG_HOT_FIT ((AG_SMEM_MAX - AG_SMEM_STATIC - AG_STAGE_BYTES) / 4 / 64 * 64)
#define AG_HOT_MAX AG_HOT_FIT
#define AG_BULK_CHUNK 32768u

/* A task is one warp's work item (uint4):
 *   x = kind << 30 | first row      y = end row (ROWS) or partial slot (HUB)
 *   z = first in-edge               w = end in-edge
 * ROWS: rows [x, y) holding <= AG_WCAP in-edges, at most AG_WROWS rows,
 *       each of degree <= AG_WCAP.
 * LONG: one row x with AG_WCAP < degree (<= AG_WHUB in FAST order).
 * HUB : in-edges [z, w) of row x; y = partial base (low 20 bits) |
 *       chunk index << 20.  The row's chunk count follows from its degree. */
#define AG_T_ROWS 0u
#define AG_T_LONG 1u
#define AG_T_HUB 2u
#define AG_ROW_MASK 0x3FFFFFFFu
#define AG_SLOT_BITS 20
#define AG_SLOT_MASK ((1u << AG_SLOT_BITS) - 1u)

#define AG_MODE_PR 0
#define AG_MODE_SPMV 1
#define AG_MODE_MULTI 2   /* PageRank over a union of independent graphs,
                             each with its own convergence                  */
#define AG_MODE_DD 3      /* data-driven PageRank: a rank is replaced only
                             when it moves by at least epsilon, and only rows
                             with a changed in-neighbour (or the first pass)
                             are updated; a change is signalled by the sign
                             bit of the contribution written                */

/* push-direction and residual forms (ag_push.cu) */
#define AG_PUSH_FLOAT 0    /* push, binary32 atomic adds                      */
#define AG_PUSH_FIXED 1    /* push, 64-bit fixed-point integer adds           */
#define AG_PUSH_QUANT 2    /* push, 32-bit quantised contributions            */
#define AG_PUSH_DD 3       /* data-driven push (residuals, worklist)          */
#define AG_PUSH_PULLPUSH 4 /* data-driven pull-push                           */
#define AG_NUM_PUSH_FORMS 5
#define AG_SPMV_W_GRAPH 0 /* multiply by the uploaded weight                */
#define AG_SPMV_W_CONST 1 /* multiply by 0.0001f (graph without weights)    */
#define AG_SPMV_W_UNIT 2  /* no multiply                                    */

#define AG_MAX_HISTORY 4096

typedef struct AgControl
{
    uint32_t iter;            /* passes completed                           */
    uint32_t max_iter;
    uint32_t active_acc;      /* active vertices of the running pass        */
    uint32_t done_ctas;       /* CTAs finished in the running pass          */
    double err_acc;           /* sum of |r' - r| of the running pass        */
    double eps;
    uint32_t converged;
    uint32_t mode_read;       /* 1: this pass reads 16-bit contributions    */
    uint32_t mode_write;      /* 1: this pass writes 16-bit contributions   */
    uint32_t switch_pass;     /* first pass that reads FP32 contributions   */
    double switch_residual;
    double prev_err;
    double rank_sum;          /* FP64 sum of the normalised ranks           */
    unsigned long long t0;    /* %globaltimer at the end of the init kernel */
    uint32_t use_init;        /* warm start from init_ranks                 */
    uint32_t low_passes;      /* passes that read 16-bit contributions      */
    uint32_t stop;            /* 1 once the loop is over (stream launches)  */
    uint32_t fault;           /* nonzero: a bounded device wait ran out     */
    double last_err_sum;      /* sum of |r' - r| of the last closed pass    */
    uint32_t hist_active[AG_MAX_HISTORY];
    double hist_err[AG_MAX_HISTORY];
    unsigned long long hist_t[AG_MAX_HISTORY];
} AgControl;

/* run configuration copied into AgControl by the init kernel */
typedef struct AgRunConfig
{
    uint32_t max_iter;
    uint32_t use_init;
    double eps;
    double switch_residual;
} AgRunConfig;

typedef struct AgPullParams
{
    const uint32_t *row_off;
    const uint32_t *ids;
    const float *w;
    const uint32_t *outdeg;
    const uint4 *tasks;
    uint32_t ntasks;
    uint32_t N;
    float *rank;           /* PR: ranks; SpMV: y                               */
    const float *x;        /* SpMV input                                       */
    uint32_t whub;         /* in-edges per hub chunk of this work list         */
    uint32_t c_base;       /* row r's contribution is written at c_base + r
                              (a rank's slice of a partitioned solve)          */
    uint32_t norm_n;       /* vertex count ranks are normalised by (0: N)      */
    float *c32_0, *c32_1;
    uint16_t *c16_0, *c16_1;
    float *hub_part;
    uint32_t *hub_cnt;
    float *hub_vals;       /* EXACT order: hub rows' gathered values, at chunk
                              slot x whub + offset in the row                  */
    uint32_t *hub_pred;    /* EXACT order, per hub chunk: the biased exponent
                              of the row's stream-order sum where the chunk
                              began in the pass before (0: unknown), and
                              AG_XFELL                                         */
    uint32_t *hub_t;       /* EXACT order, AG_XWORDS per hub chunk: for each
                              round of 256 in-edges, the sum of its integer
                              steps at that exponent and at the next one
                              (AG_XNOT: does not apply)                        */
    uint32_t *steal;       /* EXACT order, AG_STEAL_WORDS words: [0] donors
                              of this pass, [1] warps done with their items,
                              then per donor its first given item + 1 (0: not
                              yet published) and its claim counter; the last
                              warp done resets them                           */
    AgControl *ctl;
    const AgRunConfig *cfg;
    const float *init_ranks;
    float base, damp;
    int wmode;             /* AG_SPMV_W_* */
    uint32_t use_cond;     /* 1: launched by the CUDA graph's WHILE node      */
    uint32_t mbar_spins;   /* polls of the hot-table copy's mbarrier before the
                              wait counts as run out (ctl->fault)              */
    uint32_t hot_n;        /* contributions (ids < hot_n) served from shared
                              memory; a multiple of 64                         */
    uint32_t hot_n16;      /* entries of the same table in 16-bit passes       */
    uint32_t warm_n;       /* gathers of ids in [hot_n, warm_n) may take L1
                              lines; colder ones bypass L1                     */
    const uint32_t *perm;  /* device row i is caller vertex perm[i]            */
    const uint32_t *inv;   /* caller vertex v is device row inv[v]             */
    float *out;            /* normalised ranks in caller order                 */
    /* union of independent graphs (AG_MODE_MULTI) */
    const uint32_t *gstart; /* first row of each graph, ngraphs + 1 entries    */
    uint32_t ngraphs;
    uint32_t *g_active;    /* per graph: active vertices of the running pass   */
    double *g_err;         /* per graph: sum |r' - r| of the running pass      */
    uint32_t *g_done;      /* per graph: 1 once converged or capped            */
    uint32_t *g_passes;    /* per graph: passes run                            */
    uint32_t *g_conv;      /* per graph: 1 if a pass had no active vertex      */
    double *g_err_last;    /* per graph: error total of its last pass          */
    /* integer pulls (ag_fixed.cu): contribution buffers (64-bit, or W-bit
     * in their first N * W/8 bytes), hub partials, the quantised forms'
     * binary32 contributions and min/max key slots (mm[0..1] minimum keys,
     * mm[2..3] maximum keys, one of each per pass parity), and the vectors of
     * the plain gather (x of any width, y 64-bit) */
    uint64_t *c64_0, *c64_1;
    uint64_t *hub_part64;
    float *cqf;
    uint32_t *qmm;
    const uint64_t *x64;
    uint64_t *y64;
    /* push and residual forms (ag_push.cu): the forward edge list sorted by
     * source (device ids), two vertex vectors (contributions and next sums,
     * or seed and pull sums), residuals, per-vertex deltas and the two
     * worklists (2N bytes, one per pass parity) */
    const uint32_t *fwd_src, *fwd_dst;
    uint32_t E;
    uint32_t honor_stop;   /* SpMV launches inside a solve loop: return once
                              the loop has stopped (stream launches)         */
    float *pa, *pb, *res, *delta;
    uint8_t *wl;
    cudaGraphConditionalHandle cond;
} AgPullParams;

/* read-only view of a device graph for the other kernels of this library */
typedef struct AgGraphView
{
    const uint32_t *row_off, *ids, *outdeg, *perm, *inv;
    uint32_t N, E;
    cudaStream_t stream;
    const uint4 *tasks;  /* the pull kernel's FAST-order work list           */
    uint32_t ntasks;
    uint32_t hub_slots;  /* hub chunks in it (slot indexes of HUB items)     */
} AgGraphView;

/* device planner of the work lists (ag_plan.cu): hub chunks, long rows not
 * split, row items, split rows */
typedef struct AgPlanTotals
{
    uint32_t hub_items, long_items, row_items, hub_rows;
} AgPlanTotals;

typedef struct AgPlanState
{
    const uint32_t *row_off, *gstart;
    uint32_t n, cap, whub, ngraphs, nseg;
    void *scratch;
    uint32_t *scan;
} AgPlanState;

/* forward and inverse CSR in device memory, caller vertex order (ag_build.cu) */
typedef struct AgDevCSR
{
    uint32_t N, E;
    uint32_t *out_deg, *in_deg;   /* N                                       */
    uint32_t *fwd_idx, *inv_idx;  /* N + 1 row starts                        */
    uint32_t *fwd_src, *fwd_dst;  /* E, sorted by source                     */
    uint32_t *inv_src, *inv_dst;  /* E, sorted by destination: inv_src holds
                                     the row (destination), inv_dst the
                                     in-neighbour (source)                   */
    float *fwd_w, *inv_w;         /* E or NULL                               */
    float max_w;
    uint32_t max_in_degree;
} AgDevCSR;

#ifdef __cplusplus
extern "C" {
#endif

/* build both CSRs from a device edge list (m < 2^31 edges); a bad endpoint
 * returns cudaErrorInvalidValue with *bad_edge = its lowest edge index */
cudaError_t ag_csr_build_device(uint32_t n, uint32_t m, const uint32_t *src, const uint32_t *dst, const float *w,
                                uint32_t flags, AgDevCSR *out, uint32_t *bad_edge, cudaStream_t s);
void ag_csr_free_device(AgDevCSR *c, cudaStream_t s);


/* count items per segment and copy the four totals to totals_host (the copy
 * is stream-ordered: wait on the stream before reading them) */
cudaError_t ag_plan_count(const uint32_t *row_off, uint32_t n, uint32_t cap, uint32_t whub, const uint32_t *gstart,
                          uint32_t ngraphs, AgPlanState *ps, uint32_t *totals_host, cudaStream_t s);
/* write both lists (the same items: hub chunks, long rows, row items; the
 * kernel's order decides how each is summed) */
cudaError_t ag_plan_write(AgPlanState *ps, const uint32_t *totals, uint4 *fast, uint4 *exact, cudaStream_t s);
void ag_plan_release(AgPlanState *ps, cudaStream_t s);
cudaError_t ag_set_u32(uint32_t *p, uint32_t v, cudaStream_t s);

struct ag_graph_s;
int32_t ag_rt_graph_view(struct ag_graph_s *g, AgGraphView *v);

/* Kernel selection (prec: 0 fp32, 1 bf16, 2 fp16; exact: stream-order sums) */
const void *ag_pull_kernel_ptr(int mode, int prec, int exact);
const void *ag_init_kernel_ptr(int prec);
const void *ag_normalize_kernel_ptr(void);
/* integer pulls: contributions of `bytes` (8, 4, 2, 1) bytes, fixed point or
 * quantised; gather = 1: only the integer sums.  Their init kernel, the
 * quantised forms' element-wise quantiser, and the dynamic shared memory of
 * the pull kernels */
const void *ag_int_kernel_ptr(int bytes, int quant, int gather);
const void *ag_int_init_kernel_ptr(int bytes, int quant);
const void *ag_quant_kernel_ptr(int bytes);
size_t ag_fixed_smem_bytes(int bytes);
/* vectors of `bytes`-byte elements into device order (y[i] = x[perm[i]]) and
 * 64-bit sums back to caller order (y[v] = x[inv[v]]); a NULL map is the
 * identity */
cudaError_t ag_permute_uint_in(const uint32_t *perm, const void *x, void *y, uint32_t n, int bytes, cudaStream_t s);
cudaError_t ag_permute_u64_out(const uint32_t *inv, const uint64_t *x, uint64_t *y, uint32_t n, cudaStream_t s);
/* forward edge list from the device inverse CSR: (fwd_src, fwd_dst) sorted by
 * source, each source's destinations in row order */
cudaError_t ag_forward_build(const uint32_t *row_off, const uint32_t *ids, uint32_t n, uint32_t e,
                             uint32_t *fwd_src, uint32_t *fwd_dst, cudaStream_t s);
/* kernels of the push and residual forms (AG_PUSH_*): stage 0 init, 1 scatter
 * or vertex phase, 2 update or edge phase, 3 quantiser (AG_PUSH_QUANT) or
 * residual seed (AG_PUSH_DD, AG_PUSH_PULLPUSH) */
const void *ag_push_kernel_ptr(int kind, int stage);
/* CTA size and dynamic shared memory of the push scatter and of the residual
 * edge phase */
void ag_push_scatter_shape(unsigned *threads, size_t *smem);
cudaError_t ag_validate_ids(const uint32_t *ids, uint64_t E, uint32_t N, uint32_t *flag, cudaStream_t s);
cudaError_t ag_relabel_layout(const uint32_t *off_old, const uint32_t *outdeg_old, uint32_t n, uint32_t *perm,
                              uint32_t *inv, uint32_t *off_new, uint32_t *outdeg_new, cudaStream_t s);
cudaError_t ag_relabel_rows(const uint32_t *perm, const uint32_t *inv, const uint32_t *off_old, const uint32_t *off_new,
                            const uint32_t *ids_old, uint32_t *ids_new, const float *w_old, float *w_new, uint32_t n,
                            uint32_t e, cudaStream_t s);
cudaError_t ag_relabel_by_out_degree(const uint32_t *off_old, const uint32_t *ids_old, const float *w_old,
                                     const uint32_t *outdeg_old, uint32_t n, uint32_t e, uint32_t *perm,
                                     uint32_t *inv, uint32_t *off_new, uint32_t *ids_new, float *w_new,
                                     uint32_t *outdeg_new, cudaStream_t s);
cudaError_t ag_permute_in(const uint32_t *perm, const float *x, float *x_new, uint32_t n, cudaStream_t s);
cudaError_t ag_permute_out(const uint32_t *inv, const float *y_new, float *y, uint32_t n, cudaStream_t s);
cudaError_t ag_pr_f64_run(const uint32_t *row_off, const uint32_t *ids, const uint32_t *outdeg, uint32_t N,
                          uint32_t max_iter, double tol, double *r, double *r2, double *c, double *maxdiff,
                          uint32_t *passes_out, cudaStream_t s);

#ifdef __cplusplus
}
#endif

#endif /* AG_DEVICE_H */
