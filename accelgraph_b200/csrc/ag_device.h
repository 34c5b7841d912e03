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
 *   hub_cnt[H]     uint32  arrival counters of split rows
 *   ctl            AgControl  iteration state read and written on the device
 */
#ifndef AG_DEVICE_H
#define AG_DEVICE_H

#include <cuda_runtime.h>
#include <stdint.h>

/* ---------------------------------------------------------- tiling */
#define AG_BLK 256        /* threads per CTA of the pull kernel             */
#define AG_CAP 2048       /* in-edges staged in shared memory per row block */
#define AG_RMAX 1024      /* rows per row block                             */
#define AG_TSEQ 32        /* FAST order: rows up to this length summed by
                             one thread in stream order                     */
#define AG_HUB 8192       /* rows longer than this are split into chunks of
                             AG_HUB in-edges processed by separate CTAs     */
#define AG_LONG_MAX 64    /* rows longer than AG_TSEQ inside one row block  */

/* task kinds (low 2 bits of task.x) */
#define AG_T_BLOCK 0u     /* y = first row, z = end row                     */
#define AG_T_ROW 1u       /* y = row (AG_CAP < degree <= AG_HUB, or any
                             degree > AG_CAP in EXACT order)                */
#define AG_T_HUB 2u       /* x >> 2 = chunk, y = row, z = partial base,
                             w = number of chunks                           */

#define AG_MODE_PR 0
#define AG_MODE_SPMV 1

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
    float *c32_0, *c32_1;
    uint16_t *c16_0, *c16_1;
    float *hub_part;
    uint32_t *hub_cnt;
    AgControl *ctl;
    const AgRunConfig *cfg;
    const float *init_ranks;
    float base, damp;
    int wmode;             /* AG_SPMV_W_* */
    cudaGraphConditionalHandle cond;
} AgPullParams;

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel selection (prec: 0 fp32, 1 bf16, 2 fp16; exact: stream-order sums) */
const void *ag_pull_kernel_ptr(int mode, int prec, int exact);
const void *ag_init_kernel_ptr(int prec);
const void *ag_normalize_kernel_ptr(void);
cudaError_t ag_validate_ids(const uint32_t *ids, uint64_t E, uint32_t N, uint32_t *flag, cudaStream_t s);
cudaError_t ag_pr_f64_run(const uint32_t *row_off, const uint32_t *ids, const uint32_t *outdeg, uint32_t N,
                          uint32_t max_iter, double tol, double *r, double *r2, double *c, double *maxdiff,
                          uint32_t *passes_out, cudaStream_t s);

#ifdef __cplusplus
}
#endif

#endif /* AG_DEVICE_H */
