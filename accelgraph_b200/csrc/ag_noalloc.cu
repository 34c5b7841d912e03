/*
 * ag_noalloc.cu -- SpMV pull over a caller-owned inverse CSR with no device
 * allocation at all.
 *
 * Who needs it: callers that may not allocate device memory once they are
 * running.  Examples are a host framework that owns every byte of device
 * memory and hands out fixed buffers at start-up, and a latency-critical
 * path where a cudaMalloc (which can synchronise the whole device) is not
 * acceptable.  Such callers pass their own device buffers for every input
 * and output; the only scratch the product needs is the list of rows too
 * long for one warp, and that list lives in the fixed-size array below.
 *
 * Scratch: ag_noalloc_scratch, a file-scope __device__ array.  Every GPU that
 * loads this library holds it (AG_NOALLOC_SCRATCH_WORDS words, 256 KB plus a
 * header) until the process exits.  Word 0 counts the long rows, words from
 * AG_NOALLOC_HEADER on list them.  In host code the array's name only stands
 * for the symbol; the device address is obtained once per device with
 * cudaGetSymbolAddress on the first call made with that device current, so
 * that first call should come before any stream capture.  The address is kept
 * for the life of the process: a call after cudaDeviceReset (which unloads
 * the module) is not supported.  Every call shares the array and keeps the
 * previous call's contents: the count is cleared at the start of each call,
 * and two calls whose work overlaps on the GPU race on the list (issue them
 * on one stream, or serialise them).
 *
 * Work split: kernel 1 gives each row of <= AG_NOALLOC_SPLIT in-edges to one
 * warp (lane-strided partial sums, fixed xor tree) and appends every longer
 * row to the list; kernel 2 gives each listed row to one CTA (thread-strided
 * partials, fixed-order CTA reduction).  Results do not depend on the list
 * order.  A long row that finds the list full (only when the caller's
 * num_edges understates the graph) is summed by its warp in kernel 1 instead:
 * slower, never dropped.  Arithmetic per edge matches the pull kernel: one
 * binary32 multiply w * x[u] (no multiply in unit mode), then binary32 adds.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "ag_internal.h"

#define AG_NOALLOC_SPLIT 4096u          /* rows longer than this go to kernel 2    */
#define AG_NOALLOC_MAX_LONG 65536u      /* listed long rows (so E <= 2^28 always fits) */
#define AG_NOALLOC_HEADER 64u           /* words before the list (word 0: count)   */
#define AG_NOALLOC_SCRATCH_WORDS (AG_NOALLOC_HEADER + AG_NOALLOC_MAX_LONG)
#define AG_NOALLOC_BLK 256

static __device__ __align__(256) uint32_t ag_noalloc_scratch[AG_NOALLOC_SCRATCH_WORDS];

/* value of in-edge j with source u */
__device__ __forceinline__ float ag_na_term(const float *x, const float *w, uint32_t mode, uint32_t j, uint32_t u)
{
    const float xv = __ldg(x + u);
    if (mode & AG_SPMV_UNIT)
        return xv;
    return __fmul_rn(w ? __ldg(w + j) : 0.0001f, xv);
}

__device__ __forceinline__ float ag_na_warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void __launch_bounds__(AG_NOALLOC_BLK) ag_na_rows_kernel(uint32_t n, const uint32_t *row_off,
                                                                     const uint32_t *ids, const float *w,
                                                                     const float *x, float *y, uint32_t mode,
                                                                     uint32_t *scratch)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const uint32_t b = __ldg(row_off + r), e = __ldg(row_off + r + 1);
        if (e - b > AG_NOALLOC_SPLIT) {
            uint32_t k = 0;
            if (lane == 0) {
                k = atomicAdd(scratch, 1u);
                if (k < AG_NOALLOC_MAX_LONG)
                    scratch[AG_NOALLOC_HEADER + k] = r;
            }
            /* listed: kernel 2 sums it; the list is full: this warp does */
            if (__shfl_sync(0xffffffffu, k, 0) < AG_NOALLOC_MAX_LONG)
                continue;
        }
        float s = 0.0f;
        for (uint32_t j = b + lane; j < e; j += 32)
            s = __fadd_rn(s, ag_na_term(x, w, mode, j, __ldg(ids + j)));
        s = ag_na_warp_sum(s);
        if (lane == 0)
            y[r] = s;
    }
}

__global__ void __launch_bounds__(AG_NOALLOC_BLK) ag_na_long_kernel(const uint32_t *row_off, const uint32_t *ids,
                                                                     const float *w, const float *x, float *y,
                                                                     uint32_t mode, const uint32_t *scratch)
{
    __shared__ float sh[AG_NOALLOC_BLK / 32];
    const uint32_t count = min(*((volatile const uint32_t *)scratch), AG_NOALLOC_MAX_LONG);
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t r = scratch[AG_NOALLOC_HEADER + i];
        const uint32_t b = __ldg(row_off + r), e = __ldg(row_off + r + 1);
        float s = 0.0f;
        for (uint32_t j = b + threadIdx.x; j < e; j += blockDim.x)
            s = __fadd_rn(s, ag_na_term(x, w, mode, j, __ldg(ids + j)));
        s = ag_na_warp_sum(s);
        if ((threadIdx.x & 31) == 0)
            sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = sh[0];
            for (int k = 1; k < AG_NOALLOC_BLK / 32; ++k)
                t = __fadd_rn(t, sh[k]);
            y[r] = t;
        }
        __syncthreads();
    }
}

/* device address of the scratch array and the SM count, looked up once per
 * device (atomic: concurrent first calls from several host threads store the
 * same values) */
#define AG_NOALLOC_MAX_DEVICES 64
static std::atomic<uint32_t *> g_na_scratch[AG_NOALLOC_MAX_DEVICES];
static std::atomic<int> g_na_sms[AG_NOALLOC_MAX_DEVICES];

static ag_status_t na_scratch(uint32_t **out, int *sms)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ag_set_error(AG_ERR_NO_DEVICE, "ag_spmv_pull_noalloc: no current device: %s", cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= AG_NOALLOC_MAX_DEVICES)
        return ag_set_error(AG_ERR_UNSUPPORTED, "ag_spmv_pull_noalloc: device %d beyond %d", dev,
                            AG_NOALLOC_MAX_DEVICES);
    uint32_t *cached = g_na_scratch[dev].load(std::memory_order_acquire);
    if (!cached) {
        void *p = nullptr;
        int n = 0;
        e = cudaGetSymbolAddress(&p, ag_noalloc_scratch);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || !p || n <= 0) {
            cudaGetLastError();
            return ag_set_error(AG_ERR_CUDA, "ag_spmv_pull_noalloc: device set-up failed: %s",
                                cudaGetErrorString(e));
        }
        g_na_sms[dev].store(n, std::memory_order_relaxed);
        cached = (uint32_t *)p;
        g_na_scratch[dev].store(cached, std::memory_order_release);
    }
    *out = cached;
    *sms = g_na_sms[dev].load(std::memory_order_relaxed);
    return AG_OK;
}

extern "C" ag_status_t ag_spmv_pull_noalloc(uint32_t num_vertices, uint32_t num_edges, const uint32_t *row_off,
                                            const uint32_t *ids, const float *w, const float *x, float *y,
                                            uint32_t mode, void *stream)
{
    ag_clear_error();
    if (num_vertices == 0)
        return AG_OK;
    if (!row_off || !x || !y || (num_edges && !ids))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_pull_noalloc: NULL argument");
    if (mode & ~AG_SPMV_UNIT)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_spmv_pull_noalloc: mode %u: only AG_SPMV_GRAPH_WEIGHTS (0) and "
                            "AG_SPMV_UNIT (1); the stream-order form (AG_SPMV_EXACT) needs ag_spmv_pull", mode);
    if ((uint64_t)num_edges > (uint64_t)AG_NOALLOC_MAX_LONG * AG_NOALLOC_SPLIT)
        return ag_set_error(AG_ERR_UNSUPPORTED,
                            "ag_spmv_pull_noalloc: %u in-edges exceed the fixed scratch (at most %llu edges: "
                            "%u rows longer than %u)",
                            num_edges, (unsigned long long)AG_NOALLOC_MAX_LONG * AG_NOALLOC_SPLIT,
                            AG_NOALLOC_MAX_LONG, AG_NOALLOC_SPLIT);
    uint32_t *scratch = nullptr;
    int sms = 0;
    ag_status_t st = na_scratch(&scratch, &sms);
    if (st != AG_OK)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        uint64_t blocks = ((uint64_t)num_vertices * 32 + AG_NOALLOC_BLK - 1) / AG_NOALLOC_BLK;
        if (blocks > (uint64_t)sms * 16)
            blocks = (uint64_t)sms * 16;
        ag_na_rows_kernel<<<(unsigned)blocks, AG_NOALLOC_BLK, 0, s>>>(num_vertices, row_off, ids, w, x, y, mode,
                                                                       scratch);
        ag_na_long_kernel<<<(unsigned)sms * 4, AG_NOALLOC_BLK, 0, s>>>(row_off, ids, w, x, y, mode, scratch);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ag_set_error(AG_ERR_CUDA, "ag_spmv_pull_noalloc: launch failed: %s", cudaGetErrorString(e));
    }
    return AG_OK;
}
