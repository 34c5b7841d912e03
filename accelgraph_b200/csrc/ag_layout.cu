/*
 * ag_layout.cu -- upload-time device layout of the inverse CSR.
 *
 * Vertices are relabelled by descending forward out-degree (ties keep the
 * caller's id order; stable radix sort): new id i holds old vertex perm[i],
 * inv[old] = i.  The gather reads c[u] once per out-edge of u, so after the
 * relabelling the most-read contributions sit in one dense prefix of the
 * contribution vector.  The pull kernel copies that prefix into shared memory
 * each pass (one TMA bulk copy) and serves those gathers from it; the rest hit
 * a contribution vector whose hot lines are packed together in L2.
 *
 * Rows are permuted the same way (row i of the device CSR is old vertex
 * perm[i]) and every in-neighbour id is mapped through inv.  Each row keeps
 * its edges in the caller's stream order, so the stream-order sums (and the
 * EXACT order's bit-identity with a sequential loop) are unchanged: only
 * where a value is fetched from moves.
 */
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ag_device.h"

__global__ void ag_iota_kernel(uint32_t *a, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = i;
}

__global__ void ag_inverse_perm_kernel(const uint32_t *perm, uint32_t *inv, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        inv[perm[i]] = i;
}

/* new in-degree (n+1 entries, last 0 for the scan) and new out-degree */
__global__ void ag_permuted_degrees_kernel(const uint32_t *perm, const uint32_t *off_old,
                                           const uint32_t *outdeg_old, uint32_t *deg_new,
                                           uint32_t *outdeg_new, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            deg_new[n] = 0;
            continue;
        }
        const uint32_t o = perm[i];
        deg_new[i] = off_old[o + 1] - off_old[o];
        outdeg_new[i] = outdeg_old[o];
    }
}

/* Rows copied in the new order, mapping ids through inv, rows keeping their
 * edge order.  The new edge array is cut into segments of AG_COPY_SEG
 * positions, one warp per segment, so that a row of any length is spread
 * over many warps.  A warp finds the row holding its first position by a
 * binary search of the new row starts, then walks its positions 32 at a time
 * (coalesced stores) over a window of 32 consecutive rows: each lane holds
 * one row's old start and new start, and a position's row is found by a
 * five-step binary search over the lanes (shuffles).  When the window's rows
 * end before the segment does, the window moves on. */
#define AG_COPY_SEG 2048u

__global__ void ag_copy_rows_kernel(const uint32_t *perm, const uint32_t *inv, const uint32_t *off_old,
                                    const uint32_t *off_new, const uint32_t *ids_old, uint32_t *ids_new,
                                    const float *w_old, float *w_new, uint32_t n, uint32_t e)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nseg = (e + AG_COPY_SEG - 1) / AG_COPY_SEG;
    for (uint32_t seg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; seg < nseg; seg += nw) {
        const uint32_t p0 = seg * AG_COPY_SEG;
        const uint32_t p1 = min(e, p0 + AG_COPY_SEG);
        /* the last row starting at or before p0 (rows 0 .. n-1; off_new[n] = e > p0) */
        uint32_t lo = 0, hi = n - 1;
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo + 1) >> 1);
            if (off_new[mid] <= p0)
                lo = mid;
            else
                hi = mid - 1;
        }
        uint32_t rbase = lo, jb = p0;
        while (jb < p1) {
            const uint32_t i = rbase + lane;
            /* lanes past the last row start at e, so no position maps to them */
            const uint32_t dst = off_new[i < n ? i : n];
            const uint32_t src = i < n ? off_old[perm[i]] : 0u;
            const uint32_t wend = off_new[rbase + 32 < n ? rbase + 32 : n];
            const uint32_t stop = min(p1, wend);
            for (; jb < stop; jb += 32) {
                const uint32_t j = jb + lane;
                /* the last lane whose row starts at or before j owns it (an
                 * empty row shares its start with the next row, which wins) */
                uint32_t l = 0;
#pragma unroll
                for (uint32_t step = 16; step >= 1; step >>= 1) {
                    const uint32_t cand = l + step;
                    if (__shfl_sync(0xffffffffu, dst, cand) <= j)
                        l = cand;
                }
                const uint32_t k = __shfl_sync(0xffffffffu, src, l) + (j - __shfl_sync(0xffffffffu, dst, l));
                if (j < stop) {
                    ids_new[j] = inv[ids_old[k]];
                    if (w_new)
                        w_new[j] = w_old[k];
                }
            }
            jb = stop;
            rbase += 32;
        }
    }
}

/* x_new[i] = x[perm[i]] */
__global__ void ag_permute_in_kernel(const uint32_t *perm, const float *x, float *x_new, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x_new[i] = x[perm[i]];
}

/* y[v] = y_new[inv[v]] */
__global__ void ag_permute_out_kernel(const uint32_t *inv, const float *y_new, float *y, uint32_t n)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        y[v] = y_new[inv[v]];
}

static unsigned grid_for(uint64_t n, unsigned per_block)
{
    uint64_t g = (n + per_block - 1) / per_block;
    if (g > ag_sm_grid(16))
        g = ag_sm_grid(16);
    return g ? (unsigned)g : 1u;
}

/* The relabelled layout, from the degrees alone.  Inputs (device):
 * off_old[n+1], outdeg_old[n].  Outputs (device, allocated by the caller):
 * perm[n], inv[n], off_new[n+1], outdeg_new[n].  Scratch is taken from the
 * stream-ordered pool.  It needs no in-edge, so it can run while the in-edges
 * are still being copied to the device. */
extern "C" cudaError_t ag_relabel_layout(const uint32_t *off_old, const uint32_t *outdeg_old, uint32_t n,
                                         uint32_t *perm, uint32_t *inv, uint32_t *off_new, uint32_t *outdeg_new,
                                         cudaStream_t s)
{
    cudaError_t err;
    if (n == 0)
        return cudaMemsetAsync(off_new, 0, sizeof(uint32_t), s);
    uint32_t *iota = nullptr, *keys_out = nullptr, *deg_new = nullptr;
    void *tmp = nullptr;
    size_t tmp_sort = 0, tmp_scan = 0;
    err = cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_sort, outdeg_old, (uint32_t *)nullptr,
                                                    (const uint32_t *)nullptr, perm, (int)n, 0, 32, s);
    if (err != cudaSuccess)
        return err;
    err = cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, (const uint32_t *)nullptr, off_new, (int)n + 1, s);
    if (err != cudaSuccess)
        return err;
    const size_t tmp_bytes = tmp_sort > tmp_scan ? tmp_sort : tmp_scan;
    if ((err = cudaMallocAsync((void **)&iota, (size_t)n * 4, s)) != cudaSuccess)
        return err;
    if ((err = cudaMallocAsync((void **)&keys_out, (size_t)n * 4, s)) != cudaSuccess)
        goto done;
    if ((err = cudaMallocAsync((void **)&deg_new, (size_t)(n + 1) * 4, s)) != cudaSuccess)
        goto done;
    if ((err = cudaMallocAsync(&tmp, tmp_bytes ? tmp_bytes : 16, s)) != cudaSuccess)
        goto done;
    ag_iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(iota, n);
    {
        size_t tb = tmp_bytes;
        err = cub::DeviceRadixSort::SortPairsDescending(tmp, tb, outdeg_old, keys_out, iota, perm, (int)n, 0, 32, s);
        if (err != cudaSuccess)
            goto done;
    }
    ag_inverse_perm_kernel<<<grid_for(n, 256), 256, 0, s>>>(perm, inv, n);
    ag_permuted_degrees_kernel<<<grid_for((uint64_t)n + 1, 256), 256, 0, s>>>(perm, off_old, outdeg_old, deg_new,
                                                                            outdeg_new, n);
    {
        size_t tb = tmp_bytes;
        err = cub::DeviceScan::ExclusiveSum(tmp, tb, deg_new, off_new, (int)n + 1, s);
        if (err != cudaSuccess)
            goto done;
    }
    err = cudaGetLastError();
done:
    if (iota)
        cudaFreeAsync(iota, s);
    if (keys_out)
        cudaFreeAsync(keys_out, s);
    if (deg_new)
        cudaFreeAsync(deg_new, s);
    if (tmp)
        cudaFreeAsync(tmp, s);
    return err;
}

/* The relabelled rows: every row copied to its new place, its in-neighbour
 * ids mapped through inv (and its weights copied), in stream order. */
extern "C" cudaError_t ag_relabel_rows(const uint32_t *perm, const uint32_t *inv, const uint32_t *off_old,
                                       const uint32_t *off_new, const uint32_t *ids_old, uint32_t *ids_new,
                                       const float *w_old, float *w_new, uint32_t n, uint32_t e, cudaStream_t s)
{
    if (n == 0 || e == 0)
        return cudaSuccess;
    ag_copy_rows_kernel<<<grid_for(((uint64_t)e + AG_COPY_SEG - 1) / AG_COPY_SEG * 32, 256), 256, 0, s>>>(
        perm, inv, off_old, off_new, ids_old, ids_new, w_old, w_new, n, e);
    return cudaGetLastError();
}

/* Layout and rows in one call (device-resident inputs). */
extern "C" cudaError_t ag_relabel_by_out_degree(const uint32_t *off_old, const uint32_t *ids_old, const float *w_old,
                                                const uint32_t *outdeg_old, uint32_t n, uint32_t e, uint32_t *perm,
                                                uint32_t *inv, uint32_t *off_new, uint32_t *ids_new, float *w_new,
                                                uint32_t *outdeg_new, cudaStream_t s)
{
    cudaError_t err = ag_relabel_layout(off_old, outdeg_old, n, perm, inv, off_new, outdeg_new, s);
    if (err != cudaSuccess)
        return err;
    return ag_relabel_rows(perm, inv, off_old, off_new, ids_old, ids_new, w_old, w_new, n, e, s);
}

extern "C" cudaError_t ag_permute_in(const uint32_t *perm, const float *x, float *x_new, uint32_t n, cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    ag_permute_in_kernel<<<grid_for(n, 256), 256, 0, s>>>(perm, x, x_new, n);
    return cudaGetLastError();
}

extern "C" cudaError_t ag_permute_out(const uint32_t *inv, const float *y_new, float *y, uint32_t n, cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    ag_permute_out_kernel<<<grid_for(n, 256), 256, 0, s>>>(inv, y_new, y, n);
    return cudaGetLastError();
}
