/*
 * ag_build.cu -- forward and inverse CSR built from an edge list on the
 * device.
 *
 * The result is the host builder's (graph_host.c, ag_graph_from_edges) array
 * for array, bit for bit, for the same build flags:
 *   - AG_BUILD_SORT / AG_BUILD_DEDUPE: edges sorted by (source, destination)
 *     with a stable radix sort of the packed key src << nb | dst, so equal
 *     keys keep their input order; DEDUPE then drops self loops and every
 *     repeat of a key (the first occurrence stays, with its weight);
 *   - neither: a stable sort by source only, so each row keeps the input
 *     order of its edges;
 *   - the inverse CSR is a stable sort of the forward order by destination:
 *     inverse rows list sources in forward order (ascending when sorted);
 *   - row starts have N + 1 entries (the last is E); out- and in-degrees are
 *     their differences; max_weight is the largest weight above zero (0.0f
 *     without weights or without a positive one).
 * The sorts are CUB device radix sorts (stable LSD); row starts come from
 * the sorted row ids by binary search, one thread per row.
 */
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "accelgraph_b200.h"
#include "ag_device.h"

static int bits_for(uint64_t max_value)
{
    int b = 1;
    while (b < 64 && (max_value >> b) != 0)
        b++;
    return b;
}

static unsigned grid_for(uint64_t n, unsigned per_block)
{
    uint64_t b = (n + per_block - 1) / per_block;
    if (b < 1)
        b = 1;
    if (b > 65535u * 16u)
        b = 65535u * 16u;
    return (unsigned)b;
}

/* lowest edge index with an endpoint >= n (flag[0] = UINT32_MAX: none) */
__global__ void ag_build_validate_kernel(const uint32_t *src, const uint32_t *dst, uint32_t m, uint32_t n,
                                         uint32_t *flag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        if (src[i] >= n || dst[i] >= n)
            atomicMin(flag, i);
}

__global__ void ag_build_keys_pair_kernel(const uint32_t *src, const uint32_t *dst, uint32_t m, int nb,
                                          unsigned long long *keys, uint32_t *idx)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        keys[i] = ((unsigned long long)src[i] << nb) | dst[i];
        idx[i] = i;
    }
}

__global__ void ag_build_iota_kernel(uint32_t *idx, uint32_t m)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        idx[i] = i;
}

/* keep flag of a sorted key: not a self loop and not a repeat */
__global__ void ag_build_dedupe_flags_kernel(const unsigned long long *keys, uint32_t m, int nb, uint32_t *keep)
{
    const unsigned long long mask = (1ull << nb) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        const bool loop = (k >> nb) == (k & mask);
        keep[i] = (!loop && (i == 0 || keys[i - 1] != k)) ? 1u : 0u;
    }
}

__global__ void ag_build_compact_kernel(const unsigned long long *keys, const uint32_t *idx, const uint32_t *keep,
                                        const uint32_t *pos, uint32_t m, unsigned long long *keys_out,
                                        uint32_t *idx_out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        if (keep[i]) {
            keys_out[pos[i]] = keys[i];
            idx_out[pos[i]] = idx[i];
        }
}

/* forward arrays from the sorted keys (pair keys, or source keys plus the
 * original destinations) and the original edge index of each position */
__global__ void ag_build_forward_kernel(const unsigned long long *keys64, const uint32_t *keys32,
                                        const uint32_t *idx, const uint32_t *dst_in, const float *w_in, uint32_t e,
                                        int nb, uint32_t *fsrc, uint32_t *fdst, float *fw)
{
    const unsigned long long mask = (1ull << nb) - 1ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) {
        uint32_t s, d;
        if (keys64) {
            s = (uint32_t)(keys64[i] >> nb);
            d = (uint32_t)(keys64[i] & mask);
        } else {
            s = keys32[i];
            d = dst_in[idx[i]];
        }
        fsrc[i] = s;
        fdst[i] = d;
        if (fw)
            fw[i] = w_in[idx[i]];
    }
}

/* starts[v] = first position whose row id is >= v, for v in [0, n]
 * (binary search of the sorted row ids; rows without edges cost nothing
 * extra however long their runs) */
__global__ void ag_build_row_starts_kernel(const uint32_t *rows, uint32_t e, uint32_t n, uint32_t *starts)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = e;
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if (rows[mid] < v)
                lo = mid + 1;
            else
                hi = mid;
        }
        starts[v] = lo;
    }
}

__global__ void ag_build_degrees_kernel(const uint32_t *starts, uint32_t n, uint32_t *deg)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        deg[v] = starts[v + 1] - starts[v];
}

__global__ void ag_build_inverse_kernel(const uint32_t *perm, const uint32_t *fsrc, const float *fw, uint32_t e,
                                        uint32_t *idst, float *iw)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < e; j += gridDim.x * blockDim.x) {
        const uint32_t f = perm[j];
        idst[j] = fsrc[f];
        if (iw)
            iw[j] = fw[f];
    }
}

/* largest weight above zero, as the host builder's running maximum from
 * 0.0f (NaN never taken) */
struct AgPositiveMax
{
    __device__ __forceinline__ float operator()(float a, float b) const
    {
        a = (a > 0.0f) ? a : 0.0f;
        b = (b > 0.0f) ? b : 0.0f;
        return a > b ? a : b;
    }
};

struct AgUMax
{
    __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

extern "C" void ag_csr_free_device(AgDevCSR *c, cudaStream_t s)
{
    void *ptrs[] = {c->out_deg, c->in_deg, c->fwd_idx, c->inv_idx, c->fwd_src,
                    c->fwd_dst, c->inv_src, c->inv_dst, c->fwd_w, c->inv_w};
    for (void *p : ptrs)
        if (p)
            cudaFreeAsync(p, s);
    memset(c, 0, sizeof(*c));
}

#define BUILD_CUDA(call)                                                                       \
    do {                                                                                       \
        err = (call);                                                                          \
        if (err != cudaSuccess)                                                                \
            goto done;                                                                         \
    } while (0)

extern "C" cudaError_t ag_csr_build_device(uint32_t n, uint32_t m, const uint32_t *src, const uint32_t *dst,
                                           const float *w, uint32_t flags, AgDevCSR *out, uint32_t *bad_edge,
                                           cudaStream_t s)
{
    cudaError_t err = cudaSuccess;
    const bool sorted = (flags & (AG_BUILD_SORT | AG_BUILD_DEDUPE)) != 0;
    const bool dedupe = (flags & AG_BUILD_DEDUPE) != 0;
    const int nb = bits_for(n > 0 ? (uint64_t)(n - 1) : 0);
    unsigned long long *k64a = nullptr, *k64b = nullptr;
    uint32_t *k32 = nullptr, *idxa = nullptr, *idxb = nullptr, *keep = nullptr, *pos = nullptr, *flag = nullptr;
    uint32_t *hbuf = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, need = 0;
    uint32_t e = m;
    memset(out, 0, sizeof(*out));
    *bad_edge = UINT32_MAX;
    out->N = n;
    const unsigned B = 256;

    BUILD_CUDA(cudaMallocHost((void **)&hbuf, 4 * sizeof(uint32_t)));
    /* scratch: sort keys and values, twice; keep flags and positions */
    BUILD_CUDA(cudaMallocAsync((void **)&flag, 16, s));
    BUILD_CUDA(cudaMemsetAsync(flag, 0xFF, 4, s));
    if (m) {
        ag_build_validate_kernel<<<grid_for(m, B), B, 0, s>>>(src, dst, m, n, flag);
        BUILD_CUDA(cudaGetLastError());
    }
    BUILD_CUDA(cudaMemcpyAsync(hbuf, flag, 4, cudaMemcpyDeviceToHost, s));
    BUILD_CUDA(cudaStreamSynchronize(s));
    if (hbuf[0] != UINT32_MAX) {
        *bad_edge = hbuf[0];
        err = cudaErrorInvalidValue;
        goto done;
    }

    /* scratch sizes of the three sorts and the scan */
    if (sorted) {
        BUILD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, (const unsigned long long *)nullptr,
                                                   (unsigned long long *)nullptr, (const uint32_t *)nullptr,
                                                   (uint32_t *)nullptr, (int)m, 0, 2 * nb, s));
        tmp_bytes = need;
    }
    BUILD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                               (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)m, 0, nb, s));
    tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
    BUILD_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, need, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                             (int)m + 1, s));
    tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
    BUILD_CUDA(cub::DeviceReduce::Reduce(nullptr, need, (const float *)nullptr, (float *)nullptr, (int)m,
                                         AgPositiveMax(), 0.0f, s));
    tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
    BUILD_CUDA(cub::DeviceReduce::Reduce(nullptr, need, (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n,
                                         AgUMax(), 0u, s));
    tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
    BUILD_CUDA(cudaMallocAsync(&tmp, tmp_bytes ? tmp_bytes : 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&idxa, (size_t)m * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&idxb, (size_t)m * 4 + 16, s));

    /* forward order */
    if (sorted) {
        BUILD_CUDA(cudaMallocAsync((void **)&k64a, (size_t)m * 8 + 16, s));
        BUILD_CUDA(cudaMallocAsync((void **)&k64b, (size_t)m * 8 + 16, s));
        if (m) {
            ag_build_keys_pair_kernel<<<grid_for(m, B), B, 0, s>>>(src, dst, m, nb, k64a, idxa);
            BUILD_CUDA(cudaGetLastError());
            size_t tb = tmp_bytes;
            BUILD_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, k64a, k64b, idxa, idxb, (int)m, 0, 2 * nb, s));
        }
        /* sorted keys and original indexes now in k64b / idxb */
        if (dedupe && m) {
            BUILD_CUDA(cudaMallocAsync((void **)&keep, ((size_t)m + 1) * 4, s));
            BUILD_CUDA(cudaMallocAsync((void **)&pos, ((size_t)m + 1) * 4, s));
            BUILD_CUDA(cudaMemsetAsync(keep + m, 0, 4, s));
            ag_build_dedupe_flags_kernel<<<grid_for(m, B), B, 0, s>>>(k64b, m, nb, keep);
            BUILD_CUDA(cudaGetLastError());
            size_t tb = tmp_bytes;
            BUILD_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, keep, pos, (int)m + 1, s));
            ag_build_compact_kernel<<<grid_for(m, B), B, 0, s>>>(k64b, idxb, keep, pos, m, k64a, idxa);
            BUILD_CUDA(cudaGetLastError());
            BUILD_CUDA(cudaMemcpyAsync(hbuf, pos + m, 4, cudaMemcpyDeviceToHost, s));
            BUILD_CUDA(cudaStreamSynchronize(s));
            e = hbuf[0];
            /* compacted keys and indexes now in k64a / idxa */
            unsigned long long *tk = k64a;
            k64a = k64b;
            k64b = tk;
            uint32_t *ti = idxa;
            idxa = idxb;
            idxb = ti;
        }
    } else {
        BUILD_CUDA(cudaMallocAsync((void **)&k32, (size_t)m * 4 + 16, s));
        if (m) {
            ag_build_iota_kernel<<<grid_for(m, B), B, 0, s>>>(idxa, m);
            BUILD_CUDA(cudaGetLastError());
            size_t tb = tmp_bytes;
            BUILD_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, src, k32, idxa, idxb, (int)m, 0, nb, s));
        }
    }
    /* k64b (pair keys) or k32 (sources) + idxb: e edges in forward order */
    out->E = e;
    BUILD_CUDA(cudaMallocAsync((void **)&out->out_deg, (size_t)n * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->in_deg, (size_t)n * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->fwd_idx, (size_t)n * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->inv_idx, (size_t)n * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->fwd_src, (size_t)e * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->fwd_dst, (size_t)e * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->inv_src, (size_t)e * 4 + 16, s));
    BUILD_CUDA(cudaMallocAsync((void **)&out->inv_dst, (size_t)e * 4 + 16, s));
    if (w) {
        BUILD_CUDA(cudaMallocAsync((void **)&out->fwd_w, (size_t)e * 4 + 16, s));
        BUILD_CUDA(cudaMallocAsync((void **)&out->inv_w, (size_t)e * 4 + 16, s));
    }
    if (e) {
        ag_build_forward_kernel<<<grid_for(e, B), B, 0, s>>>(sorted ? k64b : nullptr, sorted ? nullptr : k32, idxb,
                                                             dst, w, e, nb, out->fwd_src, out->fwd_dst, out->fwd_w);
        BUILD_CUDA(cudaGetLastError());
        ag_build_row_starts_kernel<<<grid_for((uint64_t)n + 1, B), B, 0, s>>>(out->fwd_src, e, n, out->fwd_idx);
        BUILD_CUDA(cudaGetLastError());
        /* inverse: stable sort of the forward order by destination */
        ag_build_iota_kernel<<<grid_for(e, B), B, 0, s>>>(idxa, e);
        BUILD_CUDA(cudaGetLastError());
        size_t tb = tmp_bytes;
        BUILD_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, out->fwd_dst, out->inv_src, idxa, idxb, (int)e, 0, nb,
                                                   s));
        ag_build_inverse_kernel<<<grid_for(e, B), B, 0, s>>>(idxb, out->fwd_src, out->fwd_w, e, out->inv_dst,
                                                             out->inv_w);
        BUILD_CUDA(cudaGetLastError());
        ag_build_row_starts_kernel<<<grid_for((uint64_t)n + 1, B), B, 0, s>>>(out->inv_src, e, n, out->inv_idx);
        BUILD_CUDA(cudaGetLastError());
    } else {
        BUILD_CUDA(cudaMemsetAsync(out->fwd_idx, 0, (size_t)n * 4 + 4, s));
        BUILD_CUDA(cudaMemsetAsync(out->inv_idx, 0, (size_t)n * 4 + 4, s));
    }
    if (n) {
        ag_build_degrees_kernel<<<grid_for(n, B), B, 0, s>>>(out->fwd_idx, n, out->out_deg);
        BUILD_CUDA(cudaGetLastError());
        ag_build_degrees_kernel<<<grid_for(n, B), B, 0, s>>>(out->inv_idx, n, out->in_deg);
        BUILD_CUDA(cudaGetLastError());
    }
    /* largest weight and largest in-degree */
    {
        float *dmax = reinterpret_cast<float *>(flag + 1);
        uint32_t *dmaxd = flag + 2;
        BUILD_CUDA(cudaMemsetAsync(flag + 1, 0, 8, s));
        size_t tb = tmp_bytes;
        if (w && e)
            BUILD_CUDA(cub::DeviceReduce::Reduce(tmp, tb, out->fwd_w, dmax, (int)e, AgPositiveMax(), 0.0f, s));
        tb = tmp_bytes;
        if (n)
            BUILD_CUDA(cub::DeviceReduce::Reduce(tmp, tb, out->in_deg, dmaxd, (int)n, AgUMax(), 0u, s));
        BUILD_CUDA(cudaMemcpyAsync(hbuf, flag + 1, 8, cudaMemcpyDeviceToHost, s));
        BUILD_CUDA(cudaStreamSynchronize(s));
        float mw;
        memcpy(&mw, hbuf, 4);
        out->max_w = mw > 0.0f ? mw : 0.0f;
        out->max_in_degree = hbuf[1];
    }
done:
    if (k64a)
        cudaFreeAsync(k64a, s);
    if (k64b)
        cudaFreeAsync(k64b, s);
    if (k32)
        cudaFreeAsync(k32, s);
    if (idxa)
        cudaFreeAsync(idxa, s);
    if (idxb)
        cudaFreeAsync(idxb, s);
    if (keep)
        cudaFreeAsync(keep, s);
    if (pos)
        cudaFreeAsync(pos, s);
    if (flag)
        cudaFreeAsync(flag, s);
    if (tmp)
        cudaFreeAsync(tmp, s);
    if (err != cudaSuccess)
        ag_csr_free_device(out, s);
    if (hbuf) {
        cudaStreamSynchronize(s);
        cudaFreeHost(hbuf);
    }
    return err;
}
