/*
 * gather_probe.cu -- device probe of random 4-byte gather rates, the quantity
 * that bounds a pull pass (every in-edge is one random gather).  A measuring
 * aid, not part of the library: bench.py --workload gather-probe builds it into
 * its own libgather_probe.so (tests/probe/) and calls gather_probe_rates.
 *
 * Each probe kernel runs one 1024-thread CTA per SM (clusters of 8 for the
 * distributed case); every thread issues 256 x 8 gathers with indexes from an
 * integer hash masked to the table size, so every access is in range.
 * Results are gathers per second for: shared memory (64 KB table), global
 * memory with L1-resident (256 KB), L2-resident (64 MB) and HBM-resident
 * (256 MB) working sets, L2-resident through the texture path, and
 * distributed shared memory across an 8-CTA cluster (8 x 160 KB).
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cg = cooperative_groups;

#define AG_PB_BLK 1024
#define AG_PB_ITERS 256
#define AG_PB_CL 8
#define AG_PB_P 40960

__device__ __forceinline__ uint32_t ag_pb_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

extern __shared__ float ag_pb_tab[];

template <int MODE>
__global__ void __launch_bounds__(AG_PB_BLK, 1) ag_pb_kernel(const float *src, uint32_t mask, float *out,
                                                              cudaTextureObject_t tex)
{
    if (MODE == 0) {
        for (uint32_t i = threadIdx.x; i <= mask; i += AG_PB_BLK)
            ag_pb_tab[i] = src[i];
        __syncthreads();
    }
    float acc = 0.f;
    uint32_t h = blockIdx.x * AG_PB_BLK + threadIdx.x;
    for (int it = 0; it < AG_PB_ITERS; ++it) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            h = ag_pb_hash(h + q);
            const uint32_t i = h & mask;
            if (MODE == 0)
                v[q] = ag_pb_tab[i];
            else if (MODE == 1)
                v[q] = __ldg(src + i);
            else
                v[q] = tex1Dfetch<float>(tex, (int)i);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            acc += v[q];
    }
    out[blockIdx.x * AG_PB_BLK + threadIdx.x] = acc;
}

__global__ void __cluster_dims__(AG_PB_CL, 1, 1) __launch_bounds__(AG_PB_BLK, 1)
    ag_pb_cluster_kernel(const float *src, float *out)
{
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t crank = cl.block_rank();
    for (uint32_t i = threadIdx.x; i < AG_PB_P; i += AG_PB_BLK)
        ag_pb_tab[i] = src[crank * AG_PB_P + i];
    cl.sync();
    float acc = 0.f;
    uint32_t h = blockIdx.x * AG_PB_BLK + threadIdx.x;
    for (int it = 0; it < AG_PB_ITERS; ++it) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            h = ag_pb_hash(h + q);
            const uint32_t g = h % (AG_PB_CL * AG_PB_P);
            float *rp = cl.map_shared_rank(ag_pb_tab, g / AG_PB_P);
            v[q] = rp[g % AG_PB_P];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            acc += v[q];
    }
    out[blockIdx.x * AG_PB_BLK + threadIdx.x] = acc;
    cl.sync();
}

/* rates[0..5] = gathers/s from: shared memory, L1-resident, L2-resident,
 * HBM-resident, L2-resident through textures, cluster shared memory, on the
 * current device.  Returns 0 or the failing call's cudaError_t. */
extern "C" int gather_probe_rates(double *rates)
{
    if (!rates)
        return (int)cudaErrorInvalidValue;
    int dev = 0, nsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return (int)e;
    cudaStream_t s = nullptr;
    if ((e = cudaStreamCreate(&s)) != cudaSuccess)
        return (int)e;
    const uint32_t n = 1u << 26; /* 256 MB */
    float *src = nullptr, *out = nullptr;
    cudaTextureObject_t tex = 0;
    cudaEvent_t a = nullptr, b = nullptr;
    e = cudaMalloc((void **)&src, (size_t)n * 4);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&out, (size_t)nsm * AG_PB_BLK * 4);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(src, 0, (size_t)n * 4, s);
    if (e == cudaSuccess) {
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypeLinear;
        rd.res.linear.devPtr = src;
        rd.res.linear.desc = cudaCreateChannelDesc<float>();
        rd.res.linear.sizeInBytes = (size_t)n * 4;
        cudaTextureDesc td = {};
        td.readMode = cudaReadModeElementType;
        e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    }
    if (e == cudaSuccess)
        e = cudaEventCreate(&a);
    if (e == cudaSuccess)
        e = cudaEventCreate(&b);
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(ag_pb_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(ag_pb_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     AG_PB_P * 4);
    }
    const double per_thread = (double)AG_PB_ITERS * 8;
    for (int t = 0; t < 6 && e == cudaSuccess; ++t) {
        float ms = 0.f;
        int grid = nsm;
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(a, s);
            switch (t) {
            case 0: ag_pb_kernel<0><<<nsm, AG_PB_BLK, 65536, s>>>(src, (1u << 14) - 1, out, tex); break;
            case 1: ag_pb_kernel<1><<<nsm, AG_PB_BLK, 0, s>>>(src, (1u << 16) - 1, out, tex); break;
            case 2: ag_pb_kernel<1><<<nsm, AG_PB_BLK, 0, s>>>(src, (1u << 24) - 1, out, tex); break;
            case 3: ag_pb_kernel<1><<<nsm, AG_PB_BLK, 0, s>>>(src, n - 1, out, tex); break;
            case 4: ag_pb_kernel<2><<<nsm, AG_PB_BLK, 0, s>>>(src, (1u << 24) - 1, out, tex); break;
            default:
                grid = (nsm / AG_PB_CL) * AG_PB_CL;
                ag_pb_cluster_kernel<<<grid, AG_PB_BLK, AG_PB_P * 4, s>>>(src, out);
                break;
            }
            if (e == cudaSuccess)
                e = cudaGetLastError();
            if (e == cudaSuccess)
                e = cudaEventRecord(b, s);
            if (e == cudaSuccess)
                e = cudaEventSynchronize(b);
            if (e == cudaSuccess)
                e = cudaEventElapsedTime(&ms, a, b);
        }
        rates[t] = (double)grid * AG_PB_BLK * per_thread / (ms * 1e-3);
    }
    if (tex)
        cudaDestroyTextureObject(tex);
    if (a)
        cudaEventDestroy(a);
    if (b)
        cudaEventDestroy(b);
    cudaFree(src);
    cudaFree(out);
    cudaStreamDestroy(s);
    if (e != cudaSuccess)
        cudaGetLastError();
    return (int)e;
}
