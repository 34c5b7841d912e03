/*
 * ag_mem.h -- cache-policy loads and stores shared by the pull kernels.
 *
 * A pull pass streams the in-neighbour ids once (L1 no-allocate, first to
 * leave L2), gathers the pass's read-only contribution vector at random (kept
 * in L2; ids of the warm tier may take L1 lines, colder ones do not, so they
 * cannot displace warm lines), and reads each row's offsets, degree and rank
 * once (no L1 line).
 */
#ifndef AG_MEM_H
#define AG_MEM_H
#include <cuda_runtime.h>
#include <stdint.h>

__device__ __forceinline__ uint64_t ag_policy_evict_first()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ uint64_t ag_policy_evict_last()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

/* streamed once per pass: keep it out of L1, first to leave L2 */
__device__ __forceinline__ uint4 ag_ld_stream_u4(const uint4 *p, uint64_t pol)
{
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float4 ag_ld_stream_f4(const float4 *p, uint64_t pol)
{
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(pol));
    return v;
}

/* random gather of the pass's read-only contribution vector: keep it in L2 */
__device__ __forceinline__ float ag_ld_gather_f32(const float *p, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

/* cold gather: beyond the warm tier, do not displace warm lines from L1 */
__device__ __forceinline__ float ag_ld_cold_f32(const float *p, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint16_t ag_ld_cold_u16(const uint16_t *p, uint64_t pol)
{
    uint16_t v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
    return v;
}

/* per-row data read once per pass: bypass L1 */
__device__ __forceinline__ uint32_t ag_ld_row_u32(const uint32_t *p)
{
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

/* rank: read and later written by the same lane in the same kernel, so the
 * coherent path, still without an L1 line */
__device__ __forceinline__ float ag_ld_rank(const float *p)
{
    float v;
    asm volatile("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint16_t ag_ld_gather_u16(const uint16_t *p, uint64_t pol)
{
    uint16_t v;
    asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ void ag_st_keep_f32(float *p, float v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

__device__ __forceinline__ void ag_st_keep_u16(uint16_t *p, uint16_t v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.u16 [%0], %1, %2;" ::"l"(p), "h"(v), "l"(pol) : "memory");
}

__device__ __forceinline__ unsigned long long ag_globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* integer gathers of 8-, 16-, 32- or 64-bit elements, zero-extended; l1:
 * whether the line may be allocated in L1 */
template <typename T> __device__ __forceinline__ uint64_t ag_ld_gather_uint(const T *p, uint64_t pol, bool l1)
{
    if constexpr (sizeof(T) == 8) {
        unsigned long long v;
        if (l1)
            asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
        else
            asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
        return v;
    } else {
        uint32_t v;
        if constexpr (sizeof(T) == 4) {
            if (l1)
                asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
            else
                asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
        } else if constexpr (sizeof(T) == 2) {
            if (l1)
                asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
            else
                asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
        } else {
            if (l1)
                asm("ld.global.nc.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
            else
                asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
        }
        return v;
    }
}

/* one streamed 32-bit id (long rows): no L1 line, first to leave L2 */
__device__ __forceinline__ uint32_t ag_ld_stream_u32(const uint32_t *p, uint64_t pol)
{
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

#endif /* AG_MEM_H */
