/*
 * ag_pull.cu -- sm_100a kernels of the pull PageRank / SpMV hot path.
 *
 * One pull pass (reference: the host contribution loop pageRank.c:1026-1033,
 * the accelerator gather of the cu_PageRank CSR PULL compute units, whose arithmetic the RTL
 * testbench pins in pagerank_kernel_tb.sv:303-314, and the host update loop
 * pageRank.c:1055-1069) is ONE kernel launch here:
 *
 *   s[v]  = c[u0] + c[u1] + ...     over v's inverse row, binary32
 *   r'[v] = base + damp * s[v]      binary32 multiply, then add (no FMA)
 *   err   = |r'[v] - r[v]|          binary32 subtract, compared in binary64
 *   c'[v] = r'[v] / out_degree[v]   next pass's contribution (0 if no out-edge)
 *
 * with the pass's error sum (binary64) and active count reduced per CTA and
 * the last CTA to finish closing the pass: it records the pass, decides
 * whether another pass runs and sets the CUDA-graph WHILE condition.
 *
 * Work decomposition (planned once per graph on the host, see ag_runtime.cu):
 *   row block : consecutive rows holding <= AG_CAP in-edges.  Phase 1 streams
 *               the block's ids with 16-byte loads (L1 no-allocate, L2
 *               evict-first) and gathers c[id] (L2 evict-last) into shared
 *               memory -- every gather of the block is independent, so the
 *               loads overlap.  Phase 2 reduces each row from shared memory:
 *               one thread per row in stream order for rows of <= AG_TSEQ
 *               edges (bit-identical to the reference's sequential sum), one
 *               warp per longer row (lane-strided partial sums + xor tree).
 *   long row  : AG_CAP < degree <= AG_HUB, one CTA, lane-strided partials and
 *               a fixed-order CTA reduction.
 *   hub chunk : rows > AG_HUB split into AG_HUB chunks on separate CTAs; the
 *               last chunk to arrive sums the chunk partials in chunk order.
 * In EXACT order every row is summed in stream order by one thread.
 * All reductions have a fixed order: results do not depend on scheduling.
 */
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "ag_device.h"

#define AG_NW (AG_BLK / 32)

/* ------------------------------------------------------ memory access */
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

/* 16-bit contribution formats of the precision form */
template <int PREC>
__device__ __forceinline__ float ag_low_to_f32(uint16_t h)
{
    if (PREC == 1)
        return __uint_as_float(((uint32_t)h) << 16);
    return __half2float(__ushort_as_half(h));
}

template <int PREC>
__device__ __forceinline__ uint16_t ag_f32_to_low(float f)
{
    if (PREC == 1)
        return __bfloat16_as_ushort(__float2bfloat16_rn(f));
    return __half_as_ushort(__float2half_rn(f));
}

/* ----------------------------------------------------- reductions */
__device__ __forceinline__ float ag_warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double ag_warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t ag_warp_sum_u(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* fixed-order CTA sum; the result is valid in thread 0 */
__device__ __forceinline__ float ag_block_sum_f(float v, float *sh)
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = ag_warp_sum_f(v);
    if (lane == 0)
        sh[warp] = v;
    __syncthreads();
    float s = 0.0f;
    if (threadIdx.x == 0) {
        s = sh[0];
#pragma unroll
        for (int w = 1; w < AG_NW; ++w)
            s = __fadd_rn(s, sh[w]);
    }
    __syncthreads();
    return s;
}

/* ------------------------------------------------------------- kernel */
template <int MODE, int PREC, bool EXACT>
struct AgPass
{
    const AgPullParams &p;
    uint64_t pol_first, pol_last;
    const float *c_in32;
    const uint16_t *c_in16;
    float *c_out32;
    uint16_t *c_out16;
    uint32_t read_low, write_low;
    double eps;
    double my_err;
    uint32_t my_active;

    __device__ __forceinline__ AgPass(const AgPullParams &pp) : p(pp)
    {
        pol_first = ag_policy_evict_first();
        pol_last = ag_policy_evict_last();
        my_err = 0.0;
        my_active = 0;
        read_low = write_low = 0;
        eps = 0.0;
        c_in32 = nullptr;
        c_in16 = nullptr;
        c_out32 = nullptr;
        c_out16 = nullptr;
        if (MODE == AG_MODE_PR) {
            const uint32_t pass = p.ctl->iter;
            eps = p.ctl->eps;
            if (PREC != 0) {
                read_low = p.ctl->mode_read;
                write_low = p.ctl->mode_write;
            }
            const bool odd = (pass & 1u) != 0;
            c_in32 = odd ? p.c32_1 : p.c32_0;
            c_out32 = odd ? p.c32_0 : p.c32_1;
            c_in16 = odd ? p.c16_1 : p.c16_0;
            c_out16 = odd ? p.c16_0 : p.c16_1;
        }
    }

    /* value gathered for in-edge j with source u (weight wj for SpMV) */
    __device__ __forceinline__ float gather(uint32_t u, float wj) const
    {
        if (MODE == AG_MODE_SPMV) {
            const float xv = ag_ld_gather_f32(p.x + u, pol_last);
            if (p.wmode == AG_SPMV_W_UNIT)
                return xv;
            return __fmul_rn(wj, xv);
        }
        if (PREC != 0 && read_low)
            return ag_low_to_f32<PREC>(ag_ld_gather_u16(c_in16 + u, pol_last));
        return ag_ld_gather_f32(c_in32 + u, pol_last);
    }

    /* the reference's per-vertex update for a finished row sum */
    __device__ __forceinline__ void finish(uint32_t r, float s)
    {
        if (MODE == AG_MODE_SPMV) {
            p.rank[r] = s;
            return;
        }
        const float rp = p.rank[r];
        const float rn = __fadd_rn(p.base, __fmul_rn(p.damp, s));
        p.rank[r] = rn;
        const double err = (double)fabsf(__fsub_rn(rn, rp));
        my_err += err;
        my_active += (err >= eps) ? 1u : 0u;
        const uint32_t od = p.outdeg[r];
        const float c = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
        if (PREC != 0 && write_low)
            ag_st_keep_u16(c_out16 + r, ag_f32_to_low<PREC>(c), pol_last);
        else
            ag_st_keep_f32(c_out32 + r, c, pol_last);
    }

    /* phase 1: vals[j - eb] = gathered value of in-edge j, j in [eb, ee) */
    __device__ __forceinline__ void stage(float *vals, uint32_t eb, uint32_t ee) const
    {
        const uint4 *ids4 = reinterpret_cast<const uint4 *>(p.ids);
        const float4 *w4 = reinterpret_cast<const float4 *>(p.w);
        const uint32_t q1 = (ee + 3u) >> 2;
        for (uint32_t q = (eb >> 2) + threadIdx.x; q < q1; q += AG_BLK) {
            const uint4 u = ag_ld_stream_u4(ids4 + q, pol_first);
            float4 wv = make_float4(0.0001f, 0.0001f, 0.0001f, 0.0001f);
            if (MODE == AG_MODE_SPMV && p.wmode == AG_SPMV_W_GRAPH)
                wv = ag_ld_stream_f4(w4 + q, pol_first);
            const uint32_t j0 = q << 2;
            const bool in0 = j0 >= eb && j0 < ee;
            const bool in1 = j0 + 1 >= eb && j0 + 1 < ee;
            const bool in2 = j0 + 2 >= eb && j0 + 2 < ee;
            const bool in3 = j0 + 3 < ee && j0 + 3 >= eb;
            float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
            if (in0) v0 = gather(u.x, wv.x);
            if (in1) v1 = gather(u.y, wv.y);
            if (in2) v2 = gather(u.z, wv.z);
            if (in3) v3 = gather(u.w, wv.w);
            if (in0) vals[j0 - eb] = v0;
            if (in1) vals[j0 + 1 - eb] = v1;
            if (in2) vals[j0 + 2 - eb] = v2;
            if (in3) vals[j0 + 3 - eb] = v3;
        }
    }

    /* lane-strided partial sum of in-edges [eb, ee) straight from memory:
     * each thread adds its own 4-edge groups in edge order */
    __device__ __forceinline__ float strided_partial(uint32_t eb, uint32_t ee) const
    {
        const uint4 *ids4 = reinterpret_cast<const uint4 *>(p.ids);
        const float4 *w4 = reinterpret_cast<const float4 *>(p.w);
        const uint32_t q1 = (ee + 3u) >> 2;
        float s = 0.0f;
        for (uint32_t q = (eb >> 2) + threadIdx.x; q < q1; q += AG_BLK) {
            const uint4 u = ag_ld_stream_u4(ids4 + q, pol_first);
            float4 wv = make_float4(0.0001f, 0.0001f, 0.0001f, 0.0001f);
            if (MODE == AG_MODE_SPMV && p.wmode == AG_SPMV_W_GRAPH)
                wv = ag_ld_stream_f4(w4 + q, pol_first);
            const uint32_t j0 = q << 2;
            const bool in0 = j0 >= eb && j0 < ee;
            const bool in1 = j0 + 1 >= eb && j0 + 1 < ee;
            const bool in2 = j0 + 2 >= eb && j0 + 2 < ee;
            const bool in3 = j0 + 3 < ee && j0 + 3 >= eb;
            float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
            if (in0) v0 = gather(u.x, wv.x);
            if (in1) v1 = gather(u.y, wv.y);
            if (in2) v2 = gather(u.z, wv.z);
            if (in3) v3 = gather(u.w, wv.w);
            if (in0) s = __fadd_rn(s, v0);
            if (in1) s = __fadd_rn(s, v1);
            if (in2) s = __fadd_rn(s, v2);
            if (in3) s = __fadd_rn(s, v3);
        }
        return s;
    }
};

template <int MODE, int PREC, bool EXACT>
__global__ void __launch_bounds__(AG_BLK) ag_pull_kernel(const AgPullParams p)
{
    __shared__ float vals[AG_CAP];
    __shared__ uint16_t s_long[AG_LONG_MAX];
    __shared__ uint32_t s_nlong;
    __shared__ float s_redf[AG_NW];
    __shared__ double s_redd[AG_NW];
    __shared__ uint32_t s_redu[AG_NW];
    __shared__ uint32_t s_last;

    AgPass<MODE, PREC, EXACT> ps(p);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (uint32_t t = blockIdx.x; t < p.ntasks; t += gridDim.x) {
        const uint4 task = p.tasks[t];
        const uint32_t kind = task.x & 3u;
        if (kind == AG_T_BLOCK) {
            const uint32_t rb = task.y, re = task.z;
            const uint32_t eb = p.row_off[rb], ee = p.row_off[re];
            if (!EXACT && tid == 0)
                s_nlong = 0;
            ps.stage(vals, eb, ee);
            __syncthreads();
            for (uint32_t i = tid; i < re - rb; i += AG_BLK) {
                const uint32_t r = rb + i;
                const uint32_t o0 = p.row_off[r] - eb, o1 = p.row_off[r + 1] - eb;
                if (EXACT || o1 - o0 <= AG_TSEQ) {
                    /* stream order: the accumulator restarts with the first
                     * value and adds the rest one by one */
                    float s = 0.0f;
                    if (o1 > o0) {
                        s = vals[o0];
                        for (uint32_t j = o0 + 1; j < o1; ++j)
                            s = __fadd_rn(s, vals[j]);
                    }
                    ps.finish(r, s);
                } else {
                    const uint32_t k = atomicAdd(&s_nlong, 1u);
                    s_long[k] = (uint16_t)i;
                }
            }
            if (!EXACT) {
                __syncthreads();
                const uint32_t nl = s_nlong;
                for (uint32_t k = warp; k < nl; k += AG_NW) {
                    const uint32_t r = rb + s_long[k];
                    const uint32_t o0 = p.row_off[r] - eb, o1 = p.row_off[r + 1] - eb;
                    float s = 0.0f;
                    for (uint32_t j = o0 + lane; j < o1; j += 32)
                        s = __fadd_rn(s, vals[j]);
                    s = ag_warp_sum_f(s);
                    if (lane == 0)
                        ps.finish(r, s);
                }
            }
            __syncthreads();
        } else if (kind == AG_T_ROW) {
            const uint32_t r = task.y;
            const uint32_t eb = p.row_off[r], ee = p.row_off[r + 1];
            if (EXACT) {
                float s = 0.0f;
                for (uint32_t cb = eb; cb < ee; cb += AG_CAP) {
                    const uint32_t ce = min(ee, cb + (uint32_t)AG_CAP);
                    ps.stage(vals, cb, ce);
                    __syncthreads();
                    if (tid == 0) {
                        uint32_t j = 0;
                        if (cb == eb) {
                            s = vals[0];
                            j = 1;
                        }
                        for (; j < ce - cb; ++j)
                            s = __fadd_rn(s, vals[j]);
                    }
                    __syncthreads();
                }
                if (tid == 0)
                    ps.finish(r, s);
            } else {
                float s = ps.strided_partial(eb, ee);
                s = ag_block_sum_f(s, s_redf);
                if (tid == 0)
                    ps.finish(r, s);
            }
            __syncthreads();
        } else {
            /* hub chunk (FAST order only) */
            const uint32_t chunk = task.x >> 2, r = task.y, pbase = task.z, nch = task.w;
            const uint32_t rb0 = p.row_off[r], re0 = p.row_off[r + 1];
            const uint32_t cb = rb0 + chunk * (uint32_t)AG_HUB;
            const uint32_t ce = min(re0, cb + (uint32_t)AG_HUB);
            float s = ps.strided_partial(cb, ce);
            s = ag_block_sum_f(s, s_redf);
            if (tid == 0) {
                p.hub_part[pbase + chunk] = s;
                __threadfence();
                const uint32_t prev = atomicAdd(&p.hub_cnt[pbase], 1u);
                if (prev == nch - 1) {
                    __threadfence();
                    float tot = __ldcg(p.hub_part + pbase);
                    for (uint32_t c = 1; c < nch; ++c)
                        tot = __fadd_rn(tot, __ldcg(p.hub_part + pbase + c));
                    p.hub_cnt[pbase] = 0;
                    ps.finish(r, tot);
                }
            }
            __syncthreads();
        }
    }

    if (MODE != AG_MODE_PR)
        return;

    /* close the pass: CTA totals, then the last CTA records the pass and
     * sets the loop condition */
    {
        const double e = ag_warp_sum_d(ps.my_err);
        const uint32_t a = ag_warp_sum_u(ps.my_active);
        if (lane == 0) {
            s_redd[warp] = e;
            s_redu[warp] = a;
        }
        __syncthreads();
        if (tid == 0) {
            double be = 0.0;
            uint32_t ba = 0;
            for (int w = 0; w < AG_NW; ++w) {
                be += s_redd[w];
                ba += s_redu[w];
            }
            if (be != 0.0)
                atomicAdd(&p.ctl->err_acc, be);
            if (ba)
                atomicAdd(&p.ctl->active_acc, ba);
            __threadfence();
            const uint32_t ticket = atomicAdd(&p.ctl->done_ctas, 1u);
            s_last = (ticket == gridDim.x - 1) ? 1u : 0u;
        }
        __syncthreads();
    }
    if (s_last && tid == 0) {
        __threadfence();
        AgControl *c = p.ctl;
        volatile AgControl *vc = c;
        const uint32_t P = vc->iter;
        const uint32_t active = vc->active_acc;
        const double err = vc->err_acc / (double)p.N;
        if (P < AG_MAX_HISTORY) {
            c->hist_active[P] = active;
            c->hist_err[P] = err;
            c->hist_t[P] = ag_globaltimer();
        }
        bool conv = (active == 0);
        if (PREC != 0) {
            const uint32_t read_low = vc->mode_read;
            uint32_t next_write = vc->mode_write;
            if (read_low)
                c->low_passes = vc->low_passes + 1;
            /* leave 16-bit storage once the residual is small, once it stops
             * falling, or once the 16-bit map has reached its fixed point */
            if (next_write && (err < vc->switch_residual || conv || (P >= 2 && err >= 0.98 * vc->prev_err)))
                next_write = 0;
            /* convergence only counts on FP32 contributions */
            if (read_low)
                conv = false;
            c->mode_read = vc->mode_write;
            c->mode_write = next_write;
            if (c->mode_read == 0 && vc->switch_pass == 0)
                c->switch_pass = P + 1;
        }
        c->prev_err = err;
        c->iter = P + 1;
        c->converged = conv ? 1u : 0u;
        const bool cont = !conv && (P + 1 < vc->max_iter);
        c->active_acc = 0;
        c->err_acc = 0.0;
        c->done_ctas = 0;
        __threadfence();
        cudaGraphSetConditional(p.cond, cont ? 1u : 0u);
    }
}

/* init: r = base (or the warm start), first contributions, control reset */
template <int PREC>
__global__ void __launch_bounds__(AG_BLK) ag_pr_init_kernel2(const AgPullParams p, const AgRunConfig run)
{
    const uint64_t pol_last = ag_policy_evict_last();
    for (uint32_t v = blockIdx.x * AG_BLK + threadIdx.x; v < p.N; v += gridDim.x * AG_BLK) {
        const float r0 = run.use_init ? p.init_ranks[v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        const float c = od ? __fdiv_rn(r0, __uint2float_rn(od)) : 0.0f;
        if (PREC != 0)
            ag_st_keep_u16(p.c16_0 + v, ag_f32_to_low<PREC>(c), pol_last);
        else
            ag_st_keep_f32(p.c32_0 + v, c, pol_last);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        AgControl *c = p.ctl;
        c->iter = 0;
        c->max_iter = run.max_iter;
        c->active_acc = 0;
        c->done_ctas = 0;
        c->err_acc = 0.0;
        c->eps = run.eps;
        c->converged = 0;
        c->mode_read = PREC != 0 ? 1u : 0u;
        c->mode_write = PREC != 0 ? 1u : 0u;
        c->switch_pass = 0;
        c->switch_residual = run.switch_residual;
        c->prev_err = 1e300;
        c->rank_sum = 0.0;
        c->use_init = run.use_init;
        c->low_passes = 0;
        c->t0 = ag_globaltimer();
        cudaGraphSetConditional(p.cond, (run.max_iter > 0 && p.N > 0) ? 1u : 0u);
    }
}

/* ranks / N in binary32 (pageRank.c:1079-1085), FP64 sum */
__global__ void __launch_bounds__(AG_BLK) ag_normalize_kernel(const AgPullParams p)
{
    __shared__ double sh[AG_NW];
    const float fN = __uint2float_rn(p.N);
    double s = 0.0;
    for (uint32_t v = blockIdx.x * AG_BLK + threadIdx.x; v < p.N; v += gridDim.x * AG_BLK) {
        const float r = __fdiv_rn(p.rank[v], fN);
        p.rank[v] = r;
        s += (double)r;
    }
    s = ag_warp_sum_d(s);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < AG_NW; ++w)
            t += sh[w];
        atomicAdd(&p.ctl->rank_sum, t);
    }
}

/* ------------------------------------------------ upload-time checks */
__global__ void ag_validate_ids_kernel(const uint32_t *ids, uint64_t E, uint32_t N, uint32_t *flag)
{
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < E; j += (uint64_t)gridDim.x * blockDim.x) {
        if (ids[j] >= N) {
            atomicOr(flag, 1u);
            atomicMin(flag + 1, (uint32_t)j);
        }
    }
}

/* ------------------------------------------------- FP64 oracle kernels */
__global__ void ag_f64_contrib(uint32_t N, const double *r, const uint32_t *outdeg, double *c)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
        const uint32_t od = outdeg[v];
        c[v] = od ? r[v] / (double)od : 0.0;
    }
}

__global__ void ag_f64_pull(uint32_t N, const uint32_t *row_off, const uint32_t *ids, const double *c,
                            const double *r, double *rn, unsigned long long *maxdiff)
{
    const double damp = (double)0.85f;
    const double base = (double)(1.0f - 0.85f);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = wid; v < N; v += nw) {
        double s = 0.0;
        for (uint32_t j = row_off[v] + lane; j < row_off[v + 1]; j += 32)
            s += c[ids[j]];
        s = ag_warp_sum_d(s);
        if (lane == 0) {
            const double x = base + damp * s;
            const double d = fabs(x - r[v]);
            rn[v] = x;
            /* non-negative doubles order like their bit patterns */
            atomicMax(maxdiff, (unsigned long long)__double_as_longlong(d));
        }
    }
}

__global__ void ag_f64_fill(uint32_t N, double *r, double v0)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x)
        r[v] = v0;
}

/* ------------------------------------------------------- host glue */
extern "C" const void *ag_pull_kernel_ptr(int mode, int prec, int exact)
{
    if (mode == AG_MODE_SPMV)
        return exact ? (const void *)ag_pull_kernel<AG_MODE_SPMV, 0, true>
                     : (const void *)ag_pull_kernel<AG_MODE_SPMV, 0, false>;
    switch (prec) {
    case 1:
        return exact ? (const void *)ag_pull_kernel<AG_MODE_PR, 1, true> : (const void *)ag_pull_kernel<AG_MODE_PR, 1, false>;
    case 2:
        return exact ? (const void *)ag_pull_kernel<AG_MODE_PR, 2, true> : (const void *)ag_pull_kernel<AG_MODE_PR, 2, false>;
    default:
        return exact ? (const void *)ag_pull_kernel<AG_MODE_PR, 0, true> : (const void *)ag_pull_kernel<AG_MODE_PR, 0, false>;
    }
}

extern "C" const void *ag_init_kernel_ptr(int prec)
{
    switch (prec) {
    case 1: return (const void *)ag_pr_init_kernel2<1>;
    case 2: return (const void *)ag_pr_init_kernel2<2>;
    default: return (const void *)ag_pr_init_kernel2<0>;
    }
}

extern "C" const void *ag_normalize_kernel_ptr(void) { return (const void *)ag_normalize_kernel; }

extern "C" cudaError_t ag_validate_ids(const uint32_t *ids, uint64_t E, uint32_t N, uint32_t *flag, cudaStream_t s)
{
    if (E == 0)
        return cudaSuccess;
    uint64_t blocks = (E + 255) / 256;
    if (blocks > 148 * 32)
        blocks = 148 * 32;
    ag_validate_ids_kernel<<<(unsigned)blocks, 256, 0, s>>>(ids, E, N, flag);
    return cudaGetLastError();
}

extern "C" cudaError_t ag_pr_f64_run(const uint32_t *row_off, const uint32_t *ids, const uint32_t *outdeg, uint32_t N,
                                     uint32_t max_iter, double tol, double *r, double *r2, double *c,
                                     double *maxdiff_dev, uint32_t *passes_out, cudaStream_t s)
{
    const unsigned gb = 148 * 8;
    double *const r_final = r;
    uint32_t it = 0;
    cudaError_t e;
    ag_f64_fill<<<gb, 256, 0, s>>>(N, r, (double)(1.0f - 0.85f));
    for (it = 0; it < max_iter; ++it) {
        unsigned long long h = 0;
        ag_f64_contrib<<<gb, 256, 0, s>>>(N, r, outdeg, c);
        cudaMemsetAsync(maxdiff_dev, 0, sizeof(unsigned long long), s);
        ag_f64_pull<<<gb, 256, 0, s>>>(N, row_off, ids, c, r, r2, (unsigned long long *)maxdiff_dev);
        e = cudaMemcpyAsync(&h, maxdiff_dev, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess)
            return e;
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return e;
        { double *t = r; r = r2; r2 = t; }
        double md;
        memcpy(&md, &h, sizeof(md));
        if (md <= tol) {
            ++it;
            break;
        }
    }
    /* the final ranks always end in the caller's first buffer */
    if (r != r_final) {
        e = cudaMemcpyAsync(r_final, r, (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess)
            return e;
    }
    *passes_out = it;
    return cudaGetLastError();
}
