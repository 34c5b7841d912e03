/*
 * ag_fixed.cu -- 64-bit fixed-point pull (the reference's pushpull 2,
 * 02_capi_graph/src/algorithms/capi/pageRank.c:1276-1453).
 *
 * Per pass the reference converts every contribution r[v] / out_degree[v]
 * (binary32 division) to 64-bit fixed point, the accelerator sums each row's
 * contributions as integers modulo 2^64 (its FixedPoint contract,
 * pagerank_kernel_tb.sv:13-16), and the host forms
 * r' = base + damp * to_double(sum) in binary64, stored in binary32.  The
 * conversions are OpenGraph's (absent from the reference checkout); they are
 * restated as 32 fractional bits, the conversion to fixed point truncating
 * toward zero.
 *
 * The first AG_FX_HOT values of the gathered vector (the most-gathered
 * after the upload's relabelling by out-degree) are copied into shared
 * memory at the start of each pass.
 *
 * Integer sums do not depend on their order, so one kernel serves both
 * orders and its results are the same bits whatever the work split: a row
 * item's values are staged in shared memory by the whole warp and each lane
 * sums its row, long rows are summed warp-strided, hub rows in chunks whose
 * partials the last chunk adds.  The
 * update, residual, stop test, per-pass record and the loop's WHILE
 * condition follow the FP32 pull kernel.  GATHER mode only sums: y[r] = the
 * row's sum of x (rows without in-edges give 0).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "ag_device.h"

#define AG_FX_ONE 4294967296.0 /* 2^32: fixed-point unit */

__device__ __forceinline__ uint64_t ag_d2fixed(double x)
{
    return (uint64_t)__double2ll_rz(__dmul_rn(x, AG_FX_ONE));
}

__device__ __forceinline__ double ag_fixed2d(uint64_t x)
{
    return __ddiv_rn(__ll2double_rn((long long)x), AG_FX_ONE);
}

__device__ __forceinline__ uint64_t ag_warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* one warp's stage: a row item's AG_WCAP in-edges start anywhere in their
 * first 16-byte quad, so they span up to AG_WCAP + 3 slots */
#define AG_FX_WSTRIDE (AG_WCAP + 4)
#define AG_FX_HOT 8192u /* entries of the shared-memory table (64 KB) */
extern __shared__ __align__(16) uint64_t ag_fx_stage[];

template <bool GATHER>
__global__ void __launch_bounds__(AG_BLK, 1) ag_fixed_kernel(const AgPullParams p)
{
    __shared__ double s_redd[AG_WARPS];
    __shared__ uint32_t s_redu[AG_WARPS];
    __shared__ uint32_t s_last;
    if (!GATHER && !p.use_cond && *((volatile uint32_t *)&p.ctl->stop))
        return;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nwarps = gridDim.x * AG_WARPS;
    uint64_t *vals = ag_fx_stage + (size_t)warp * AG_FX_WSTRIDE;
    uint64_t *hot = ag_fx_stage + (size_t)AG_WARPS * AG_FX_WSTRIDE;
    const uint32_t pass = GATHER ? 0u : p.ctl->iter;
    const uint64_t *cin = GATHER ? p.x64 : ((pass & 1u) ? p.c64_1 : p.c64_0);
    /* the most-gathered values (the first ids after the relabelling by
     * out-degree) are copied into shared memory once per pass */
    const uint32_t hot_n = min(p.N, (uint32_t)AG_FX_HOT);
    for (uint32_t i = tid; i < hot_n; i += AG_BLK)
        hot[i] = __ldg(cin + i);
    __syncthreads();
    auto gather = [&](uint32_t u) -> uint64_t { return u < hot_n ? hot[u] : __ldg(cin + u); };
    uint64_t *cout = (pass & 1u) ? p.c64_0 : p.c64_1;
    const double eps = GATHER ? 0.0 : p.ctl->eps;
    double my_err = 0.0;
    uint32_t my_active = 0;

    /* the reference's update of row r from its fixed-point sum; rp and od
     * are the row's previous rank and out-degree, loaded ahead of time */
    auto finish = [&](uint32_t r, uint64_t s, float rp, uint32_t od) {
        if (GATHER) {
            p.y64[r] = s;
            return;
        }
        const float rn = __double2float_rn(__dadd_rn((double)p.base, __dmul_rn((double)p.damp, ag_fixed2d(s))));
        const double err = (double)fabsf(__fsub_rn(rn, rp));
        my_err += err;
        my_active += (err >= eps) ? 1u : 0u;
        p.rank[r] = rn;
        cout[r] = od ? ag_d2fixed((double)__fdiv_rn(rn, __uint2float_rn(od))) : 0ull;
    };

    /* the next item's descriptor is requested before the current item runs */
    uint32_t t = blockIdx.x * AG_WARPS + warp;
    uint4 task_n = t < p.ntasks ? __ldg(p.tasks + t) : make_uint4(0, 0, 0, 0);
    for (; t < p.ntasks; t += nwarps) {
        const uint4 task = task_n;
        if (t + nwarps < p.ntasks)
            task_n = __ldg(p.tasks + t + nwarps);
        const uint32_t kind = task.x >> 30;
        const uint32_t r0 = task.x & AG_ROW_MASK;
        if (kind == AG_T_ROWS) {
            /* the warp stages the item's values: 16-byte id loads, four
             * gathers in flight per quad, slot j - (eb & ~3) for in-edge j;
             * then each lane sums its row from shared memory */
            const uint32_t eb = task.z, ee = task.w, q0 = eb >> 2, q1 = (ee + 3u) >> 2;
            const uint32_t r = r0 + lane;
            uint32_t o0 = ee, o1 = ee, od = 0;
            float rp = 0.0f;
            if (r < task.y) {
                o0 = __ldg(p.row_off + r);
                o1 = __ldg(p.row_off + r + 1);
                if (!GATHER) {
                    rp = p.rank[r];
                    od = __ldg(p.outdeg + r);
                }
            }
            for (uint32_t qa = q0 + lane; qa < q1; qa += 64) {
                /* two quads per lane and round: eight gathers in flight */
                const uint32_t qb = qa + 32;
                const uint4 ia = __ldg(reinterpret_cast<const uint4 *>(p.ids) + qa);
                const uint4 ib = qb < q1 ? __ldg(reinterpret_cast<const uint4 *>(p.ids) + qb) : make_uint4(0, 0, 0, 0);
                const uint32_t ja = qa << 2, jb = qb << 2;
                uint64_t v[8];
                v[0] = (ja >= eb && ja < ee) ? gather(ia.x) : 0ull;
                v[1] = (ja + 1 >= eb && ja + 1 < ee) ? gather(ia.y) : 0ull;
                v[2] = (ja + 2 >= eb && ja + 2 < ee) ? gather(ia.z) : 0ull;
                v[3] = (ja + 3 < ee) ? gather(ia.w) : 0ull;
                v[4] = (jb < ee) ? gather(ib.x) : 0ull;
                v[5] = (jb + 1 < ee) ? gather(ib.y) : 0ull;
                v[6] = (jb + 2 < ee) ? gather(ib.z) : 0ull;
                v[7] = (jb + 3 < ee) ? gather(ib.w) : 0ull;
                uint64_t *q = vals + ((qa - q0) << 2);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    q[k] = v[k];
                if (qb < q1) {
                    q = vals + ((qb - q0) << 2);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        q[k] = v[4 + k];
                }
            }
            __syncwarp();
            if (r < task.y) {
                uint64_t s = 0;
                for (uint32_t j = o0; j < o1; ++j)
                    s += vals[j - (q0 << 2)];
                finish(r, s, rp, od);
            }
        } else {
            float rp = 0.0f;
            uint32_t od = 0;
            if (!GATHER && lane == 0 && kind == AG_T_LONG) {
                rp = p.rank[r0];
                od = __ldg(p.outdeg + r0);
            }
            uint64_t s = 0;
#pragma unroll 4
            for (uint32_t j = task.z + lane; j < task.w; j += 32)
                s += gather(__ldg(p.ids + j));
            s = ag_warp_sum_u64(s);
            if (kind == AG_T_LONG) {
                if (lane == 0)
                    finish(r0, s, rp, od);
            } else if (lane == 0) {
                /* hub chunk: the last chunk to arrive adds the partials */
                const uint32_t pbase = task.y & AG_SLOT_MASK, chunk = task.y >> AG_SLOT_BITS;
                const uint32_t deg = __ldg(p.row_off + r0 + 1) - __ldg(p.row_off + r0);
                const uint32_t nch = (deg + p.whub - 1) / p.whub;
                p.hub_part64[pbase + chunk] = s;
                __threadfence();
                const uint32_t prev = atomicAdd(&p.hub_cnt[pbase], 1u);
                if (prev == nch - 1) {
                    __threadfence();
                    uint64_t tot = 0;
                    for (uint32_t c = 0; c < nch; ++c)
                        tot += __ldcg((const unsigned long long *)p.hub_part64 + pbase + c);
                    p.hub_cnt[pbase] = 0;
                    finish(r0, tot, GATHER ? 0.0f : p.rank[r0], GATHER ? 0u : __ldg(p.outdeg + r0));
                }
            }
        }
        __syncwarp();
    }
    if (GATHER)
        return;

    /* close the pass: CTA totals, then the last CTA records the pass and sets
     * the loop condition */
    {
        double e = my_err;
        uint32_t a = my_active;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            a += __shfl_xor_sync(0xffffffffu, a, o);
        }
        if (lane == 0) {
            s_redd[warp] = e;
            s_redu[warp] = a;
        }
        __syncthreads();
        if (tid == 0) {
            double be = 0.0;
            uint32_t ba = 0;
            for (int w = 0; w < AG_WARPS; ++w) {
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
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            c->hist_t[P] = t;
        }
        const bool conv = active == 0;
        c->prev_err = err;
        c->last_err_sum = vc->err_acc;
        c->iter = P + 1;
        c->converged = conv ? 1u : 0u;
        const bool cont = !conv && (P + 1 < vc->max_iter);
        c->active_acc = 0;
        c->err_acc = 0.0;
        c->done_ctas = 0;
        c->stop = cont ? 0u : 1u;
        __threadfence();
        if (p.use_cond)
            cudaGraphSetConditional(p.cond, cont ? 1u : 0u);
    }
}

/* init: r = base (or the warm start), first fixed-point contributions,
 * control reset */
__global__ void __launch_bounds__(AG_SBLK) ag_fixed_init_kernel(const AgPullParams p, const AgRunConfig run)
{
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        const float r0 = run.use_init ? p.init_ranks[p.perm ? p.perm[v] : v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        p.c64_0[v] = od ? ag_d2fixed((double)__fdiv_rn(r0, __uint2float_rn(od))) : 0ull;
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
        c->mode_read = 0;
        c->mode_write = 0;
        c->switch_pass = 0;
        c->switch_residual = run.switch_residual;
        c->prev_err = 1e300;
        c->rank_sum = 0.0;
        c->use_init = run.use_init;
        c->low_passes = 0;
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        c->t0 = t;
        c->stop = (run.max_iter > 0 && p.N > 0) ? 0u : 1u;
        if (p.use_cond)
            cudaGraphSetConditional(p.cond, (run.max_iter > 0 && p.N > 0) ? 1u : 0u);
    }
}

/* 64-bit vectors between caller order and device order */
__global__ void ag_permute_in_u64_kernel(const uint32_t *perm, const uint64_t *x, uint64_t *x_new, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x_new[i] = x[perm ? perm[i] : i];
}

__global__ void ag_permute_out_u64_kernel(const uint32_t *inv, const uint64_t *y_new, uint64_t *y, uint32_t n)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        y[v] = y_new[inv ? inv[v] : v];
}

extern "C" const void *ag_fixed_kernel_ptr(int gather)
{
    return gather ? (const void *)ag_fixed_kernel<true> : (const void *)ag_fixed_kernel<false>;
}

extern "C" const void *ag_fixed_init_kernel_ptr(void) { return (const void *)ag_fixed_init_kernel; }

extern "C" cudaError_t ag_permute_u64(const uint32_t *map, const uint64_t *x, uint64_t *y, uint32_t n, int out,
                                      cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    unsigned blocks = (n + 255) / 256;
    if (blocks > 148 * 16)
        blocks = 148 * 16;
    if (out)
        ag_permute_out_u64_kernel<<<blocks, 256, 0, s>>>(map, x, y, n);
    else
        ag_permute_in_u64_kernel<<<blocks, 256, 0, s>>>(map, x, y, n);
    return cudaGetLastError();
}

/* dynamic shared memory of the fixed-point kernel (the warps' stages) */
extern "C" size_t ag_fixed_smem_bytes(void)
{
    return ((size_t)AG_WARPS * AG_FX_WSTRIDE + AG_FX_HOT) * sizeof(uint64_t);
}
