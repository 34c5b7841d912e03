/*
 * ag_intpass.h -- device helpers shared by the integer pulls (ag_fixed.cu)
 * and the push forms (ag_push.cu): the fixed-point conversions, the
 * quantiser, the order-preserving keys of the quantised forms' min/max, the
 * control reset of an init kernel and the close of a pass.
 *
 * The conversions restate OpenGraph's fixedPoint.h and quantization.h
 * (absent from the reference checkout):
 *   64-bit fixed point  32 fractional bits, to fixed point truncating toward
 *                       zero, back exact up to binary64 rounding
 *   W-bit fixed point   W/2 fractional bits; to fixed point the exact binary32
 *                       product truncated toward zero, kept modulo 2^W; back
 *                       the 64-bit sum rounded once to binary32 and scaled
 *   W-bit quantiser     scale = (max - min) / (2^W - 1) in binary32,
 *                       q = round-half-even(c / scale) clamped to
 *                       [0, 2^W - 1], zero point 0; a zero scale gives 0
 */
#ifndef AG_INTPASS_H
#define AG_INTPASS_H
#include <cuda_runtime.h>
#include <stdint.h>

#include "ag_device.h"

#define AG_FX_ONE 4294967296.0 /* 2^32: 64-bit fixed-point unit */

__device__ __forceinline__ uint64_t ag_d2fixed(double x)
{
    return (uint64_t)__double2ll_rz(__dmul_rn(x, AG_FX_ONE));
}

__device__ __forceinline__ double ag_fixed2d(uint64_t x)
{
    return __ddiv_rn(__ll2double_rn((long long)x), AG_FX_ONE);
}

template <typename T> __device__ __forceinline__ T ag_to_fixed(float x)
{
    constexpr float one = (float)(1u << (4 * sizeof(T)));
    return (T)(unsigned long long)__float2ll_rz(__fmul_rn(x, one));
}

template <typename T> __device__ __forceinline__ float ag_from_fixed(uint64_t s)
{
    constexpr float one = (float)(1u << (4 * sizeof(T)));
    return __fdiv_rn(__ull2float_rn(s), one);
}

/* order-preserving 32-bit keys of binary32 values (for atomic min/max) */
__device__ __forceinline__ uint32_t ag_fkey(float f)
{
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float ag_fkey_value(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

/* scale of the contributions whose min/max keys are in slot `slot`
 * (mm[0..1] minimum keys, mm[2..3] maximum keys); 0 for an empty slot */
template <typename T> __device__ __forceinline__ float ag_quant_scale(const uint32_t *mm, uint32_t slot)
{
    constexpr float levels = (float)((1ull << (8 * sizeof(T))) - 1ull);
    const uint32_t kmin = mm[slot], kmax = mm[2 + slot];
    if (kmin > kmax)
        return 0.0f;
    return __fdiv_rn(__fsub_rn(ag_fkey_value(kmax), ag_fkey_value(kmin)), levels);
}

template <typename T> __device__ __forceinline__ T ag_quantize(float x, float scale)
{
    constexpr unsigned long long top = (1ull << (8 * sizeof(T))) - 1ull;
    if (!(scale > 0.0f))
        return (T)0;
    const float q = rintf(__fdiv_rn(x, scale));
    if (!(q > 0.0f))
        return (T)0;
    if (q >= (float)top)
        return (T)top;
    return (T)(unsigned long long)q;
}

__device__ __forceinline__ uint64_t ag_warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* fold a CTA of NW warps' min/max keys into slot 0 of mm (init kernels) */
template <int NW> __device__ __forceinline__ void ag_fold_minmax_slot0(uint32_t *mm, uint32_t mn, uint32_t mx)
{
    __shared__ uint32_t s_mn[NW], s_mx[NW];
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0) {
        s_mn[threadIdx.x >> 5] = mn;
        s_mx[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NW; ++w) {
            mn = min(mn, s_mn[w]);
            mx = max(mx, s_mx[w]);
        }
        if (mn != 0xFFFFFFFFu)
            atomicMin(&mm[0], mn);
        if (mx)
            atomicMax(&mm[2], mx);
    }
}

/* control block of a new solve (one thread) */
__device__ __forceinline__ void ag_reset_control(const AgPullParams &p, const AgRunConfig &run)
{
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

/* Close a pass: every thread of the CTA (NW warps) calls this after its last
 * element with its share of the pass's error and activity (and, for the
 * quantised forms, the min/max keys of the next contributions).  The CTA's
 * totals go to the control block; the last CTA to arrive records the pass,
 * clears the quantised forms' min/max slot of this pass (every CTA read it
 * at its start), decides whether another pass runs and sets the loop
 * condition.  err_per_n: the recorded error is the sum divided by N (pull and
 * push forms) rather than the sum itself (residual forms). */
template <int NW>
__device__ __forceinline__ void ag_close_pass(const AgPullParams &p, double err, uint32_t active, bool quant, uint32_t mn,
                              uint32_t mx, bool err_per_n)
{
    __shared__ double s_e[NW];
    __shared__ uint32_t s_a[NW], s_mn[NW], s_mx[NW];
    __shared__ uint32_t s_last;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        err += __shfl_xor_sync(0xffffffffu, err, o);
        active += __shfl_xor_sync(0xffffffffu, active, o);
    }
    if (quant) {
        mn = __reduce_min_sync(0xffffffffu, mn);
        mx = __reduce_max_sync(0xffffffffu, mx);
    }
    if (lane == 0) {
        s_e[warp] = err;
        s_a[warp] = active;
        s_mn[warp] = mn;
        s_mx[warp] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double be = 0.0;
        uint32_t ba = 0, bmn = 0xFFFFFFFFu, bmx = 0u;
        for (int w = 0; w < NW; ++w) {
            be += s_e[w];
            ba += s_a[w];
            bmn = min(bmn, s_mn[w]);
            bmx = max(bmx, s_mx[w]);
        }
        if (be != 0.0)
            atomicAdd(&p.ctl->err_acc, be);
        if (ba)
            atomicAdd(&p.ctl->active_acc, ba);
        if (quant) {
            const uint32_t nslot = (p.ctl->iter + 1u) & 1u;
            if (bmn != 0xFFFFFFFFu)
                atomicMin(&p.qmm[nslot], bmn);
            if (bmx)
                atomicMax(&p.qmm[2 + nslot], bmx);
        }
        __threadfence();
        const uint32_t ticket = atomicAdd(&p.ctl->done_ctas, 1u);
        s_last = (ticket == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        AgControl *c = p.ctl;
        volatile AgControl *vc = c;
        const uint32_t P = vc->iter;
        const uint32_t act = vc->active_acc;
        const double e = err_per_n ? vc->err_acc / (double)p.N : vc->err_acc;
        if (P < AG_MAX_HISTORY) {
            c->hist_active[P] = act;
            c->hist_err[P] = e;
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            c->hist_t[P] = t;
        }
        if (quant) {
            p.qmm[P & 1u] = 0xFFFFFFFFu;
            p.qmm[2 + (P & 1u)] = 0u;
        }
        const bool conv = act == 0;
        c->prev_err = e;
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

#endif /* AG_INTPASS_H */
