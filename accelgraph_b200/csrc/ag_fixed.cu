/*
 * ag_fixed.cu -- integer pulls: the reference's fixed-point and quantised
 * PageRank forms (02_capi_graph/src/algorithms/capi/pageRank.c):
 *   pushpull 2        64-bit fixed point          :1276-1453
 *   pushpull 9/10/11  32/16/8-bit fixed point     :1455-1991
 *   pushpull 4/12/13  32/16/8-bit quantised       :2119-2677
 *
 * Per pass the reference turns every contribution r[v] / out_degree[v]
 * (binary32 division) into a W-bit integer, the accelerator sums each row's
 * integers zero-extended into 64 bits modulo 2^64 (its FixedPoint and
 * Quantized contracts, pagerank_kernel_tb.sv:13-19), and the host forms the
 * new rank from the sum:
 *   64-bit fixed   r' = base + damp * to_double(sum) in binary64, stored in
 *                  binary32; 32 fractional bits, conversion truncating
 *   W-bit fixed    r' = base + damp * to_float(sum) in binary32; W/2
 *                  fractional bits (Q16.16, Q8.8, Q4.4), conversion
 *                  truncating, the sum rounded once to binary32
 *   W-bit quant    r' = base + damp * (scale * (float)sum) in binary32, with
 *                  scale = (max - min) / (2^W - 1) over the pass's float
 *                  contributions, q = round-half-even(c / scale) clamped to
 *                  [0, 2^W - 1], zero point 0 (pageRank.c:2225-2226)
 * The conversions and the quantiser are OpenGraph's (absent from the
 * reference checkout) and are restated as above.
 *
 * The quantised forms need the minimum and maximum of all contributions
 * before any of them is quantised: the pull kernel writes binary32
 * contributions and folds their order-preserving keys into a min/max slot
 * (one per pass parity); a separate element-wise kernel, the first node of
 * the next loop iteration, quantises them with the scale of that slot.
 *
 * The first 64 KB of the gathered vector (the most-gathered ids after the
 * upload's relabelling by out-degree: 8K 64-bit, 16K 32-bit, 32K 16-bit or
 * 64K 8-bit values) are copied into shared memory at the start of each pass.
 *
 * Integer sums do not depend on their order, so one kernel serves both
 * orders and its results are the same bits whatever the work split: a row
 * item's values are staged in shared memory by the whole warp and each lane
 * sums its row, long rows are summed warp-strided, hub rows in chunks whose
 * partials the last chunk adds.  The update, residual, stop test, per-pass
 * record and the loop's WHILE condition follow the FP32 pull kernel.  GATHER
 * mode only sums: y[r] = the row's sum of x (rows without in-edges give 0).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "ag_device.h"
#include "ag_intpass.h"
#include "ag_mem.h"

#define AG_INT_FIXED 0
#define AG_INT_QUANT 1

/* one warp's stage: a row item's AG_WCAP in-edges start anywhere in their
 * first 16-byte quad, so they span up to AG_WCAP + 3 slots */
#define AG_FX_WSTRIDE (AG_WCAP + 4)
#define AG_FX_HOT_BYTES 65536u /* shared-memory table of the gathered vector */
/* cache policy of the integer kernels (tuning builds may override):
 *   AG_FX_IDS_NA    1: ids streamed without L1 lines, first out of L2
 *   AG_FX_ROW_NA    1: row offsets, degrees and ranks read without L1 lines
 *   AG_FX_GATHER    0: plain read-only gathers; 1: every gather may take an
 *                   L1 line, kept in L2; 2: only the warm tier takes L1 lines */
#ifndef AG_FX_IDS_NA
#define AG_FX_IDS_NA 1
#endif
#ifndef AG_FX_ROW_NA
#define AG_FX_ROW_NA 1
#endif
#ifndef AG_FX_GATHER
#define AG_FX_GATHER 2
#endif
extern __shared__ __align__(16) uint64_t ag_fx_stage[];

/* T: contribution type (uint64_t, uint32_t, uint16_t, uint8_t); KIND:
 * AG_INT_FIXED or AG_INT_QUANT (narrow T only); GATHER: sums only */
template <typename T, int KIND, bool GATHER>
__global__ void __launch_bounds__(AG_BLK, 1) ag_int_kernel(const AgPullParams p)
{
    constexpr bool WIDE = sizeof(T) == 8;
    constexpr bool QUANT = KIND == AG_INT_QUANT;
    constexpr uint32_t HOT = AG_FX_HOT_BYTES / sizeof(T);
    /* staged values: one element each, so 32 bits hold the narrow ones */
    using S = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;
    if (!GATHER && !p.use_cond && *((volatile uint32_t *)&p.ctl->stop))
        return;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nwarps = gridDim.x * AG_WARPS;
    S *vals = reinterpret_cast<S *>(ag_fx_stage) + (size_t)warp * AG_FX_WSTRIDE;
    T *hot = reinterpret_cast<T *>(reinterpret_cast<S *>(ag_fx_stage) + (size_t)AG_WARPS * AG_FX_WSTRIDE);
    const uint32_t pass = GATHER ? 0u : p.ctl->iter;
    /* quantised forms read one buffer (re-quantised between passes); fixed
     * forms ping-pong */
    const T *cin = reinterpret_cast<const T *>(GATHER ? p.x64 : (QUANT || !(pass & 1u)) ? p.c64_0 : p.c64_1);
    T *cout = reinterpret_cast<T *>((pass & 1u) ? p.c64_0 : p.c64_1);
    /* the most-gathered values (the first ids after the relabelling by
     * out-degree) are copied into shared memory once per pass, 16 bytes at a
     * time (the buffers hold at least 16 bytes past their last element) */
    const uint32_t hot_n = min(p.N, HOT);
    {
        const uint32_t nvec = (hot_n * (uint32_t)sizeof(T) + 15u) >> 4;
        const uint4 *src = reinterpret_cast<const uint4 *>(cin);
        uint4 *dst = reinterpret_cast<uint4 *>(hot);
        for (uint32_t i = tid; i < nvec; i += AG_BLK)
            dst[i] = __ldg(src + i);
    }
    __syncthreads();
    /* ids streamed once (no L1 line, first out of L2); gathers kept in L2,
     * and below the warm tier (the same bytes of the vector as the FP32
     * pull's tier, so 4 / sizeof(T) times its entries) allowed into L1 */
    const uint64_t pol_first = ag_policy_evict_first(), pol_last = ag_policy_evict_last();
    const uint32_t warm_n = (uint32_t)min((uint64_t)p.warm_n * 4u / sizeof(T), (uint64_t)p.N);
    auto gather = [&](uint32_t u) -> uint64_t {
        if (u < hot_n)
            return (uint64_t)hot[u];
        if (AG_FX_GATHER == 0)
            return (uint64_t)__ldg(cin + u);
        return ag_ld_gather_uint<T>(cin + u, pol_last, AG_FX_GATHER == 1 || u < warm_n);
    };
    auto ld_row = [&](const uint32_t *q) -> uint32_t { return AG_FX_ROW_NA ? ag_ld_row_u32(q) : __ldg(q); };
    auto ld_rank = [&](const float *q) -> float { return AG_FX_ROW_NA ? ag_ld_rank(q) : *q; };
    float qscale = 0.0f;
    if constexpr (QUANT && !GATHER)
        qscale = ag_quant_scale<T>(p.qmm, pass & 1u);
    const double eps = GATHER ? 0.0 : p.ctl->eps;
    double my_err = 0.0;
    uint32_t my_active = 0, my_mn = 0xFFFFFFFFu, my_mx = 0u;

    /* the reference's update of row r from its integer sum; rp and od are the
     * row's previous rank and out-degree, loaded ahead of time */
    auto finish = [&](uint32_t r, uint64_t s, float rp, uint32_t od) {
        if (GATHER) {
            p.y64[r] = s;
            return;
        }
        float rn;
        if constexpr (WIDE)
            rn = __double2float_rn(__dadd_rn((double)p.base, __dmul_rn((double)p.damp, ag_fixed2d(s))));
        else if constexpr (QUANT)
            rn = __fadd_rn(p.base, __fmul_rn(p.damp, __fmul_rn(qscale, __ull2float_rn(s))));
        else
            rn = __fadd_rn(p.base, __fmul_rn(p.damp, ag_from_fixed<T>(s)));
        const double err = (double)fabsf(__fsub_rn(rn, rp));
        my_err += err;
        my_active += (err >= eps) ? 1u : 0u;
        p.rank[r] = rn;
        if constexpr (QUANT) {
            const float c = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
            p.cqf[r] = c;
            const uint32_t k = ag_fkey(c);
            my_mn = min(my_mn, k);
            my_mx = max(my_mx, k);
        } else if constexpr (WIDE) {
            cout[r] = od ? ag_d2fixed((double)__fdiv_rn(rn, __uint2float_rn(od))) : 0ull;
        } else {
            cout[r] = od ? ag_to_fixed<T>(__fdiv_rn(rn, __uint2float_rn(od))) : (T)0;
        }
    };

    /* a pair of 16-byte id quads per lane: quads qa and qa + 32 */
    struct IdPair
    {
        uint4 a, b;
    };
    const uint4 *ids4 = reinterpret_cast<const uint4 *>(p.ids);
    auto ld_quad = [&](uint32_t q) -> uint4 { return AG_FX_IDS_NA ? ag_ld_stream_u4(ids4 + q, pol_first) : __ldg(ids4 + q); };
    auto load_pair = [&](uint32_t qa, uint32_t q1) -> IdPair {
        IdPair r;
        r.a = qa < q1 ? ld_quad(qa) : make_uint4(0, 0, 0, 0);
        r.b = qa + 32 < q1 ? ld_quad(qa + 32) : make_uint4(0, 0, 0, 0);
        return r;
    };
    /* the lane's first pair of an item's in-edges [eb, ee) */
    auto prefetch = [&](uint32_t eb, uint32_t ee) -> IdPair { return load_pair((eb >> 2) + lane, (ee + 3u) >> 2); };
    /* the eight values of a pair; in-edges outside [eb, ee) give 0 */
    auto gather8 = [&](const IdPair &q, uint32_t qa, uint32_t eb, uint32_t ee, S *v) {
        const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
        v[0] = (ja >= eb && ja < ee) ? (S)gather(q.a.x) : (S)0;
        v[1] = (ja + 1 >= eb && ja + 1 < ee) ? (S)gather(q.a.y) : (S)0;
        v[2] = (ja + 2 >= eb && ja + 2 < ee) ? (S)gather(q.a.z) : (S)0;
        v[3] = (ja + 3 >= eb && ja + 3 < ee) ? (S)gather(q.a.w) : (S)0;
        v[4] = (jb >= eb && jb < ee) ? (S)gather(q.b.x) : (S)0;
        v[5] = (jb + 1 >= eb && jb + 1 < ee) ? (S)gather(q.b.y) : (S)0;
        v[6] = (jb + 2 >= eb && jb + 2 < ee) ? (S)gather(q.b.z) : (S)0;
        v[7] = (jb + 3 >= eb && jb + 3 < ee) ? (S)gather(q.b.w) : (S)0;
    };

    /* each warp walks its items with a stride of all warps; the first id
     * pair of the next item is requested before the current one is gathered,
     * summed and written, so it is in flight meanwhile */
    uint32_t t = blockIdx.x * AG_WARPS + warp;
    uint4 task = t < p.ntasks ? __ldg(p.tasks + t) : make_uint4(0, 0, 0, 0);
    IdPair pf = prefetch(task.z, task.w);
    while (t < p.ntasks) {
        const uint32_t tn = t + nwarps;
        const uint4 task_n = tn < p.ntasks ? __ldg(p.tasks + tn) : make_uint4(0, 0, 0, 0);
        const uint32_t kind = task.x >> 30;
        const uint32_t r0 = task.x & AG_ROW_MASK;
        const uint32_t eb = task.z, ee = task.w;
        IdPair pn;
        if (kind == AG_T_ROWS) {
            /* one row per lane: its bounds, previous rank and out-degree load
             * first; the warp stages the item's values (slot j - eb for
             * in-edge j), then each lane sums its row if it is short, the
             * whole warp each long one */
            const uint32_t r = r0 + lane;
            const bool live = r < task.y;
            uint32_t o0 = ee, o1 = ee, od = 0;
            float rp = 0.0f;
            if (live) {
                o0 = ld_row(p.row_off + r);
                o1 = ld_row(p.row_off + r + 1);
                if (!GATHER) {
                    rp = ld_rank(p.rank + r);
                    od = ld_row(p.outdeg + r);
                }
            }
            pn = prefetch(task_n.z, task_n.w);
            {
                const uint32_t q1 = (ee + 3u) >> 2;
                uint32_t qa = (eb >> 2) + lane;
                IdPair cur = pf;
                while (qa < q1) {
                    S v[8];
                    gather8(cur, qa, eb, ee, v);
                    if (qa + 64 < q1)
                        cur = load_pair(qa + 64, q1);
                    const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (ja + k >= eb && ja + k < ee)
                            vals[ja + k - eb] = v[k];
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (jb + k >= eb && jb + k < ee)
                            vals[jb + k - eb] = v[4 + k];
                    qa += 64;
                }
            }
            __syncwarp();
            o0 -= eb;
            o1 -= eb;
            uint64_t s = 0;
            const bool is_long = o1 - o0 > AG_TSEQ;
            if (!is_long)
                for (uint32_t j = o0; j < o1; ++j)
                    s += (uint64_t)vals[j];
            unsigned m = __ballot_sync(0xffffffffu, is_long);
            while (m) {
                const int src = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t a = __shfl_sync(0xffffffffu, o0, src);
                const uint32_t b = __shfl_sync(0xffffffffu, o1, src);
                uint64_t ts = 0;
                for (uint32_t j = a + lane; j < b; j += 32)
                    ts += (uint64_t)vals[j];
                ts = ag_warp_sum_u64(ts);
                if ((int)lane == src)
                    s = ts;
            }
            if (live)
                finish(r, s, rp, od);
        } else {
            float rp = 0.0f;
            uint32_t od = 0;
            if (!GATHER && lane == 0 && kind == AG_T_LONG) {
                rp = ld_rank(p.rank + r0);
                od = ld_row(p.outdeg + r0);
            }
            pn = prefetch(task_n.z, task_n.w);
            /* warp-strided partial sums straight from memory: the values of
             * one round are added while the next round's gathers travel and
             * the ids of the round after load */
            uint64_t s = 0;
            {
                const uint32_t q1 = (ee + 3u) >> 2;
                uint32_t qa = (eb >> 2) + lane;
                if constexpr (sizeof(S) == 8) {
                    /* 64-bit values take twice the registers: one round in
                     * flight */
                    IdPair cur = pf;
                    while (qa < q1) {
                        const IdPair nx = load_pair(qa + 64, q1);
                        S v[8];
                        gather8(cur, qa, eb, ee, v);
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            s += (uint64_t)v[k];
                        cur = nx;
                        qa += 64;
                    }
                } else if (qa < q1) {
                    S v[8];
                    gather8(pf, qa, eb, ee, v);
                    IdPair nxt = load_pair(qa + 64, q1);
                    while (qa < q1) {
                        const uint32_t qn = qa + 64;
                        const IdPair nn = load_pair(qn + 64, q1);
                        S vn[8];
                        gather8(nxt, qn, eb, ee, vn);
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            s += (uint64_t)v[k];
                            v[k] = vn[k];
                        }
                        nxt = nn;
                        qa = qn;
                    }
                }
            }
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
        pf = pn;
        task = task_n;
        t = tn;
    }
    if (GATHER)
        return;

    /* close the pass: CTA totals (and the quantised forms' min/max keys of
     * the next contributions), then the last CTA records the pass and sets
     * the loop condition */
    ag_close_pass<AG_WARPS>(p, my_err, my_active, QUANT, my_mn, my_mx, true);
}

/* init: r = base (or the warm start), first contributions (quantised forms:
 * binary32 contributions and their min/max keys in slot 0, which the graph
 * clears before this kernel), control reset */
template <typename T, int KIND>
__global__ void __launch_bounds__(AG_SBLK) ag_int_init_kernel(const AgPullParams p, const AgRunConfig run)
{
    constexpr bool WIDE = sizeof(T) == 8;
    constexpr bool QUANT = KIND == AG_INT_QUANT;
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        const float r0 = run.use_init ? p.init_ranks[p.perm ? p.perm[v] : v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        if constexpr (QUANT) {
            const float c = od ? __fdiv_rn(r0, __uint2float_rn(od)) : 0.0f;
            p.cqf[v] = c;
            const uint32_t k = ag_fkey(c);
            mn = min(mn, k);
            mx = max(mx, k);
        } else if constexpr (WIDE) {
            p.c64_0[v] = od ? ag_d2fixed((double)__fdiv_rn(r0, __uint2float_rn(od))) : 0ull;
        } else {
            reinterpret_cast<T *>(p.c64_0)[v] = od ? ag_to_fixed<T>(__fdiv_rn(r0, __uint2float_rn(od))) : (T)0;
        }
    }
    if (QUANT)
        ag_fold_minmax_slot0<AG_SBLK / 32>(p.qmm, mn, mx);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        ag_reset_control(p, run);
}

/* quantise the binary32 contributions with the scale of this pass's min/max
 * slot.  One wave of CTAs; each thread takes groups of four contributions,
 * AG_QK groups a round, and issues all of a round's 16-byte loads before it
 * needs the scale, so that the loads are in flight together; each group is
 * stored with one 4-, 8- or 16-byte store. */
#define AG_QK 4
template <typename T> __global__ void __launch_bounds__(AG_SBLK) ag_quant_kernel(const AgPullParams p)
{
    if (!p.use_cond && *((volatile uint32_t *)&p.ctl->stop))
        return;
    T *q = reinterpret_cast<T *>(p.c64_0);
    const uint32_t n4 = p.N >> 2;
    const uint32_t stride = gridDim.x * AG_SBLK;
    const float4 *src = reinterpret_cast<const float4 *>(p.cqf);
    bool have_scale = false;
    float scale = 0.0f;
    for (uint32_t i0 = blockIdx.x * AG_SBLK + threadIdx.x; i0 < n4; i0 += AG_QK * stride) {
        float4 f[AG_QK];
#pragma unroll
        for (int k = 0; k < AG_QK; ++k)
            if (i0 + k * stride < n4)
                f[k] = __ldg(src + i0 + k * stride);
        if (!have_scale) {
            scale = ag_quant_scale<T>(p.qmm, p.ctl->iter & 1u);
            have_scale = true;
        }
#pragma unroll
        for (int k = 0; k < AG_QK; ++k) {
            const uint32_t i = i0 + k * stride;
            if (i >= n4)
                break;
            const T a = ag_quantize<T>(f[k].x, scale), b = ag_quantize<T>(f[k].y, scale);
            const T c = ag_quantize<T>(f[k].z, scale), d = ag_quantize<T>(f[k].w, scale);
            if constexpr (sizeof(T) == 4)
                reinterpret_cast<uint4 *>(q)[i] = make_uint4(a, b, c, d);
            else if constexpr (sizeof(T) == 2)
                reinterpret_cast<uint2 *>(q)[i] =
                    make_uint2((uint32_t)a | ((uint32_t)b << 16), (uint32_t)c | ((uint32_t)d << 16));
            else
                reinterpret_cast<uint32_t *>(q)[i] =
                    (uint32_t)a | ((uint32_t)b << 8) | ((uint32_t)c << 16) | ((uint32_t)d << 24);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < (p.N & 3u)) {
        const uint32_t v = (n4 << 2) + threadIdx.x;
        q[v] = ag_quantize<T>(p.cqf[v], ag_quant_scale<T>(p.qmm, p.ctl->iter & 1u));
    }
}

/* vectors between caller order and device order: W-bit in, 64-bit out */
template <typename T> __global__ void ag_permute_in_kernel(const uint32_t *perm, const T *x, T *x_new, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x_new[i] = x[perm ? perm[i] : i];
}

__global__ void ag_permute_out_u64_kernel(const uint32_t *inv, const uint64_t *y_new, uint64_t *y, uint32_t n)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        y[v] = y_new[inv ? inv[v] : v];
}

extern "C" const void *ag_int_kernel_ptr(int bytes, int quant, int gather)
{
    if (gather) {
        switch (bytes) {
        case 1: return (const void *)ag_int_kernel<uint8_t, AG_INT_FIXED, true>;
        case 2: return (const void *)ag_int_kernel<uint16_t, AG_INT_FIXED, true>;
        case 4: return (const void *)ag_int_kernel<uint32_t, AG_INT_FIXED, true>;
        default: return (const void *)ag_int_kernel<uint64_t, AG_INT_FIXED, true>;
        }
    }
    switch (bytes) {
    case 1: return quant ? (const void *)ag_int_kernel<uint8_t, AG_INT_QUANT, false>
                         : (const void *)ag_int_kernel<uint8_t, AG_INT_FIXED, false>;
    case 2: return quant ? (const void *)ag_int_kernel<uint16_t, AG_INT_QUANT, false>
                         : (const void *)ag_int_kernel<uint16_t, AG_INT_FIXED, false>;
    case 4: return quant ? (const void *)ag_int_kernel<uint32_t, AG_INT_QUANT, false>
                         : (const void *)ag_int_kernel<uint32_t, AG_INT_FIXED, false>;
    default: return (const void *)ag_int_kernel<uint64_t, AG_INT_FIXED, false>;
    }
}

extern "C" const void *ag_int_init_kernel_ptr(int bytes, int quant)
{
    switch (bytes) {
    case 1: return quant ? (const void *)ag_int_init_kernel<uint8_t, AG_INT_QUANT>
                         : (const void *)ag_int_init_kernel<uint8_t, AG_INT_FIXED>;
    case 2: return quant ? (const void *)ag_int_init_kernel<uint16_t, AG_INT_QUANT>
                         : (const void *)ag_int_init_kernel<uint16_t, AG_INT_FIXED>;
    case 4: return quant ? (const void *)ag_int_init_kernel<uint32_t, AG_INT_QUANT>
                         : (const void *)ag_int_init_kernel<uint32_t, AG_INT_FIXED>;
    default: return (const void *)ag_int_init_kernel<uint64_t, AG_INT_FIXED>;
    }
}

extern "C" const void *ag_quant_kernel_ptr(int bytes)
{
    switch (bytes) {
    case 1: return (const void *)ag_quant_kernel<uint8_t>;
    case 2: return (const void *)ag_quant_kernel<uint16_t>;
    default: return (const void *)ag_quant_kernel<uint32_t>;
    }
}

static unsigned ag_elem_blocks(uint32_t n)
{
    unsigned blocks = (n + 255) / 256;
    return blocks > ag_sm_grid(16) ? ag_sm_grid(16) : blocks;
}

extern "C" cudaError_t ag_permute_uint_in(const uint32_t *perm, const void *x, void *y, uint32_t n, int bytes,
                                          cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    const unsigned blocks = ag_elem_blocks(n);
    switch (bytes) {
    case 1: ag_permute_in_kernel<uint8_t><<<blocks, 256, 0, s>>>(perm, (const uint8_t *)x, (uint8_t *)y, n); break;
    case 2: ag_permute_in_kernel<uint16_t><<<blocks, 256, 0, s>>>(perm, (const uint16_t *)x, (uint16_t *)y, n); break;
    case 4: ag_permute_in_kernel<uint32_t><<<blocks, 256, 0, s>>>(perm, (const uint32_t *)x, (uint32_t *)y, n); break;
    default: ag_permute_in_kernel<uint64_t><<<blocks, 256, 0, s>>>(perm, (const uint64_t *)x, (uint64_t *)y, n); break;
    }
    return cudaGetLastError();
}

extern "C" cudaError_t ag_permute_u64_out(const uint32_t *inv, const uint64_t *x, uint64_t *y, uint32_t n,
                                          cudaStream_t s)
{
    if (n == 0)
        return cudaSuccess;
    ag_permute_out_u64_kernel<<<ag_elem_blocks(n), 256, 0, s>>>(inv, x, y, n);
    return cudaGetLastError();
}

/* dynamic shared memory of the integer kernels of `bytes`-byte elements (the
 * warps' stages, 64-bit for 64-bit elements and 32-bit otherwise, and the
 * 64 KB table) */
extern "C" size_t ag_fixed_smem_bytes(int bytes)
{
    return (size_t)AG_WARPS * AG_FX_WSTRIDE * (bytes == 8 ? 8u : 4u) + AG_FX_HOT_BYTES;
}
