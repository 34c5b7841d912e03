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
 * Work decomposition (planned once per graph on the host, see ag_runtime.cu).
 * Every task is one WARP's work item; warps of a persistent grid take tasks
 * in a fixed stride and never wait for each other inside a pass, so the SM
 * always holds warps in every phase (loading ids, gathering, reducing):
 *   rows : up to 32 consecutive rows holding <= AG_WCAP in-edges.  The warp
 *          streams the ids with 16-byte loads (L1 no-allocate, L2
 *          evict-first), gathers c[id] (L2 evict-last) into its slice of
 *          shared memory -- up to 256 independent gathers in flight -- while
 *          each lane's row bounds, previous rank and out-degree load in the
 *          background.  A lane then sums its row in stream order (rows of
 *          <= AG_TSEQ edges: bit-identical to the reference's sequential
 *          sum); longer rows are summed by the whole warp (lane-strided
 *          partials + xor tree).  The update runs lane-parallel.
 *   long : one row of (item cap) < degree <= (hub chunk), warp-strided partials
 *          straight from memory + xor tree.
 *   hub  : longer rows split into hub-chunk-sized pieces on separate warps;
 *          the last chunk to arrive sums the chunk partials in chunk order.
 * In EXACT order every row is summed in stream order by one lane; a hub
 * row's chunks store their gathered values in a staging array, and the last
 * chunk to arrive adds them in stream order.
 * All reductions have a fixed order: results do not depend on scheduling.
 */
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "ag_device.h"
#include "ag_mem.h"

#define AG_SNW (AG_SBLK / 32)

/* ---------------------------------------------- TMA bulk copy to smem */
__device__ __forceinline__ uint32_t ag_smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ag_mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ag_smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void ag_mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ag_smem_addr(bar)), "r"(bytes)
                 : "memory");
}

/* one bulk global->shared copy (16-byte aligned, size a multiple of 16)
 * completing on the CTA's mbarrier */
__device__ __forceinline__ void ag_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     ag_smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(ag_smem_addr(bar))
                 : "memory");
}

/* bounded wait for the mbarrier phase to complete; false if the limit ran
 * out first */
__device__ __forceinline__ bool ag_mbar_wait(uint64_t *bar, uint32_t phase, uint32_t limit)
{
    const uint32_t a = ag_smem_addr(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(phase)
                     : "memory");
        if (done)
            return true;
    }
    return false;
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

/* ------------------------------------------------------------- kernel */
template <int MODE, int PREC, bool EXACT, bool LOW = false>
struct AgPass
{
    const AgPullParams &p;
    uint64_t pol_first, pol_last;
    const float *c_in32;
    const uint16_t *c_in16;
    float *c_out32;
    uint16_t *c_out16;
    /* this pass reads 16-bit contributions (fixed per kernel body, so that
     * the 16-bit and 32-bit passes each get their own loads and registers) */
    static constexpr bool read_low = PREC != 0 && LOW;
    uint32_t write_low;
    double eps;
    double my_err;
    uint32_t my_active;
    const float *hot32;     /* shared-memory copy of the first hot_n values */
    const uint16_t *hot16;
    uint32_t hot_n;
    bool dd_all;              /* data-driven mode: the first pass, where every row is active */

    __device__ __forceinline__ AgPass(const AgPullParams &pp) : p(pp)
    {
        hot32 = nullptr;
        hot16 = nullptr;
        hot_n = 0;
        pol_first = ag_policy_evict_first();
        pol_last = ag_policy_evict_last();
        my_err = 0.0;
        my_active = 0;
        write_low = 0;
        eps = 0.0;
        c_in32 = nullptr;
        c_in16 = nullptr;
        c_out32 = nullptr;
        c_out16 = nullptr;
        dd_all = false;
        if (MODE != AG_MODE_SPMV) {
            const uint32_t pass = p.ctl->iter;
            eps = p.ctl->eps;
            if (PREC != 0)
                write_low = p.ctl->mode_write;
            const bool odd = (pass & 1u) != 0;
            c_in32 = odd ? p.c32_1 : p.c32_0;
            c_out32 = odd ? p.c32_0 : p.c32_1;
            c_in16 = odd ? p.c16_1 : p.c16_0;
            c_out16 = odd ? p.c16_0 : p.c16_1;
            if (MODE == AG_MODE_DD)
                dd_all = pass == 0;
        }
    }

    /* the vector this pass gathers from, and its element size */
    __device__ __forceinline__ const void *gather_source() const
    {
        if (MODE == AG_MODE_SPMV)
            return p.x;
        if (PREC != 0 && read_low)
            return c_in16;
        return c_in32;
    }

    __device__ __forceinline__ uint32_t gather_elem_bytes() const { return (PREC != 0 && read_low) ? 2u : 4u; }

    /* value gathered for an in-edge with source u (weight wj for SpMV):
     * from the shared-memory table when u is hot, else from global memory */
    __device__ __forceinline__ float gather(uint32_t u, float wj) const
    {
        if (MODE == AG_MODE_SPMV) {
            const float xv = (u < hot_n) ? hot32[u]
                             : (u < p.warm_n ? ag_ld_gather_f32(p.x + u, pol_last) : ag_ld_cold_f32(p.x + u, pol_last));
            if (p.wmode == AG_SPMV_W_UNIT)
                return xv;
            return __fmul_rn(wj, xv);
        }
        if (PREC != 0 && read_low)
            return ag_low_to_f32<PREC>((u < hot_n) ? hot16[u]
                                       : (u < p.warm_n ? ag_ld_gather_u16(c_in16 + u, pol_last)
                                                       : ag_ld_cold_u16(c_in16 + u, pol_last)));
        return (u < hot_n) ? hot32[u]
                           : (u < p.warm_n ? ag_ld_gather_f32(c_in32 + u, pol_last) : ag_ld_cold_f32(c_in32 + u, pol_last));
    }

    /* the reference's per-vertex update for a finished row sum; rp and od
     * are the row's previous rank and out-degree, loaded ahead of time */
    __device__ __forceinline__ void finish(uint32_t r, float s, float rp, uint32_t od)
    {
        if (MODE == AG_MODE_SPMV) {
            p.rank[r] = s;
            return;
        }
        const float rn = __fadd_rn(p.base, __fmul_rn(p.damp, s));
        p.rank[r] = rn;
        const double err = (double)fabsf(__fsub_rn(rn, rp));
        my_err += err;
        my_active += (err >= eps) ? 1u : 0u;
        const float c = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
        if (PREC != 0 && write_low)
            ag_st_keep_u16(c_out16 + r, ag_f32_to_low<PREC>(c), pol_last);
        else
            ag_st_keep_f32(c_out32 + p.c_base + r, c, pol_last);
    }

    /* Data-driven mode (the reference's worklist pull, pageRank.c:2810-2969).
     * A row is on the worklist of a pass when the pass is the first or one of
     * its in-neighbours changed in the pass before.  A vertex that changes
     * writes its next contribution with the sign bit set (contributions are
     * otherwise never negative), so a row learns that from the values it
     * gathers anyway: it sums their magnitudes, which are the reference's
     * contributions bit for bit, and ORs their sign bits.  Nothing is
     * scattered to out-neighbours. */
    static __device__ __forceinline__ uint32_t dd_neg(float v) { return __float_as_uint(v) >> 31; }

    /* the update of a row (pageRank.c:2896-2916): rows off the worklist and
     * rows that moved by less than epsilon keep rank and contribution (sign
     * cleared); an active row's residual always counts */
    __device__ __forceinline__ void finish_dd(uint32_t r, float s, float rp, uint32_t od, bool act)
    {
        if (act) {
            const float rn = __fadd_rn(p.base, __fmul_rn(p.damp, s));
            const double err = (double)fabsf(__fsub_rn(rn, rp));
            my_err += err;
            if (err >= eps) {
                p.rank[r] = rn;
                const float c = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
                ag_st_keep_f32(c_out32 + r, __uint_as_float(__float_as_uint(c) | 0x80000000u), pol_last);
                ++my_active;
                return;
            }
        }
        ag_st_keep_f32(c_out32 + r, fabsf(__ldg(c_in32 + r)), pol_last);
    }

    /* two 16-byte groups of in-edges per lane: quads qa and qa + 32 (ids and,
     * for a weighted SpMV, weights); quads at or past q1 read as zero */
    struct Pair
    {
        uint4 a, b;
        float4 wa, wb;
    };

    __device__ __forceinline__ Pair load_pair(uint32_t qa, uint32_t q1) const
    {
        const uint4 *ids4 = reinterpret_cast<const uint4 *>(p.ids);
        const float4 *w4 = reinterpret_cast<const float4 *>(p.w);
        Pair r;
        r.a = make_uint4(0, 0, 0, 0);
        r.b = make_uint4(0, 0, 0, 0);
        r.wa = make_float4(0.0001f, 0.0001f, 0.0001f, 0.0001f);
        r.wb = r.wa;
        const bool ha = qa < q1, hb = qa + 32 < q1;
        if (ha)
            r.a = ag_ld_stream_u4(ids4 + qa, pol_first);
        if (hb)
            r.b = ag_ld_stream_u4(ids4 + qa + 32, pol_first);
        if (MODE == AG_MODE_SPMV && p.wmode == AG_SPMV_W_GRAPH) {
            if (ha)
                r.wa = ag_ld_stream_f4(w4 + qa, pol_first);
            if (hb)
                r.wb = ag_ld_stream_f4(w4 + qa + 32, pol_first);
        }
        return r;
    }

    /* first pair of a task's edge range, issued one task ahead */
    __device__ __forceinline__ Pair prefetch(uint32_t eb, uint32_t ee, uint32_t lane) const
    {
        return load_pair((eb >> 2) + lane, (ee + 3u) >> 2);
    }

    /* the eight values of a pair (in-edge j valid when eb <= j < ee) */
    __device__ __forceinline__ void gather8(const Pair &q, uint32_t qa, uint32_t eb, uint32_t ee, float *v,
                                            bool *in) const
    {
        const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            in[k] = ja + k >= eb && ja + k < ee;
            in[4 + k] = jb + k >= eb && jb + k < ee;
        }
        v[0] = in[0] ? gather(q.a.x, q.wa.x) : 0.f;
        v[1] = in[1] ? gather(q.a.y, q.wa.y) : 0.f;
        v[2] = in[2] ? gather(q.a.z, q.wa.z) : 0.f;
        v[3] = in[3] ? gather(q.a.w, q.wa.w) : 0.f;
        v[4] = in[4] ? gather(q.b.x, q.wb.x) : 0.f;
        v[5] = in[5] ? gather(q.b.y, q.wb.y) : 0.f;
        v[6] = in[6] ? gather(q.b.z, q.wb.z) : 0.f;
        v[7] = in[7] ? gather(q.b.w, q.wb.w) : 0.f;
    }

    /* first round of a warp stage, issued ahead of its use: the lane's
     * values of quads (eb >> 2) + lane and + 32 (zero outside [eb, ee)) */
    __device__ __forceinline__ void stage_issue(const Pair &first, uint32_t eb, uint32_t ee, uint32_t lane,
                                                float *v) const
    {
        bool in[8];
        gather8(first, (eb >> 2) + lane, eb, ee, v, in);
    }

    /* warp stage: vals[j - eb] = gathered value of in-edge j, j in [eb, ee).
     * `v` holds the lane's first round (stage_issue); the later rounds, if
     * any, load their ids and gather here.  A lane gathers all eight values
     * of a round before it stores any of them. */
    __device__ __forceinline__ void stage_commit(float *vals, uint32_t eb, uint32_t ee, uint32_t lane,
                                                 const float *v) const
    {
        const uint32_t q1 = (ee + 3u) >> 2;
        uint32_t qa = (eb >> 2) + lane;
        {
            const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (ja + k >= eb && ja + k < ee)
                    vals[ja + k - eb] = v[k];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (jb + k >= eb && jb + k < ee)
                    vals[jb + k - eb] = v[4 + k];
        }
        for (qa += 64; qa < q1; qa += 64) {
            const Pair cur = load_pair(qa, q1);
            float w[8];
            bool in[8];
            gather8(cur, qa, eb, ee, w, in);
            const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (in[k])
                    vals[ja + k - eb] = w[k];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (in[4 + k])
                    vals[jb + k - eb] = w[4 + k];
        }
    }

    __device__ __forceinline__ void stage(float *vals, uint32_t eb, uint32_t ee, uint32_t lane,
                                          const Pair &first) const
    {
        float v[8];
        stage_issue(first, eb, ee, lane, v);
        stage_commit(vals, eb, ee, lane, v);
    }

    /* warp-strided partial sum of in-edges [eb, ee) straight from memory;
     * the next pair is in flight while the current one is gathered and
     * added (fixed lane assignment, edge order within a lane) */
    __device__ __forceinline__ float strided_partial(uint32_t eb, uint32_t ee, uint32_t lane,
                                                     const Pair &first, uint32_t &neg) const
    {
        /* two rounds of gathers in flight: the values of round k are added
         * while those of round k + 1 travel and the ids of round k + 2 load.
         * In-edges outside [eb, ee) gather nothing and add +0.0, which leaves
         * this (tree-ordered) partial sum unchanged. */
        const uint32_t q1 = (ee + 3u) >> 2;
        uint32_t qa = (eb >> 2) + lane;
        float s = 0.0f;
        if (MODE == AG_MODE_SPMV) {
            /* weighted pairs take twice the registers: one round in flight */
            Pair cur = first;
            while (qa < q1) {
                const Pair nx = load_pair(qa + 64, q1);
                float v[8];
                bool in[8];
                gather8(cur, qa, eb, ee, v, in);
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (in[k])
                        s = __fadd_rn(s, v[k]);
                cur = nx;
                qa += 64;
            }
            return s;
        }
        if (qa >= q1)
            return s;
        float v[8];
        bool in[8];
        gather8(first, qa, eb, ee, v, in);
        Pair nxt = load_pair(qa + 64, q1);
        while (qa < q1) {
            const uint32_t qn = qa + 64;
            const Pair nn = load_pair(qn + 64, q1);
            float vn[8];
            gather8(nxt, qn, eb, ee, vn, in);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (MODE == AG_MODE_DD) {
                    neg |= dd_neg(v[k]);
                    s = __fadd_rn(s, fabsf(v[k]));
                } else {
                    s = __fadd_rn(s, v[k]);
                }
                v[k] = vn[k];
            }
            nxt = nn;
            qa = qn;
        }
        return s;
    }

    /* EXACT-order hub chunk: the gathered values of in-edges [eb, ee) of a
     * row starting at o0, stored at dst[j - o0] (coalesced) */
    __device__ __forceinline__ void stage_global(float *dst, uint32_t o0, uint32_t eb, uint32_t ee, uint32_t lane,
                                                 const Pair &first) const
    {
        const uint32_t q1 = (ee + 3u) >> 2;
        uint32_t qa = (eb >> 2) + lane;
        Pair cur = first;
        while (qa < q1) {
            const Pair nx = load_pair(qa + 64, q1);
            float v[8];
            bool in[8];
            gather8(cur, qa, eb, ee, v, in);
            const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (in[k])
                    dst[ja + k - o0] = v[k];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (in[4 + k])
                    dst[jb + k - o0] = v[4 + k];
            cur = nx;
            qa += 64;
        }
    }

    /* ---------------------------------------------------------------
     * EXACT order of a hub row: the stream-order binary32 sum
     * ((v0 + v1) + v2) + ... of up to millions of values, bit for bit,
     * without a chain of that many adds on one warp.
     *
     * While the running sum s is a positive normal number of biased exponent
     * e, it is M * 2^(e-150) with an integer M in [2^23, 2^24).  The binary32
     * add s + v rounds to M' = M + rint(x), x = v / 2^(e-150), as long as the
     * exact sum stays in the binade and x is not a tie (x = k + 1/2, where
     * the result is the even neighbour, which depends on M).  So within a
     * binade a run of adds is one integer add of its steps, and the steps of
     * a run can be summed in any order, by any warp.
     *
     * A hub row is split into chunks on separate warps, and a chunk into
     * rounds of 256 in-edges (round k of in-edges [eb, ee): those at or past
     * eb in [(eb & ~3) + 256 k, + 256)).
     *  - The first chunk sums its own in-edges in stream order (ordered_sum)
     *    and stores the sum.
     *  - Every other chunk stages its values and, for each round, sums the
     *    integer steps at the binade e where the chunk began in the pass
     *    before and at e + 1 (hub_steps).  A total does not apply when a
     *    step is a tie, 2^22 or more, or not from a finite non-negative
     *    value.
     *  - The last chunk to arrive walks the rounds in order (hub_compose).
     *    When s is in binade e or e + 1, the matching total applies and
     *    M plus the total stays below 2^24, the round is one integer add
     *    (no partial sum can leave the binade: the steps are >= 0).
     *    Otherwise the round's staged values are added one by one.  It then
     *    records where each chunk began, for the next pass.
     * Data-driven passes stage the values with their sign tags and sum the
     * magnitudes. */

    /* s rebuilt from its exponent bits and M (M in [2^23, 2^24)) */
    static __device__ __forceinline__ float exact_make(uint32_t ex, uint32_t m)
    {
        return __uint_as_float((ex << 23) | (m & 0x7fffffu));
    }

    /* 2^(150-e) for a biased exponent e in [24, 254] */
    static __device__ __forceinline__ float exact_scale(uint32_t e) { return __uint_as_float((277u - e) << 23); }

    /* the step of x (a value in units of s's last place) and whether it
     * breaks the integer form: a tie, too large, negative or not finite */
    static __device__ __forceinline__ uint32_t exact_step(float x, bool &bad)
    {
        bad |= !((x >= 0.0f) & (x < 4194304.0f)) | (__fsub_rn(x, floorf(x)) == 0.5f);
        return (uint32_t)__float2int_rn(x);
    }

    /* whether a hub chunk after the first stages its gathered values, from
     * its record of the pass before (hub_pred): when its starting binade is
     * unknown or it had a round added value by value.  The composing warp
     * re-gathers an unstaged round if it needs one after all.  SpMV and
     * 16-bit passes always stage. */
    static __device__ __forceinline__ bool hub_staged(uint32_t pr)
    {
        const uint32_t e = pr & 0xffu;
        return MODE == AG_MODE_SPMV || PREC != 0 || e < 24u || e > 253u || (pr & AG_XFELL) != 0u;
    }

    /* EXACT-order hub chunk after the first: stages (when `stage`) the
     * gathered values of in-edges [eb, ee) of the row starting at o0 at
     * dst[j - o0], and writes
     * per round the totals of its integer steps at binade e and e + 1
     * (words[2k], words[2k+1]; AG_XNOT when they do not apply or e is
     * unknown) and the chunk's sign tag (words[AG_XWORDS - 1]). */
    __device__ __forceinline__ void hub_steps(float *dst, uint32_t o0, uint32_t eb, uint32_t ee, uint32_t lane,
                                              const Pair &first, uint32_t e, bool stage, uint32_t *words) const
    {
        const uint32_t q1 = (ee + 3u) >> 2;
        const bool known = (e >= 24u) & (e <= 253u);
        const float sc = known ? exact_scale(e) : 0.0f;
        uint32_t neg = 0;
        /* round k's values v (quads qa and qa + 32): staged when asked, and
         * their integer steps summed.  Values outside [eb, ee) gather as +0,
         * whose step is 0. */
        auto round = [&](uint32_t k, uint32_t qa, const float *v) {
            if (stage) {
                const uint32_t ja = qa << 2, jb = (qa + 32) << 2;
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (ja + i >= eb && ja + i < ee)
                        dst[ja + i - o0] = v[i];
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (jb + i >= eb && jb + i < ee)
                        dst[jb + i - o0] = v[4 + i];
            }
            if (known && k < AG_XROUNDS) {
                uint32_t t0 = 0, t1 = 0;
                bool b0 = false, b1 = false;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float x = v[i];
                    if (MODE == AG_MODE_DD) {
                        neg |= dd_neg(x);
                        x = fabsf(x);
                    }
                    const float x0 = __fmul_rn(x, sc);
                    /* one binade up: half the units (exact, or a value far
                     * below one unit either way) */
                    const float x1 = __fmul_rn(x0, 0.5f);
                    t0 += exact_step(x0, b0);
                    t1 += exact_step(x1, b1);
                }
                /* a total of 2^24 or more cannot stay in a binade */
                t0 = __reduce_add_sync(0xffffffffu, min(t0, 1u << 24));
                t1 = __reduce_add_sync(0xffffffffu, min(t1, 1u << 24));
                b0 = __any_sync(0xffffffffu, b0 | (t0 >= (1u << 24)));
                b1 = __any_sync(0xffffffffu, b1 | (t1 >= (1u << 24)));
                if (lane == 0) {
                    words[2 * k] = b0 ? AG_XNOT : t0;
                    words[2 * k + 1] = b1 ? AG_XNOT : t1;
                }
            } else if (MODE == AG_MODE_DD) {
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    neg |= dd_neg(v[i]);
            }
        };
        /* the loop runs on the round's first quad, the same in every lane:
         * the warp reductions need all 32 lanes (lanes past the range load
         * and gather nothing) */
        uint32_t q0 = eb >> 2;
        if (MODE == AG_MODE_SPMV) {
            /* weighted pairs take twice the registers: one round in flight */
            Pair cur = first;
            for (uint32_t k = 0; q0 < q1; ++k, q0 += 64) {
                const uint32_t qa = q0 + lane;
                const Pair nx = load_pair(qa + 64, q1);
                float v[8];
                bool in[8];
                gather8(cur, qa, eb, ee, v, in);
                round(k, qa, v);
                cur = nx;
            }
        } else {
            /* two rounds of gathers in flight, as in strided_partial: round
             * k's steps are summed while round k + 1's values travel and
             * round k + 2's ids load */
            float v[8];
            {
                bool in[8];
                gather8(first, q0 + lane, eb, ee, v, in);
            }
            Pair nxt = load_pair(q0 + lane + 64, q1);
            for (uint32_t k = 0; q0 < q1; ++k, q0 += 64) {
                const uint32_t qa = q0 + lane;
                const Pair nn = load_pair(qa + 128, q1);
                float vn[8];
                {
                    bool in[8];
                    gather8(nxt, qa + 64, eb, ee, vn, in);
                }
                round(k, qa, v);
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    v[i] = vn[i];
                nxt = nn;
            }
        }
        if (!known && lane < AG_XROUNDS)
            words[2 * lane] = words[2 * lane + 1] = AG_XNOT;
        if (MODE == AG_MODE_DD) {
            neg = __any_sync(0xffffffffu, neg) ? 1u : 0u;
            if (lane == 0)
                words[AG_XWORDS - 1] = neg;
        }
    }

    /* EXACT-order hub row, on the warp of its last chunk to arrive: the
     * stream-order sum of its deg in-edges (row start o0, chunks of
     * p.whub at slots pbase + c) from the first chunk's sum, the other
     * chunks' round totals and, where a total does not apply, the staged
     * values (row_vals[j - o0]) added one by one through the warp's
     * shared-memory slice.  Records each chunk's starting binade for the
     * next pass.  Data-driven passes OR the sign tags into `neg`. */
    struct XSum
    {
        float s;
        uint32_t neg;
    };

    /* static, with plain arguments: a call of a member would need the
     * kernel's parameter block in local memory */
    static __device__ __noinline__ XSum hub_compose(const uint32_t *hub_part, const uint32_t *hub_t,
                                                    uint32_t *hub_pred, const float *row_vals, const uint32_t *ids,
                                                    const float *c_in, float *vals, uint32_t whub, uint32_t o0,
                                                    uint32_t deg, uint32_t pbase, uint32_t nch, uint32_t lane)
    {
        uint32_t neg = 0;
        float s = __uint_as_float(__ldcg(hub_part + pbase));
        if (MODE == AG_MODE_DD) {
            neg |= dd_neg(s);
            s = fabsf(s);
        }
        const uint32_t *wp = hub_t + (size_t)(pbase + 1) * AG_XWORDS;
        uint32_t wa = __ldcg(wp + lane), wb = __ldcg(wp + 32 + lane);
        uint32_t pr = __ldcg(hub_pred + pbase + 1);
        for (uint32_t c = 1; c < nch; ++c) {
            /* the next chunk's words travel while this one is composed */
            uint32_t na = 0, nb = 0, npr = 0;
            if (c + 1 < nch) {
                const uint32_t *wn = hub_t + (size_t)(pbase + c + 1) * AG_XWORDS;
                na = __ldcg(wn + lane);
                nb = __ldcg(wn + 32 + lane);
                npr = __ldcg(hub_pred + pbase + c + 1);
            }
            if (MODE == AG_MODE_DD)
                neg |= __shfl_sync(0xffffffffu, wb, 31) & 1u;
            const uint32_t e = pr & 0xffu;
            const uint32_t e_start = __float_as_uint(s) >> 23;
            bool fell = false;
            const uint32_t cb = o0 + c * whub, ce = min(o0 + deg, cb + whub), base = cb & ~3u;
            const uint32_t nr = (ce - base + 255u) >> 8;
            for (uint32_t k = 0; k < nr; ++k) {
                const uint32_t lo = max(cb, base + 256u * k), hi = min(ce, base + 256u * (k + 1u));
                const uint32_t w0 = __shfl_sync(0xffffffffu, k < 16u ? wa : wb, (int)((2u * k) & 31u));
                const uint32_t w1 = __shfl_sync(0xffffffffu, k < 16u ? wa : wb, (int)((2u * k + 1u) & 31u));
                const uint32_t sb = __float_as_uint(s), ex = sb >> 23;
                uint32_t w = AG_XNOT;
                if (k < AG_XROUNDS && e != 0u)
                    w = ex == e ? w0 : (ex == e + 1u ? w1 : AG_XNOT);
                const uint32_t m = ((sb & 0x7fffffu) | 0x800000u) + (w & 0x1ffffffu);
                if (!(w & AG_XNOT) && (ex >= 24u) & (ex <= 254u) && m < (1u << 24)) {
                    s = exact_make(ex, m);
                } else {
                    /* this round's values, one by one: staged by the chunk,
                     * or gathered again (contribution of each in-edge's
                     * source; the hot table holds copies of the same values) */
                    __syncwarp();
                    if (hub_staged(pr)) {
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const uint32_t j = lo + lane + 32u * i;
                            vals[lane + 32u * i] = j < hi ? __ldcg(row_vals + (j - o0)) : 0.0f;
                        }
                    } else {
                        uint32_t u[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const uint32_t j = lo + lane + 32u * i;
                            u[i] = j < hi ? __ldg(ids + j) : 0u;
                        }
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const uint32_t j = lo + lane + 32u * i;
                            vals[lane + 32u * i] = j < hi ? __ldcg(c_in + u[i]) : 0.0f;
                        }
                    }
                    __syncwarp();
                    if (lane == 0)
                        s = seq_sum(vals, 0, hi - lo, s, false, neg);
                    s = __shfl_sync(0xffffffffu, s, 0);
                    fell = true;
                }
            }
            if (lane == 0)
                hub_pred[pbase + c] = e_start | (fell ? AG_XFELL : 0u);
            wa = na;
            wb = nb;
            pr = npr;
        }
        return XSum{s, neg};
    }

    /* the stream-order sum of vals[a, b) (the warp's shared-memory slice)
     * by the calling lane alone, continuing s, or starting with vals[a] when
     * `first`: four values per 16-byte shared load once the index is
     * aligned, one binary32 add after another.  Data-driven passes add the
     * magnitudes and OR the sign tags into `neg`. */
    static __device__ __forceinline__ float seq_sum(const float *vals, uint32_t a, uint32_t b, float s, bool first,
                                                    uint32_t &neg)
    {
        auto val = [&](float v) {
            if (MODE == AG_MODE_DD) {
                neg |= dd_neg(v);
                v = fabsf(v);
            }
            return v;
        };
        uint32_t j = a;
        if (first && j < b) {
            s = val(vals[j]);
            ++j;
        }
        for (; j < b && (j & 3u); ++j)
            s = __fadd_rn(s, val(vals[j]));
        for (; j + 8u <= b; j += 8u) {
            const float4 q0 = reinterpret_cast<const float4 *>(vals)[j >> 2];
            const float4 q1 = reinterpret_cast<const float4 *>(vals)[(j >> 2) + 1];
            s = __fadd_rn(s, val(q0.x));
            s = __fadd_rn(s, val(q0.y));
            s = __fadd_rn(s, val(q0.z));
            s = __fadd_rn(s, val(q0.w));
            s = __fadd_rn(s, val(q1.x));
            s = __fadd_rn(s, val(q1.y));
            s = __fadd_rn(s, val(q1.z));
            s = __fadd_rn(s, val(q1.w));
        }
        for (; j < b; ++j)
            s = __fadd_rn(s, val(vals[j]));
        return s;
    }

    /* EXACT-order long row: the stream-order sum of in-edges [eb, ee) on one
     * warp.  Rounds of 256 in-edges (after the first, each starting on a
     * 16-byte group) are staged in the warp's shared-memory slice by the row
     * items' stage (16-byte id loads, eight gathers in flight per lane);
     * lane 0 adds a round one value after another while the next round's
     * gathers travel.  Rows this short cross a binade in most rounds, where
     * the integer way of the hub rows falls back to its slower forms; the
     * lane's chain costs about 1.25 instructions per value.  `first` is the
     * range's first id pair; the sum is lane 0's. */
    __device__ __forceinline__ float ordered_sum(float *vals, uint32_t eb, uint32_t ee, uint32_t lane,
                                                 const Pair &first, uint32_t &neg) const
    {
        uint32_t cb = eb, ce = min(ee, (eb & ~3u) + (uint32_t)AG_WCAP);
        /* the ids of a round are requested one round before its gathers */
        Pair ids = prefetch(ce, min(ee, ce + (uint32_t)AG_WCAP), lane);
        stage(vals, cb, ce, lane, first);
        float s = 0.0f;
        for (;;) {
            __syncwarp();
            const uint32_t nb = ce, ne = min(ee, ce + (uint32_t)AG_WCAP);
            if (nb >= ee) {
                if (lane == 0)
                    s = seq_sum(vals, 0, ce - cb, s, cb == eb, neg);
                return s;
            }
            /* the next round's gathers travel while this one is added */
            float w[8];
            stage_issue(ids, nb, ne, lane, w);
            ids = prefetch(ne, min(ee, ne + (uint32_t)AG_WCAP), lane);
            if (lane == 0)
                s = seq_sum(vals, 0, ce - cb, s, cb == eb, neg);
            __syncwarp();
            stage_commit(vals, nb, ne, lane, w);
            cb = nb;
            ce = ne;
        }
    }
};

extern __shared__ __align__(128) unsigned char ag_dsmem[];

/* EXACT-order work sharing.  A warp that sums a long hub row in stream order
 * would still own every nwarps-th item after it, and the pass would wait for
 * it.  So before the sum it publishes the rest of its stride as a donor
 * entry; warps that have run out of items claim them one at a time with an
 * atomic counter, and so does the donor once its sum is done.  State lives
 * in lane 0 of each warp. */
struct AgSteal
{
    int donor = -1;        /* this warp's donor entry                        */
    bool stealing = false; /* the warp's own stride is used up               */
    uint32_t probe = 0;    /* donor entries found empty so far               */
};

/* item k of donor d (nwarps apart), or ntasks once the entry is used up */
static __device__ __forceinline__ uint32_t ag_steal_claim(uint32_t *steal, uint32_t d, uint32_t nwarps,
                                                          uint32_t ntasks)
{
    volatile uint32_t *vs = steal;
    const uint32_t b1 = vs[2 + 2 * d], k = vs[3 + 2 * d];
    if (b1 == 0 || (uint64_t)(b1 - 1u) + (uint64_t)k * nwarps >= ntasks)
        return ntasks;
    const uint64_t item = (b1 - 1u) + (uint64_t)atomicAdd(steal + 3 + 2 * d, 1u) * nwarps;
    return item < ntasks ? (uint32_t)item : ntasks;
}

/* the item after t for warp w (lane 0): its own stride, then its donor
 * entry, then other donors' entries (at most AG_STEAL_PROBES of them,
 * starting at one picked by w); ntasks when there is none */
static __device__ __forceinline__ uint32_t ag_steal_next(uint32_t *steal, AgSteal &st, uint32_t t, uint32_t w,
                                                         uint32_t nwarps, uint32_t ntasks)
{
    if (st.donor >= 0) {
        const uint32_t it = ag_steal_claim(steal, (uint32_t)st.donor, nwarps, ntasks);
        if (it < ntasks)
            return it;
        st.donor = -1;
        st.stealing = true;
    } else if (!st.stealing) {
        if ((uint64_t)t + nwarps < ntasks)
            return t + nwarps;
        st.stealing = true;
    }
    const uint32_t n = min(*((volatile uint32_t *)steal), (uint32_t)AG_STEAL_CAP);
    for (; st.probe < min(n, (uint32_t)AG_STEAL_PROBES); ++st.probe) {
        const uint32_t it = ag_steal_claim(steal, (w + st.probe) % n, nwarps, ntasks);
        if (it < ntasks)
            return it;
    }
    return ntasks;
}

/* one pull pass on this CTA; LOW: the pass reads 16-bit contributions */
template <int MODE, int PREC, bool EXACT, bool LOW>
__device__ __forceinline__ void ag_pull_body(const AgPullParams &p, double *s_redd, uint32_t *s_redu,
                                             uint32_t &s_last, uint64_t &s_bar)
{
    AgPass<MODE, PREC, EXACT, LOW> ps(p);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float *vals = reinterpret_cast<float *>(ag_dsmem) + warp * AG_WCAP;
    unsigned char *hot = ag_dsmem + AG_STAGE_BYTES;
    const uint32_t nwarps = gridDim.x * AG_WARPS;

    /* hot table: the first hot_n values of the gathered vector, one TMA bulk
     * copy per 32 KB, completing on an mbarrier that every thread waits on
     * (bounded; a wait that runs out is reported through ctl->fault) */
    if (p.hot_n) {
        /* 16-bit passes hold twice the entries in the same bytes */
        const uint32_t hn = ps.gather_elem_bytes() == 2 ? p.hot_n16 : p.hot_n;
        const uint32_t bytes = hn * ps.gather_elem_bytes();
        if (tid == 0) {
            ag_mbar_init(&s_bar, 1);
            ag_mbar_expect_tx(&s_bar, bytes);
            const unsigned char *src = reinterpret_cast<const unsigned char *>(ps.gather_source());
            for (uint32_t off = 0; off < bytes; off += AG_BULK_CHUNK)
                ag_bulk_g2s(hot + off, src + off, min(AG_BULK_CHUNK, bytes - off), &s_bar);
        }
        __syncthreads();
        if (!ag_mbar_wait(&s_bar, 0, p.mbar_spins)) {
            if (p.ctl)
                atomicOr(&p.ctl->fault, 1u);
            /* the copies may still be in flight: give them a long, bounded
             * second chance before this CTA can exit */
            ag_mbar_wait(&s_bar, 0, 1u << 24);
        }
        ps.hot32 = reinterpret_cast<const float *>(hot);
        ps.hot16 = reinterpret_cast<const uint16_t *>(hot);
        ps.hot_n = hn;
    }

    /* each warp walks its tasks with a stride of all warps; the first id
     * pair of the next task is requested before the current task is
     * gathered, reduced and written, so it is in flight meanwhile */
    uint32_t t = blockIdx.x * AG_WARPS + warp;
    uint4 task = t < p.ntasks ? p.tasks[t] : make_uint4(0, 0, 0, 0);
    typename AgPass<MODE, PREC, EXACT, LOW>::Pair pf = ps.prefetch(task.z, task.w, lane);
    AgSteal steal;
    while (t < p.ntasks) {
        uint32_t tn = t + nwarps;
        if (EXACT) {
            if (lane == 0)
                tn = ag_steal_next(p.steal, steal, t, blockIdx.x * AG_WARPS + warp, nwarps, p.ntasks);
            tn = __shfl_sync(0xffffffffu, tn, 0);
        }
        const uint4 task_n = tn < p.ntasks ? p.tasks[tn] : make_uint4(0, 0, 0, 0);
        const uint32_t kind = task.x >> 30;
        const uint32_t r0 = task.x & AG_ROW_MASK;
        const uint32_t eb = task.z, ee = task.w;
        uint32_t gid = 0;
        if (MODE == AG_MODE_MULTI) {
            /* the item's graph; items of finished graphs are skipped */
            uint32_t lo = 0, hi = p.ngraphs;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(p.gstart + mid) <= r0)
                    lo = mid;
                else
                    hi = mid;
            }
            gid = lo;
            if (*((volatile uint32_t *)(p.g_done + gid))) {
                pf = ps.prefetch(task_n.z, task_n.w, lane);
                task = task_n;
                t = tn;
                continue;
            }
        }
        if (MODE == AG_MODE_DD && kind == AG_T_ROWS) {
            /* data-driven: the sums are those of the plain pull over the
             * gathered magnitudes; a row is active when the pass is the first
             * or a gathered value carries the sign of a change */
            const uint32_t r = r0 + lane;
            const bool live = r < task.y;
            uint32_t o0 = ee, o1 = ee, od = 0;
            float rp = 0.0f;
            if (live) {
                o0 = ag_ld_row_u32(p.row_off + r);
                o1 = ag_ld_row_u32(p.row_off + r + 1);
                rp = ag_ld_rank(p.rank + r);
                od = ag_ld_row_u32(p.outdeg + r);
            }
            const typename AgPass<MODE, PREC, EXACT, LOW>::Pair pn = ps.prefetch(task_n.z, task_n.w, lane);
            ps.stage(vals, eb, ee, lane, pf);
            __syncwarp();
            o0 -= eb;
            o1 -= eb;
            float s = 0.0f;
            uint32_t neg = 0;
            bool is_long = false;
            if (EXACT) {
                s = ps.seq_sum(vals, o0, o1, 0.0f, true, neg);
            } else if (o1 - o0 <= AG_TSEQ) {
                if (o1 > o0) {
                    float v = vals[o0];
                    neg = ps.dd_neg(v);
                    s = fabsf(v);
                    for (uint32_t j = o0 + 1; j < o1; ++j) {
                        v = vals[j];
                        neg |= ps.dd_neg(v);
                        s = __fadd_rn(s, fabsf(v));
                    }
                }
            } else {
                is_long = true;
            }
            if (!EXACT) {
                unsigned m = __ballot_sync(0xffffffffu, is_long);
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t a = __shfl_sync(0xffffffffu, o0, src);
                    const uint32_t b = __shfl_sync(0xffffffffu, o1, src);
                    float tsum = 0.0f;
                    uint32_t tneg = 0;
                    for (uint32_t j = a + lane; j < b; j += 32) {
                        const float v = vals[j];
                        tneg |= ps.dd_neg(v);
                        tsum = __fadd_rn(tsum, fabsf(v));
                    }
                    tsum = ag_warp_sum_f(tsum);
                    tneg = __any_sync(0xffffffffu, tneg) ? 1u : 0u;
                    if ((int)lane == src) {
                        s = tsum;
                        neg = tneg;
                    }
                }
            }
            if (live)
                ps.finish_dd(r, s, rp, od, ps.dd_all || neg);
            __syncwarp();
            pf = pn;
        } else if (kind == AG_T_ROWS) {
            /* one row per lane; its bounds, previous rank and out-degree are
             * loaded first so that they arrive while the stage runs */
            const uint32_t r = r0 + lane;
            const bool live = r < task.y;
            uint32_t o0 = ee, o1 = ee, od = 0;
            float rp = 0.0f;
            if (live) {
                o0 = ag_ld_row_u32(p.row_off + r);
                o1 = ag_ld_row_u32(p.row_off + r + 1);
                if (MODE != AG_MODE_SPMV) {
                    rp = ag_ld_rank(p.rank + r);
                    od = ag_ld_row_u32(p.outdeg + r);
                }
            }
            const typename AgPass<MODE, PREC, EXACT, LOW>::Pair pn = ps.prefetch(task_n.z, task_n.w, lane);
            ps.stage(vals, eb, ee, lane, pf);
            __syncwarp();
            o0 -= eb;
            o1 -= eb;
            float s = 0.0f;
            bool is_long = false;
            if (EXACT) {
                /* stream order, rows of any length: 16-byte shared loads */
                uint32_t nn = 0;
                s = ps.seq_sum(vals, o0, o1, 0.0f, true, nn);
            } else if (o1 - o0 <= AG_TSEQ) {
                /* stream order: the accumulator restarts with the first value
                 * and adds the rest one by one */
                if (o1 > o0) {
                    s = vals[o0];
                    for (uint32_t j = o0 + 1; j < o1; ++j)
                        s = __fadd_rn(s, vals[j]);
                }
            } else {
                is_long = true;
            }
            if (!EXACT) {
                /* rows of AG_TSEQ+1 .. AG_WCAP in-edges: the whole warp sums
                 * each one (lane-strided partials, xor tree) */
                unsigned m = __ballot_sync(0xffffffffu, is_long);
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t a = __shfl_sync(0xffffffffu, o0, src);
                    const uint32_t b = __shfl_sync(0xffffffffu, o1, src);
                    float tsum = 0.0f;
                    for (uint32_t j = a + lane; j < b; j += 32)
                        tsum = __fadd_rn(tsum, vals[j]);
                    tsum = ag_warp_sum_f(tsum);
                    if ((int)lane == src)
                        s = tsum;
                }
            }
            if (live)
                ps.finish(r, s, rp, od);
            __syncwarp();
            pf = pn;
        } else if (kind == AG_T_LONG) {
            float rp = 0.0f;
            uint32_t od = 0;
            if (MODE != AG_MODE_SPMV && lane == 0) {
                rp = p.rank[r0];
                od = p.outdeg[r0];
            }
            const typename AgPass<MODE, PREC, EXACT, LOW>::Pair pn = ps.prefetch(task_n.z, task_n.w, lane);
            float s;
            uint32_t neg = 0;
            if (EXACT) {
                s = ps.ordered_sum(vals, eb, ee, lane, pf, neg);
            } else {
                s = ps.strided_partial(eb, ee, lane, pf, neg);
                s = ag_warp_sum_f(s);
            }
            if (MODE == AG_MODE_DD) {
                const bool act = ps.dd_all || __any_sync(0xffffffffu, neg);
                if (lane == 0)
                    ps.finish_dd(r0, s, rp, od, act);
            } else if (lane == 0) {
                ps.finish(r0, s, rp, od);
            }
            __syncwarp();
            pf = pn;
        } else if (EXACT) {
            /* hub chunk, EXACT order: the first chunk sums its in-edges in
             * stream order, the others stage their values and sum their
             * integer steps per round; the row's last chunk to arrive
             * composes the row (hub_compose) */
            const uint32_t pbase = task.y & AG_SLOT_MASK, chunk = task.y >> AG_SLOT_BITS;
            const uint32_t o0 = eb - chunk * p.whub;
            float *row_vals = p.hub_vals + (size_t)pbase * p.whub;
            const typename AgPass<MODE, PREC, EXACT, LOW>::Pair pn = ps.prefetch(task_n.z, task_n.w, lane);
            if (chunk == 0) {
                uint32_t neg0 = 0;
                const float s0 = ps.ordered_sum(vals, eb, ee, lane, pf, neg0);
                if (lane == 0) {
                    /* data-driven: the sign bit carries the chunk's tag */
                    const uint32_t bits = __float_as_uint(s0) | (MODE == AG_MODE_DD && neg0 ? 0x80000000u : 0u);
                    reinterpret_cast<uint32_t *>(p.hub_part)[pbase] = bits;
                }
            } else {
                const uint32_t pred = __ldcg(p.hub_pred + pbase + chunk);
                ps.hub_steps(row_vals, o0, eb, ee, lane, pf, pred & 0xffu, ps.hub_staged(pred),
                             p.hub_t + (size_t)(pbase + chunk) * AG_XWORDS);
            }
            __threadfence();
            __syncwarp();
            uint32_t last = 0;
            const uint32_t deg = p.row_off[r0 + 1] - o0;
            const uint32_t nch = (deg + p.whub - 1) / p.whub;
            if (lane == 0)
                last = atomicAdd(&p.hub_cnt[pbase], 1u) == nch - 1 ? 1u : 0u;
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                __threadfence();
                if (lane == 0 && deg >= AG_STEAL_MIN && steal.donor < 0 && !steal.stealing &&
                    (uint64_t)tn + nwarps < p.ntasks) {
                    /* give away the items after the next one */
                    const uint32_t d = atomicAdd(p.steal, 1u);
                    if (d < AG_STEAL_CAP) {
                        p.steal[3 + 2 * d] = 0;
                        __threadfence();
                        atomicExch(p.steal + 2 + 2 * d, tn + nwarps + 1u);
                        steal.donor = (int)d;
                    }
                }
                const typename AgPass<MODE, PREC, EXACT, LOW>::XSum xs = AgPass<MODE, PREC, EXACT, LOW>::hub_compose(
                    reinterpret_cast<const uint32_t *>(p.hub_part), p.hub_t, p.hub_pred, row_vals, p.ids, ps.c_in32,
                    vals, p.whub, o0, deg, pbase, nch, lane);
                const float tot = xs.s;
                const uint32_t neg = xs.neg;
                if (lane == 0) {
                    p.hub_cnt[pbase] = 0;
                    float rp = 0.0f;
                    uint32_t od = 0;
                    if (MODE != AG_MODE_SPMV) {
                        rp = p.rank[r0];
                        od = p.outdeg[r0];
                    }
                    if (MODE == AG_MODE_DD)
                        ps.finish_dd(r0, tot, rp, od, ps.dd_all || neg);
                    else
                        ps.finish(r0, tot, rp, od);
                }
            }
            __syncwarp();
            pf = pn;
        } else {
            /* hub chunk, FAST order: chunk partials, added in chunk order */
            const uint32_t pbase = task.y & AG_SLOT_MASK, chunk = task.y >> AG_SLOT_BITS;
            uint32_t deg = 0;
            if (lane == 0)
                deg = p.row_off[r0 + 1] - p.row_off[r0];
            const typename AgPass<MODE, PREC, EXACT, LOW>::Pair pn = ps.prefetch(task_n.z, task_n.w, lane);
            /* data-driven: each chunk's partial carries the sign of a change
             * among its in-neighbours; the last chunk ORs them */
            uint32_t neg = 0;
            float s = ps.strided_partial(eb, ee, lane, pf, neg);
            s = ag_warp_sum_f(s);
            if (MODE == AG_MODE_DD && __any_sync(0xffffffffu, neg))
                s = __uint_as_float(__float_as_uint(s) | 0x80000000u);
            if (lane == 0) {
                const uint32_t nch = (deg + p.whub - 1) / p.whub;
                p.hub_part[pbase + chunk] = s;
                __threadfence();
                const uint32_t prev = atomicAdd(&p.hub_cnt[pbase], 1u);
                if (prev == nch - 1) {
                    __threadfence();
                    float tot = __ldcg(p.hub_part + pbase);
                    uint32_t any = 0;
                    if (MODE == AG_MODE_DD) {
                        any = ps.dd_neg(tot);
                        tot = fabsf(tot);
                    }
                    for (uint32_t c = 1; c < nch; ++c) {
                        const float part = __ldcg(p.hub_part + pbase + c);
                        if (MODE == AG_MODE_DD)
                            any |= ps.dd_neg(part);
                        tot = __fadd_rn(tot, MODE == AG_MODE_DD ? fabsf(part) : part);
                    }
                    p.hub_cnt[pbase] = 0;
                    float rp = 0.0f;
                    uint32_t od = 0;
                    if (MODE != AG_MODE_SPMV) {
                        rp = p.rank[r0];
                        od = p.outdeg[r0];
                    }
                    if (MODE == AG_MODE_DD)
                        ps.finish_dd(r0, tot, rp, od, ps.dd_all || any);
                    else
                        ps.finish(r0, tot, rp, od);
                }
            }
            __syncwarp();
            pf = pn;
        }
        if (MODE == AG_MODE_MULTI) {
            /* the item's totals go to its graph */
            const double e = ag_warp_sum_d(ps.my_err);
            const uint32_t a = ag_warp_sum_u(ps.my_active);
            if (lane == 0) {
                if (e != 0.0)
                    atomicAdd(p.g_err + gid, e);
                if (a)
                    atomicAdd(p.g_active + gid, a);
            }
            ps.my_err = 0.0;
            ps.my_active = 0;
        }
        task = task_n;
        t = tn;
    }

    if (EXACT) {
        /* the last warp out clears the donor table for the next pass, its
         * lanes taking every 32nd entry */
        uint32_t out = 0;
        if (lane == 0) {
            __threadfence();
            out = atomicAdd(p.steal + 1, 1u) == nwarps - 1 ? 1u : 0u;
        }
        if (__shfl_sync(0xffffffffu, out, 0)) {
            __threadfence();
            const uint32_t n = min(*((volatile uint32_t *)p.steal), (uint32_t)AG_STEAL_CAP);
            for (uint32_t d = lane; d < n; d += 32)
                p.steal[2 + 2 * d] = 0;
            __syncwarp();
            if (lane == 0) {
                p.steal[0] = 0;
                p.steal[1] = 0;
            }
            __threadfence();
        }
    }

    if (MODE == AG_MODE_SPMV)
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
    if (MODE == AG_MODE_MULTI) {
        if (!s_last)
            return;
        /* every thread of the last CTA closes the pass of some graphs */
        __threadfence();
        AgControl *c = p.ctl;
        volatile AgControl *vc = c;
        const uint32_t P = vc->iter;
        const uint32_t max_iter = vc->max_iter;
        int running = 0;
        for (uint32_t g = tid; g < p.ngraphs; g += blockDim.x) {
            if (*((volatile uint32_t *)(p.g_done + g)))
                continue;
            const uint32_t a = *((volatile uint32_t *)(p.g_active + g));
            const uint32_t np = p.g_passes[g] + 1;
            const double n_g = (double)(__ldg(p.gstart + g + 1) - __ldg(p.gstart + g));
            p.g_passes[g] = np;
            p.g_err_last[g] = *((volatile double *)(p.g_err + g)) / (n_g > 0 ? n_g : 1.0);
            p.g_active[g] = 0;
            p.g_err[g] = 0.0;
            if (a == 0) {
                p.g_conv[g] = 1;
                p.g_done[g] = 1;
            } else if (np >= max_iter) {
                p.g_done[g] = 1;
            } else {
                running = 1;
            }
        }
        running = __syncthreads_or(running);
        if (tid == 0) {
            if (P < AG_MAX_HISTORY)
                c->hist_t[P] = ag_globaltimer();
            c->iter = P + 1;
            c->done_ctas = 0;
            c->converged = running ? 0u : 1u;
            c->stop = running ? 0u : 1u;
            __threadfence();
            if (p.use_cond)
                cudaGraphSetConditional(p.cond, running ? 1u : 0u);
        }
        return;
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

template <int MODE, int PREC, bool EXACT>
__global__ void __launch_bounds__(AG_BLK, AG_CTAS_PER_SM) ag_pull_kernel(const AgPullParams p)
{
    __shared__ double s_redd[AG_WARPS];
    __shared__ uint32_t s_redu[AG_WARPS];
    __shared__ uint32_t s_last;
    __shared__ __align__(8) uint64_t s_bar;

    /* stream launches (profiling) run a fixed number of kernels: the ones
     * after the loop has ended return at once */
    if ((MODE != AG_MODE_SPMV || p.honor_stop) && !p.use_cond && *((volatile uint32_t *)&p.ctl->stop))
        return;
    if constexpr (PREC != 0) {
        /* the storage this pass reads, set by the pass before */
        if (*((volatile uint32_t *)&p.ctl->mode_read)) {
            ag_pull_body<MODE, PREC, EXACT, true>(p, s_redd, s_redu, s_last, s_bar);
            return;
        }
    }
    ag_pull_body<MODE, PREC, EXACT, false>(p, s_redd, s_redu, s_last, s_bar);
}

/* init: r = base (or the warm start), first contributions, control reset */
template <int PREC>
__global__ void __launch_bounds__(AG_SBLK) ag_pr_init_kernel2(const AgPullParams p, const AgRunConfig run)
{
    const uint64_t pol_last = ag_policy_evict_last();
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        /* device row v is caller vertex perm[v]; the warm start is in caller order */
        const float r0 = run.use_init ? p.init_ranks[p.perm ? p.perm[v] : v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        const float c = od ? __fdiv_rn(r0, __uint2float_rn(od)) : 0.0f;
        if (PREC != 0)
            ag_st_keep_u16(p.c16_0 + v, ag_f32_to_low<PREC>(c), pol_last);
        else
            ag_st_keep_f32(p.c32_0 + p.c_base + v, c, pol_last);
    }
    for (uint32_t g = blockIdx.x * AG_SBLK + threadIdx.x; g < p.ngraphs; g += gridDim.x * AG_SBLK) {
        p.g_active[g] = 0;
        p.g_err[g] = 0.0;
        p.g_done[g] = (run.max_iter > 0 && p.gstart[g + 1] > p.gstart[g]) ? 0u : 1u;
        p.g_passes[g] = 0;
        p.g_conv[g] = 0;
        p.g_err_last[g] = 0.0;
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
        c->stop = (run.max_iter > 0 && p.N > 0) ? 0u : 1u;
        c->fault = 0;
        if (p.use_cond)
            cudaGraphSetConditional(p.cond, (run.max_iter > 0 && p.N > 0) ? 1u : 0u);
    }
}

/* ranks / N in binary32 (pageRank.c:1079-1085), back in caller order, FP64 sum */
__global__ void __launch_bounds__(AG_SBLK) ag_normalize_kernel(const AgPullParams p)
{
    __shared__ double sh[AG_SNW];
    const float fN = __uint2float_rn(p.N);
    double s = 0.0;
    const float fNn = p.norm_n ? __uint2float_rn(p.norm_n) : fN;
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        float div = fNn;
        if (p.ngraphs) {
            /* each graph of a union is normalised by its own vertex count */
            uint32_t lo = 0, hi = p.ngraphs;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(p.gstart + mid) <= v)
                    lo = mid;
                else
                    hi = mid;
            }
            div = __uint2float_rn(__ldg(p.gstart + lo + 1) - __ldg(p.gstart + lo));
        }
        const float r = __fdiv_rn(p.rank[p.inv ? p.inv[v] : v], div);
        p.out[v] = r;
        s += (double)r;
    }
    s = ag_warp_sum_d(s);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < AG_SNW; ++w)
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
    if (mode == AG_MODE_MULTI)
        return exact ? (const void *)ag_pull_kernel<AG_MODE_MULTI, 0, true>
                     : (const void *)ag_pull_kernel<AG_MODE_MULTI, 0, false>;
    if (mode == AG_MODE_DD)
        return exact ? (const void *)ag_pull_kernel<AG_MODE_DD, 0, true>
                     : (const void *)ag_pull_kernel<AG_MODE_DD, 0, false>;
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
    if (blocks > ag_sm_grid(32))
        blocks = ag_sm_grid(32);
    ag_validate_ids_kernel<<<(unsigned)blocks, 256, 0, s>>>(ids, E, N, flag);
    return cudaGetLastError();
}

extern "C" cudaError_t ag_pr_f64_run(const uint32_t *row_off, const uint32_t *ids, const uint32_t *outdeg, uint32_t N,
                                     uint32_t max_iter, double tol, double *r, double *r2, double *c,
                                     double *maxdiff_dev, uint32_t *passes_out, cudaStream_t s)
{
    const unsigned gb = ag_sm_grid(8);
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
