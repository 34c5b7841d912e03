/*
 * ag_push.cu -- push-direction and residual PageRank forms of the
 * reference's dispatcher (02_capi_graph/src/algorithms/capi/pageRank.c):
 *   pushpull 1  push, binary32                 :1111-1272
 *   pushpull 3  push, 64-bit fixed point       :1992-2118
 *   pushpull 5  push, 32-bit quantised         :2678-2809
 *   pushpull 7  data-driven push (residuals)   :2971-3127
 *   pushpull 8  data-driven pull-push          :3128-3325
 *
 * The reference runs these on many OpenMP threads (or the FPGA's push unit),
 * with atomic or unsynchronised adds into the destination: their add order,
 * and for the residual forms which updates a vertex sees, are not fixed.  The
 * device forms here are instances of that behaviour:
 *
 * Push (1, 3, 5): one thread per forward edge (a source-sorted edge list
 * built on the device from the relabelled inverse CSR) adds the source's
 * contribution into next[destination] with an atomic add.  The fixed-point
 * form adds 64-bit integers, whose sums are exact and identical to the 64-bit
 * fixed-point pull's.  The binary32 forms add into a binary64 accumulator,
 * rounded once to binary32 by the update: atomic binary32 adds land in a new
 * order every pass, and a rank whose ulp exceeds epsilon (un-normalised hub
 * ranks) would then change by an ulp every pass and never pass the residual
 * test, whereas the binary64 sum's order moves only bits that the rounding
 * drops.  An element-wise kernel then forms r' = base + damp * next (binary64
 * for fixed point, as the pull), the residual, the next contributions and
 * clears next; its last CTA closes the pass.  The quantised form first
 * replaces every contribution c by scale * q(c), the value the reference adds
 * per edge (zero point 0).
 *
 * Residual forms (7, 8): a vertex phase takes each worklist vertex's
 * residual (atomic exchange with 0, so that no concurrent add is lost),
 * forms its new rank (7: r + residual; 8: base + damp * the pull over its
 * in-edges of the contributions at the start of the pass -- the interleaving
 * of the reference's loop in which every read precedes every write), adds
 * |r'/n - r/n| to the pass's error and stores delta = damp * (residual /
 * out_degree); an edge phase, one thread per forward edge of a worklist
 * source, adds delta to the destination's residual (atomic, returning the
 * previous value) and, when the residual crosses epsilon (|prev + delta| >=
 * epsilon and prev <= epsilon), counts an activation and puts the
 * destination on the next worklist (8 adds delta a second time, as the
 * reference does).  A self-edge adds nothing: the reference sets the
 * residual to 0 after the vertex's own adds, so only its crossing test, made
 * on the residual the vertex phase took, remains.  The edge phase's last CTA
 * closes the pass; the loop stops after a pass without activations.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/cub.cuh>

#include "ag_device.h"
#include "ag_intpass.h"
#include "ag_mem.h"

#define AG_PNW (AG_SBLK / 32)
#define AG_PUSH_BLK 1024     /* threads of a scatter CTA (one per SM)        */
#define AG_PUSH_HOT 8192u    /* destinations summed in shared memory (64 KB) */
#define AG_RES_HOT 8192u     /* residual destinations summed in shared memory
                                (32 KB; the same table space) */

__device__ __forceinline__ double ag_push_warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* the CTA's sum of one double per thread, valid in thread 0 */
__device__ double ag_push_block_sum_d(double v)
{
    __shared__ double s_v[AG_PNW];
    v = ag_push_warp_sum_d(v);
    if ((threadIdx.x & 31) == 0)
        s_v[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < AG_PNW; ++w)
            t += s_v[w];
    return t;
}

__device__ __forceinline__ bool ag_push_stopped(const AgPullParams &p)
{
    return !p.use_cond && *((volatile uint32_t *)&p.ctl->stop);
}

/* ---------------------------------------------------------------- init */
/* push forms: r = base (or the warm start), next = 0, first contributions
 * (quantised: binary32 and their min/max keys in slot 0, which the graph
 * clears first) */
template <int KIND>
__global__ void __launch_bounds__(AG_SBLK) ag_push_init_kernel(const AgPullParams p, const AgRunConfig run)
{
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        const float r0 = run.use_init ? p.init_ranks[p.perm ? p.perm[v] : v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        p.c64_1[v] = 0ull; /* the next sums: 64-bit integer or binary64 zero */
        if (KIND == AG_PUSH_FIXED) {
            p.c64_0[v] = od ? ag_d2fixed((double)__fdiv_rn(r0, __uint2float_rn(od))) : 0ull;
        } else {
            const float c = od ? __fdiv_rn(r0, __uint2float_rn(od)) : 0.0f;
            p.pa[v] = c;
            if (KIND == AG_PUSH_QUANT) {
                const uint32_t k = ag_fkey(c);
                mn = min(mn, k);
                mx = max(mx, k);
            }
        }
    }
    if (KIND == AG_PUSH_QUANT)
        ag_fold_minmax_slot0<AG_PNW>(p.qmm, mn, mx);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        ag_reset_control(p, run);
}

/* residual forms: x[v] = 1 / out_degree[v] (0 without out-edges), the
 * vector whose stream-order in-row sums give the first residuals; the sums'
 * vector starts at 0 */
__global__ void __launch_bounds__(AG_SBLK) ag_residual_seed_kernel(const AgPullParams p)
{
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        const uint32_t od = p.outdeg[v];
        p.pa[v] = od ? __fdiv_rn(1.0f, __uint2float_rn(od)) : 0.0f;
        p.pb[v] = 0.0f;
    }
}

/* residual forms: res = ((1 - damp) * damp) * sum, r = base (or the warm
 * start), every vertex on the first worklist, contributions r / out_degree
 * for the pull-push form's first pull, control reset */
__global__ void __launch_bounds__(AG_SBLK) ag_residual_init_kernel(const AgPullParams p, const AgRunConfig run)
{
    const float k = __fmul_rn(p.base, p.damp);
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        p.res[v] = __fmul_rn(k, p.pb[v]);
        const float r0 = run.use_init ? p.init_ranks[p.perm ? p.perm[v] : v] : p.base;
        p.rank[v] = r0;
        const uint32_t od = p.outdeg[v];
        p.pa[v] = od ? __fdiv_rn(r0, __uint2float_rn(od)) : 0.0f;
        p.wl[v] = 1;
        p.wl[p.N + v] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        ag_reset_control(p, run);
}

/* ---------------------------------------------------------------- push */
/* quantised push: every contribution becomes scale * q(c), the value the
 * reference adds along each of the source's edges */
__global__ void __launch_bounds__(AG_SBLK) ag_push_quant_kernel(const AgPullParams p)
{
    if (ag_push_stopped(p))
        return;
    const float scale = ag_quant_scale<uint32_t>(p.qmm, p.ctl->iter & 1u);
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK)
        p.pa[v] = __fmul_rn(scale, __uint2float_rn(ag_quantize<uint32_t>(p.pa[v], scale)));
}

/* One thread per forward edge: next[dst] += c[src] (64-bit integer, or
 * binary64 for the binary32 forms).  The first AG_PUSH_HOT destinations (the
 * most-read vertices after the relabelling by out-degree, and in power-law
 * graphs the in-hubs) are summed first in a shared-memory table of the CTA
 * and added to next once per CTA: adds to one hub otherwise queue at the one
 * L2 slice that holds it.  A persistent grid of AG_PUSH_BLK-thread CTAs. */
template <int KIND> __global__ void __launch_bounds__(AG_PUSH_BLK) ag_push_scatter_kernel(const AgPullParams p)
{
    extern __shared__ __align__(16) unsigned long long ag_push_hot[];
    if (ag_push_stopped(p))
        return;
    const uint32_t hot_n = min(p.N, (uint32_t)AG_PUSH_HOT);
    for (uint32_t i = threadIdx.x; i < hot_n; i += AG_PUSH_BLK)
        ag_push_hot[i] = 0ull;
    __syncthreads();
    const uint64_t pol_first = ag_policy_evict_first();
    const uint32_t stride = gridDim.x * AG_PUSH_BLK;
    for (uint32_t j = blockIdx.x * AG_PUSH_BLK + threadIdx.x; j < p.E; j += stride) {
        const uint32_t v = ag_ld_stream_u32(p.fwd_src + j, pol_first);
        const uint32_t u = ag_ld_stream_u32(p.fwd_dst + j, pol_first);
        /* separate shared and global adds: a pointer to either would make a
         * generic atomic that returns its value instead of a reduction */
        if (KIND == AG_PUSH_FIXED) {
            const unsigned long long c = p.c64_0[v];
            if (u < hot_n)
                atomicAdd(ag_push_hot + u, c);
            else
                atomicAdd((unsigned long long *)p.c64_1 + u, c);
        } else {
            const double c = (double)p.pa[v];
            if (u < hot_n)
                atomicAdd(reinterpret_cast<double *>(ag_push_hot) + u, c);
            else
                atomicAdd(reinterpret_cast<double *>(p.c64_1) + u, c);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hot_n; i += AG_PUSH_BLK) {
        const unsigned long long t = ag_push_hot[i];
        if (t == 0ull) /* +0.0 or integer 0: nothing to add */
            continue;
        if (KIND == AG_PUSH_FIXED)
            atomicAdd((unsigned long long *)p.c64_1 + i, t);
        else
            atomicAdd(reinterpret_cast<double *>(p.c64_1) + i, __longlong_as_double((long long)t));
    }
}

/* element-wise update of the push forms; the last CTA closes the pass */
template <int KIND> __global__ void __launch_bounds__(AG_SBLK) ag_push_update_kernel(const AgPullParams p)
{
    if (ag_push_stopped(p))
        return;
    const double eps = p.ctl->eps;
    double my_err = 0.0;
    uint32_t my_active = 0, mn = 0xFFFFFFFFu, mx = 0u;
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        float rn;
        if (KIND == AG_PUSH_FIXED) {
            const uint64_t s = p.c64_1[v];
            p.c64_1[v] = 0ull;
            rn = __double2float_rn(__dadd_rn((double)p.base, __dmul_rn((double)p.damp, ag_fixed2d(s))));
        } else {
            double *nd = reinterpret_cast<double *>(p.c64_1);
            const float s = __double2float_rn(nd[v]);
            nd[v] = 0.0;
            rn = __fadd_rn(p.base, __fmul_rn(p.damp, s));
        }
        const float rp = p.rank[v];
        const double err = (double)fabsf(__fsub_rn(rn, rp));
        my_err += err;
        my_active += (err >= eps) ? 1u : 0u;
        p.rank[v] = rn;
        const uint32_t od = p.outdeg[v];
        if (KIND == AG_PUSH_FIXED) {
            p.c64_0[v] = od ? ag_d2fixed((double)__fdiv_rn(rn, __uint2float_rn(od))) : 0ull;
        } else {
            const float c = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
            p.pa[v] = c;
            if (KIND == AG_PUSH_QUANT) {
                const uint32_t k = ag_fkey(c);
                mn = min(mn, k);
                mx = max(mx, k);
            }
        }
    }
    ag_close_pass<AG_PNW>(p, my_err, my_active, KIND == AG_PUSH_QUANT, mn, mx, true);
}

/* ------------------------------------------------------------ residual */
/* vertex phase: worklist vertices take their residual, form the new rank,
 * add to the pass's error and store their delta and the residual taken (pb,
 * for the crossing test of a self-edge); the previous pass's worklist (the
 * buffer the edge phase fills next) is cleared */
template <bool PULLPUSH> __global__ void __launch_bounds__(AG_SBLK) ag_residual_vertex_kernel(const AgPullParams p)
{
    if (ag_push_stopped(p))
        return;
    const uint32_t pass = p.ctl->iter;
    const uint8_t *wl_cur = p.wl + (size_t)(pass & 1u) * p.N;
    uint8_t *wl_old = p.wl + (size_t)((pass + 1u) & 1u) * p.N;
    const float fN = __uint2float_rn(p.N);
    double my_err = 0.0;
    for (uint32_t v = blockIdx.x * AG_SBLK + threadIdx.x; v < p.N; v += gridDim.x * AG_SBLK) {
        wl_old[v] = 0;
        if (!wl_cur[v])
            continue;
        const float old = p.rank[v];
        const float res = atomicExch(p.res + v, 0.0f);
        /* pull-push: the pull over v's in-edges of the start-of-pass
         * contributions (pb, from the pass's first kernel) */
        const float rn = PULLPUSH ? __fadd_rn(p.base, __fmul_rn(p.damp, p.pb[v])) : __fadd_rn(res, old);
        my_err += (double)fabsf(__fsub_rn(__fdiv_rn(rn, fN), __fdiv_rn(old, fN)));
        p.rank[v] = rn;
        p.pb[v] = res;
        const uint32_t od = p.outdeg[v];
        /* without out-edges the delta is never read */
        p.delta[v] = od ? __fmul_rn(p.damp, __fdiv_rn(res, __uint2float_rn(od))) : 0.0f;
        if (PULLPUSH)
            p.pa[v] = od ? __fdiv_rn(rn, __uint2float_rn(od)) : 0.0f;
    }
    /* the error joins the pass's record (one atomic per CTA); the edge phase
     * closes the pass */
    const double e = ag_push_block_sum_d(my_err);
    if (threadIdx.x == 0 && e != 0.0)
        atomicAdd(&p.ctl->err_acc, e);
}

/* Edge phase: one thread per forward edge of a worklist source (a
 * persistent grid of AG_PUSH_BLK-thread CTAs).  In the data-driven push the
 * first AG_RES_HOT destinations (the in-hubs of power-law graphs) are summed
 * first in a shared-memory table of the CTA and added to the residual once per
 * CTA, with the crossing test on that add: residuals only grow within a pass,
 * so exactly one add takes a residual across epsilon whether the adds come
 * one edge at a time or one CTA at a time, and the activations and the next
 * worklist are the same.  The pull-push adds each crossing edge's delta a
 * second time, so every one of its edges adds on its own. */
template <bool PULLPUSH> __global__ void __launch_bounds__(AG_PUSH_BLK) ag_residual_edge_kernel(const AgPullParams p)
{
    extern __shared__ __align__(16) unsigned long long ag_push_hot[];
    float *hot = reinterpret_cast<float *>(ag_push_hot);
    if (ag_push_stopped(p))
        return;
    const uint32_t pass = p.ctl->iter;
    const uint8_t *wl_cur = p.wl + (size_t)(pass & 1u) * p.N;
    uint8_t *wl_next = p.wl + (size_t)((pass + 1u) & 1u) * p.N;
    const double eps = p.ctl->eps;
    const uint32_t hot_n = PULLPUSH ? 0u : min(p.N, (uint32_t)AG_RES_HOT);
    for (uint32_t i = threadIdx.x; i < hot_n; i += AG_PUSH_BLK)
        hot[i] = 0.0f;
    __syncthreads();
    const uint64_t pol_first = ag_policy_evict_first();
    uint32_t my_act = 0;
    auto crosses = [&](float prev, float add) {
        return (double)fabsf(__fadd_rn(prev, add)) >= eps && (double)prev <= eps;
    };
    const uint32_t stride = gridDim.x * AG_PUSH_BLK;
    for (uint32_t j = blockIdx.x * AG_PUSH_BLK + threadIdx.x; j < p.E; j += stride) {
        const uint32_t v = ag_ld_stream_u32(p.fwd_src + j, pol_first);
        if (!wl_cur[v])
            continue;
        const uint32_t u = ag_ld_stream_u32(p.fwd_dst + j, pol_first);
        const float dl = p.delta[v];
        if (u < hot_n && u != v) {
            atomicAdd(hot + u, dl);
            continue;
        }
        const float prev = u == v ? p.pb[v] : atomicAdd(p.res + u, dl);
        if (crosses(prev, dl)) {
            ++my_act;
            if (PULLPUSH && u != v)
                atomicAdd(p.res + u, dl);
            wl_next[u] = 1;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hot_n; i += AG_PUSH_BLK) {
        const float t = hot[i];
        if (t == 0.0f)
            continue;
        const float prev = atomicAdd(p.res + i, t);
        if (crosses(prev, t)) {
            ++my_act;
            wl_next[i] = 1;
        }
    }
    ag_close_pass<AG_PUSH_BLK / 32>(p, 0.0, my_act, false, 0xFFFFFFFFu, 0u, false);
}

/* --------------------------------------------------- forward edge list */
/* rows[j] = the row holding in-edge j (binary search of the row starts) */
__global__ void ag_edge_rows_kernel(const uint32_t *row_off, uint32_t n, uint32_t e, uint32_t *rows)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < e; j += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n; /* row_off[lo] <= j < row_off[hi] */
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(row_off + mid) <= j)
                lo = mid;
            else
                hi = mid;
        }
        rows[j] = lo;
    }
}

extern "C" cudaError_t ag_forward_build(const uint32_t *row_off, const uint32_t *ids, uint32_t n, uint32_t e,
                                        uint32_t *fwd_src, uint32_t *fwd_dst, cudaStream_t s)
{
    if (e == 0)
        return cudaSuccess;
    uint32_t *rows = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int bits = 1;
    while (bits < 32 && (1ull << bits) < (uint64_t)n)
        ++bits;
    cudaError_t err = cudaMallocAsync((void **)&rows, (size_t)e * 4, s);
    if (err != cudaSuccess)
        return err;
    unsigned blocks = (e + 255) / 256;
    if (blocks > ag_sm_grid(32))
        blocks = ag_sm_grid(32);
    ag_edge_rows_kernel<<<blocks, 256, 0, s>>>(row_off, n, e, rows);
    err = cudaGetLastError();
    /* stable by source: each source's destinations stay in row order */
    if (err == cudaSuccess)
        err = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, ids, fwd_src, rows, fwd_dst, (int)e, 0, bits, s);
    if (err == cudaSuccess)
        err = cudaMallocAsync(&tmp, tmp_bytes, s);
    if (err == cudaSuccess)
        err = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, ids, fwd_src, rows, fwd_dst, (int)e, 0, bits, s);
    if (tmp)
        cudaFreeAsync(tmp, s);
    cudaFreeAsync(rows, s);
    return err;
}

/* launch shape of the push scatter and of the residual edge phase: threads
 * per CTA, dynamic shared memory */
extern "C" void ag_push_scatter_shape(unsigned *threads, size_t *smem)
{
    *threads = AG_PUSH_BLK;
    *smem = (size_t)AG_PUSH_HOT * 8;
}

extern "C" const void *ag_push_kernel_ptr(int kind, int stage)
{
    /* stage 0 init, 1 scatter / vertex phase, 2 update / edge phase,
     * 3 quantiser (kind 2) or seed (kinds 3, 4) */
    switch (kind) {
    case AG_PUSH_FLOAT:
        return stage == 0   ? (const void *)ag_push_init_kernel<AG_PUSH_FLOAT>
               : stage == 1 ? (const void *)ag_push_scatter_kernel<AG_PUSH_FLOAT>
                            : (const void *)ag_push_update_kernel<AG_PUSH_FLOAT>;
    case AG_PUSH_FIXED:
        return stage == 0   ? (const void *)ag_push_init_kernel<AG_PUSH_FIXED>
               : stage == 1 ? (const void *)ag_push_scatter_kernel<AG_PUSH_FIXED>
                            : (const void *)ag_push_update_kernel<AG_PUSH_FIXED>;
    case AG_PUSH_QUANT:
        return stage == 0   ? (const void *)ag_push_init_kernel<AG_PUSH_QUANT>
               : stage == 1 ? (const void *)ag_push_scatter_kernel<AG_PUSH_QUANT>
               : stage == 2 ? (const void *)ag_push_update_kernel<AG_PUSH_QUANT>
                            : (const void *)ag_push_quant_kernel;
    case AG_PUSH_DD:
        return stage == 0   ? (const void *)ag_residual_init_kernel
               : stage == 1 ? (const void *)ag_residual_vertex_kernel<false>
               : stage == 2 ? (const void *)ag_residual_edge_kernel<false>
                            : (const void *)ag_residual_seed_kernel;
    default:
        return stage == 0   ? (const void *)ag_residual_init_kernel
               : stage == 1 ? (const void *)ag_residual_vertex_kernel<true>
               : stage == 2 ? (const void *)ag_residual_edge_kernel<true>
                            : (const void *)ag_residual_seed_kernel;
    }
}
