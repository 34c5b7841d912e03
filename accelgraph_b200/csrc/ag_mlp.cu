/*
 * ag_mlp.cu -- learned warm start for the pull PageRank: per-vertex degree
 * features, and a small MLP (8 -> 64 -> 64 -> 1, ReLU) that predicts the
 * log of a vertex's un-normalised rank, with hand-written training and
 * inference kernels.
 *
 * Features of vertex v (in-neighbours u over the inverse CSR), all log1p:
 *   f0 in-degree(v)            f1 out-degree(v)
 *   f2 sum in-degree(u)        f3 sum out-degree(u)          (2-hop degrees)
 *   f4 min out-degree(u)       f5 max out-degree(u)          (0 without u)
 *   f6 sum 1/out-degree(u)     (one pull pass from uniform ranks)
 *   f7 max in-degree(u)
 *
 * Precision: master weights are binary32; the forward pass of training and
 * inference uses their bfloat16 rounding (round to nearest even) with binary32
 * accumulation; gradients are taken with respect to the bfloat16 weights and
 * applied to the binary32 masters (Adam).
 *
 * Training step (mini-batch of B samples):
 *   k1  one thread per sample: forward, loss, and the per-sample backward
 *       signals dh2 = d loss / d pre-activation of layer 2 (masked by ReLU),
 *       dh1 likewise for layer 1; stores x, h1, h2, dh1, dh2 and d3.
 *   k2  one CTA per chunk of 128 samples: the weight gradients as
 *       chunk-local sums over samples staged in shared memory
 *       (dW2 = dh2^T h1, dW1 = dh1^T x, dW3 = d3 h2, biases), added to the
 *       global gradient with one atomic per weight per chunk.
 *   k3  Adam update of the 4801 parameters, refresh of the bfloat16 copies.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "ag_device.h"
#include "ag_internal.h"
#include "ag_rng.h"

#define AG_MLP_IN 8
#define AG_MLP_H 64
/* parameter layout (binary32 masters): W1[64][8] b1[64] W2[64][64] b2[64] w3[64] b3 */
#define AG_MLP_OFF_W1 0
#define AG_MLP_OFF_B1 (AG_MLP_OFF_W1 + AG_MLP_H * AG_MLP_IN)
#define AG_MLP_OFF_W2 (AG_MLP_OFF_B1 + AG_MLP_H)
#define AG_MLP_OFF_B2 (AG_MLP_OFF_W2 + AG_MLP_H * AG_MLP_H)
#define AG_MLP_OFF_W3 (AG_MLP_OFF_B2 + AG_MLP_H)
#define AG_MLP_OFF_B3 (AG_MLP_OFF_W3 + AG_MLP_H)
#define AG_MLP_NPARAM (AG_MLP_OFF_B3 + 1)
#define AG_MLP_BLK 128
#define AG_MLP_CHUNK 128

struct ag_mlp_s
{
    float *w;        /* masters (device)              */
    __nv_bfloat16 *wb; /* bfloat16 copies (device)    */
    float *g;        /* gradient accumulator          */
    float *m, *v;    /* Adam moments                  */
    float *buf;      /* per-sample training signals   */
    uint32_t buf_cap;
    float *part;     /* per-chunk gradient sums       */
    uint32_t part_cap; /* chunks                      */
    float *loss;     /* device scalar                 */
    uint32_t step;
};

/* ---------------------------------------------------------- features */
/* (in-degree, out-degree) of every vertex, device order: one 8-byte gather
 * per in-edge instead of three */
__global__ void ag_deg2_kernel(AgGraphView gv, uint2 *deg2)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < gv.N; v += gridDim.x * blockDim.x)
        deg2[v] = make_uint2(gv.row_off[v + 1] - gv.row_off[v], gv.outdeg[v]);
}

/* Per-row statistics of the in-neighbours u, all integers so that they
 * come out the same in any order and on any split of the row: sums of u's
 * in- and out-degree, the sum of 1/out-degree(u) in fixed point (2^40 units,
 * one binary32 reciprocal per edge), and the extremes of the degrees. */
struct AgFeatAcc
{
    unsigned long long s_in, s_out, s_c;
    uint32_t mx_in, mx_out, mn_out;
};

#define AG_FEAT_FIX 1099511627776.0 /* 2^40 */

__device__ __forceinline__ AgFeatAcc ag_feat_zero()
{
    AgFeatAcc a;
    a.s_in = a.s_out = a.s_c = 0ull;
    a.mx_in = a.mx_out = 0u;
    a.mn_out = 0xFFFFFFFFu;
    return a;
}

__device__ __forceinline__ void ag_feat_edge(uint2 d, AgFeatAcc &a)
{
    a.s_in += d.x;
    a.s_out += d.y;
    a.s_c += d.y ? __double2ull_rn((double)__frcp_rn((float)d.y) * AG_FEAT_FIX) : 0ull;
    a.mx_in = max(a.mx_in, d.x);
    a.mx_out = max(a.mx_out, d.y);
    a.mn_out = min(a.mn_out, d.y);
}

__device__ __forceinline__ AgFeatAcc ag_feat_warp(AgFeatAcc a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a.s_in += __shfl_xor_sync(0xffffffffu, a.s_in, o);
        a.s_out += __shfl_xor_sync(0xffffffffu, a.s_out, o);
        a.s_c += __shfl_xor_sync(0xffffffffu, a.s_c, o);
    }
    a.mx_in = __reduce_max_sync(0xffffffffu, a.mx_in);
    a.mx_out = __reduce_max_sync(0xffffffffu, a.mx_out);
    a.mn_out = __reduce_min_sync(0xffffffffu, a.mn_out);
    return a;
}

/* the warp's lane-strided pass over in-edges [b, e) */
__device__ __forceinline__ AgFeatAcc ag_feat_range(const AgGraphView &gv, const uint2 *deg2, uint32_t b, uint32_t e,
                                                   uint32_t lane)
{
    AgFeatAcc a = ag_feat_zero();
    uint32_t j = b + lane;
    for (; j + 96 < e; j += 128) {
        const uint32_t u0 = __ldg(gv.ids + j), u1 = __ldg(gv.ids + j + 32), u2 = __ldg(gv.ids + j + 64),
                       u3 = __ldg(gv.ids + j + 96);
        const uint2 d0 = __ldg(deg2 + u0), d1 = __ldg(deg2 + u1), d2 = __ldg(deg2 + u2), d3 = __ldg(deg2 + u3);
        ag_feat_edge(d0, a);
        ag_feat_edge(d1, a);
        ag_feat_edge(d2, a);
        ag_feat_edge(d3, a);
    }
    for (; j < e; j += 32)
        ag_feat_edge(__ldg(deg2 + __ldg(gv.ids + j)), a);
    return ag_feat_warp(a);
}

/* the eight features of a vertex, written in caller order (two 16-byte
 * stores when the output is 16-byte aligned) */
__device__ __forceinline__ void ag_features_store(const AgGraphView &gv, float *X, uint32_t v, uint32_t deg,
                                                  const AgFeatAcc &a, bool vec)
{
    const uint32_t dst = gv.perm ? gv.perm[v] : v;
    float *x = X + (size_t)dst * AG_MLP_IN;
    const float4 lo = make_float4(log1pf((float)deg), log1pf((float)gv.outdeg[v]), log1pf((float)a.s_in),
                                  log1pf((float)a.s_out));
    const float4 hi = make_float4(log1pf(deg ? (float)a.mn_out : 0.0f), log1pf((float)a.mx_out),
                                  log1pf((float)((double)a.s_c * (1.0 / AG_FEAT_FIX))), log1pf((float)a.mx_in));
    if (vec) {
        reinterpret_cast<float4 *>(x)[0] = lo;
        reinterpret_cast<float4 *>(x)[1] = hi;
    } else {
        x[0] = lo.x;
        x[1] = lo.y;
        x[2] = lo.z;
        x[3] = lo.w;
        x[4] = hi.x;
        x[5] = hi.y;
        x[6] = hi.z;
        x[7] = hi.w;
    }
}

/* All features in one pass over the pull kernel's work list, so that the
 * gathers are balanced as the pull's are (a warp per item):
 *  - row items: one row per lane; rows of up to 32 in-edges by their lane
 *    (four gathers in flight), longer ones by the whole warp;
 *  - long rows: the whole warp;
 *  - hub chunks: the whole warp, then integer atomics into the row's slot
 *    (acc: three sums, ext: two maxima, the complemented minimum, and the
 *    in-edges seen); the chunk that completes the row writes it. */
__global__ void __launch_bounds__(256) ag_features_items_kernel(AgGraphView gv, const uint2 *deg2,
                                                                unsigned long long *acc, uint32_t *ext, float *X)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const bool vec = (reinterpret_cast<uintptr_t>(X) & 15u) == 0;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < gv.ntasks; t += nw) {
        const uint4 task = gv.tasks[t];
        const uint32_t kind = task.x >> 30, r0 = task.x & AG_ROW_MASK;
        if (kind == AG_T_ROWS) {
            const uint32_t r = r0 + lane;
            const bool live = r < task.y;
            uint32_t b = 0, e = 0;
            if (live) {
                b = gv.row_off[r];
                e = gv.row_off[r + 1];
            }
            AgFeatAcc a = ag_feat_zero();
            const bool mine = live && e - b <= 32;
            if (mine) {
                uint32_t j = b;
                for (; j + 4 <= e; j += 4) {
                    const uint32_t u0 = __ldg(gv.ids + j), u1 = __ldg(gv.ids + j + 1), u2 = __ldg(gv.ids + j + 2),
                                   u3 = __ldg(gv.ids + j + 3);
                    const uint2 d0 = __ldg(deg2 + u0), d1 = __ldg(deg2 + u1), d2 = __ldg(deg2 + u2),
                                d3 = __ldg(deg2 + u3);
                    ag_feat_edge(d0, a);
                    ag_feat_edge(d1, a);
                    ag_feat_edge(d2, a);
                    ag_feat_edge(d3, a);
                }
                for (; j < e; ++j)
                    ag_feat_edge(__ldg(deg2 + __ldg(gv.ids + j)), a);
            }
            unsigned m = __ballot_sync(0xffffffffu, live && !mine);
            while (m) {
                const int src = __ffs(m) - 1;
                m &= m - 1;
                const AgFeatAcc w =
                    ag_feat_range(gv, deg2, __shfl_sync(0xffffffffu, b, src), __shfl_sync(0xffffffffu, e, src), lane);
                if ((int)lane == src)
                    a = w;
            }
            if (live)
                ag_features_store(gv, X, r, e - b, a, vec);
        } else if (kind == AG_T_LONG) {
            const AgFeatAcc w = ag_feat_range(gv, deg2, task.z, task.w, lane);
            if (lane == 0)
                ag_features_store(gv, X, r0, task.w - task.z, w, vec);
        } else {
            const AgFeatAcc w = ag_feat_range(gv, deg2, task.z, task.w, lane);
            if (lane == 0) {
                const uint32_t slot = task.y & AG_SLOT_MASK;
                unsigned long long *ac = acc + (size_t)slot * 3;
                uint32_t *ex = ext + (size_t)slot * 4;
                atomicAdd(ac, w.s_in);
                atomicAdd(ac + 1, w.s_out);
                atomicAdd(ac + 2, w.s_c);
                atomicMax(ex, w.mx_in);
                atomicMax(ex + 1, w.mx_out);
                atomicMax(ex + 2, 0xFFFFFFFFu - w.mn_out);
                __threadfence();
                const uint32_t deg = gv.row_off[r0 + 1] - gv.row_off[r0];
                const uint32_t seen = atomicAdd(ex + 3, task.w - task.z) + (task.w - task.z);
                if (seen == deg) {
                    /* every chunk of the row is in: the row's totals */
                    __threadfence();
                    AgFeatAcc a;
                    a.s_in = __ldcg(ac);
                    a.s_out = __ldcg(ac + 1);
                    a.s_c = __ldcg(ac + 2);
                    a.mx_in = __ldcg(ex);
                    a.mx_out = __ldcg(ex + 1);
                    a.mn_out = 0xFFFFFFFFu - __ldcg(ex + 2);
                    ag_features_store(gv, X, r0, deg, a, vec);
                }
            }
        }
    }
}

/* ------------------------------------------------------------ MLP math */
__device__ __forceinline__ void ag_mlp_load_weights(const __nv_bfloat16 *wb, float *sw)
{
    for (uint32_t i = threadIdx.x; i < AG_MLP_NPARAM; i += blockDim.x)
        sw[i] = __bfloat162float(wb[i]);
    __syncthreads();
}

/* layer 1 and 2 activations of one sample */
__device__ __forceinline__ void ag_mlp_hidden(const float *sw, const float *x, float *h1, float *h2)
{
#pragma unroll 8
    for (int j = 0; j < AG_MLP_H; ++j) {
        float a = sw[AG_MLP_OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < AG_MLP_IN; ++i)
            a = fmaf(sw[AG_MLP_OFF_W1 + j * AG_MLP_IN + i], x[i], a);
        h1[j] = fmaxf(a, 0.0f);
    }
#pragma unroll 4
    for (int k = 0; k < AG_MLP_H; ++k) {
        float a = sw[AG_MLP_OFF_B2 + k];
#pragma unroll
        for (int j = 0; j < AG_MLP_H; ++j)
            a = fmaf(sw[AG_MLP_OFF_W2 + k * AG_MLP_H + j], h1[j], a);
        h2[k] = fmaxf(a, 0.0f);
    }
}

__device__ __forceinline__ float ag_mlp_out(const float *sw, const float *h2)
{
    float y = sw[AG_MLP_OFF_B3];
#pragma unroll
    for (int k = 0; k < AG_MLP_H; ++k)
        y = fmaf(sw[AG_MLP_OFF_W3 + k], h2[k], y);
    return y;
}

/* Inference: one sample per thread and no loop over samples, so that the
 * compiler cannot hoist the shared-memory weights into registers across
 * samples.  The first hidden layer stays in registers (its loops are fully
 * unrolled, every index a constant) and the output layer is folded into the
 * loop over the second layer's units, so no activation array lives in local
 * memory.  Sums run in the same order as ag_mlp_hidden / ag_mlp_out. */
__global__ void __launch_bounds__(AG_MLP_BLK) ag_mlp_infer_kernel(const __nv_bfloat16 *wb, const float *X, uint32_t n,
                                                                  float *Y)
{
    __shared__ __align__(16) float sw[AG_MLP_NPARAM];
    ag_mlp_load_weights(wb, sw);
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    float x[AG_MLP_IN];
#pragma unroll
    for (int i = 0; i < AG_MLP_IN; ++i)
        x[i] = X[(size_t)s * AG_MLP_IN + i];
    float h1[AG_MLP_H];
#pragma unroll
    for (int j = 0; j < AG_MLP_H; ++j) {
        float a = sw[AG_MLP_OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < AG_MLP_IN; ++i)
            a = fmaf(sw[AG_MLP_OFF_W1 + j * AG_MLP_IN + i], x[i], a);
        h1[j] = fmaxf(a, 0.0f);
    }
    float y = sw[AG_MLP_OFF_B3];
#pragma unroll 1
    for (int k = 0; k < AG_MLP_H; ++k) {
        float a = sw[AG_MLP_OFF_B2 + k];
#pragma unroll
        for (int j = 0; j < AG_MLP_H; ++j)
            a = fmaf(sw[AG_MLP_OFF_W2 + k * AG_MLP_H + j], h1[j], a);
        y = fmaf(sw[AG_MLP_OFF_W3 + k], fmaxf(a, 0.0f), y);
    }
    Y[s] = y;
}

/* ------------------------------------------------ tensor-core inference */
/* The warm start's prediction on the tensor cores: one warp per tile of 16
 * vertices, mma.sync m16n8k16 with bfloat16 operands and binary32
 * accumulation.  A binary32 activation a is split into a bfloat16 head
 * hi = bf16(a) and tail lo = bf16(a - hi), and hi * w + lo * w is formed
 * exactly in the accumulator, so the products see about 16 significant bits
 * of a instead of 8 (the weights are bfloat16 in both forward passes).
 *  layer 1: K = 16 holds the 8 features' heads and their 8 tails, B = W1^T
 *           twice; 8 MMAs give the 16 x 64 pre-activations, bias and ReLU in
 *           binary32.
 *  layer 2: the layer-1 accumulator fragments are exactly the A fragments of
 *           the next product (columns 16 ks .. 16 ks + 15 are n-tiles 2 ks and
 *           2 ks + 1); heads and tails, B = W2^T: 2 x 4 k-steps x 8 n-tiles =
 *           64 MMAs.
 *  output:  bias, ReLU and the 64-weight dot product on the accumulators, a
 *           sum over the 4 lanes that share a row.
 * The sums run in another order than ag_mlp_forward's, and the tails lose
 * the last bits: the prediction agrees with the binary32 forward pass to
 * about 1e-4 in log-rank.  Fragment layouts: PTX ISA, mma.m16n8k16 for
 * .bf16. */
__device__ __forceinline__ uint32_t ag_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

/* the bfloat16 tails of a pair: a - bf16(a) */
__device__ __forceinline__ uint32_t ag_bf16x2_tail(float a, float b)
{
    return ag_bf16x2(a - __bfloat162float(__float2bfloat16_rn(a)), b - __bfloat162float(__float2bfloat16_rn(b)));
}

__device__ __forceinline__ void ag_mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                            uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

#define AG_MLP_TC_BLK 256
__global__ void __launch_bounds__(AG_MLP_TC_BLK) ag_mlp_infer_tc_kernel(const __nv_bfloat16 *wb, const float *X,
                                                                        uint32_t n, float *Y)
{
    /* W1 and W2 as bfloat16 pairs along the input index: pair p of output o
     * holds inputs 2p, 2p+1 (the B fragment's element order) */
    __shared__ uint32_t sw1[AG_MLP_H * AG_MLP_IN / 2];
    __shared__ uint32_t sw2[AG_MLP_H * AG_MLP_H / 2];
    __shared__ float sb1[AG_MLP_H], sb2[AG_MLP_H], sw3[AG_MLP_H];
    __shared__ float sb3;
    const uint32_t *wp = reinterpret_cast<const uint32_t *>(wb);
    for (uint32_t i = threadIdx.x; i < AG_MLP_H * AG_MLP_IN / 2; i += blockDim.x)
        sw1[i] = wp[AG_MLP_OFF_W1 / 2 + i];
    for (uint32_t i = threadIdx.x; i < AG_MLP_H * AG_MLP_H / 2; i += blockDim.x)
        sw2[i] = wp[AG_MLP_OFF_W2 / 2 + i];
    for (uint32_t i = threadIdx.x; i < AG_MLP_H; i += blockDim.x) {
        sb1[i] = __bfloat162float(wb[AG_MLP_OFF_B1 + i]);
        sb2[i] = __bfloat162float(wb[AG_MLP_OFF_B2 + i]);
        sw3[i] = __bfloat162float(wb[AG_MLP_OFF_W3 + i]);
    }
    if (threadIdx.x == 0)
        sb3 = __bfloat162float(wb[AG_MLP_OFF_B3]);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const uint32_t nwarps = gridDim.x * (AG_MLP_TC_BLK / 32);
    for (uint32_t tile = blockIdx.x * (AG_MLP_TC_BLK / 32) + (threadIdx.x >> 5); (uint64_t)tile * 16 < n;
         tile += nwarps) {
        const uint32_t r0 = tile * 16 + gid, r1 = r0 + 8;
        /* features of rows r0 and r1, columns 2 tig and 2 tig + 1 */
        float2 x0 = make_float2(0.f, 0.f), x1 = x0;
        if (r0 < n)
            x0 = *reinterpret_cast<const float2 *>(X + (size_t)r0 * AG_MLP_IN + 2 * tig);
        if (r1 < n)
            x1 = *reinterpret_cast<const float2 *>(X + (size_t)r1 * AG_MLP_IN + 2 * tig);
        const uint32_t xa0 = ag_bf16x2(x0.x, x0.y), xa1 = ag_bf16x2(x1.x, x1.y);
        const uint32_t xt0 = ag_bf16x2_tail(x0.x, x0.y), xt1 = ag_bf16x2_tail(x1.x, x1.y);
        /* layer 1: n-tile t gives units 8 t .. 8 t + 7; K 0-7 heads, 8-15 tails */
        float h[8][4];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            h[t][0] = h[t][1] = h[t][2] = h[t][3] = 0.0f;
            const uint32_t w1 = sw1[(8 * t + gid) * (AG_MLP_IN / 2) + tig];
            ag_mma_bf16(h[t], xa0, xa1, xt0, xt1, w1, w1);
            const uint32_t c = 8 * t + 2 * tig;
            h[t][0] = fmaxf(h[t][0] + sb1[c], 0.0f);
            h[t][1] = fmaxf(h[t][1] + sb1[c + 1], 0.0f);
            h[t][2] = fmaxf(h[t][2] + sb1[c], 0.0f);
            h[t][3] = fmaxf(h[t][3] + sb1[c + 1], 0.0f);
        }
        /* layer 2 and the output layer, one n-tile of 8 units at a time */
        float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            const uint32_t *w2 = sw2 + (8 * t + gid) * (AG_MLP_H / 2);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint32_t b0 = w2[8 * ks + tig], b1 = w2[8 * ks + 4 + tig];
                ag_mma_bf16(acc, ag_bf16x2(h[2 * ks][0], h[2 * ks][1]), ag_bf16x2(h[2 * ks][2], h[2 * ks][3]),
                            ag_bf16x2(h[2 * ks + 1][0], h[2 * ks + 1][1]),
                            ag_bf16x2(h[2 * ks + 1][2], h[2 * ks + 1][3]), b0, b1);
                ag_mma_bf16(acc, ag_bf16x2_tail(h[2 * ks][0], h[2 * ks][1]),
                            ag_bf16x2_tail(h[2 * ks][2], h[2 * ks][3]),
                            ag_bf16x2_tail(h[2 * ks + 1][0], h[2 * ks + 1][1]),
                            ag_bf16x2_tail(h[2 * ks + 1][2], h[2 * ks + 1][3]), b0, b1);
            }
            const uint32_t c = 8 * t + 2 * tig;
            y0 = fmaf(sw3[c], fmaxf(acc[0] + sb2[c], 0.0f), y0);
            y0 = fmaf(sw3[c + 1], fmaxf(acc[1] + sb2[c + 1], 0.0f), y0);
            y1 = fmaf(sw3[c], fmaxf(acc[2] + sb2[c], 0.0f), y1);
            y1 = fmaf(sw3[c + 1], fmaxf(acc[3] + sb2[c + 1], 0.0f), y1);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (tig == 0) {
            if (r0 < n)
                Y[r0] = y0 + sb3;
            if (r1 < n)
                Y[r1] = y1 + sb3;
        }
    }
}

/* per-sample training signals; buf layout per sample (stride 2 + 4*64 + 8):
 * [x(8) h1(64) h2(64) dh1(64) dh2(64) d3 pad] */
#define AG_MLP_REC (AG_MLP_IN + 4 * AG_MLP_H + 2)
__global__ void __launch_bounds__(AG_MLP_BLK) ag_mlp_k1(const __nv_bfloat16 *wb, const float *X, const float *T,
                                                        uint32_t n, float scale, float *buf, float *loss)
{
    __shared__ float sw[AG_MLP_NPARAM];
    __shared__ float sl[AG_MLP_BLK / 32];
    ag_mlp_load_weights(wb, sw);
    float my_loss = 0.0f;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float x[AG_MLP_IN], h1[AG_MLP_H], h2[AG_MLP_H];
#pragma unroll
        for (int i = 0; i < AG_MLP_IN; ++i)
            x[i] = X[(size_t)s * AG_MLP_IN + i];
        ag_mlp_hidden(sw, x, h1, h2);
        const float y = ag_mlp_out(sw, h2);
        const float r = y - T[s];
        my_loss += r * r;
        const float d3 = 2.0f * r * scale; /* d (mean squared error) / d y */
        float *rec = buf + (size_t)s * AG_MLP_REC;
#pragma unroll
        for (int i = 0; i < AG_MLP_IN; ++i)
            rec[i] = x[i];
        float dh2[AG_MLP_H];
#pragma unroll
        for (int k = 0; k < AG_MLP_H; ++k) {
            dh2[k] = h2[k] > 0.0f ? d3 * sw[AG_MLP_OFF_W3 + k] : 0.0f;
            rec[AG_MLP_IN + k] = h1[k];
            rec[AG_MLP_IN + AG_MLP_H + k] = h2[k];
            rec[AG_MLP_IN + 3 * AG_MLP_H + k] = dh2[k];
        }
#pragma unroll 4
        for (int j = 0; j < AG_MLP_H; ++j) {
            float a = 0.0f;
#pragma unroll
            for (int k = 0; k < AG_MLP_H; ++k)
                a = fmaf(dh2[k], sw[AG_MLP_OFF_W2 + k * AG_MLP_H + j], a);
            rec[AG_MLP_IN + 2 * AG_MLP_H + j] = h1[j] > 0.0f ? a : 0.0f;
        }
        rec[AG_MLP_IN + 4 * AG_MLP_H] = d3;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
    if ((threadIdx.x & 31) == 0)
        sl[threadIdx.x >> 5] = my_loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < AG_MLP_BLK / 32; ++w)
            t += sl[w];
        atomicAdd(loss, t);
    }
}

/* chunk sums of the weight gradients over AG_MLP_CHUNK samples, one row of
 * part per chunk (added in chunk order by ag_mlp_k3, so that a gradient
 * does not depend on which chunk finishes first) */
__global__ void __launch_bounds__(256) ag_mlp_k2(const float *buf, uint32_t n, float *part)
{
    extern __shared__ float sm[]; /* AG_MLP_CHUNK x AG_MLP_REC */
    const uint32_t s0 = blockIdx.x * AG_MLP_CHUNK;
    const uint32_t cnt = min((uint32_t)AG_MLP_CHUNK, n - s0);
    for (uint32_t i = threadIdx.x; i < cnt * AG_MLP_REC; i += blockDim.x)
        sm[i] = buf[(size_t)s0 * AG_MLP_REC + i];
    __syncthreads();
    for (uint32_t o = threadIdx.x; o < AG_MLP_NPARAM; o += blockDim.x) {
        float a = 0.0f;
        if (o < AG_MLP_OFF_B1) { /* W1[j][i] = sum dh1[j] x[i] */
            const uint32_t j = o / AG_MLP_IN, i = o % AG_MLP_IN;
            for (uint32_t s = 0; s < cnt; ++s)
                a = fmaf(sm[s * AG_MLP_REC + AG_MLP_IN + 2 * AG_MLP_H + j], sm[s * AG_MLP_REC + i], a);
        } else if (o < AG_MLP_OFF_W2) { /* b1[j] */
            const uint32_t j = o - AG_MLP_OFF_B1;
            for (uint32_t s = 0; s < cnt; ++s)
                a += sm[s * AG_MLP_REC + AG_MLP_IN + 2 * AG_MLP_H + j];
        } else if (o < AG_MLP_OFF_B2) { /* W2[k][j] = sum dh2[k] h1[j] */
            const uint32_t k = (o - AG_MLP_OFF_W2) / AG_MLP_H, j = (o - AG_MLP_OFF_W2) % AG_MLP_H;
            for (uint32_t s = 0; s < cnt; ++s)
                a = fmaf(sm[s * AG_MLP_REC + AG_MLP_IN + 3 * AG_MLP_H + k], sm[s * AG_MLP_REC + AG_MLP_IN + j], a);
        } else if (o < AG_MLP_OFF_W3) { /* b2[k] */
            const uint32_t k = o - AG_MLP_OFF_B2;
            for (uint32_t s = 0; s < cnt; ++s)
                a += sm[s * AG_MLP_REC + AG_MLP_IN + 3 * AG_MLP_H + k];
        } else if (o < AG_MLP_OFF_B3) { /* w3[k] = sum d3 h2[k] */
            const uint32_t k = o - AG_MLP_OFF_W3;
            for (uint32_t s = 0; s < cnt; ++s)
                a = fmaf(sm[s * AG_MLP_REC + AG_MLP_IN + 4 * AG_MLP_H], sm[s * AG_MLP_REC + AG_MLP_IN + AG_MLP_H + k],
                         a);
        } else { /* b3 */
            for (uint32_t s = 0; s < cnt; ++s)
                a += sm[s * AG_MLP_REC + AG_MLP_IN + 4 * AG_MLP_H];
        }
        part[(size_t)blockIdx.x * AG_MLP_NPARAM + o] = a;
    }
}

/* the gradient: the chunk sums added in chunk order */
__global__ void ag_mlp_k3(const float *part, uint32_t nchunks, float *grad)
{
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < AG_MLP_NPARAM; o += gridDim.x * blockDim.x) {
        float a = 0.0f;
        for (uint32_t c = 0; c < nchunks; ++c)
            a += part[(size_t)c * AG_MLP_NPARAM + o];
        grad[o] = a;
    }
}

__global__ void ag_mlp_adam_kernel(float *w, __nv_bfloat16 *wb, const float *g, float *m, float *v, float lr,
                                   float b1t, float b2t)
{
    const float b1 = 0.9f, b2 = 0.999f, epsv = 1e-8f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < AG_MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / (1.0f - b1t), vh = vi / (1.0f - b2t);
        const float wi = w[i] - lr * mh / (sqrtf(vh) + epsv);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void ag_mlp_round_kernel(const float *w, __nv_bfloat16 *wb)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < AG_MLP_NPARAM; i += gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

/* init[v] = exp(prediction) in caller order, floored at base_pr */
__global__ void ag_mlp_to_ranks_kernel(const float *Y, uint32_t n, float floor_v, float *out)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[v] = fmaxf(expf(Y[v]), floor_v);
}

/* ------------------------------------------------------------- host API */
#define MCHK(call)                                                                                       \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            return ag_set_error(AG_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));            \
        }                                                                                                \
    } while (0)

static cudaStream_t mlp_stream()
{
    return (cudaStream_t)ag_stream();
}

extern "C" uint32_t ag_mlp_num_params(void) { return AG_MLP_NPARAM; }

extern "C" ag_status_t ag_mlp_create(uint64_t seed, ag_mlp_t *out)
{
    ag_clear_error();
    if (!out)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_create: NULL out");
    if (!ag_stream())
        return ag_set_error(AG_ERR_NO_DEVICE, "ag_mlp_create: no CUDA device");
    ag_mlp_s *m = new ag_mlp_s();
    memset((void *)m, 0, sizeof(*m));
    const size_t nb = AG_MLP_NPARAM * sizeof(float);
    cudaError_t e = cudaMalloc((void **)&m->w, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->wb, AG_MLP_NPARAM * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->g, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->m, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->v, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->loss, sizeof(float));
    if (e != cudaSuccess) {
        cudaGetLastError();
        ag_mlp_release(m);
        return ag_set_error(AG_ERR_OOM, "ag_mlp_create: %s", cudaGetErrorString(e));
    }
    /* He-style uniform init from the counter generator; zero biases */
    std::vector<float> w(AG_MLP_NPARAM, 0.0f);
    for (int i = 0; i < AG_MLP_NPARAM; ++i) {
        float lim = 0.0f;
        if (i < AG_MLP_OFF_B1)
            lim = sqrtf(6.0f / AG_MLP_IN);
        else if (i >= AG_MLP_OFF_W2 && i < AG_MLP_OFF_B2)
            lim = sqrtf(6.0f / AG_MLP_H);
        else if (i >= AG_MLP_OFF_W3 && i < AG_MLP_OFF_B3)
            lim = sqrtf(3.0f / AG_MLP_H);
        w[i] = lim * (2.0f * ag_u01(ag_draw64(seed, (uint64_t)i, 0)) - 1.0f);
    }
    ag_status_t st = ag_mlp_set_params(m, w.data());
    if (st != AG_OK) {
        ag_mlp_release(m);
        return st;
    }
    *out = m;
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_release(ag_mlp_t m)
{
    if (!m)
        return AG_OK;
    cudaStreamSynchronize(mlp_stream());
    cudaFree(m->w);
    cudaFree(m->wb);
    cudaFree(m->g);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->buf);
    cudaFree(m->part);
    cudaFree(m->loss);
    delete m;
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_set_params(ag_mlp_t m, const float *params)
{
    if (!m || !params)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_set_params: NULL argument");
    cudaStream_t s = mlp_stream();
    MCHK(cudaMemcpyAsync(m->w, params, AG_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    MCHK(cudaMemsetAsync(m->m, 0, AG_MLP_NPARAM * sizeof(float), s));
    MCHK(cudaMemsetAsync(m->v, 0, AG_MLP_NPARAM * sizeof(float), s));
    ag_mlp_round_kernel<<<8, 1024, 0, s>>>(m->w, m->wb);
    MCHK(cudaGetLastError());
    MCHK(cudaStreamSynchronize(s));
    m->step = 0;
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_get_params(ag_mlp_t m, float *params)
{
    if (!m || !params)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_get_params: NULL argument");
    MCHK(cudaStreamSynchronize(mlp_stream()));
    MCHK(cudaMemcpy(params, m->w, AG_MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return AG_OK;
}

extern "C" ag_status_t ag_features(ag_graph_t g, float *features)
{
    ag_clear_error();
    AgGraphView gv;
    ag_status_t st = ag_rt_graph_view(g, &gv);
    if (st != AG_OK)
        return st;
    if (!features)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_features: NULL output");
    if (gv.N == 0)
        return AG_OK;
    if (!gv.tasks)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_features: the graph has no work list");
    /* deg2, then the hub rows' slots: three 64-bit sums and four words each */
    const size_t deg2_bytes = ((size_t)gv.N * sizeof(uint2) + 255) & ~(size_t)255;
    const size_t acc_bytes = (size_t)gv.hub_slots * 3 * sizeof(unsigned long long);
    const size_t ext_bytes = (size_t)gv.hub_slots * 4 * sizeof(uint32_t);
    unsigned char *buf = nullptr;
    MCHK(cudaMallocAsync((void **)&buf, deg2_bytes + acc_bytes + ext_bytes + 16, gv.stream));
    uint2 *deg2 = reinterpret_cast<uint2 *>(buf);
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(buf + deg2_bytes);
    uint32_t *ext = reinterpret_cast<uint32_t *>(buf + deg2_bytes + acc_bytes);
    cudaError_t e = cudaSuccess;
    if (acc_bytes)
        e = cudaMemsetAsync(acc, 0, acc_bytes + ext_bytes, gv.stream);
    if (e == cudaSuccess) {
        uint64_t blocks = ((uint64_t)gv.N + 255) / 256;
        if (blocks > ag_sm_grid(16))
            blocks = ag_sm_grid(16);
        ag_deg2_kernel<<<(unsigned)blocks, 256, 0, gv.stream>>>(gv, deg2);
        uint64_t iblocks = ((uint64_t)gv.ntasks * 32 + 255) / 256;
        if (iblocks > ag_sm_grid(8))
            iblocks = ag_sm_grid(8);
        if (iblocks)
            ag_features_items_kernel<<<(unsigned)iblocks, 256, 0, gv.stream>>>(gv, deg2, acc, ext, features);
        e = cudaGetLastError();
    }
    cudaFreeAsync(buf, gv.stream);
    MCHK(e);
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_forward(ag_mlp_t m, const float *X, uint32_t n, float *Y)
{
    ag_clear_error();
    if (!m || (n && (!X || !Y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_forward: NULL argument");
    if (n == 0)
        return AG_OK;
    const uint64_t blocks = (n + AG_MLP_BLK - 1) / AG_MLP_BLK; /* one sample per thread */
    ag_mlp_infer_kernel<<<(unsigned)blocks, AG_MLP_BLK, 0, mlp_stream()>>>(m->wb, X, n, Y);
    MCHK(cudaGetLastError());
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_predict(ag_mlp_t m, const float *X, uint32_t n, float *Y)
{
    ag_clear_error();
    if (!m || (n && (!X || !Y)))
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_predict: NULL argument");
    if (n == 0)
        return AG_OK;
    uint64_t blocks = ((uint64_t)n + 16 * (AG_MLP_TC_BLK / 32) - 1) / (16 * (AG_MLP_TC_BLK / 32));
    if (blocks > ag_sm_grid(8))
        blocks = ag_sm_grid(8);
    ag_mlp_infer_tc_kernel<<<(unsigned)blocks, AG_MLP_TC_BLK, 0, mlp_stream()>>>(m->wb, X, n, Y);
    MCHK(cudaGetLastError());
    return AG_OK;
}

static ag_status_t mlp_ensure_buf(ag_mlp_t m, uint32_t n)
{
    if (m->buf_cap < n) {
        cudaFree(m->buf);
        m->buf = nullptr;
        m->buf_cap = 0;
        MCHK(cudaMalloc((void **)&m->buf, (size_t)n * AG_MLP_REC * sizeof(float)));
        m->buf_cap = n;
    }
    const uint32_t chunks = (n + AG_MLP_CHUNK - 1) / AG_MLP_CHUNK;
    if (m->part_cap < chunks) {
        cudaFree(m->part);
        m->part = nullptr;
        m->part_cap = 0;
        MCHK(cudaMalloc((void **)&m->part, (size_t)chunks * AG_MLP_NPARAM * sizeof(float)));
        m->part_cap = chunks;
    }
    return AG_OK;
}

/* gradient of the mean squared error over n samples into m->g (and *loss) */
static ag_status_t mlp_grad(ag_mlp_t m, const float *X, const float *T, uint32_t n, float *loss)
{
    ag_status_t st = mlp_ensure_buf(m, n);
    if (st != AG_OK)
        return st;
    cudaStream_t s = mlp_stream();
    MCHK(cudaMemsetAsync(m->loss, 0, sizeof(float), s));
    uint64_t blocks = (n + AG_MLP_BLK - 1) / AG_MLP_BLK;
    if (blocks > ag_sm_grid(16))
        blocks = ag_sm_grid(16);
    ag_mlp_k1<<<(unsigned)blocks, AG_MLP_BLK, 0, s>>>(m->wb, X, T, n, 1.0f / (float)n, m->buf, m->loss);
    MCHK(cudaGetLastError());
    const size_t smem = AG_MLP_CHUNK * AG_MLP_REC * sizeof(float);
    MCHK(cudaFuncSetAttribute(ag_mlp_k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t chunks = (n + AG_MLP_CHUNK - 1) / AG_MLP_CHUNK;
    ag_mlp_k2<<<chunks, 256, smem, s>>>(m->buf, n, m->part);
    ag_mlp_k3<<<(AG_MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->part, chunks, m->g);
    MCHK(cudaGetLastError());
    if (loss) {
        float h = 0.0f;
        MCHK(cudaMemcpyAsync(&h, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        MCHK(cudaStreamSynchronize(s));
        *loss = h / (float)n;
    }
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_gradients(ag_mlp_t m, const float *X, const float *T, uint32_t n, float *grad,
                                        float *loss)
{
    ag_clear_error();
    if (!m || !X || !T || n == 0)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_gradients: bad argument");
    ag_status_t st = mlp_grad(m, X, T, n, loss);
    if (st != AG_OK)
        return st;
    if (grad) {
        MCHK(cudaStreamSynchronize(mlp_stream()));
        MCHK(cudaMemcpy(grad, m->g, AG_MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    }
    return AG_OK;
}

extern "C" ag_status_t ag_mlp_train(ag_mlp_t m, const float *X, const float *T, uint32_t n, uint32_t epochs,
                                    uint32_t batch, float lr, float *final_loss)
{
    ag_clear_error();
    if (!m || !X || !T || n == 0 || batch == 0)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_train: bad argument");
    cudaStream_t s = mlp_stream();
    float last = 0.0f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        double sum = 0.0;
        uint32_t nb = 0;
        for (uint32_t b0 = 0; b0 < n; b0 += batch) {
            const uint32_t cnt = std::min<uint32_t>(batch, n - b0);
            float l = 0.0f;
            const bool want = (b0 + batch >= n); /* loss of the epoch's last batch */
            ag_status_t st = mlp_grad(m, X + (size_t)b0 * AG_MLP_IN, T + b0, cnt, want ? &l : nullptr);
            if (st != AG_OK)
                return st;
            m->step++;
            const float b1t = powf(0.9f, (float)m->step), b2t = powf(0.999f, (float)m->step);
            ag_mlp_adam_kernel<<<8, 1024, 0, s>>>(m->w, m->wb, m->g, m->m, m->v, lr, b1t, b2t);
            MCHK(cudaGetLastError());
            if (want) {
                sum += l;
                ++nb;
            }
        }
        last = nb ? (float)(sum / nb) : 0.0f;
    }
    MCHK(cudaStreamSynchronize(s));
    if (final_loss)
        *final_loss = last;
    return AG_OK;
}

/* predicted un-normalised ranks into a device array (caller order) */
extern "C" ag_status_t ag_mlp_warm_start_device(ag_graph_t g, ag_mlp_t m, float *init_dev)
{
    ag_clear_error();
    AgGraphView gv;
    ag_status_t st = ag_rt_graph_view(g, &gv);
    if (st != AG_OK)
        return st;
    if (!m || !init_dev)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_warm_start_device: NULL argument");
    if (gv.N == 0)
        return AG_OK;
    cudaStream_t s = gv.stream;
    float *X = nullptr;
    MCHK(cudaMallocAsync((void **)&X, (size_t)gv.N * AG_MLP_IN * sizeof(float), s));
    st = ag_features(g, X);
    if (st == AG_OK)
        st = ag_mlp_predict(m, X, gv.N, init_dev);
    if (st == AG_OK) {
        ag_mlp_to_ranks_kernel<<<ag_sm_grid(8), 256, 0, s>>>(init_dev, gv.N, 1.0f - Damp, init_dev);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            st = ag_set_error(AG_ERR_CUDA, "ag_mlp_warm_start_device: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(X, s);
    return st;
}

/* predicted un-normalised ranks (caller order, host) for a warm start */
extern "C" ag_status_t ag_mlp_warm_start(ag_graph_t g, ag_mlp_t m, float *init_ranks)
{
    ag_clear_error();
    AgGraphView gv;
    ag_status_t st = ag_rt_graph_view(g, &gv);
    if (st != AG_OK)
        return st;
    if (!m || !init_ranks)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_mlp_warm_start: NULL argument");
    if (gv.N == 0)
        return AG_OK;
    cudaStream_t s = gv.stream;
    float *X = nullptr, *Y = nullptr;
    MCHK(cudaMallocAsync((void **)&X, (size_t)gv.N * AG_MLP_IN * sizeof(float), s));
    MCHK(cudaMallocAsync((void **)&Y, (size_t)gv.N * sizeof(float), s));
    st = ag_features(g, X);
    if (st == AG_OK)
        st = ag_mlp_predict(m, X, gv.N, Y);
    if (st == AG_OK) {
        ag_mlp_to_ranks_kernel<<<ag_sm_grid(8), 256, 0, s>>>(Y, gv.N, 1.0f - Damp, Y);
        cudaError_t e = cudaMemcpyAsync(init_ranks, Y, (size_t)gv.N * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess)
            st = ag_set_error(AG_ERR_CUDA, "ag_mlp_warm_start: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(X, s);
    cudaFreeAsync(Y, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (st == AG_OK && e != cudaSuccess)
        st = ag_set_error(AG_ERR_CUDA, "ag_mlp_warm_start: %s", cudaGetErrorString(e));
    return st;
}
