/*
 * ag_ppr.cu -- batched personalized PageRank: k <= 64 source vertices solved
 * together as one sparse-matrix x dense-matrix product per pass.
 *
 * Column i is the pull PageRank of the reference (pageRank.c:1026-1069) with
 * the teleport concentrated on source s_i:
 *   c_i[u]  = r_i[u] / out_degree[u]            (0 without out-edges)
 *   s_i[v]  = sum over v's in-edges of c_i[u]    (binary32, stream order)
 *   r_i'[v] = b_i[v] + damp * s_i[v],  b_i[v] = (1 - damp) * N at v = s_i, else 0
 *   err     = |r_i' - r_i| in binary64 against epsilon; stop when no (v, i)
 *             pair changes by >= epsilon
 * and the result is r_i / N, as for the plain kernel.  The teleport mass
 * (1 - damp) * N keeps the un-normalised scale of the reference's ranks, so
 * the same epsilon means the same thing.
 *
 * Layout: contributions and ranks are N x 64 binary32, row-major (256 bytes
 * per vertex).  One warp owns a destination row; lane l owns columns 2l and
 * 2l + 1.  Each in-edge becomes one fully coalesced 256-byte row gather, so
 * the pass streams the gathered rows from HBM at full width (the per-edge
 * 4-byte random gather of the single-vector kernel becomes a 256-byte
 * sequential one).  Every column is summed in stream order, so each column
 * is bit-identical to a sequential binary32 loop.
 *
 * The contribution matrix of a graph of millions of vertices is far larger
 * than L2, so the gathered rows come from HBM: 256 bytes per in-edge is the
 * pass's real traffic.  The kernel therefore keeps as many row gathers in
 * flight as it can: eight per warp, a grid of exactly the resident warps,
 * and the next row's bounds and first 32 ids loading while the current row
 * is gathered, so no warp waits on the offsets -> ids -> rows chain between
 * rows.
 *
 * The loop stays on the device: after each pass a one-thread kernel counts
 * it and sets a stop flag once no (v, i) pair moved by epsilon; passes that
 * see the flag return at once, and the host reads the flag every
 * AG_PPR_CHECK passes.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "ag_device.h"
#include "ag_internal.h"

#define AG_PPR_K 64
#define AG_PPR_BLK 256
#define AG_PPR_DEPTH 8 /* row gathers in flight per warp: 62 registers, 32
                          resident warps per SM.  AG_PPR_DEPTH=16 in the
                          environment takes sixteen (80 registers, 24 warps):
                          8.56 against 7.46 ms per pass on ER 2^23, k = 64 */
#define AG_PPR_CHECK 8  /* passes between host reads of the stop flag */

/* the device-side loop state, written by ag_ppr_close_kernel */
struct AgPprState
{
    uint32_t stop;       /* set once a pass had no active pair */
    uint32_t passes;     /* passes that did work               */
    uint32_t converged;
    uint32_t pad;
    unsigned long long active_last;
    double err_last;
};

struct AgPprParams
{
    const uint32_t *row_off;
    const uint32_t *ids;
    const uint32_t *outdeg;
    uint32_t N;
    uint32_t k;
    const float *X;   /* contributions of this pass (N x 64) */
    float *Xn;        /* contributions of the next pass      */
    float *R;         /* ranks (N x 64), updated in place    */
    const uint32_t *src_rows; /* device row of each source (k entries) */
    float base_src;   /* (1 - damp) * N                       */
    float damp;
    double eps;
    unsigned long long *active; /* pairs with |r' - r| >= eps */
    double *err;      /* sum of |r' - r|                      */
    AgPprState *state;
};

__device__ __forceinline__ float2 ag_ppr_ld_row(const float *X, uint32_t u, uint32_t lane)
{
    float2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0,%1}, [%2];"
        : "=f"(v.x), "=f"(v.y)
        : "l"(X + (size_t)u * AG_PPR_K + 2 * lane));
    return v;
}

__global__ void __launch_bounds__(AG_PPR_BLK) ag_ppr_init_kernel(AgPprParams p)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t c0 = 2 * lane, c1 = c0 + 1;
    const uint32_t s0 = c0 < p.k ? p.src_rows[c0] : 0xFFFFFFFFu;
    const uint32_t s1 = c1 < p.k ? p.src_rows[c1] : 0xFFFFFFFFu;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < p.N; v += nw) {
        const uint32_t od = p.outdeg[v];
        float2 r, c;
        r.x = (v == s0) ? p.base_src : 0.0f;
        r.y = (v == s1) ? p.base_src : 0.0f;
        c.x = od ? __fdiv_rn(r.x, __uint2float_rn(od)) : 0.0f;
        c.y = od ? __fdiv_rn(r.y, __uint2float_rn(od)) : 0.0f;
        reinterpret_cast<float2 *>(p.R + (size_t)v * AG_PPR_K)[lane] = r;
        reinterpret_cast<float2 *>(p.Xn + (size_t)v * AG_PPR_K)[lane] = c;
    }
}

template <int DEPTH>
__global__ void __launch_bounds__(AG_PPR_BLK) ag_ppr_pass_kernel(AgPprParams p)
{
    __shared__ unsigned long long s_act[AG_PPR_BLK / 32];
    __shared__ double s_err[AG_PPR_BLK / 32];
    if (*(volatile const uint32_t *)&p.state->stop)
        return;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t c0 = 2 * lane, c1 = c0 + 1;
    const bool live0 = c0 < p.k, live1 = c1 < p.k;
    const uint32_t s0 = live0 ? p.src_rows[c0] : 0xFFFFFFFFu;
    const uint32_t s1 = live1 ? p.src_rows[c1] : 0xFFFFFFFFu;
    unsigned long long my_act = 0;
    double my_err = 0.0;
    /* row v's bounds and first ids, and row vn's bounds, are loaded one row
     * ahead of their use */
    uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t b = 0, e = 0, myid = 0;
    if (v < p.N) {
        b = p.row_off[v];
        e = p.row_off[v + 1];
        myid = lane < min(32u, e - b) ? p.ids[b + lane] : 0u;
    }
    uint32_t vn = v + nw, bn = 0, en = 0;
    if (vn < p.N) {
        bn = p.row_off[vn];
        en = p.row_off[vn + 1];
    }
    while (v < p.N) {
        const uint32_t od = p.outdeg[v];
        const float2 rp = reinterpret_cast<const float2 *>(p.R + (size_t)v * AG_PPR_K)[lane];
        const uint32_t myid_n = (vn < p.N && lane < min(32u, en - bn)) ? p.ids[bn + lane] : 0u;
        const uint32_t vnn = vn + nw;
        uint32_t bnn = 0, enn = 0;
        if (vnn < p.N) {
            bnn = p.row_off[vnn];
            enn = p.row_off[vnn + 1];
        }
        /* stream order; -0 + x = x for every binary32 x, so the sum starts
         * at -0 instead of at the first value, and a row without in-edges
         * still gives +0 once the teleport term (+0 or positive) is added */
        float ax = -0.0f, ay = -0.0f;
        for (uint32_t j0 = b; j0 < e; j0 += 32) {
            const uint32_t n = min(32u, e - j0);
            const uint32_t chunk = (j0 == b) ? myid : (lane < n ? p.ids[j0 + lane] : 0u);
            for (uint32_t t = 0; t < n; t += DEPTH) {
                float2 val[DEPTH];
#pragma unroll
                for (int q = 0; q < DEPTH; ++q) {
                    const uint32_t u = __shfl_sync(0xffffffffu, chunk, (t + q) & 31);
                    val[q] = (t + q < n) ? ag_ppr_ld_row(p.X, u, lane) : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int q = 0; q < DEPTH; ++q) {
                    if (t + q < n) {
                        ax = __fadd_rn(ax, val[q].x);
                        ay = __fadd_rn(ay, val[q].y);
                    }
                }
            }
        }
        float2 rn, cn;
        rn.x = __fadd_rn((v == s0) ? p.base_src : 0.0f, __fmul_rn(p.damp, ax));
        rn.y = __fadd_rn((v == s1) ? p.base_src : 0.0f, __fmul_rn(p.damp, ay));
        if (!live0)
            rn.x = 0.0f;
        if (!live1)
            rn.y = 0.0f;
        const double e0 = (double)fabsf(__fsub_rn(rn.x, rp.x));
        const double e1 = (double)fabsf(__fsub_rn(rn.y, rp.y));
        my_err += e0 + e1;
        my_act += (unsigned long long)((live0 && e0 >= p.eps) ? 1 : 0) + ((live1 && e1 >= p.eps) ? 1 : 0);
        cn.x = od ? __fdiv_rn(rn.x, __uint2float_rn(od)) : 0.0f;
        cn.y = od ? __fdiv_rn(rn.y, __uint2float_rn(od)) : 0.0f;
        reinterpret_cast<float2 *>(p.R + (size_t)v * AG_PPR_K)[lane] = rn;
        reinterpret_cast<float2 *>(p.Xn + (size_t)v * AG_PPR_K)[lane] = cn;
        v = vn;
        b = bn;
        e = en;
        myid = myid_n;
        vn = vnn;
        bn = bnn;
        en = enn;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        my_act += __shfl_xor_sync(0xffffffffu, my_act, o);
        my_err += __shfl_xor_sync(0xffffffffu, my_err, o);
    }
    if (lane == 0) {
        s_act[warp] = my_act;
        s_err[warp] = my_err;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0;
        double er = 0.0;
        for (int w = 0; w < AG_PPR_BLK / 32; ++w) {
            a += s_act[w];
            er += s_err[w];
        }
        if (a)
            atomicAdd(p.active, a);
        if (er != 0.0)
            atomicAdd(p.err, er);
    }
}

/* after each pass: count it, keep its statistics, stop when nothing moved;
 * clears the counters for the next pass */
__global__ void ag_ppr_close_kernel(AgPprParams p)
{
    AgPprState *st = p.state;
    if (!st->stop) {
        st->passes += 1;
        st->active_last = *p.active;
        st->err_last = *p.err;
        if (*p.active == 0) {
            st->stop = 1;
            st->converged = 1;
        }
    }
    *p.active = 0;
    *p.err = 0.0;
}

/* out[perm[v] * k + i] = R[v][i] / N (binary32), caller order */
__global__ void ag_ppr_output_kernel(AgPprParams p, const uint32_t *perm, float *out)
{
    const float fN = __uint2float_rn(p.N);
    const uint64_t total = (uint64_t)p.N * p.k;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(t / p.k), i = (uint32_t)(t % p.k);
        const uint32_t dst = perm ? perm[v] : v;
        out[(size_t)dst * p.k + i] = __fdiv_rn(p.R[(size_t)v * AG_PPR_K + i], fN);
    }
}

/* host side ------------------------------------------------------------ */

extern "C" ag_status_t ag_ppr_spmm(ag_graph_t g, const uint32_t *sources, uint32_t k, uint32_t max_iterations,
                                   double epsilon, float *ranks, ag_pr_result *result)
{
    ag_clear_error();
    AgGraphView gv;
    ag_status_t st = ag_rt_graph_view(g, &gv);
    if (st != AG_OK)
        return st;
    if (!sources || k == 0 || k > AG_PPR_K)
        return ag_set_error(AG_ERR_INVALID_ARG, "ag_ppr_spmm: need 1..%d sources", AG_PPR_K);
    for (uint32_t i = 0; i < k; ++i)
        if (sources[i] >= gv.N)
            return ag_set_error(AG_ERR_INVALID_ARG, "ag_ppr_spmm: source %u >= %u vertices", sources[i], gv.N);
    cudaStream_t s = gv.stream;
    const size_t mat = (size_t)gv.N * AG_PPR_K * sizeof(float);
    float *X = nullptr, *Xn = nullptr, *R = nullptr, *out = nullptr;
    uint32_t *src_dev = nullptr;
    unsigned long long *ctr = nullptr;
    AgPprState *state = nullptr;
    AgPprState hs;
    int per_sm = 0;
    void (*pass_kernel)(AgPprParams) = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<uint32_t> src_rows(k);
    cudaError_t err = cudaSuccess;
    uint32_t passes = 0, converged = 0;
    unsigned long long act_last = 0;
    double err_last = 0.0;
    float ms = 0.0f;
    AgPprParams p;
    memset(&p, 0, sizeof(p));
    /* init and output: a few waves; passes: exactly the resident CTAs, so
     * that every warp's share of rows runs at once */
    const unsigned grid_rows = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)gv.N * 32 + AG_PPR_BLK - 1) / AG_PPR_BLK, (uint64_t)ag_sm_grid(8)));
    unsigned grid_pass = grid_rows;
    memset(&hs, 0, sizeof(hs));
#define PCHK(call)                                                                                       \
    do {                                                                                                 \
        err = (call);                                                                                    \
        if (err != cudaSuccess)                                                                          \
            goto done;                                                                                   \
    } while (0)
    /* sources in device numbering */
    if (gv.inv) {
        std::vector<uint32_t> inv(gv.N);
        PCHK(cudaMemcpy(inv.data(), gv.inv, (size_t)gv.N * 4, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < k; ++i)
            src_rows[i] = inv[sources[i]];
    } else {
        for (uint32_t i = 0; i < k; ++i)
            src_rows[i] = sources[i];
    }
    PCHK(cudaMallocAsync((void **)&X, mat, s));
    PCHK(cudaMallocAsync((void **)&Xn, mat, s));
    PCHK(cudaMallocAsync((void **)&R, mat, s));
    PCHK(cudaMallocAsync((void **)&src_dev, AG_PPR_K * 4, s));
    PCHK(cudaMallocAsync((void **)&ctr, 16, s));
    PCHK(cudaMallocAsync((void **)&state, sizeof(AgPprState), s));
    PCHK(cudaMemsetAsync(ctr, 0, 16, s));
    PCHK(cudaMemsetAsync(state, 0, sizeof(AgPprState), s));
    {
        const char *d = getenv("AG_PPR_DEPTH");
        pass_kernel = (d && atoi(d) == 16) ? ag_ppr_pass_kernel<16> : ag_ppr_pass_kernel<AG_PPR_DEPTH>;
    }
    PCHK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass_kernel, AG_PPR_BLK, 0));
    grid_pass = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)gv.N * 32 + AG_PPR_BLK - 1) / AG_PPR_BLK,
                              (uint64_t)ag_sm_grid((unsigned)std::max(per_sm, 1))));
    PCHK(cudaMemcpyAsync(src_dev, src_rows.data(), (size_t)k * 4, cudaMemcpyHostToDevice, s));
    PCHK(cudaEventCreate(&e0));
    PCHK(cudaEventCreate(&e1));
    p.row_off = gv.row_off;
    p.ids = gv.ids;
    p.outdeg = gv.outdeg;
    p.N = gv.N;
    p.k = k;
    p.src_rows = src_dev;
    p.damp = Damp;
    p.base_src = (1.0f - Damp) * (float)gv.N; /* one binary32 multiply */
    p.eps = epsilon;
    p.active = ctr;
    p.err = reinterpret_cast<double *>(ctr + 1);
    p.state = state;
    PCHK(cudaEventRecord(e0, s));
    p.X = X;
    p.Xn = X; /* init writes the first contributions into X */
    p.R = R;
    ag_ppr_init_kernel<<<grid_rows, AG_PPR_BLK, 0, s>>>(p);
    PCHK(cudaGetLastError());
    for (uint32_t it = 0; it < max_iterations; ++it) {
        p.X = (it & 1) ? Xn : X;
        p.Xn = (it & 1) ? X : Xn;
        pass_kernel<<<grid_pass, AG_PPR_BLK, 0, s>>>(p);
        ag_ppr_close_kernel<<<1, 1, 0, s>>>(p);
        PCHK(cudaGetLastError());
        if ((it + 1) % AG_PPR_CHECK == 0 || it + 1 == max_iterations) {
            PCHK(cudaMemcpyAsync(&hs, state, sizeof(hs), cudaMemcpyDeviceToHost, s));
            PCHK(cudaStreamSynchronize(s));
            if (hs.stop)
                break;
        }
    }
    PCHK(cudaEventRecord(e1, s));
    passes = hs.passes;
    converged = hs.converged;
    act_last = hs.active_last;
    err_last = hs.err_last;
    if (ranks) {
        PCHK(cudaMallocAsync((void **)&out, (size_t)gv.N * k * sizeof(float), s));
        ag_ppr_output_kernel<<<ag_sm_grid(8), 256, 0, s>>>(p, gv.perm, out);
        PCHK(cudaGetLastError());
        PCHK(cudaMemcpyAsync(ranks, out, (size_t)gv.N * k * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    PCHK(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&ms, e0, e1);
    if (result) {
        memset(result, 0, sizeof(*result));
        result->passes = passes;
        result->converged = converged;
        result->iterations = converged ? passes - 1 : passes;
        result->active_last = (uint32_t)std::min<unsigned long long>(act_last, 0xFFFFFFFFull);
        result->error_total = err_last / ((double)gv.N * k);
        result->device_ms = ms;
    }
done:
    if (X)
        cudaFreeAsync(X, s);
    if (Xn)
        cudaFreeAsync(Xn, s);
    if (R)
        cudaFreeAsync(R, s);
    if (out)
        cudaFreeAsync(out, s);
    if (src_dev)
        cudaFreeAsync(src_dev, s);
    if (ctr)
        cudaFreeAsync(ctr, s);
    if (state)
        cudaFreeAsync(state, s);
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
#undef PCHK
    if (err != cudaSuccess) {
        cudaGetLastError();
        return ag_set_error(AG_ERR_CUDA, "ag_ppr_spmm: %s", cudaGetErrorString(err));
    }
    return AG_OK;
}
