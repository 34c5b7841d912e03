/*
 * ag_plan.cu -- device planner of the pull kernel's work lists.
 *
 * Both lists are built from the device row offsets in two walks of the rows:
 * one thread per segment of AG_PLAN_SEG consecutive rows counts its items,
 * the counts are scanned, and a second walk writes every item at its final
 * position.  The lists, the item kinds and their order are those of the
 * pull kernel's contract:
 *   FAST and EXACT (the same list): hub chunks (rows above hub_chunk
 *           in-edges, split in chunks), then long rows (above task_edges),
 *           then row items.  The kernel's order decides how each is summed.
 * A row item packs at most AG_WROWS consecutive rows of at most task_edges
 * in-edges each and together; it never crosses the first row of a graph of
 * a block-diagonal union, nor a segment boundary (a segment holds 512 rows,
 * so the boundary costs at most one extra item per 512 rows).  Within each
 * kind, items follow row order.  Which rows share an item never changes a
 * result: sums depend only on a row's own edges and on the row's kind.
 */
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "ag_device.h"

#define AG_PLAN_SEG 512u

struct AgPlanArgs
{
    const uint32_t *off;
    const uint32_t *gstart; /* ngraphs + 1 first rows, or NULL */
    uint32_t n, cap, whub, ngraphs, nseg;
};

/* index of the first graph start above row r (ngraphs + 1 when none) */
__device__ __forceinline__ uint32_t ag_plan_next_graph(const AgPlanArgs &a, uint32_t r)
{
    uint32_t lo = 0, hi = a.ngraphs + 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.gstart[mid] <= r)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* counts live in four arrays of nseg + 1 words: hub chunks, long rows (not
 * split), row items, split rows.  WRITE = false fills them; WRITE = true
 * reads their exclusive scans and writes the lists. */
template <bool WRITE>
__global__ void ag_plan_kernel(const AgPlanArgs a, uint32_t *cnt, const uint32_t *scan, AgPlanTotals tot,
                               uint4 *fast, uint4 *exact)
{
    const uint32_t seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= a.nseg)
        return;
    const uint32_t stride = a.nseg + 1;
    uint32_t r = seg * AG_PLAN_SEG;
    const uint32_t rend = min(a.n, r + AG_PLAN_SEG);
    uint32_t nh = 0, nl = 0, nw = 0, nhr = 0;
    uint32_t hb = 0, lb = 0, wb = 0;
    if (WRITE) {
        hb = scan[seg];
        lb = scan[stride + seg];
        wb = scan[2 * stride + seg];
    }
    uint32_t gi = a.gstart ? ag_plan_next_graph(a, r) : 0;
    while (r < rend) {
        const uint32_t o0 = a.off[r], o1 = a.off[r + 1], d = o1 - o0;
        if (d > a.cap) {
            const uint4 lng = make_uint4((AG_T_LONG << 30) | r, r + 1, o0, o1);
            if (d > a.whub) {
                const uint32_t nch = (d + a.whub - 1) / a.whub;
                if (WRITE) {
                    const uint32_t pbase = hb + nh;
                    for (uint32_t c = 0; c < nch; ++c) {
                        const uint32_t cb = o0 + c * a.whub;
                        const uint4 it =
                            make_uint4((AG_T_HUB << 30) | r, pbase | (c << AG_SLOT_BITS), cb, min(o1, cb + a.whub));
                        fast[pbase + c] = it;
                        exact[pbase + c] = it;
                    }
                }
                nh += nch;
                ++nhr;
            } else {
                if (WRITE) {
                    fast[tot.hub_items + lb + nl] = lng;
                    exact[tot.hub_items + lb + nl] = lng;
                }
                ++nl;
            }
            ++r;
            continue;
        }
        /* a row item: the first row always fits (d <= cap) */
        const uint32_t rb = r, eb = o0;
        uint32_t limit = rend;
        if (a.gstart) {
            while (gi <= a.ngraphs && a.gstart[gi] <= rb)
                ++gi;
            if (gi <= a.ngraphs)
                limit = min(limit, a.gstart[gi]);
        }
        uint32_t ee = o1;
        ++r;
        while (r < limit && r - rb < AG_WROWS) {
            const uint32_t e1 = a.off[r + 1];
            if (e1 - a.off[r] > a.cap || e1 - eb > a.cap)
                break;
            ee = e1;
            ++r;
        }
        if (WRITE) {
            const uint4 it = make_uint4((AG_T_ROWS << 30) | rb, r, eb, ee);
            fast[tot.hub_items + tot.long_items + wb + nw] = it;
            exact[tot.hub_items + tot.long_items + wb + nw] = it;
        }
        ++nw;
    }
    if (!WRITE) {
        cnt[seg] = nh;
        cnt[stride + seg] = nl;
        cnt[2 * stride + seg] = nw;
        cnt[3 * stride + seg] = nhr;
    }
}

__global__ void ag_plan_totals_kernel(const uint32_t *scan, uint32_t nseg, uint32_t *tot)
{
    const uint32_t k = threadIdx.x;
    if (k < 4)
        tot[k] = scan[k * (nseg + 1) + nseg];
}

static AgPlanArgs plan_args(const AgPlanState *ps)
{
    AgPlanArgs a;
    a.off = ps->row_off;
    a.gstart = ps->gstart;
    a.n = ps->n;
    a.cap = ps->cap;
    a.whub = ps->whub;
    a.ngraphs = ps->ngraphs;
    a.nseg = ps->nseg;
    return a;
}

extern "C" void ag_plan_release(AgPlanState *ps, cudaStream_t s)
{
    if (ps->scratch)
        cudaFreeAsync(ps->scratch, s);
    ps->scratch = nullptr;
}

extern "C" cudaError_t ag_plan_count(const uint32_t *row_off, uint32_t n, uint32_t cap, uint32_t whub,
                                     const uint32_t *gstart, uint32_t ngraphs, AgPlanState *ps,
                                     uint32_t *totals_host, cudaStream_t s)
{
    memset(ps, 0, sizeof(*ps));
    ps->row_off = row_off;
    ps->n = n;
    ps->cap = cap;
    ps->whub = whub;
    ps->gstart = gstart;
    ps->ngraphs = gstart ? ngraphs : 0;
    ps->nseg = (n + AG_PLAN_SEG - 1) / AG_PLAN_SEG;
    if (n == 0) {
        memset(totals_host, 0, 4 * sizeof(uint32_t));
        return cudaSuccess;
    }
    const size_t words = 4 * ((size_t)ps->nseg + 1);
    size_t tmp_bytes = 0;
    cudaError_t err = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (const uint32_t *)nullptr,
                                                    (uint32_t *)nullptr, (int)ps->nseg + 1, s);
    if (err != cudaSuccess)
        return err;
    tmp_bytes = (tmp_bytes + 255) & ~(size_t)255;
    const size_t bytes = 2 * words * 4 + 256 + tmp_bytes;
    if ((err = cudaMallocAsync(&ps->scratch, bytes, s)) != cudaSuccess)
        return err;
    void *tmp = ps->scratch; /* scan scratch first: 256-byte aligned */
    uint32_t *cnt = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(ps->scratch) + tmp_bytes);
    ps->scan = cnt + words;
    uint32_t *tot = ps->scan + words;
    if ((err = cudaMemsetAsync(cnt, 0, words * 4, s)) != cudaSuccess)
        return err;
    AgPlanTotals none = {0, 0, 0, 0};
    ag_plan_kernel<false><<<(ps->nseg + 127) / 128, 128, 0, s>>>(plan_args(ps), cnt, nullptr, none, nullptr, nullptr);
    for (int k = 0; k < 4; ++k) {
        size_t tb = tmp_bytes;
        err = cub::DeviceScan::ExclusiveSum(tmp, tb, cnt + (size_t)k * (ps->nseg + 1),
                                            ps->scan + (size_t)k * (ps->nseg + 1), (int)ps->nseg + 1, s);
        if (err != cudaSuccess)
            return err;
    }
    ag_plan_totals_kernel<<<1, 32, 0, s>>>(ps->scan, ps->nseg, tot);
    if ((err = cudaGetLastError()) != cudaSuccess)
        return err;
    return cudaMemcpyAsync(totals_host, tot, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
}

extern "C" cudaError_t ag_plan_write(AgPlanState *ps, const uint32_t *totals, uint4 *fast, uint4 *exact,
                                     cudaStream_t s)
{
    if (ps->n == 0)
        return cudaSuccess;
    AgPlanTotals tot = {totals[0], totals[1], totals[2], totals[3]};
    ag_plan_kernel<true><<<(ps->nseg + 127) / 128, 128, 0, s>>>(plan_args(ps), nullptr, ps->scan, tot, fast, exact);
    return cudaGetLastError();
}

__global__ void ag_set_u32_kernel(uint32_t *p, uint32_t v) { *p = v; }

/* one 32-bit store on the stream (used for the closing row offset) */
extern "C" cudaError_t ag_set_u32(uint32_t *p, uint32_t v, cudaStream_t s)
{
    ag_set_u32_kernel<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError();
}
