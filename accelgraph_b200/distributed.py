"""Row-partitioned PageRank over several GPUs (one process per GPU).

Every rank owns a contiguous range of rows, cut so that the ranges carry
about the same number of in-edges.  Vertex u of range r lives at
r * slice + (u - bounds[r]) in the contribution vector that every rank holds
in full; a pass reads that vector, writes the rank's own slice of the next
one, and the slices are then all-gathered in place (NCCL over NVLink) while
the pass statistics (active rows, sum of |r' - r|) are all-reduced on the
device.  A one-thread kernel then counts the pass and sets a device stop flag
once no row of any rank moved by epsilon; the next passes see the flag and do
nothing, and the host reads it only every few passes, so the loop has no host
round trip per pass.  Each row is still summed exactly as on one GPU (EXACT
order: the reference loop's stream order), so the partitioned solve gives the
one-GPU result bit for bit.

`solve` is the loop itself, written against callables so that the same code
drives the GPU kernels (with NCCL) and, in the tests, the CPU oracle's
row-range pass (with gloo).
"""
from __future__ import annotations

import numpy as np


def partition_bounds(in_degree, nranks: int, align: int = 64):
    """Row ranges balanced by in-edges (+1 per row, so empty rows count too);
    returns (bounds[nranks + 1], slice) with slice a multiple of `align`."""
    deg = np.asarray(in_degree, np.int64)
    n = len(deg)
    w = np.concatenate([[0], np.cumsum(deg + 1)])
    total = w[-1]
    cuts = [0]
    for r in range(1, nranks):
        cuts.append(int(np.searchsorted(w, total * r / nranks, side="left")))
    cuts.append(n)
    bounds = np.maximum.accumulate(np.array(cuts, np.int64))
    width = int(np.max(np.diff(bounds))) if nranks else 0
    slice_ = max(align, (width + align - 1) // align * align)
    return bounds.astype(np.uint32), slice_


def solve(init_fn, pass_fn, allgather_fn, allreduce_fn, close_fn, stopped_fn, result_fn, iterations, epsilon,
          check_every: int = 8):
    """The partitioned pass loop; every rank takes the same steps.

    init_fn()                   -> the two contribution buffers, this rank's
                                   first contributions written in buffer 0
    pass_fn(c_in, c_out, eps)   -> this rank's [active, err_sum] (a no-op
                                   with zero statistics once stopped), writes
                                   its slice of c_out
    allgather_fn(c)             -> fills every rank's slice of c in place
    allreduce_fn(stats)         -> sums the statistics over ranks in place
    close_fn(stats)             -> counts the pass, keeps err_sum, sets the
                                   stop flag when nothing is active
    stopped_fn()                -> whether the stop flag is set (read on the
                                   host every `check_every` passes)
    result_fn()                 -> (passes, converged, err_sum)
    Returns (iterations in the reference's sense, passes, converged, err_sum)."""
    buffers = init_fn()
    allgather_fn(buffers[0])
    for p in range(iterations):
        c_in, c_out = buffers[p & 1], buffers[(p + 1) & 1]
        stats = pass_fn(c_in, c_out, epsilon)
        allgather_fn(c_out)
        allreduce_fn(stats)
        close_fn(stats)
        if (p + 1) % check_every == 0 and stopped_fn():
            break
    passes, converged, err = result_fn()
    its = passes - 1 if converged else passes
    return its, passes, converged, err


def pagerank_rows_gpu(graph, iterations=20, epsilon=1e-4, exact=True):
    """Partitioned solve of `graph` (an accelgraph_b200.Graph every rank has
    built) over the initialised torch.distributed NCCL group, in EXACT order
    (or FAST with exact=False).  Returns this rank's normalised ranks, its row
    range and the solve statistics."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from . import AG_ORDER_EXACT, AG_ORDER_FAST, check, f32p, lib

    rank, world = dist.get_rank(), dist.get_world_size()
    bounds, slice_ = partition_bounds(graph.in_degree(), world)
    dev = torch.device("cuda", torch.cuda.current_device())
    check(lib.ag_set_stream(C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)), "ag_set_stream")
    h = C.c_void_p()
    check(lib.ag_graph_upload_rows(graph.ptr, bounds.ctypes.data_as(C.POINTER(C.c_uint32)), world, rank, slice_,
                                   0, C.byref(h)), "ag_graph_upload_rows")
    full = [torch.zeros(world * slice_, dtype=torch.float32, device=dev) for _ in range(2)]
    stats = torch.zeros(2, dtype=torch.float64, device=dev)
    state = torch.zeros(3, dtype=torch.int32, device=dev)  # stop, passes, converged
    err = torch.zeros(1, dtype=torch.float64, device=dev)
    order = AG_ORDER_EXACT if exact else AG_ORDER_FAST

    def init_fn():
        check(lib.ag_partition_init(h, full[0].data_ptr()), "ag_partition_init")
        return full

    def pass_fn(c_in, c_out, eps):
        check(lib.ag_partition_step(h, c_in.data_ptr(), c_out.data_ptr(), eps, order, stats.data_ptr(),
                                    state.data_ptr()), "ag_partition_step")
        return stats

    def allgather_fn(c):
        # in place: this rank's input is its own slice of the output
        dist.all_gather_into_tensor(c, c[rank * slice_:(rank + 1) * slice_])

    def allreduce_fn(st):
        dist.all_reduce(st)

    def close_fn(st):
        check(lib.ag_partition_close(st.data_ptr(), state.data_ptr(), err.data_ptr()), "ag_partition_close")

    def stopped_fn():
        return bool(state[0].item())

    def result_fn():
        s = state.tolist()
        return int(s[1]), bool(s[2]), float(err.item())

    its, passes, conv, err_sum = solve(init_fn, pass_fn, allgather_fn, allreduce_fn, close_fn, stopped_fn, result_fn,
                                       iterations, epsilon)
    n_local = int(bounds[rank + 1] - bounds[rank])
    local = np.empty(n_local, np.float32)
    check(lib.ag_partition_fetch(h, local.ctypes.data_as(f32p)), "ag_partition_fetch")
    lib.ag_graph_release(h)
    check(lib.ag_set_stream(None), "ag_set_stream")
    return local, (int(bounds[rank]), int(bounds[rank + 1])), {"iterations": its, "passes": passes,
                                                             "converged": conv, "error_total":
                                                             err_sum / graph.num_vertices}
