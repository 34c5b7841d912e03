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


class RowPartition:
    """This rank's rows of `graph` (an accelgraph_b200.Graph every rank has
    built) resident on its GPU, over the initialised torch.distributed NCCL
    group: the row upload and the contribution buffers are made once, and
    `solve` runs the partitioned loop on them as often as asked."""

    def __init__(self, graph):
        import ctypes as C

        import torch
        import torch.distributed as dist

        from . import check, lib

        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.bounds, self.slice = partition_bounds(graph.in_degree(), self.world)
        self.num_vertices = graph.num_vertices
        self.dev = torch.device("cuda", torch.cuda.current_device())
        # one stream for the library's kernels and torch's collectives and
        # copies, so that they run in order.  It is a stream of its own: the
        # legacy default stream (handle 0) would read as "the library's own
        # stream", which does not wait for work on the default stream.
        self.stream = torch.cuda.Stream(self.dev)
        check(lib.ag_set_stream(C.c_void_p(self.stream.cuda_stream)), "ag_set_stream")
        self.h = C.c_void_p()
        check(lib.ag_graph_upload_rows(graph.ptr, self.bounds.ctypes.data_as(C.POINTER(C.c_uint32)), self.world,
                                       self.rank, self.slice, 0, C.byref(self.h)), "ag_graph_upload_rows")
        with torch.cuda.stream(self.stream):
            self.full = [torch.zeros(self.world * self.slice, dtype=torch.float32, device=self.dev)
                         for _ in range(2)]
            self.stats = torch.zeros(2, dtype=torch.float64, device=self.dev)
            self.state = torch.zeros(3, dtype=torch.int32, device=self.dev)  # stop, passes, converged
            self.err = torch.zeros(1, dtype=torch.float64, device=self.dev)

    def solve(self, iterations=20, epsilon=1e-4, exact=True):
        """One partitioned solve; returns (iterations, passes, converged,
        error_total) of the reference's semantics."""
        import torch
        import torch.distributed as dist

        from . import AG_ORDER_EXACT, AG_ORDER_FAST, check, lib

        order = AG_ORDER_EXACT if exact else AG_ORDER_FAST
        h, full, stats, state, err, rank, sl = self.h, self.full, self.stats, self.state, self.err, self.rank, self.slice

        def init_fn():
            check(lib.ag_partition_init(h, full[0].data_ptr()), "ag_partition_init")
            return full

        def pass_fn(c_in, c_out, eps):
            check(lib.ag_partition_step(h, c_in.data_ptr(), c_out.data_ptr(), eps, order, stats.data_ptr(),
                                        state.data_ptr()), "ag_partition_step")
            return stats

        def allgather_fn(c):
            # in place: this rank's input is its own slice of the output
            dist.all_gather_into_tensor(c, c[rank * sl:(rank + 1) * sl])

        def allreduce_fn(st):
            dist.all_reduce(st)

        def close_fn(st):
            check(lib.ag_partition_close(st.data_ptr(), state.data_ptr(), err.data_ptr()), "ag_partition_close")

        def stopped_fn():
            return bool(state[0].item())

        def result_fn():
            s = state.tolist()
            return int(s[1]), bool(s[2]), float(err.item())

        with torch.cuda.stream(self.stream):
            state.zero_()
            err.zero_()
            stats.zero_()
            its, passes, conv, err_sum = solve(init_fn, pass_fn, allgather_fn, allreduce_fn, close_fn, stopped_fn,
                                               result_fn, iterations, epsilon)
        return its, passes, conv, err_sum / self.num_vertices

    def ranks(self):
        """This rank's normalised ranks and its row range."""
        from . import check, f32p, lib

        n_local = int(self.bounds[self.rank + 1] - self.bounds[self.rank])
        local = np.empty(n_local, np.float32)
        check(lib.ag_partition_fetch(self.h, local.ctypes.data_as(f32p)), "ag_partition_fetch")
        return local, (int(self.bounds[self.rank]), int(self.bounds[self.rank + 1]))

    def release(self):
        from . import check, lib

        if self.h:
            self.stream.synchronize()
            lib.ag_graph_release(self.h)
            self.h = None
            check(lib.ag_set_stream(None), "ag_set_stream")


def pagerank_rows_gpu(graph, iterations=20, epsilon=1e-4, exact=True):
    """Partitioned solve of `graph` (an accelgraph_b200.Graph every rank has
    built) over the initialised torch.distributed NCCL group, in EXACT order
    (or FAST with exact=False).  Returns this rank's normalised ranks, its row
    range and the solve statistics."""
    part = RowPartition(graph)
    try:
        its, passes, conv, err = part.solve(iterations, epsilon, exact)
        local, rows = part.ranks()
    finally:
        part.release()
    return local, rows, {"iterations": its, "passes": passes, "converged": conv, "error_total": err}
