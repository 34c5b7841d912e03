"""Row-partitioned solve on the GPU (NCCL, world size 1 on the one GPU this
suite has): the partition kernels and the NCCL all-gather plumbing against
the oracle.  The two-rank loop itself is covered on CPU (test_multirank)."""
import datetime
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rows_partition_single_rank_matches_oracle(gpu, oracle):
    ag = gpu
    import torch
    import torch.distributed as dist

    from accelgraph_b200 import distributed as agd
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = ag.Graph.rmat(13, 16)
        ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 60, 1e-4)
        # EXACT order (the default): the oracle's ranks bit for bit; the loop
        # stops on the device flag, read every 8 passes
        ranks, (rb, re), info = agd.pagerank_rows_gpu(g, iterations=60, epsilon=1e-4)
        assert (rb, re) == (0, g.num_vertices)
        assert info["iterations"] == ref["iterations"] and info["passes"] == ref["passes"]
        assert info["converged"] == (ref["iterations"] < 60)
        assert np.array_equal(ranks.view(np.uint32), ref["ranks"].view(np.uint32))
        ranks, _, info = agd.pagerank_rows_gpu(g, iterations=60, epsilon=1e-4, exact=False)
        assert np.abs(ranks.astype(np.float64) - ref["ranks"]).sum() / ref["ranks"].sum() <= 1e-5
    finally:
        dist.destroy_process_group()


def test_rows_partition_at_scale_22_repeats_the_single_gpu_solve(gpu):
    """RMAT s22 to 1e-6 (126 iterations): the partitioned loop, run twice on
    one upload, stops on the same pass as the one-GPU EXACT solve with the
    same ranks bit for bit.  The library's kernels and torch's collectives
    share one stream; on unordered streams the statistics were read before
    the pass that made them had finished."""
    ag = gpu
    import torch
    import torch.distributed as dist

    from accelgraph_b200 import distributed as agd
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = ag.Graph.rmat(22, 16, seed=27491095)
        dg = ag.DeviceGraph(g)
        want, res, _ = dg.pagerank(300, 1e-6, order=ag.AG_ORDER_EXACT)
        dg.release()
        part = agd.RowPartition(g)
        try:
            for _ in range(2):
                its, passes, conv, _ = part.solve(300, 1e-6, True)
                assert (its, passes, conv) == (res.iterations, res.passes, True)
                ranks, _ = part.ranks()
                assert np.array_equal(ranks.view(np.uint32), want.view(np.uint32))
        finally:
            part.release()
    finally:
        dist.destroy_process_group()


def test_whole_graph_entries_refuse_a_row_partition(gpu):
    """A rank's row upload names the other ranks' rows by padded global id,
    so the entries that need a whole graph (features, warm start, PPR, the
    solves and products) refuse it instead of reading or writing past their
    per-vertex arrays."""
    import ctypes as C

    import torch

    ag = gpu
    g = ag.Graph.rmat(10, 8)
    n = g.num_vertices
    bounds = np.array([0, n // 2, n], np.uint32)
    h = C.c_void_p()
    ag.check(ag.lib.ag_graph_upload_rows(g.ptr, bounds.ctypes.data_as(C.POINTER(C.c_uint32)), 2, 1, n, 0,
                                         C.byref(h)), "ag_graph_upload_rows")
    try:
        X = torch.empty((n, 8), dtype=torch.float32, device="cuda")
        assert ag.lib.ag_features(h, X.data_ptr()) == ag.AG_ERR_UNSUPPORTED
        src = np.array([0], np.uint32)
        out = np.empty(n, np.float32)
        assert ag.lib.ag_ppr_spmm(h, src.ctypes.data_as(C.POINTER(C.c_uint32)), 1, 3, C.c_double(1e-4),
                                  out.ctypes.data_as(ag.f32p), None) == ag.AG_ERR_UNSUPPORTED
        # the whole-graph solves and products too: only ag_partition_* run on it
        opts = ag.make_opts(order=ag.AG_ORDER_EXACT)
        assert ag.lib.ag_pagerank_launch(h, 5, C.c_double(1e-4), C.byref(opts)) == ag.AG_ERR_UNSUPPORTED
        x = np.ones(n, np.float32)
        assert ag.lib.ag_spmv_pull(h, x.ctypes.data_as(ag.f32p), out.ctypes.data_as(ag.f32p), 0) == \
            ag.AG_ERR_UNSUPPORTED
        r64 = np.empty(n, np.float64)
        p = C.c_uint32()
        assert ag.lib.ag_pagerank_f64(h, 5, C.c_double(1e-9), r64.ctypes.data_as(ag.f64p), C.byref(p)) == \
            ag.AG_ERR_UNSUPPORTED
    finally:
        ag.lib.ag_graph_release(h)
