"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
whole-job rate is the sum of all ranks' work over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, w = bench.reduce_time_work(10.0 + rank, 100.0 * (rank + 1))
    out[rank] = (t, w)
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_time_work_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r] == (11.0, 300.0)


def test_reduce_time_work_single_process():
    import bench
    assert bench.reduce_time_work(5.0, 7.0) == (5.0, 7.0)


def _partition_worker(rank, world, port, out):
    """The partitioned loop of accelgraph_b200.distributed on two gloo ranks:
    the product's loop (solve), in-place all-gather of the contribution
    slices, all-reduce of the pass statistics and the stop rule of
    ag_partition_close, with the oracle's row-range pass
    (oracle_partition_pass, C) in place of the GPU kernel.  The result must
    equal the single-process oracle."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import accelgraph_b200 as ag
    import oracle
    from accelgraph_b200 import distributed as agd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g = ag.Graph.rmat(11, 12)
    n = g.num_vertices
    bounds, slice_ = agd.partition_bounds(g.in_degree(), world)
    rb, re = int(bounds[rank]), int(bounds[rank + 1])
    pos = np.zeros(n, np.uint32)
    for r in range(world):
        pos[bounds[r]:bounds[r + 1]] = r * slice_ + np.arange(bounds[r + 1] - bounds[r])
    idx, deg, nb, od = g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree()
    f = np.float32
    base = f(f(1.0) - f(0.85))
    r_local = np.full(re - rb, base, np.float32)
    state = {"stop": False, "passes": 0, "converged": False, "err": 0.0}

    def init_fn():
        bufs = [torch.zeros(world * slice_, dtype=torch.float32) for _ in range(2)]
        o = od[rb:re]
        c0 = np.where(o > 0, r_local / np.maximum(o, 1).astype(np.float32), f(0.0)).astype(np.float32)
        bufs[0][rank * slice_:rank * slice_ + (re - rb)] = torch.from_numpy(c0)
        return bufs

    def pass_fn(c_in, c_out, eps):
        if state["stop"]:
            return torch.zeros(2, dtype=torch.float64)
        st = oracle.partition_pass(rb, re, idx, deg, nb, od, pos, c_in.numpy(), c_out.numpy(), r_local, eps)
        return torch.from_numpy(st)

    def allgather_fn(c):
        dist.all_gather_into_tensor(c, c[rank * slice_:(rank + 1) * slice_])

    def allreduce_fn(st):
        dist.all_reduce(st)

    def close_fn(st):
        # the rule of ag_partition_close_kernel
        if state["stop"]:
            return
        state["passes"] += 1
        state["err"] = float(st[1])
        if float(st[0]) == 0.0:
            state["stop"] = state["converged"] = True

    its, passes, conv, err = agd.solve(init_fn, pass_fn, allgather_fn, allreduce_fn, close_fn,
                                       lambda: state["stop"],
                                       lambda: (state["passes"], state["converged"], state["err"]), 30, 1e-4)
    out[rank] = (its, passes, rb, re, (r_local / f(n)).astype(np.float32).tobytes())
    dist.barrier()
    dist.destroy_process_group()


def test_partitioned_loop_two_ranks_matches_oracle():
    import numpy as np

    import accelgraph_b200 as ag
    import oracle
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    g = ag.Graph.rmat(11, 12)
    ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 30, 1e-4)
    ranks = np.zeros(g.num_vertices, np.float32)
    for r in range(2):
        its, passes, rb, re, blob = out[r]
        assert its == ref["iterations"] and passes == ref["passes"]
        ranks[rb:re] = np.frombuffer(blob, np.float32)
    assert np.array_equal(ranks, ref["ranks"])


def test_partition_bounds_balance():
    import numpy as np

    from accelgraph_b200 import distributed as agd
    deg = np.r_[np.full(100, 1000), np.zeros(10000, np.int64), np.full(5000, 3)]
    b, s = agd.partition_bounds(deg, 4)
    assert b[0] == 0 and b[-1] == len(deg) and np.all(np.diff(b) >= 0)
    w = np.add.reduceat(deg + 1, b[:-1].astype(np.int64))
    assert w.max() <= 1.6 * w.mean()
    assert s % 64 == 0 and s >= np.diff(b).max()


def test_partition_bounds_edge_cases():
    """One rank owns everything; more ranks than rows leaves some ranks
    empty, and every row still has exactly one owner."""
    import numpy as np

    from accelgraph_b200 import distributed as agd
    b, s = agd.partition_bounds(np.array([5, 0, 7]), 1)
    assert list(b) == [0, 3] and s == 64
    b, s = agd.partition_bounds(np.array([5, 0, 7]), 8)
    assert b[0] == 0 and b[-1] == 3 and len(b) == 9 and np.all(np.diff(b.astype(np.int64)) >= 0)
    owners = np.zeros(3, np.int64)
    for r in range(8):
        owners[b[r]:b[r + 1]] += 1
    assert np.all(owners == 1) and s == 64
    b, s = agd.partition_bounds(np.zeros(0, np.int64), 2)
    assert list(b) == [0, 0, 0] and s == 64
