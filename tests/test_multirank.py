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
    """The partitioned loop of accelgraph_b200.distributed on two gloo ranks,
    with a CPU pass that sums every row in stream order (binary32) over the
    padded global ids: the result must equal the single-process oracle."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import accelgraph_b200 as ag
    from accelgraph_b200 import distributed as agd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g = ag.Graph.rmat(11, 12)
    n = g.num_vertices
    bounds, slice_ = agd.partition_bounds(g.in_degree(), world)
    rb, re = int(bounds[rank]), int(bounds[rank + 1])
    owner = np.zeros(n, np.int64)
    for r in range(world):
        owner[bounds[r]:bounds[r + 1]] = r * slice_ + np.arange(bounds[r + 1] - bounds[r])
    idx, deg, nb, od = g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree()
    f = np.float32
    base, damp = f(f(1.0) - f(0.85)), f(0.85)
    r_local = np.full(re - rb, base, np.float32)

    def contrib(v_local):
        o = od[rb + v_local]
        return f(r_local[v_local] / f(o)) if o else f(0.0)

    def init_fn(_):
        bufs = [torch.zeros(world * slice_, dtype=torch.float32) for _ in range(2)]
        for i in range(re - rb):
            bufs[0][rank * slice_ + i] = float(contrib(i))
        return bufs

    def pass_fn(c_in, c_out, eps):
        cin = c_in.numpy()
        active, err = 0, 0.0
        for i in range(re - rb):
            v = rb + i
            s = f(0.0)
            for j in range(idx[v], idx[v] + deg[v]):
                s = f(s + cin[owner[nb[j]]])
            new = f(base + f(damp * s))
            e = abs(float(f(new - r_local[i])))
            err += e
            active += e >= eps
            r_local[i] = new
            c_out[rank * slice_ + i] = float(contrib(i))
        return torch.tensor([float(active), err], dtype=torch.float64)

    def allgather_fn(c):
        parts = [torch.zeros(slice_, dtype=torch.float32) for _ in range(world)]
        dist.all_gather(parts, c[rank * slice_:(rank + 1) * slice_].clone())
        c.copy_(torch.cat(parts))

    def allreduce_fn(st):
        dist.all_reduce(st)
        return int(st[0].item()), float(st[1].item())

    its, passes, conv, err = agd.solve(rank, world, slice_, init_fn, pass_fn, allgather_fn, allreduce_fn, 30, 1e-4)
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
