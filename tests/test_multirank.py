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
