"""64-bit fixed-point pull on the GPU (the reference's pushpull 2): the integer
gather reproduces the testbench's FixedPoint-context goldens bit for bit, and
the solve equals the oracle (and the reference's own code, where compiled) bit
for bit in both orders and on every tile shape, integer sums having no order."""
import ctypes as C

import numpy as np
import pytest

from conftest import fixed_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("i", range(13))
def test_fixed_gather_matches_rtl_golden(gpu, rtl, i):
    ag = gpu
    run = rtl["pagerank_fixed_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, x = fixed_inputs(run, fx)
    if n == 0:
        return
    od = np.zeros(len(deg), np.uint32)
    od[n:] = 1
    g = ag.Graph.from_inverse_csr(len(deg), deg, idx, nb, od)
    y = ag.DeviceGraph(g).gather_u64(x)
    for row in run["rows"]:
        assert "%016x" % int(y[row["v"]]) == row["golden"], (run["fixture"], run["class"], row["v"])
    assert (y[deg == 0] == 0).all()


def test_fixed_gather_wraps_modulo_2_64(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(12, 16, seed=2)
    rng = np.random.default_rng(0)
    x = rng.integers(0, 2**64 - 1, g.num_vertices, dtype=np.uint64, endpoint=True)
    y = ag.DeviceGraph(g).gather_u64(x)
    assert np.array_equal(y, oracle.gather_u64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), x))


@pytest.mark.parametrize("scale,ef,eps", [(10, 16, 1e-4), (13, 16, 1e-6)])
def test_fixed64_pull_matches_oracle(gpu, oracle, scale, ef, eps):
    ag = gpu
    g = ag.Graph.rmat(scale, ef, seed=scale + 40)
    ref = oracle.pagerank_fixed64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 300, eps)
    dg = ag.DeviceGraph(g)
    for tiles in ((256, 2048, 16384, 65536), (32, 32, 0, 0)):
        dg.set_tiles(*tiles)
        for order in (ag.AG_ORDER_FAST, ag.AG_ORDER_EXACT):
            r, res, hist = dg.pagerank(300, eps, precision=ag.AG_PREC_FIXED64, order=order, history=300)
            assert res.iterations == ref["iterations"], (tiles, order)
            assert np.array_equal(hist["active"], ref["active"]), (tiles, order)
            assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32)), (tiles, order)


def test_fixed64_pull_matches_reference_code_and_dispatch(gpu, oracle, capfd):
    ag = gpu
    from oracle import refcode
    g = ag.Graph.rmat(12, 8, seed=77)
    args = ag.default_arguments(200, 1e-6)
    args.pushpull = 2
    st = ag.lib.pageRankGraphCSR(C.byref(args), g.ptr)
    ranks = ag.stats_ranks(st)
    iters = st.contents.iterations
    ag.lib.freePageRankStats(st)
    assert "Starting Page Rank Pull FP_64" in capfd.readouterr().out
    ref = oracle.pagerank_fixed64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 200, 1e-6)
    assert iters == ref["iterations"] and np.array_equal(ranks, ref["ranks"])
    if refcode.available():
        rc = refcode.pagerank_fixed64(C.byref(args), g.ptr, g.num_vertices)
        assert iters == rc["iterations"] and np.array_equal(ranks.view(np.uint32), rc["ranks"].view(np.uint32))
