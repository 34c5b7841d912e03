"""Narrow integer pulls on the GPU: the reference's 32/16/8-bit fixed-point
pulls (pushpull 9, 10, 11; pageRank.c:1455-1991) and 32/16/8-bit quantised
pulls (pushpull 4, 12, 13; pageRank.c:2119-2677).

The zero-extending integer gather reproduces the testbench's Quantized-context
goldens bit for bit; each solve equals the oracle (and the reference's own
code, where compiled) bit for bit: iteration count, per-pass active counts and
every rank, in both orders, on two tile shapes, in graph and stream launch."""
import ctypes as C

import numpy as np
import pytest

from conftest import fixed_inputs

pytestmark = pytest.mark.gpu

FORMS = [4, 5, 6, 7, 8, 9]  # AG_PREC_FIXED32 .. AG_PREC_QUANT8


def _oracle(ag, oracle, g, prec, iterations, eps):
    quant, width = ag.NARROW_FORM[prec]
    return oracle.pagerank_narrow(quant, width, g.in_edges_idx(), g.in_degree(), g.in_neighbours(),
                                  g.out_degree(), iterations, eps)


@pytest.mark.parametrize("i", range(13))
def test_quant_gather_matches_rtl_golden(gpu, rtl, i):
    ag = gpu
    run = rtl["pagerank_quant_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, x = fixed_inputs(run, fx, np.uint32)
    if n == 0:
        return
    od = np.zeros(len(deg), np.uint32)
    od[n:] = 1
    g = ag.Graph.from_inverse_csr(len(deg), deg, idx, nb, od)
    y = ag.DeviceGraph(g).gather_uint(x)
    for row in run["rows"]:
        assert "%016x" % int(y[row["v"]]) == row["golden"], (run["fixture"], run["class"], row["v"])
    assert (y[deg == 0] == 0).all()


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint32, np.uint64])
def test_gather_uint_matches_oracle(gpu, oracle, dtype):
    ag = gpu
    g = ag.Graph.rmat(13, 16, seed=5)
    rng = np.random.default_rng(1)
    x = rng.integers(0, np.iinfo(dtype).max, g.num_vertices, dtype=dtype, endpoint=True)
    y = ag.DeviceGraph(g).gather_uint(x)
    assert np.array_equal(y, oracle.gather_uint(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), x))


@pytest.mark.parametrize("prec", FORMS)
@pytest.mark.parametrize("scale,ef,eps", [(10, 16, 1e-4), (13, 16, 1e-6)])
def test_narrow_pull_matches_oracle(gpu, oracle, prec, scale, ef, eps):
    ag = gpu
    g = ag.Graph.rmat(scale, ef, seed=scale + 50)
    ref = _oracle(ag, oracle, g, prec, 300, eps)
    dg = ag.DeviceGraph(g)
    for tiles in ((256, 2048, 16384, 65536), (32, 32, 0, 0)):
        dg.set_tiles(*tiles)
        for order in (ag.AG_ORDER_FAST, ag.AG_ORDER_EXACT):
            r, res, hist = dg.pagerank(300, eps, precision=prec, order=order, history=300)
            assert res.iterations == ref["iterations"], (tiles, order)
            assert np.array_equal(hist["active"], ref["active"]), (tiles, order)
            assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32)), (tiles, order)


@pytest.mark.parametrize("prec", FORMS)
def test_narrow_pull_stream_launch(gpu, oracle, prec, monkeypatch):
    """The profiling launch (one kernel per pass, passes after convergence
    returning at once) gives the graph launch's bits."""
    ag = gpu
    g = ag.Graph.rmat(11, 8, seed=9)
    ref = _oracle(ag, oracle, g, prec, 120, 1e-6)
    monkeypatch.setenv("AG_LAUNCH_MODE", "stream")
    r, res, _ = ag.DeviceGraph(g).pagerank(120, 1e-6, precision=prec)
    assert res.iterations == ref["iterations"]
    assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))


@pytest.mark.parametrize("prec", FORMS)
def test_narrow_pull_edge_shapes(gpu, oracle, prec):
    """Vertex counts that are not a multiple of 4 (the quantiser's tail),
    isolated vertices, sinks, a graph without edges, and a graph smaller than
    the shared-memory table."""
    ag = gpu
    src = np.array([0, 0, 1, 2, 2, 3, 5, 5, 5, 7, 8, 8], np.uint32)
    dst = np.array([1, 2, 2, 0, 3, 3, 1, 2, 4, 7, 9, 0], np.uint32)
    cases = [ag.Graph.from_edges(11, src, dst), ag.Graph.from_edges(7, np.zeros(0, np.uint32), np.zeros(0, np.uint32)),
             ag.Graph.er(4099, 6, seed=2)]
    for g in cases:
        ref = _oracle(ag, oracle, g, prec, 50, 1e-7)
        r, res, _ = ag.DeviceGraph(g).pagerank(50, 1e-7, precision=prec)
        assert res.iterations == ref["iterations"], g.num_vertices
        assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32)), g.num_vertices


@pytest.mark.parametrize("prec", FORMS)
def test_narrow_dispatch_matches_reference_code(gpu, oracle, prec, capfd):
    """pageRankGraphCSR with the reference's pushpull code runs the form and
    prints its title; ranks equal the oracle and the reference's own host code
    (compiled with the emulated gather) bit for bit."""
    ag = gpu
    from oracle import refcode
    quant, width = ag.NARROW_FORM[prec]
    g = ag.Graph.rmat(12, 8, seed=78)
    args = ag.default_arguments(200, 1e-6)
    args.pushpull = ag.PUSHPULL_OF_PREC[prec]
    st = ag.lib.pageRankGraphCSR(C.byref(args), g.ptr)
    ranks = ag.stats_ranks(st)
    iters = st.contents.iterations
    ag.lib.freePageRankStats(st)
    title = ("Starting Page Rank Pull Quant_%d" % width) if quant else \
        ("Starting Page Rank Pull FP_%d (tolerance/epsilon)" % width)
    assert title in capfd.readouterr().out
    ref = _oracle(ag, oracle, g, prec, 200, 1e-6)
    assert iters == ref["iterations"] and np.array_equal(ranks.view(np.uint32), ref["ranks"].view(np.uint32))
    if refcode.available():
        rc = refcode.pagerank_narrow(quant, width, C.byref(args), g.ptr, g.num_vertices)
        assert iters == rc["iterations"] and np.array_equal(ranks.view(np.uint32), rc["ranks"].view(np.uint32))


def test_narrow_forms_reject_partitions(gpu):
    """A row partition holds only its rows' contributions: the integer pulls
    (which need every contribution, and the quantised forms their global
    minimum and maximum) refuse it with AG_ERR_UNSUPPORTED."""
    ag = gpu
    from accelgraph_b200.distributed import partition_bounds
    g = ag.Graph.rmat(10, 8, seed=1)
    bounds, slice_ = partition_bounds(g.in_degree(), 2)
    h = C.c_void_p()
    ag.check(ag.lib.ag_graph_upload_rows(g.ptr, bounds.ctypes.data_as(C.POINTER(C.c_uint32)), 2, 0, slice_, 0,
                                         C.byref(h)), "ag_graph_upload_rows")
    try:
        for prec in FORMS:
            o = ag.make_opts(prec)
            assert ag.lib.ag_pagerank_launch(h, 10, 1e-4, C.byref(o)) == ag.AG_ERR_UNSUPPORTED, prec
    finally:
        ag.lib.ag_graph_release(h)
