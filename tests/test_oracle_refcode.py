"""The oracle against the reference's own host code.

oracle/refcode runs the reference's unmodified pageRankPullGraphCSR and
SPMVPullGraphCSR (pageRank.c:942-1109, SPMV.c:622-751, compiled here with a
CPU emulation of the accelerator gather).  The oracle's restatement of those
loops must give the same ranks bit for bit and the same iteration counts; the
SpMV input vector and product must match bit for bit too.  Skipped where the
reference source was not available to compile the library."""
import ctypes as C

import numpy as np
import pytest


@pytest.fixture(scope="module")
def refcode():
    from oracle import refcode as rc
    if not rc.available():
        pytest.skip("reference pull calls not compiled (reference source absent)")
    return rc


def _graphs(ag):
    yield "rmat10_ef16", ag.Graph.rmat(10, 16, seed=3)
    yield "rmat12_ef8", ag.Graph.rmat(12, 8, seed=4)
    yield "er4096_d8", ag.Graph.er(4096, 8, seed=5)
    # a graph with isolated vertices, sinks and sources
    src = np.array([0, 0, 1, 2, 2, 3, 5, 5, 5, 7, 8, 8], np.uint32)
    dst = np.array([1, 2, 2, 0, 3, 3, 1, 2, 4, 7, 9, 0], np.uint32)
    yield "small_mixed", ag.Graph.from_edges(11, src, dst)


@pytest.mark.parametrize("iterations,epsilon", [(20, 1e-4), (200, 1e-6), (3, 1e-12), (300, 0.0)])
def test_oracle_pagerank_equals_reference_code(ag, oracle, refcode, iterations, epsilon):
    for name, g in _graphs(ag):
        args = ag.default_arguments(iterations, epsilon)
        ref = refcode.pagerank_pull(C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(),
                                    iterations, epsilon)
        assert ref["damp"] == np.float32(0.85) and ref["base_pr"] == np.float32(1.0) - np.float32(0.85)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        # the reference sums the residual with an OpenMP reduction (any order)
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
        # one gather per pass run: the converging pass counts
        assert ref["gathers"] == mine["passes"], name


def test_oracle_spmv_equals_reference_code(ag, oracle, refcode):
    for name, g in _graphs(ag):
        args = ag.default_arguments(1, 1e-4)
        ref = refcode.spmv_pull(C.byref(args), g.ptr, g.num_vertices)
        x = oracle.spmv_input(g.out_degree())
        assert np.array_equal(ref["x"].view(np.uint32), x.view(np.uint32)), name
        y = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), None, x)
        assert np.array_equal(ref["y"].view(np.uint32), y.view(np.uint32)), name
        assert ref["iterations"] == 1


@pytest.mark.parametrize("iterations,epsilon", [(20, 1e-4), (300, 1e-6), (5, 1e-12)])
def test_oracle_data_driven_equals_reference_code(ag, oracle, refcode, iterations, epsilon):
    """The worklist pull (pushpull 6, pageRank.c:2810-2969): ranks bit for bit
    and iteration counts equal to the reference's own CPU code."""
    for name, g in _graphs(ag):
        args = ag.default_arguments(iterations, epsilon)
        args.pushpull = 6
        ref = refcode.pagerank_dd(C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_dd(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_edges_idx(),
                                  g.out_degree(), g.out_neighbours(), iterations, epsilon)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
        # the worklist shrinks: the data-driven solve differs from the topology-driven one
        if epsilon >= 1e-6 and name.startswith("rmat"):
            assert (mine["active"][1:] <= g.num_vertices).all()


@pytest.mark.parametrize("iterations,epsilon", [(20, 1e-4), (300, 1e-6)])
def test_oracle_fixed64_equals_reference_code(ag, oracle, refcode, iterations, epsilon):
    """The 64-bit fixed-point pull (pushpull 2): the oracle restatement equals
    the reference's own host code bit for bit (same stand-in conversions)."""
    for name, g in _graphs(ag):
        args = ag.default_arguments(iterations, epsilon)
        args.pushpull = 2
        ref = refcode.pagerank_fixed64(C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_fixed64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(),
                                       iterations, epsilon)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
        assert ref["gathers"] == mine["passes"], name


@pytest.mark.parametrize("quant", [False, True])
@pytest.mark.parametrize("width", [32, 16, 8])
def test_oracle_narrow_equals_reference_code(ag, oracle, refcode, quant, width):
    """The narrow integer pulls (fixed point pushpull 9/10/11, quantised
    pushpull 4/12/13): the oracle restatement equals the reference's own host
    code bit for bit, iteration count and per-pass gathers included."""
    iterations, epsilon = 60, 1e-6
    for name, g in _graphs(ag):
        args = ag.default_arguments(iterations, epsilon)
        ref = refcode.pagerank_narrow(quant, width, C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_narrow(quant, width, g.in_edges_idx(), g.in_degree(), g.in_neighbours(),
                                      g.out_degree(), iterations, epsilon)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
        assert ref["gathers"] == mine["passes"], name


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_oracle_push_equals_reference_code(ag, oracle, refcode, kind, capfd):
    """The push forms (pushpull 1, 3, 5) on one thread: the oracle restatement
    equals the reference's own host code bit for bit."""
    for name, g in _graphs(ag):
        args = ag.default_arguments(80, 1e-6)
        args.ker_numThreads = 1
        ref = refcode.pagerank_push(kind, C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_push(kind, g.out_edges_idx(), g.out_degree(), g.out_neighbours(), 80, 1e-6)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
    capfd.readouterr()


def test_oracle_push_float_equals_pull(ag, oracle):
    """One source after the other, each next[u] receives its contributions in
    increasing source order: the inverse row's stream order.  The sequential
    push is therefore the pull, bit for bit (and the 64-bit fixed-point push
    the 64-bit fixed-point pull)."""
    for name, g in _graphs(ag):
        push = oracle.pagerank_push(0, g.out_edges_idx(), g.out_degree(), g.out_neighbours(), 100, 1e-7)
        pull = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 100, 1e-7)
        assert push["iterations"] == pull["iterations"], name
        assert np.array_equal(push["ranks"].view(np.uint32), pull["ranks"].view(np.uint32)), name
        pfx = oracle.pagerank_push(1, g.out_edges_idx(), g.out_degree(), g.out_neighbours(), 100, 1e-7)
        fx = oracle.pagerank_fixed64(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 100, 1e-7)
        assert pfx["iterations"] == fx["iterations"], name
        assert np.array_equal(pfx["ranks"].view(np.uint32), fx["ranks"].view(np.uint32)), name


@pytest.mark.parametrize("pull_push", [False, True])
def test_oracle_residual_equals_reference_code(ag, oracle, refcode, pull_push, capfd):
    """The data-driven push (pushpull 7) and pull-push (pushpull 8) on one
    thread: the oracle restatement equals the reference's own code bit for
    bit."""
    for name, g in _graphs(ag):
        args = ag.default_arguments(100, 1e-6)
        args.ker_numThreads = 1
        ref = refcode.pagerank_residual(pull_push, C.byref(args), g.ptr, g.num_vertices)
        mine = oracle.pagerank_residual(pull_push, g.in_edges_idx(), g.in_degree(), g.in_neighbours(),
                                        g.out_edges_idx(), g.out_degree(), g.out_neighbours(), 100, 1e-6)
        assert ref["iterations"] == mine["iterations"], name
        assert np.array_equal(ref["ranks"].view(np.uint32), mine["ranks"].view(np.uint32)), name
        assert abs(ref["error_total"] - mine["error_total"]) <= 1e-12 + 1e-9 * abs(mine["error_total"]), name
    capfd.readouterr()
