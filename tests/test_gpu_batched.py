"""Batched forms on the GPU: personalized PageRank of k sources as one SpMM
pass, checked against the CPU oracle (every column in stream order, so the
result is bit-identical)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,k", [("er", 8), ("er", 64), ("rmat", 64), ("rmat", 5)])
def test_ppr_spmm_matches_oracle(gpu, oracle, kind, k):
    ag = gpu
    g = ag.Graph.er(4096, 16) if kind == "er" else ag.Graph.rmat(12, 16)
    rng = np.random.default_rng(1000)
    sources = rng.choice(g.num_vertices, size=k, replace=False).astype(np.uint32)
    dg = ag.DeviceGraph(g)
    r, res = dg.ppr(sources, iterations=60, epsilon=1e-6)
    ro, it, passes = oracle.ppr(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), sources,
                                iterations=60, epsilon=1e-6)
    assert res.passes == passes and res.iterations == it
    assert np.array_equal(r, ro)
    # each column carries the teleport of its own source
    for i, s in enumerate(sources):
        assert r[s, i] == r[:, i].max()


def test_ppr_spmm_rejects_bad_sources(gpu):
    ag = gpu
    g = ag.Graph.er(256, 4)
    dg = ag.DeviceGraph(g)
    with pytest.raises(ag.AGError):
        dg.ppr(np.arange(65, dtype=np.uint32))
    with pytest.raises(ag.AGError):
        dg.ppr(np.array([256], np.uint32))


def _uneven_graphs(ag, count=12, seed=7):
    rng = np.random.default_rng(seed)
    gs = []
    for i in range(count):
        scale = int(rng.integers(6, 12))
        ef = int(rng.integers(4, 20))
        gs.append(ag.Graph.rmat(scale, ef, seed=1000 + i))
    gs.append(ag.Graph.from_edges(5, [0, 1, 2], [1, 2, 3]))          # chain: converges fast
    gs.append(ag.Graph.from_edges(3, [], []))                         # no edges
    return gs


@pytest.mark.parametrize("order", [0, 1])
def test_multigraph_matches_per_graph_oracle(gpu, oracle, order):
    ag = gpu
    gs = _uneven_graphs(ag)
    mg = ag.MultiGraph(gs)
    parts, info = mg.pagerank(iterations=200, epsilon=1e-6, order=order)
    for i, g in enumerate(gs):
        ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 200, 1e-6)
        if order == 1:
            assert info["iterations"][i] == ref["iterations"], i
            assert info["passes"][i] == ref["passes"], i
            assert np.array_equal(parts[i], ref["ranks"]), i
        else:
            assert abs(int(info["iterations"][i]) - ref["iterations"]) <= max(10, ref["iterations"] // 10)
            den = max(np.abs(ref["ranks"]).sum(), 1e-30)
            assert np.abs(parts[i].astype(np.float64) - ref["ranks"]).sum() / den <= 1e-5


def test_multigraph_iteration_cap_per_graph(gpu, oracle):
    ag = gpu
    gs = _uneven_graphs(ag, count=4, seed=9)
    mg = ag.MultiGraph(gs)
    parts, info = mg.pagerank(iterations=7, epsilon=1e-9, order=1)
    for i, g in enumerate(gs):
        ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 7, 1e-9)
        assert info["iterations"][i] == ref["iterations"] and np.array_equal(parts[i], ref["ranks"])
