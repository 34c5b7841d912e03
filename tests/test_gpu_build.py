"""Graph preprocessing on the GPU: ag_graph_build_csr gives the host
builder's CSR array for array, bit for bit, for every build flag, with and
without weights; ag_graph_build goes from an edge list straight to a device
graph whose PageRank equals the oracle's on the host-built graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _edges(n, m, seed, loops=True):
    rng = np.random.default_rng(seed)
    # skewed endpoints give repeats, long rows and empty rows
    src = (rng.pareto(1.2, m) * 3).astype(np.int64) % n
    dst = rng.integers(0, n, m)
    if loops:
        k = m // 20
        dst[:k] = src[:k]
    w = rng.random(m, dtype=np.float32)
    return src.astype(np.uint32), dst.astype(np.uint32), w


def _arrays(g):
    el = g.g.sorted_edges_array.contents
    iel = g.g.inverse_sorted_edges_array.contents
    out = {
        "out_degree": g.out_degree(), "in_degree": g.in_degree(),
        "out_idx": np.ctypeslib.as_array(g.g.vertices.contents.edges_idx, shape=(g.num_vertices + 1,)).copy(),
        "in_idx": np.ctypeslib.as_array(g.g.inverse_vertices.contents.edges_idx, shape=(g.num_vertices + 1,)).copy(),
        "out_src": g.out_sources(), "out_dst": g.out_neighbours(),
        "in_src": g.in_owners(), "in_dst": g.in_neighbours(),
    }
    if el.edges_array_weight:
        out["out_w"] = np.ctypeslib.as_array(el.edges_array_weight, shape=(g.num_edges,)).view(np.uint32).copy()
        out["in_w"] = np.ctypeslib.as_array(iel.edges_array_weight, shape=(g.num_edges,)).view(np.uint32).copy()
    return out


def _same(ag, a, b):
    assert a.num_vertices == b.num_vertices and a.num_edges == b.num_edges
    assert a.g.avg_degree == b.g.avg_degree
    assert np.float32(a.g.max_weight).view(np.uint32) == np.float32(b.g.max_weight).view(np.uint32)
    xa, xb = _arrays(a), _arrays(b)
    assert xa.keys() == xb.keys()
    for k in xa:
        assert np.array_equal(xa[k], xb[k]), k


@pytest.mark.parametrize("n,m,seed", [(1000, 20000, 1), (4096, 3000, 2), (70000, 400000, 3)])
def test_build_csr_matches_host_builder(gpu, n, m, seed):
    ag = gpu
    src, dst, w = _edges(n, m, seed)
    for flags in (0, ag.AG_BUILD_SORT, ag.AG_BUILD_DEDUPE, ag.AG_BUILD_DEDUPE | ag.AG_BUILD_SORT,
                  ag.AG_BUILD_SYMMETRIC, ag.AG_BUILD_DEDUPE | ag.AG_BUILD_SYMMETRIC):
        for weight in (None, w):
            host = ag.Graph.from_edges(n, src, dst, weight, flags)
            dev = ag.Graph.build_gpu(n, src, dst, weight, flags)
            _same(ag, dev, host)


def test_build_csr_edge_cases(gpu):
    ag = gpu
    # no edges
    host = ag.Graph.from_edges(5, np.zeros(0, np.uint32), np.zeros(0, np.uint32), None, ag.AG_BUILD_DEDUPE)
    dev = ag.Graph.build_gpu(5, np.zeros(0, np.uint32), np.zeros(0, np.uint32), None, ag.AG_BUILD_DEDUPE)
    _same(ag, dev, host)
    # only self loops: all dropped by dedupe
    s = np.array([0, 1, 2, 2], np.uint32)
    host = ag.Graph.from_edges(3, s, s, None, ag.AG_BUILD_DEDUPE)
    dev = ag.Graph.build_gpu(3, s, s, None, ag.AG_BUILD_DEDUPE)
    _same(ag, dev, host)
    assert dev.num_edges == 0
    # one vertex, repeated edges kept without dedupe
    z = np.zeros(7, np.uint32)
    _same(ag, ag.Graph.build_gpu(1, z, z, None, 0), ag.Graph.from_edges(1, z, z, None, 0))
    # an endpoint outside the vertex range is rejected with its edge index
    with pytest.raises(ag.AGError):
        ag.Graph.build_gpu(4, np.array([0, 1, 9], np.uint32), np.array([1, 2, 3], np.uint32))
    assert "edge 2" in ag.lib.ag_last_error().decode()


def test_build_from_device_tensors(gpu):
    ag = gpu
    import torch
    src, dst, w = _edges(5000, 60000, 7)
    ts, td, tw = (torch.from_numpy(a.astype(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (src, dst, w))
    dev = ag.Graph.build_gpu(5000, ts, td, tw, ag.AG_BUILD_DEDUPE)
    host = ag.Graph.from_edges(5000, src, dst, w, ag.AG_BUILD_DEDUPE)
    _same(ag, dev, host)


def test_device_graph_from_edges_pagerank(gpu, oracle):
    """Edge list -> device graph with no host CSR: EXACT-order PageRank equals
    the oracle on the host-built CSR, and SpMV with the built weights equals
    the device graph uploaded from the host CSR."""
    ag = gpu
    src, dst, w = _edges(30000, 300000, 11)
    host = ag.Graph.from_edges(30000, src, dst, w, ag.AG_BUILD_DEDUPE)
    ref = oracle.pagerank_pull(host.in_edges_idx(), host.in_degree(), host.in_neighbours(), host.out_degree(),
                               100, 1e-6)
    dg = ag.DeviceGraph.from_edges(30000, src, dst, w)
    assert dg.num_edges == host.num_edges
    r, res, _ = dg.pagerank(100, 1e-6, order=ag.AG_ORDER_EXACT)
    assert res.iterations == ref["iterations"] and np.array_equal(r, ref["ranks"])
    x = np.random.default_rng(1).random(30000, dtype=np.float32)
    y_built = dg.spmv(x, ag.AG_SPMV_GRAPH_WEIGHTS | ag.AG_SPMV_EXACT)
    y_up = ag.DeviceGraph(host, weights=True).spmv(x, ag.AG_SPMV_GRAPH_WEIGHTS | ag.AG_SPMV_EXACT)
    assert np.array_equal(y_built, y_up)
