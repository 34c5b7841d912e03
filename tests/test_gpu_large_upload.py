"""Uploads of host graphs of a million in-edges and more: the in-edges travel
on the upload's copy stream while the relabelled layout and the work lists are
built from the degrees.  An EXACT-order solve and an EXACT-order weighted
product equal the oracle bit for bit, and a bad in-edge anywhere in the array
is reported with its own index, without a fault."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_large_upload_pagerank_exact(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(17, 16, seed=17)
    assert g.num_edges >= 1 << 20
    ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 60, 1e-7)
    r, res, _ = ag.DeviceGraph(g).pagerank(60, 1e-7, order=ag.AG_ORDER_EXACT)
    assert res.iterations == ref["iterations"]
    assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))


def test_large_upload_weighted_spmv_exact(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(17, 16, seed=18, flags=ag.AG_BUILD_DEDUPE | ag.AG_BUILD_WEIGHTS)
    dg = ag.DeviceGraph(g, weights=True)
    x = np.empty(g.num_vertices, np.float32)
    ag.lib.ag_fill_uniform(x.ctypes.data_as(ag.f32p), g.num_vertices, 27491095 + 2)
    y = dg.spmv(x, mode=ag.AG_SPMV_EXACT)
    yo = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.in_weights(), x)
    assert np.array_equal(y, yo)


@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_large_upload_reports_bad_edge(gpu, where):
    """A bad in-edge near the start, the middle or the end is rejected (no
    fault), with its index in the message; the library stays usable."""
    ag = gpu
    n, e = 1 << 16, (1 << 20) + 777
    rng = np.random.default_rng(5)
    deg = np.full(n, e // n, np.uint32)
    deg[: e - int(deg.sum())] += 1
    idx = np.concatenate([[0], np.cumsum(deg)[:-1]]).astype(np.uint32)
    nb = rng.integers(0, n, e, dtype=np.uint32)
    bad = {"first": 3, "middle": e // 2 + 5, "last": e - 2}[where]
    nb[bad] = n + 9
    g = ag.Graph.from_inverse_csr(n, deg, idx, nb, np.ones(n, np.uint32))
    with pytest.raises(ag.AGError) as exc:
        ag.DeviceGraph(g)
    assert exc.value.status == ag.AG_ERR_INVALID_GRAPH
    assert "in-edge %d names" % bad in str(exc.value)
    ok = ag.Graph.rmat(10, 8, seed=1)
    r, res, _ = ag.DeviceGraph(ok).pagerank(20, 1e-4)
    assert res.passes > 0 and np.isfinite(r).all()
