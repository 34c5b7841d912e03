"""The target configurations on the GPU against the CPU oracle, at full size.

C1  R-MAT s16 ef16, PageRank to eps 1e-4, at most 20 passes.
C2  R-MAT s22 ef16 (4,194,304 vertices, 65,245,291 in-edges): PageRank to eps
    1e-6, and one weighted SpMV product with edge weights and x uniform in
    [0, 1).
C3  R-MAT s24 ef16 (16,777,216 vertices, about 2.6e8 in-edges): plain FP32
    PageRank to eps 1e-6.

EXACT order sums every row in the reference loop's stream order: ranks,
iteration count and the number of vertices still moving by eps or more in
every pass equal the oracle's (the restatement of pageRank.c:942-1109 and the
sequential binary32 gather of the compute units) bit for bit.  FAST order
stays within 1e-5 relative L1 of the oracle's ranks, the tolerance asked of
binary32 results; its iteration count may differ by a few passes at eps
1e-6.  The SpMV product follows SPMV.c:1200-1224.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 27491095
TOL = 1e-5


def _rel(a, b):
    return float(np.abs(a.astype(np.float64) - b).sum() / np.abs(b.astype(np.float64)).sum())


def _pagerank_case(ag, oracle, scale, iterations, eps):
    g = ag.Graph.rmat(scale, 16, seed=SEED, flags=ag.AG_BUILD_DEDUPE)
    ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), iterations, eps)
    dg = ag.DeviceGraph(g)
    r, res, hist = dg.pagerank(iterations, eps, order=ag.AG_ORDER_EXACT, history=iterations)
    assert res.iterations == ref["iterations"] and res.passes == ref["passes"]
    assert np.array_equal(hist["active"], ref["active"])
    assert np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))
    rf, resf, _ = dg.pagerank(iterations, eps)
    assert _rel(rf, ref["ranks"]) <= TOL
    dg.release()
    return g, ref


def test_c1_rmat16_pagerank(gpu, oracle):
    _, ref = _pagerank_case(gpu, oracle, 16, 20, 1e-4)
    assert ref["passes"] <= 20


def test_c2_rmat22_pagerank(gpu, oracle):
    g, ref = _pagerank_case(gpu, oracle, 22, 300, 1e-6)
    assert g.num_edges == 65_245_291 and ref["iterations"] < 300


def test_c2_rmat22_weighted_spmv(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(22, 16, seed=SEED, flags=ag.AG_BUILD_DEDUPE | ag.AG_BUILD_WEIGHTS)
    n = g.num_vertices
    x = np.empty(n, np.float32)
    ag.lib.ag_fill_uniform(x.ctypes.data_as(ag.f32p), n, SEED + 1)
    w = g.in_weights()
    assert w.min() >= 0.0 and w.max() < 1.0 and x.min() >= 0.0 and x.max() < 1.0
    yo = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), w, x)
    dg = ag.DeviceGraph(g, weights=True)
    ye = dg.spmv(x, mode=ag.AG_SPMV_EXACT)
    assert np.array_equal(ye.view(np.uint32), yo.view(np.uint32))
    assert _rel(dg.spmv(x), yo) <= TOL


def test_c3_rmat24_pagerank(gpu, oracle):
    g, ref = _pagerank_case(gpu, oracle, 24, 300, 1e-6)
    assert g.num_vertices == 1 << 24 and ref["iterations"] < 300
