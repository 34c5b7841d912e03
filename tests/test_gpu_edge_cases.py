"""Degenerate and extreme inputs through every form on the GPU: empty graphs,
graphs without edges, a single hub row far above the split size, dangling
vertices, and the largest in-degree a row item can hold."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pull(oracle, g, it, eps):
    return oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), it, eps)


def _dd(oracle, g, it, eps):
    return oracle.pagerank_dd(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_edges_idx(),
                              g.out_degree(), g.out_neighbours(), it, eps)


def test_graph_without_edges(gpu, oracle):
    ag = gpu
    g = ag.Graph.from_edges(5, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    dg = ag.DeviceGraph(g)
    for order in (ag.AG_ORDER_FAST, ag.AG_ORDER_EXACT):
        r, res, _ = dg.pagerank(20, 1e-4, order=order)
        ref = _pull(oracle, g, 20, 1e-4)
        assert res.iterations == ref["iterations"] == 0 and np.array_equal(r, ref["ranks"])
        r, res, _ = dg.pagerank(20, 1e-4, order=order, data_driven=True)
        ref = _dd(oracle, g, 20, 1e-4)
        assert res.iterations == ref["iterations"] and np.array_equal(r, ref["ranks"])
    y = dg.spmv(np.ones(5, np.float32), ag.AG_SPMV_UNIT)
    assert np.array_equal(y, np.zeros(5, np.float32))
    ranks, info = dg.ppr(np.array([0, 3], np.uint32), iterations=10, epsilon=1e-6)
    assert ranks.shape == (5, 2) and np.isfinite(ranks).all()


def test_graph_without_vertices(gpu):
    ag = gpu
    g = ag.Graph.from_edges(0, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    dg = ag.DeviceGraph(g)
    r, res, _ = dg.pagerank(20, 1e-4)
    assert r.size == 0 and res.passes == 0
    r, res, _ = dg.pagerank(20, 1e-4, data_driven=True)
    assert r.size == 0 and res.passes == 0
    assert dg.tasks().shape == (0, 4)


def _rel(a, b):
    return np.abs(a.astype(np.float64) - b).sum() / np.abs(b).sum()


def test_one_huge_hub_row(gpu, oracle):
    """Every vertex points at vertex 0 (in-degree N - 1, far above the 2048-edge
    split) and at one random other vertex.  EXACT order equals the stream-order
    oracle bit for bit.  Summed in stream order in binary32, the hub row's
    200,000 terms drift by about 3e-4 relative; FAST order sums it in chunks
    and a tree, so FAST must be at least as close to the FP64 fixpoint."""
    ag = gpu
    n = 200_000
    rng = np.random.default_rng(4)
    src = np.concatenate([np.arange(1, n), np.arange(n)]).astype(np.uint32)
    dst = np.concatenate([np.zeros(n - 1), rng.integers(0, n, n)]).astype(np.uint32)
    g = ag.Graph.from_edges(n, src, dst, None, ag.AG_BUILD_DEDUPE)
    assert g.in_degree().max() >= n - 2
    dg = ag.DeviceGraph(g)
    r64, _ = dg.pagerank_f64(3000, 1e-14)
    for dd, ref in ((False, _pull(oracle, g, 100, 1e-6)), (True, _dd(oracle, g, 100, 1e-6))):
        r, res, _ = dg.pagerank(100, 1e-6, order=ag.AG_ORDER_EXACT, data_driven=dd)
        assert res.iterations == ref["iterations"] and np.array_equal(r, ref["ranks"]), dd
        r, res, _ = dg.pagerank(100, 1e-6, data_driven=dd)
        assert abs(int(res.iterations) - ref["iterations"]) <= 20, dd
        assert _rel(r, r64) <= _rel(ref["ranks"], r64) + 1e-6, dd


def test_exact_order_hub_rows_give_their_work_away(gpu, oracle):
    """Four hub rows of 9,000 to 150,000 in-edges among 600,000 short rows,
    about four row items per warp.  A warp that sums a hub row of at least
    32,768 in-edges in stream order gives the rest of its work list to warps
    that run out of items.  Every row is still summed once, in stream order,
    so EXACT PageRank over many passes (the donor table is cleared between
    passes) and an EXACT weighted product equal the oracle bit for bit."""
    ag = gpu
    n = 600_000
    rng = np.random.default_rng(21)
    src, dst = [rng.integers(0, n, 6 * n)], [rng.integers(0, n, 6 * n)]
    for v, d in ((7, 150_000), (70_000, 40_000), (300_001, 9_000), (599_999, 20_000)):
        src.append(rng.choice(n, size=d, replace=False))
        dst.append(np.full(d, v))
    src = np.concatenate(src).astype(np.uint32)
    dst = np.concatenate(dst).astype(np.uint32)
    w = rng.random(src.size, dtype=np.float32)
    g = ag.Graph.from_edges(n, src, dst, w, ag.AG_BUILD_DEDUPE)
    assert np.sort(g.in_degree())[-2] >= 32768
    dg = ag.DeviceGraph(g, weights=True)
    assert dg.tasks(True).shape[0] > 2 * 148 * 32
    ref = _pull(oracle, g, 40, 1e-9)
    r, res, _ = dg.pagerank(40, 1e-9, order=ag.AG_ORDER_EXACT)
    assert res.iterations == ref["iterations"] and np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))
    x = np.empty(n, np.float32)
    ag.lib.ag_fill_uniform(x.ctypes.data_as(ag.f32p), n, 27491095 + 3)
    yo = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.in_weights(), x)
    for _ in range(3):
        assert np.array_equal(dg.spmv(x, mode=ag.AG_SPMV_EXACT).view(np.uint32), yo.view(np.uint32))


@pytest.mark.parametrize("kind", ["mixed_signs", "ties", "magnitudes", "infinity"])
def test_exact_order_sum_of_hard_values(gpu, oracle, kind):
    """EXACT-order sums of values where binary32 rounding is delicate: signs
    that cancel, multiples of 1/8 that round ties, magnitudes from 2^-140 to
    1e30, and +inf.  Rows of 33 to 20,000 in-edges take every summation path
    (per-lane sums in row items, long rows, hub rows whose chunks stage their
    values for one warp's chain).  The unit-weight product equals the
    one-by-one binary32 sum bit for bit."""
    ag = gpu
    rng = np.random.default_rng(33)
    n = 30_000
    src, dst = [rng.integers(0, n, 4 * n)], [rng.integers(0, n, 4 * n)]
    for v, d in enumerate((40, 100, 256, 300, 1000, 2048, 2100, 5000, 20_000, 33)):
        src.append(rng.choice(n, size=d, replace=False))
        dst.append(np.full(d, v))
    g = ag.Graph.from_edges(n, np.concatenate(src).astype(np.uint32), np.concatenate(dst).astype(np.uint32), None,
                            ag.AG_BUILD_DEDUPE)
    if kind == "mixed_signs":
        x = rng.uniform(-1, 1, n)
    elif kind == "ties":
        x = rng.integers(-8, 9, n) * 0.125
        x[::5] = 2.0 ** rng.integers(-30, 10, x[::5].size)
    elif kind == "magnitudes":
        x = rng.standard_normal(n) * 10.0 ** rng.integers(-30, 31, n)
        x[::11] = 2.0 ** -140
        x[::13] = 0.0
    else:
        x = rng.random(n)
        x[rng.integers(0, n, 40)] = np.inf
    x = x.astype(np.float32)
    y = ag.DeviceGraph(g).spmv(x, mode=ag.AG_SPMV_UNIT | ag.AG_SPMV_EXACT)
    yo = oracle.gather(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), x)
    assert not np.isnan(yo).any()
    assert np.array_equal(y.view(np.uint32), yo.view(np.uint32))


def test_dangling_vertices_and_row_item_limits(gpu, oracle):
    """Rows of exactly 256 and 257 in-edges (the row-item limit and the first
    long row), 32 and 33 (the per-lane stream-order limit), and vertices with
    no out-edges whose rank mass is dropped as the reference drops it."""
    ag = gpu
    rng = np.random.default_rng(9)
    n = 4096
    src, dst = [], []
    for v, d in ((1, 256), (2, 257), (3, 32), (4, 33), (5, 2048), (6, 2049)):
        s = rng.choice(np.arange(100, n), size=d, replace=False)
        src.append(s)
        dst.append(np.full(d, v))
    # a random background, with vertices 3000.. left without out-edges
    s = rng.integers(0, 3000, 20000)
    src.append(s)
    dst.append(rng.integers(0, n, 20000))
    g = ag.Graph.from_edges(n, np.concatenate(src).astype(np.uint32), np.concatenate(dst).astype(np.uint32),
                            None, ag.AG_BUILD_DEDUPE)
    dg = ag.DeviceGraph(g)
    ref = _pull(oracle, g, 200, 1e-7)
    r, res, _ = dg.pagerank(200, 1e-7, order=ag.AG_ORDER_EXACT)
    assert res.iterations == ref["iterations"] and np.array_equal(r, ref["ranks"])
    assert r.sum() < 1.0  # dangling mass is not redistributed
