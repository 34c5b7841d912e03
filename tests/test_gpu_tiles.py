"""Tile shapes and the autotuner: any shape gives EXACT-order results that
are bit-identical to the oracle, and the tuner keeps a valid shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_set_tiles_keeps_exact_results(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(13, 16)
    ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 60, 1e-6)
    dg = ag.DeviceGraph(g)
    for cap, chunk, hot in ((128, 1024, 0), (256, 4096, 8192), (64, 512, 16384)):
        dg.set_tiles(cap, chunk, hot, 65536)
        t = dg.tiles()
        assert (t.task_edges, t.hub_chunk) == (cap, chunk)
        r, res, _ = dg.pagerank(60, 1e-6, order=ag.AG_ORDER_EXACT)
        assert res.iterations == ref["iterations"] and np.array_equal(r, ref["ranks"])
        r, res, _ = dg.pagerank(60, 1e-6)
        assert np.abs(r.astype(np.float64) - ref["ranks"]).sum() / ref["ranks"].sum() <= 1e-5


def test_set_tiles_rejects_bad_shapes(gpu):
    ag = gpu
    dg = ag.DeviceGraph(ag.Graph.rmat(8, 8))
    with pytest.raises(ag.AGError):
        dg.set_tiles(512, 2048, 0, 0)
    with pytest.raises(ag.AGError):
        dg.set_tiles(256, 128, 0, 0)


def test_autotune_and_cache(gpu, oracle, tmp_path, monkeypatch):
    ag = gpu
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("AG_TUNE_CACHE", str(cache))
    g = ag.Graph.rmat(14, 16)
    dg = ag.DeviceGraph(g)
    best, us = dg.autotune(passes=4)
    assert us > 0 and 32 <= best.task_edges <= 256 and best.hub_chunk >= best.task_edges
    assert cache.read_text().count("\n") == 1
    dg2 = ag.DeviceGraph(g)
    best2, us2 = dg2.autotune(passes=4)  # served from the cache file
    assert (best2.task_edges, best2.hub_chunk, best2.hot_entries) == (best.task_edges, best.hub_chunk,
                                                                       best.hot_entries)
    assert cache.read_text().count("\n") == 1
    ref = oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), 40, 1e-6)
    r, res, _ = dg2.pagerank(40, 1e-6, order=ag.AG_ORDER_EXACT)
    assert np.array_equal(r, ref["ranks"])


def test_multigraph_autotune(gpu):
    ag = gpu
    gs = [ag.Graph.rmat(s, 8, seed=s) for s in (8, 9, 10, 11)]
    mg = ag.MultiGraph(gs)
    best, us = mg.autotune(passes=4)
    assert best.hot_entries == 0 and us > 0
    parts, info = mg.pagerank(100, 1e-6)
    assert info["converged"].all()
