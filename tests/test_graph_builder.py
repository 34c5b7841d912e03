"""Host graph substrate: edge list -> forward and inverse CSR, generators,
binary edge-list reader.  Checked against an independent numpy derivation:
degrees, offsets and neighbour arrays must be bit-exact."""
import numpy as np
import pytest


def numpy_csr(n, src, dst, w=None, dedupe=False, sort=False):
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    idx = np.arange(len(src))
    if dedupe:
        keep = src != dst
        src, dst, idx = src[keep], dst[keep], idx[keep]
        key = src * n + dst
        order = np.lexsort((idx, key))
        key, src, dst, idx = key[order], src[order], dst[order], idx[order]
        first = np.ones(len(key), bool)
        first[1:] = key[1:] != key[:-1]
        src, dst, idx = src[first], dst[first], idx[first]
    elif sort:
        order = np.lexsort((idx, dst, src))
        src, dst, idx = src[order], dst[order], idx[order]
    else:
        order = np.argsort(src, kind="stable")
        src, dst, idx = src[order], dst[order], idx[order]
    # inverse: stable by destination of the forward order
    inv = np.argsort(dst, kind="stable")
    out_deg = np.bincount(src, minlength=n).astype(np.uint32)
    in_deg = np.bincount(dst, minlength=n).astype(np.uint32)
    res = {
        "out_deg": out_deg, "in_deg": in_deg,
        "out_idx": np.concatenate([[0], np.cumsum(out_deg)[:-1]]).astype(np.uint32) if n else out_deg,
        "in_idx": np.concatenate([[0], np.cumsum(in_deg)[:-1]]).astype(np.uint32) if n else in_deg,
        "out_src": src.astype(np.uint32), "out_dst": dst.astype(np.uint32),
        "in_owner": dst[inv].astype(np.uint32), "in_nb": src[inv].astype(np.uint32),
    }
    if w is not None:
        w = np.asarray(w, np.float32)
        res["out_w"] = w[idx]
        res["in_w"] = w[idx][inv]
    return res


def assert_graph_equals(g, ref):
    assert np.array_equal(g.out_degree(), ref["out_deg"])
    assert np.array_equal(g.in_degree(), ref["in_deg"])
    assert np.array_equal(g.out_edges_idx(), ref["out_idx"])
    assert np.array_equal(g.in_edges_idx(), ref["in_idx"])
    assert np.array_equal(g.out_sources(), ref["out_src"])
    assert np.array_equal(g.out_neighbours(), ref["out_dst"])
    assert np.array_equal(g.in_owners(), ref["in_owner"])
    assert np.array_equal(g.in_neighbours(), ref["in_nb"])
    if "in_w" in ref:
        assert np.array_equal(g.in_weights(), ref["in_w"])


@pytest.mark.parametrize("flags", [0, 2, 1])
def test_from_edges_matches_numpy(ag, flags):
    rng = np.random.default_rng(11)
    n, e = 300, 5000
    src = rng.integers(0, n, e)
    dst = rng.integers(0, n, e)
    src[:40] = dst[:40]  # self loops
    src[40:80], dst[40:80] = src[80:120], dst[80:120]  # duplicates
    w = rng.random(e).astype(np.float32)
    g = ag.Graph.from_edges(n, src, dst, w, flags=flags)
    ref = numpy_csr(n, src, dst, w, dedupe=bool(flags & 1), sort=bool(flags & 2))
    assert g.num_edges == len(ref["out_src"])
    assert_graph_equals(g, ref)


def test_rtl_fixtures_build(ag, rtl):
    for fx in rtl["fixtures"]:
        g = ag.Graph.from_edges(fx["num_vertices"], fx["src"], fx["dst"], fx["weight"] or None, flags=0)
        ref = numpy_csr(fx["num_vertices"], fx["src"], fx["dst"], fx["weight"] or None)
        assert_graph_equals(g, ref)
        assert list(g.in_degree()) == [len(r) for r in fx["inverse_neighbours"]]
        # same multiset of in-neighbours per row as the testbench derivation
        off = g.in_offsets()
        nb = g.in_neighbours()
        for v, row in enumerate(fx["inverse_neighbours"]):
            assert sorted(nb[off[v]:off[v + 1]].tolist()) == sorted(row)


def test_graphbrew_edge_file(ag, rtl, tmp_path):
    gb = rtl["graphbrew"]
    raw = np.stack([np.array(gb["src"], np.uint32), np.array(gb["dst"], np.uint32)], 1)
    assert raw.nbytes == 152  # 04_test_graphs/TEST/graphbrew/graph.bin
    p = tmp_path / "graph.bin"
    raw.tofile(p)
    g = ag.Graph.read_edge_file(p, flags=1)
    n = int(raw.max()) + 1
    assert g.num_vertices == n == 13
    ref = numpy_csr(n, raw[:, 0], raw[:, 1], dedupe=True)
    assert_graph_equals(g, ref)


def test_rmat_properties(ag):
    g = ag.Graph.rmat(12, 16)
    g2 = ag.Graph.rmat(12, 16)
    assert g.num_vertices == 4096
    assert g.num_edges == g2.num_edges and np.array_equal(g.in_neighbours(), g2.in_neighbours())
    src, dst = g.out_sources(), g.out_neighbours()
    assert np.all(src != dst)
    key = src.astype(np.int64) * 4096 + dst
    assert np.all(np.diff(key) > 0)  # sorted, no duplicates
    # skew: a = 0.57 puts most edges on low ids
    assert g.out_degree()[:64].sum() > 10 * g.out_degree()[-64:].sum()
    g3 = ag.Graph.rmat(12, 16, seed=1)
    assert not np.array_equal(g3.in_neighbours()[:1000], g.in_neighbours()[:1000])


def test_er_properties(ag):
    g = ag.Graph.er(1 << 12, 16)
    assert g.num_vertices == 4096
    assert 0.95 * 16 * 4096 < g.num_edges <= 16 * 4096
    deg = g.in_degree()
    assert deg.max() < 60


def test_weights_follow_edges(ag):
    g = ag.Graph.rmat(8, 8, flags=ag.AG_BUILD_DEDUPE | ag.AG_BUILD_WEIGHTS)
    w = g.in_weights()
    assert w is not None and np.all((w >= 0) & (w < 1))
    # the inverse weight of (u -> v) equals the forward weight of (u -> v)
    fw = {(int(s), int(d)): x for s, d, x in zip(g.out_sources(), g.out_neighbours(),
                                                  np.ctypeslib.as_array(
                                                      g.g.sorted_edges_array.contents.edges_array_weight,
                                                      shape=(g.num_edges,)))}
    for v, u, x in zip(g.in_owners()[:500], g.in_neighbours()[:500], w[:500]):
        assert fw[(int(u), int(v))] == x


def test_invalid_edges_rejected(ag):
    with pytest.raises(ag.AGError):
        ag.Graph.from_edges(4, [0, 5], [1, 2])


def test_empty_graph(ag):
    g = ag.Graph.from_edges(0, [], [])
    assert g.num_vertices == 0 and g.num_edges == 0
    g = ag.Graph.from_edges(5, [], [])
    assert g.num_edges == 0 and np.all(g.in_degree() == 0)
