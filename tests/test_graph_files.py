"""Graph files in the reference's format codes (-z/-c: text edge list, binary
edge list, serialised CSR) and the symmetrize option (-s), on the host
substrate.  Text and binary reads build the same CSR as ag_graph_from_edges on
the same edges; a serialised CSR reads back array for array."""
import numpy as np
import pytest


def _arrays(g):
    n, e = g.num_vertices, g.num_edges
    gc = g.g
    out = {
        "out_degree": g.out_degree().copy(), "in_degree": g.in_degree().copy(),
        "out_idx": np.ctypeslib.as_array(gc.vertices.contents.edges_idx, shape=(n + 1,)).copy() if n else None,
        "in_idx": np.ctypeslib.as_array(gc.inverse_vertices.contents.edges_idx, shape=(n + 1,)).copy() if n else None,
        "out_src": g.out_sources().copy(), "out_dst": g.out_neighbours().copy(),
        "in_src": g.in_owners().copy(), "in_dst": g.in_neighbours().copy(),
    }
    el = gc.sorted_edges_array.contents
    if el.edges_array_weight:
        out["out_w"] = np.ctypeslib.as_array(el.edges_array_weight, shape=(e,)).view(np.uint32).copy()
        iel = gc.inverse_sorted_edges_array.contents
        out["in_w"] = np.ctypeslib.as_array(iel.edges_array_weight, shape=(e,)).view(np.uint32).copy()
    return out


def _same(a, b):
    assert (a.num_vertices, a.num_edges, a.g.avg_degree) == (b.num_vertices, b.num_edges, b.g.avg_degree)
    assert np.float32(a.g.max_weight) == np.float32(b.g.max_weight)
    xa, xb = _arrays(a), _arrays(b)
    assert xa.keys() == xb.keys()
    for k in xa:
        if xa[k] is None:
            assert xb[k] is None
        else:
            assert np.array_equal(xa[k], xb[k]), k


def test_graphbrew_text_and_binary(ag, rtl, tmp_path):
    """The reference's 19-edge test graph (04_test_graphs/TEST/graphbrew),
    written as a tab/space text list like its graph.org and as 8-byte
    binary records, reads back as the same graph."""
    src = np.array(rtl["graphbrew"]["src"], np.uint32)
    dst = np.array(rtl["graphbrew"]["dst"], np.uint32)
    n = int(max(src.max(), dst.max())) + 1
    txt = tmp_path / "g.txt"
    txt.write_text("# graphbrew\n" + "".join(f"{s}\t{d}\n" if i % 2 else f"{s}   {d}\r\n"
                                             for i, (s, d) in enumerate(zip(src, dst))) + "\n")
    binf = tmp_path / "g.bin"
    np.stack([src, dst], 1).astype(np.uint32).tofile(binf)
    for flags in (0, ag.AG_BUILD_DEDUPE):
        want = ag.Graph.from_edges(n, src, dst, None, flags)
        _same(ag.Graph.read(txt, ag.AG_FILE_TEXT, False, flags), want)
        _same(ag.Graph.read(binf, ag.AG_FILE_BINARY, False, flags), want)


@pytest.mark.parametrize("weighted", [False, True])
def test_write_read_round_trips(ag, tmp_path, weighted):
    g = ag.Graph.rmat(10, 8, flags=ag.AG_BUILD_DEDUPE | (ag.AG_BUILD_WEIGHTS if weighted else 0))
    src, dst = g.out_sources().copy(), g.out_neighbours().copy()
    w = None
    if weighted:
        w = np.ctypeslib.as_array(g.g.sorted_edges_array.contents.edges_array_weight, shape=(g.num_edges,)).copy()
    n = int(max(src.max(), dst.max())) + 1
    for fmt in (ag.AG_FILE_TEXT, ag.AG_FILE_BINARY):
        f = tmp_path / f"g{fmt}"
        g.write(f, fmt)
        back = ag.Graph.read(f, fmt, weighted, ag.AG_BUILD_DEDUPE)
        _same(back, ag.Graph.from_edges(n, src, dst, w, ag.AG_BUILD_DEDUPE))
    f = tmp_path / "g.agcsr"
    g.write(f, ag.AG_FILE_CSR)
    back = ag.Graph.read(f, ag.AG_FILE_CSR)
    _same(back, g)


def test_csr_file_rejects_damage(ag, tmp_path):
    g = ag.Graph.rmat(8, 8)
    f = tmp_path / "g.agcsr"
    g.write(f, ag.AG_FILE_CSR)
    raw = f.read_bytes()
    (tmp_path / "short").write_bytes(raw[:-4])
    (tmp_path / "magic").write_bytes(b"XX" + raw[2:])
    for name in ("short", "magic"):
        with pytest.raises(ag.AGError):
            ag.Graph.read(tmp_path / name, ag.AG_FILE_CSR)


def test_text_rejects_bad_lines(ag, tmp_path):
    for body in ("0 1\n2\n", "0 1 x\n", "0 -1\n", "0 1 0.5\n"):
        f = tmp_path / "bad.txt"
        f.write_text(body)
        with pytest.raises(ag.AGError):
            ag.Graph.read(f, ag.AG_FILE_TEXT, False)
    f = tmp_path / "w.txt"
    f.write_text("0 1 0.25\n1 2 2.5e-1\n")
    g = ag.Graph.read(f, ag.AG_FILE_TEXT, True)
    assert g.num_edges == 2 and np.float32(g.g.max_weight) == np.float32(0.25)


def test_symmetrize_appends_reverse_edges(ag):
    rng = np.random.default_rng(3)
    src = rng.integers(0, 300, 2000).astype(np.uint32)
    dst = rng.integers(0, 300, 2000).astype(np.uint32)
    w = rng.random(2000, dtype=np.float32)
    for flags in (0, ag.AG_BUILD_DEDUPE):
        sym = ag.Graph.from_edges(300, src, dst, w, flags | ag.AG_BUILD_SYMMETRIC)
        ref = ag.Graph.from_edges(300, np.concatenate([src, dst]), np.concatenate([dst, src]),
                                  np.concatenate([w, w]), flags)
        _same(sym, ref)
    sym = ag.Graph.from_edges(300, src, dst, None, ag.AG_BUILD_DEDUPE | ag.AG_BUILD_SYMMETRIC)
    assert np.array_equal(sym.out_degree(), sym.in_degree())
