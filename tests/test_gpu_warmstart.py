"""Learned warm start: feature kernel, MLP forward and gradients against the
float64 CPU oracle, training on GPU PageRank results, and the gain of the
trained network over uniform starting ranks on a held-out graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np_features(g):
    """Independent numpy derivation of the eight features."""
    n = g.num_vertices
    indeg = g.in_degree().astype(np.float64)
    outdeg = g.out_degree().astype(np.float64)
    off = g.in_offsets()
    nb = g.in_neighbours()
    X = np.zeros((n, 8))
    for v in range(n):
        u = nb[off[v]:off[v + 1]]
        X[v, 0] = indeg[v]
        X[v, 1] = outdeg[v]
        if len(u):
            X[v, 2] = indeg[u].sum()
            X[v, 3] = outdeg[u].sum()
            X[v, 4] = outdeg[u].min()
            X[v, 5] = outdeg[u].max()
            X[v, 6] = np.where(outdeg[u] > 0, 1.0 / np.maximum(outdeg[u], 1), 0.0).sum()
            X[v, 7] = indeg[u].max()
    return np.log1p(X)


def test_features_match_numpy(gpu):
    ag = gpu
    from accelgraph_b200 import warmstart as ws
    g = ag.Graph.rmat(10, 8)
    dg = ag.DeviceGraph(g)
    X = ws.features(dg).cpu().numpy()
    np.testing.assert_allclose(X, _np_features(g), rtol=2e-6, atol=2e-6)


@pytest.mark.parametrize("tiles", [None, (64, 128)])
def test_features_of_split_rows_and_unaligned_output(gpu, tiles):
    """Rows of every kind the work list has (short, up to 256, up to the hub
    chunk, split into chunks), with the default tiles and with 128-edge hub
    chunks that split every row above 128 in-edges; the output written once
    16-byte aligned and once 4 bytes off."""
    import ctypes as C

    import torch

    ag = gpu
    rng = np.random.default_rng(11)
    n = 6000
    src = [rng.integers(0, n, 40000)]
    dst = [rng.integers(0, n, 40000)]
    for v, d in zip((5, 17, 300, 4001, 5999), (100, 700, 2500, 5000, 5999)):
        src.append(rng.choice(n, size=d, replace=False))
        dst.append(np.full(d, v))
    g = ag.Graph.from_edges(n, np.concatenate(src), np.concatenate(dst), flags=ag.AG_BUILD_DEDUPE)
    assert int(g.in_degree().max()) > 2048
    dg = ag.DeviceGraph(g)
    if tiles:
        dg.set_tiles(tiles[0], tiles[1])
    want = _np_features(g)
    buf = torch.empty(n * 8 + 4, dtype=torch.float32, device="cuda")
    for off in (0, 1):
        ag.check(ag.lib.ag_features(dg.h, buf.data_ptr() + 4 * off), "ag_features")
        torch.cuda.synchronize()
        X = buf[off:off + n * 8].cpu().numpy().reshape(n, 8)
        np.testing.assert_allclose(X, want, rtol=2e-6, atol=2e-6)


def test_mlp_forward_and_gradients_match_oracle(gpu):
    ag = gpu
    import torch

    from accelgraph_b200 import warmstart as ws
    from oracle import mlp as omlp
    m = ws.MLP(seed=5)
    p = m.params
    assert p.size == omlp.NPARAM
    rng = np.random.default_rng(0)
    X = rng.random((3000, 8)).astype(np.float32) * 3.0
    T = rng.normal(0.5, 1.0, 3000).astype(np.float32)
    Xd = torch.from_numpy(X).cuda()
    Td = torch.from_numpy(T).cuda()
    y = m.forward(Xd).cpu().numpy()
    y_ref, _ = omlp.forward(p, X)
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-4)
    g, loss = m.gradients(Xd, Td)
    g_ref, loss_ref = omlp.gradients(p, X, T)
    assert abs(loss - loss_ref) <= 1e-4 * max(1.0, loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    # per parameter group as well
    for a, b in ((omlp.OFF_W1, omlp.OFF_B1), (omlp.OFF_W2, omlp.OFF_B2), (omlp.OFF_W3, omlp.OFF_B3)):
        assert np.linalg.norm(g[a:b] - g_ref[a:b]) <= 1e-3 * np.linalg.norm(g_ref[a:b]) + 1e-7


def test_training_is_deterministic(gpu):
    """Two networks from the same seed, trained on the same samples, end with
    the same parameters bit for bit: the gradient's chunk sums are added in
    chunk order, not in the order the chunks finish."""
    ag = gpu
    import torch

    from accelgraph_b200 import warmstart as ws
    rng = np.random.default_rng(4)
    X = torch.from_numpy(rng.normal(size=(20_000, 8)).astype(np.float32)).cuda()
    T = torch.from_numpy(rng.normal(size=20_000).astype(np.float32)).cuda()
    params = []
    for _ in range(2):
        m = ws.MLP(seed=3)
        m.train(X, T, epochs=2, batch=4096, lr=2e-3)
        params.append(m.params.view(np.uint32))
        m.release()
    assert np.array_equal(params[0], params[1])


def test_tensor_core_prediction_matches_forward(gpu):
    """The warm start's prediction (mma.sync with bfloat16 head and tail of
    every feature and activation, binary32 accumulation) agrees with the
    binary32-activation forward pass that training and the oracle use to 1e-3
    relative, for sample counts that are not multiples of the 16-row tile."""
    ag = gpu
    import torch

    from accelgraph_b200 import warmstart as ws
    m = ws.MLP(seed=7)
    rng = np.random.default_rng(2)
    for n in (1, 15, 16, 17, 1000, 40_003):
        X = torch.from_numpy((rng.random((n, 8)) * 6.0).astype(np.float32)).cuda()
        y = m.forward(X).cpu().numpy()
        yp = m.predict(X).cpu().numpy()
        assert np.all(np.isfinite(yp))
        assert np.max(np.abs(yp - y) / np.maximum(1.0, np.abs(y))) <= 1e-3, n


def test_training_reduces_loss_and_warm_start_gains(gpu, oracle):
    """Train on GPU PageRank results of small seeded graphs; on a held-out
    graph the warm start needs fewer passes than uniform starting ranks and
    still meets the same epsilon and accuracy."""
    ag = gpu
    from accelgraph_b200 import warmstart as ws
    specs = ws.training_graph_specs(count=24, scales=(10, 12), seed=11)
    X, T = ws.build_training_set(specs, per_graph=2048)
    m = ws.MLP(seed=3)
    _, loss0 = m.gradients(X, T)
    loss = m.train(X, T, epochs=40, batch=2048, lr=3e-3)
    assert loss < 0.5 * loss0
    g = ag.Graph.rmat(13, 16, seed=999)
    dg = ag.DeviceGraph(g)
    cmp = ws.compare(dg, m, iterations=300, epsilon=1e-6)
    assert cmp["warm"]["passes"] < cmp["uniform"]["passes"]
    r64, _ = dg.pagerank_f64(3000, 1e-14)
    e_u = np.abs(cmp["ranks_uniform"] - r64).sum() / r64.sum()
    e_w = np.abs(cmp["ranks_warm"] - r64).sum() / r64.sum()
    assert e_w <= max(2 * e_u, 1e-6)
