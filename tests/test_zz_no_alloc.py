"""The SpMV entry point that allocates nothing (ag_spmv_pull_noalloc).

It serves callers that may not allocate device memory once running: every
input and output is a device buffer the caller already owns, and the only
scratch is a fixed array inside the library.  Checked through the C ABI, on
two calls in a row, against the regular SpMV entry point (ag_spmv_pull, which
plans and allocates its own buffers) and against the CPU oracle's product
(SPMV.c:1200-1224; 0.0001f per edge without weights), within the tolerance of
the other SpMV tests (1e-5 relative L1).  This file is collected last on
purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L1 = 1e-5


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def _graph(ag):
    rng = np.random.default_rng(21)
    n = 20000
    src = [rng.integers(0, n, 300000)]
    dst = [rng.integers(0, n, 300000)]
    # rows longer than the 4096-edge split, so the scratch list is used
    for v, d in zip((3, 77, 1234, 9999, 19998), (4097, 5000, 10000, 15000, 19999)):
        src.append(rng.choice(n, size=d, replace=False))
        dst.append(np.full(d, v))
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    w = rng.random(len(src)).astype(np.float32)
    return ag.Graph.from_edges(n, src, dst, w, flags=ag.AG_BUILD_DEDUPE)


def _device_csr(g, dev):
    import torch
    off = torch.from_numpy(g.in_offsets().astype(np.int64).astype(np.int32)).to(dev)
    ids = torch.from_numpy(g.in_neighbours().astype(np.int32)).to(dev)
    w = torch.from_numpy(np.ascontiguousarray(g.in_weights())).to(dev)
    return off, ids, w


@pytest.mark.parametrize("mode,weighted", [(0, True), (0, False), (1, True)])
def test_noalloc_matches_regular_entry_point_and_oracle(gpu, oracle, mode, weighted):
    ag = gpu
    import torch

    g = _graph(ag)
    n, e = g.num_vertices, g.num_edges
    assert int(g.in_degree().max()) > 4096
    x = np.random.default_rng(3).random(n).astype(np.float32)
    if mode == 1:
        ref = oracle.gather(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), x)
    else:
        ref = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(),
                               g.in_weights() if weighted else None, x)
    want = ag.DeviceGraph(g, weights=weighted).spmv(x, mode=mode)
    assert rel_l1(want, ref) <= REL_L1

    dev = torch.device("cuda", 0)
    off, ids, w = _device_csr(g, dev)
    xd = torch.from_numpy(x).to(dev)
    stream = torch.cuda.current_stream(dev)
    outs = []
    for _ in range(2):
        yd = torch.full((n,), float("nan"), dtype=torch.float32, device=dev)
        st = ag.lib.ag_spmv_pull_noalloc(n, e, off.data_ptr(), ids.data_ptr(), w.data_ptr() if weighted else None,
                                         xd.data_ptr(), yd.data_ptr(), mode, stream.cuda_stream)
        assert st == 0, ag.lib.ag_last_error()
        torch.cuda.synchronize(dev)
        outs.append(yd.cpu().numpy())
    for y in outs:
        assert np.all(np.isfinite(y))
        assert rel_l1(y, want) <= REL_L1
        assert rel_l1(y, ref) <= REL_L1
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_oversized_input_and_unknown_modes(gpu):
    """Real (small) device buffers: the checks run before any launch, and y
    is left as it was."""
    ag = gpu
    import torch

    dev = torch.device("cuda", 0)
    n = 10
    off = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    ids = torch.zeros(4, dtype=torch.int32, device=dev)
    x = torch.ones(n, dtype=torch.float32, device=dev)
    y = torch.full((n,), 7.0, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = ag.lib.ag_spmv_pull_noalloc(n, (1 << 28) + 1, off.data_ptr(), ids.data_ptr(), None, x.data_ptr(),
                                     y.data_ptr(), 0, stream)
    assert st == ag.AG_ERR_UNSUPPORTED
    assert b"exceed" in ag.lib.ag_last_error()
    st = ag.lib.ag_spmv_pull_noalloc(n, 0, off.data_ptr(), ids.data_ptr(), None, x.data_ptr(), y.data_ptr(),
                                     ag.AG_SPMV_EXACT, stream)
    assert st == ag.AG_ERR_INVALID_ARG
    torch.cuda.synchronize(dev)
    assert torch.equal(y, torch.full((n,), 7.0, dtype=torch.float32, device=dev))
