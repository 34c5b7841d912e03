"""Pin the CPU oracle against the reference's own golden vectors.

The reference stores no end-to-end PageRank or SpMV outputs; what it pins is
the per-vertex gather arithmetic of its RTL testbench (stream-order binary32
sums, pagerank_kernel_tb.sv:303-314, spmv_kernel_tb.sv:349-359) on 13 hand
authored fixtures (graph_fixture_pkg.sv:37-107).  Every testbench run must be
reproduced bit for bit by the oracle's gather / SpMV restatement.
"""
import numpy as np
import pytest

from conftest import f32_from_hex, fixture_csr, hex_of, run_inputs


def _check_rows(run, y):
    for row in run["rows"]:
        got = hex_of(y[row["v"]])
        want = row["golden"]
        # -0.0 and +0.0 compare equal: the oracle accumulates from 0.0f as the
        # reference's C loop does, the accelerator restarts on the first value
        if got != want:
            assert np.float32(y[row["v"]]) == f32_from_hex(want), (run["fixture"], run["class"], row["v"], got, want)


def test_fixture_registry_shape(rtl):
    assert len(rtl["fixtures"]) == 13
    names = [f["name"] for f in rtl["fixtures"]]
    assert names[0] == "FX_EMPTY" and names[-1] == "FX_SINK"
    for fx in rtl["fixtures"]:
        n, deg, idx, nb, w, od = fixture_csr(fx)
        assert int(deg.sum()) == len(fx["src"]) == int(od.sum())


@pytest.mark.parametrize("i", range(13))
def test_oracle_pagerank_gather_matches_rtl_golden(rtl, oracle, i):
    run = rtl["pagerank_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, w, od, x, pos = run_inputs(run, fx, weighted=False)
    if n == 0:
        return
    with np.errstate(over="ignore"):
        y = oracle.spmv_pull(idx, deg, nb, w, x) if pos else oracle.gather(idx, deg, nb, x)
    _check_rows(run, y)
    # vertices with no in-edge are never written and stay zero
    for v in range(n):
        if deg[v] == 0:
            assert y[v] == 0.0


@pytest.mark.parametrize("i", range(14))
def test_oracle_spmv_matches_rtl_golden(rtl, oracle, i):
    run = rtl["spmv_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, w, od, x, pos = run_inputs(run, fx, weighted=True)
    if n == 0:
        return
    with np.errstate(over="ignore"):
        y = oracle.spmv_pull(idx, deg, nb, w, x)
    _check_rows(run, y)


def test_oracle_fp_exception_rows(rtl, oracle):
    for case in rtl["fp_exception_rows"]:
        vals = np.array([f32_from_hex(h) for h in case["values"]], np.float32)
        # one vertex whose two in-edges come from vertices 1 and 2
        x = np.array([0.0, vals[0], vals[1]], np.float32)
        with np.errstate(over="ignore"):
            y = oracle.gather(np.array([0, 2, 2], np.uint32), np.array([2, 0, 0], np.uint32),
                              np.array([1, 2], np.uint32), x)
        assert np.float32(y[0]) == f32_from_hex(case["golden"])


def test_oracle_pagerank_matches_python_restatement(oracle):
    """The C oracle's full loop equals a literal Python transcription of
    pageRank.c:1021-1085 on a small graph (binary32 via numpy scalars)."""
    rng = np.random.default_rng(7)
    n, e = 40, 160
    src = rng.integers(0, n, e).astype(np.uint32)
    dst = rng.integers(0, n, e).astype(np.uint32)
    order = np.lexsort((src, dst))
    src, dst = src[order], dst[order]
    in_deg = np.bincount(dst, minlength=n).astype(np.uint32)
    in_idx = np.concatenate([[0], np.cumsum(in_deg)[:-1]]).astype(np.uint32)
    out_deg = np.bincount(src, minlength=n).astype(np.uint32)
    res = oracle.pagerank_pull(in_idx, in_deg, src, out_deg, iterations=30, epsilon=1e-6, threads=1)

    f = np.float32
    damp, base = f(0.85), f(f(1.0) - f(0.85))
    pr = [base] * n
    it_final = 30
    for it in range(30):
        contrib = [(pr[v] / f(out_deg[v])) if out_deg[v] else f(0.0) for v in range(n)]
        nxt = []
        for v in range(n):
            s = f(0.0)
            for j in range(in_idx[v], in_idx[v] + in_deg[v]):
                s = f(s + contrib[src[j]])
            nxt.append(s)
        active = 0
        for v in range(n):
            prev = pr[v]
            new = f(base + f(damp * nxt[v]))
            pr[v] = new
            if abs(float(f(new - prev))) >= 1e-6:
                active += 1
        if active == 0:
            it_final = it
            break
    want = np.array([f(p / f(n)) for p in pr], np.float32)
    assert res["iterations"] == it_final
    assert np.array_equal(res["ranks"], want)


def test_oracle_f64_fixpoint_is_a_fixpoint(oracle):
    rng = np.random.default_rng(3)
    n, e = 200, 1500
    src = rng.integers(0, n, e).astype(np.uint32)
    dst = rng.integers(0, n, e).astype(np.uint32)
    order = np.lexsort((src, dst))
    src, dst = src[order], dst[order]
    in_deg = np.bincount(dst, minlength=n).astype(np.uint32)
    in_idx = np.concatenate([[0], np.cumsum(in_deg)[:-1]]).astype(np.uint32)
    out_deg = np.bincount(src, minlength=n).astype(np.uint32)
    r, passes = oracle.pagerank_f64(in_idx, in_deg, src, out_deg, max_iter=2000, tol=1e-15)
    assert passes < 2000
    # one more application of the map leaves it unchanged
    rr = r * n
    c = np.where(out_deg > 0, rr / np.maximum(out_deg, 1), 0.0)
    s = np.zeros(n)
    np.add.at(s, dst, c[src])
    nxt = float(np.float32(1.0) - np.float32(0.85)) + float(np.float32(0.85)) * s
    assert np.max(np.abs(nxt - rr)) < 1e-12


@pytest.mark.parametrize("i", range(13))
def test_oracle_fixed_gather_matches_rtl_golden(rtl, oracle, i):
    """FixedPoint context: exact integer sums of 64-bit contributions, wrapping
    modulo 2^64 (pagerank_kernel_tb.sv:13-16, 256-263, 312)."""
    from conftest import fixed_inputs
    run = rtl["pagerank_fixed_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, x = fixed_inputs(run, fx)
    y = oracle.gather_u64(idx, deg, nb, x)
    for row in run["rows"]:
        assert "%016x" % int(y[row["v"]]) == row["golden"], (run["fixture"], run["class"], row["v"])
    for v in range(n):
        if deg[v] == 0:
            assert y[v] == 0


@pytest.mark.parametrize("i", range(13))
def test_oracle_quant_gather_matches_rtl_golden(rtl, oracle, i):
    """Quantized context: 32-bit contributions zero-extended into exact 64-bit
    sums (pagerank_kernel_tb.sv:17-19, 256-263, 312)."""
    from conftest import fixed_inputs
    run = rtl["pagerank_quant_runs"][i]
    fx = rtl["fixtures"][run["fixture_id"]]
    n, deg, idx, nb, x = fixed_inputs(run, fx, np.uint32)
    y = oracle.gather_uint(idx, deg, nb, x)
    for row in run["rows"]:
        assert "%016x" % int(y[row["v"]]) == row["golden"], (run["fixture"], run["class"], row["v"])
    for v in range(n):
        if deg[v] == 0:
            assert y[v] == 0


@pytest.mark.parametrize("width", [8, 16, 32, 64])
def test_oracle_gather_uint_widths(oracle, width):
    """Every element width zero-extends: the same values gathered as 8-, 16-,
    32- and 64-bit elements give the same sums, and equal a numpy sum."""
    rng = np.random.default_rng(width)
    n, e = 300, 2400
    src = rng.integers(0, n, e).astype(np.uint32)
    dst = rng.integers(0, n, e).astype(np.uint32)
    order = np.lexsort((src, dst))
    src, dst = src[order], dst[order]
    deg = np.bincount(dst, minlength=n).astype(np.uint32)
    idx = np.concatenate([[0], np.cumsum(deg)[:-1]]).astype(np.uint32)
    t = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[width]
    x = rng.integers(0, np.iinfo(t).max, n, dtype=t, endpoint=True)
    y = oracle.gather_uint(idx, deg, src, x)
    want = np.zeros(n, np.uint64)
    with np.errstate(over="ignore"):
        np.add.at(want, dst, x[src].astype(np.uint64))
    assert np.array_equal(y, want)
