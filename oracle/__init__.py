"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker or the timed CPU baseline.  The
product package accelgraph_b200 never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "ag_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


def _load() -> C.CDLL:
    build()
    lib = C.CDLL(str(LIB))
    lib.oracle_gather.argtypes = [C.c_uint32, u32p, u32p, u32p, f32p, f32p, C.c_int]
    lib.oracle_spmv_pull.argtypes = [C.c_uint32, u32p, u32p, u32p, f32p, f32p, f32p, C.c_int]
    lib.oracle_spmv_input.argtypes = [C.c_uint32, u32p, f32p]
    lib.oracle_spmv_checksum.argtypes = [C.c_uint32, f32p]
    lib.oracle_spmv_checksum.restype = C.c_double
    lib.oracle_pagerank_pull.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, C.c_double, f32p, f32p,
                                         u32p, f64p, f64p, u32p, f64p, f64p, C.c_int]
    lib.oracle_pagerank_pull.restype = C.c_uint32
    u64p = C.POINTER(C.c_uint64)
    lib.oracle_gather_u64.argtypes = [C.c_uint32, u32p, u32p, u32p, u64p, u64p, C.c_int]
    lib.oracle_pagerank_fixed64.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, C.c_double, f32p,
                                            u32p, f64p, u32p, C.c_int]
    lib.oracle_pagerank_fixed64.restype = C.c_uint32
    lib.oracle_gather_uint.argtypes = [C.c_uint32, u32p, u32p, u32p, C.c_void_p, C.c_uint32, u64p, C.c_int]
    lib.oracle_pagerank_narrow.argtypes = [C.c_int, C.c_int, C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32,
                                           C.c_double, f32p, u32p, f64p, u32p, C.c_int]
    lib.oracle_pagerank_narrow.restype = C.c_uint32
    lib.oracle_pagerank_push.argtypes = [C.c_int, C.c_uint32, u32p, u32p, u32p, C.c_uint32, C.c_double, f32p, u32p,
                                         f64p, u32p]
    lib.oracle_pagerank_push.restype = C.c_uint32
    lib.oracle_pagerank_residual.argtypes = [C.c_int, C.c_uint32, u32p, u32p, u32p, u32p, u32p, u32p, C.c_uint32,
                                             C.c_double, f32p, u32p, f64p, u32p]
    lib.oracle_pagerank_residual.restype = C.c_uint32
    lib.oracle_pagerank_dd.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, u32p, u32p, C.c_uint32, C.c_double,
                                       f32p, u32p, f64p, u32p, C.c_int]
    lib.oracle_pagerank_dd.restype = C.c_uint32
    lib.oracle_pagerank_f64.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, C.c_double, f64p, C.c_int]
    lib.oracle_pagerank_f64.restype = C.c_uint32
    lib.oracle_ppr.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, C.c_double, f32p,
                               u32p, C.c_int]
    lib.oracle_ppr.restype = C.c_uint32
    lib.oracle_max_threads.restype = C.c_int
    lib.oracle_rmat_inverse.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                        u32p, u32p, u32p, u32p]
    lib.oracle_rmat_inverse.restype = C.c_uint64
    lib.oracle_partition_pass.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p, u32p, f32p, f32p, f32p,
                                          C.c_double, f64p]
    return lib


lib = _load()


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _csr(in_idx, in_deg, in_nb):
    return (np.ascontiguousarray(in_idx, np.uint32), np.ascontiguousarray(in_deg, np.uint32),
            np.ascontiguousarray(in_nb, np.uint32))


def rmat_inverse(scale, edge_factor, seed, a=0.57, b=0.19, c=0.19):
    """Seeded R-MAT graph (self loops and duplicates dropped) as the arrays
    the pull oracle reads: dict(in_idx, in_deg, in_nb, out_deg, num_edges)."""
    n = 1 << scale
    m = edge_factor * n
    in_idx = np.zeros(n + 1, np.uint32)
    in_deg = np.zeros(n, np.uint32)
    in_nb = np.zeros(max(m, 1), np.uint32)
    out_deg = np.zeros(n, np.uint32)
    e = lib.oracle_rmat_inverse(scale, edge_factor, a, b, c, seed, _p(in_idx, u32p), _p(in_deg, u32p),
                                _p(in_nb, u32p), _p(out_deg, u32p))
    if e == 2 ** 64 - 1:
        raise MemoryError("oracle_rmat_inverse: allocation failed")
    return {"in_idx": in_idx, "in_deg": in_deg, "in_nb": in_nb[:e], "out_deg": out_deg, "num_edges": int(e)}


def partition_pass(rb, re, in_idx, in_deg, in_nb, out_deg, pos, c_in_full, c_out_full, rank_local, eps):
    """One pull pass over rows [rb, re) of a row partition (contribution of u
    at pos[u]); updates rank_local and the rows' entries of c_out_full in
    place; returns [active rows, sum of |r' - r|]."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    pos = np.ascontiguousarray(pos, np.uint32)
    for a in (c_in_full, c_out_full, rank_local):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    stats = np.zeros(2, np.float64)
    lib.oracle_partition_pass(rb, re, _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(out_deg, u32p),
                              _p(pos, u32p), _p(c_in_full, f32p), _p(c_out_full, f32p), _p(rank_local, f32p), eps,
                              _p(stats, f64p))
    return stats


def gather(in_idx, in_deg, in_nb, x, threads=0):
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros(len(in_deg), np.float32)
    lib.oracle_gather(len(in_deg), _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(x, f32p),
                      _p(y, f32p), threads)
    return y


def spmv_pull(in_idx, in_deg, in_nb, w, x, threads=0):
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    x = np.ascontiguousarray(x, np.float32)
    w = None if w is None else np.ascontiguousarray(w, np.float32)
    y = np.zeros(len(in_deg), np.float32)
    lib.oracle_spmv_pull(len(in_deg), _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(w, f32p),
                         _p(x, f32p), _p(y, f32p), threads)
    return y


def spmv_input(out_deg):
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    x = np.zeros(len(out_deg), np.float32)
    lib.oracle_spmv_input(len(out_deg), _p(out_deg, u32p), _p(x, f32p))
    return x


def spmv_checksum(y):
    y = np.ascontiguousarray(y, np.float32)
    return lib.oracle_spmv_checksum(len(y), _p(y, f32p))


def pagerank_pull(in_idx, in_deg, in_nb, out_deg, iterations=20, epsilon=1e-4, init=None, threads=0):
    """Returns dict(ranks, iterations, passes, error_total, rank_sum, active, error, seconds)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    n = len(in_deg)
    init = None if init is None else np.ascontiguousarray(init, np.float32)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    rs = C.c_double()
    cap = max(iterations, 1)
    ha = np.zeros(cap, np.uint32)
    he = np.zeros(cap, np.float64)
    hs = np.zeros(cap, np.float64)
    passes = lib.oracle_pagerank_pull(n, _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(out_deg, u32p),
                                      iterations, epsilon, _p(init, f32p), _p(ranks, f32p), C.byref(it),
                                      C.byref(et), C.byref(rs), _p(ha, u32p), _p(he, f64p), _p(hs, f64p), threads)
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "rank_sum": rs.value, "active": ha[:passes], "error": he[:passes], "seconds": hs[:passes]}


def gather_u64(in_idx, in_deg, in_nb, x, threads=0):
    """Fixed-point gather: integer sums modulo 2^64 (rows without in-edges 0)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    x = np.ascontiguousarray(x, np.uint64)
    y = np.zeros(len(in_deg), np.uint64)
    u64p = C.POINTER(C.c_uint64)
    lib.oracle_gather_u64(len(in_deg), _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(x, u64p),
                          _p(y, u64p), threads)
    return y


def pagerank_fixed64(in_idx, in_deg, in_nb, out_deg, iterations=20, epsilon=1e-4, threads=0):
    """64-bit fixed-point pull (pageRank.c:1276-1453). Returns dict(ranks,
    iterations, passes, error_total, active)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    n = len(in_deg)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    ha = np.zeros(max(iterations, 1), np.uint32)
    passes = lib.oracle_pagerank_fixed64(n, _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(out_deg, u32p),
                                         iterations, epsilon, _p(ranks, f32p), C.byref(it), C.byref(et),
                                         _p(ha, u32p), threads)
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "active": ha[:passes]}


_UINT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def gather_uint(in_idx, in_deg, in_nb, x, threads=0):
    """Integer gather of 8/16/32/64-bit elements (the dtype of x) zero-extended
    into 64-bit sums modulo 2^64 (rows without in-edges 0)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    x = np.ascontiguousarray(x)
    if x.dtype not in [np.dtype(t) for t in _UINT.values()]:
        raise TypeError("gather_uint: x must be uint8, uint16, uint32 or uint64")
    y = np.zeros(len(in_deg), np.uint64)
    lib.oracle_gather_uint(len(in_deg), _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p),
                           x.ctypes.data_as(C.c_void_p), x.dtype.itemsize, _p(y, C.POINTER(C.c_uint64)), threads)
    return y


def pagerank_narrow(quant, width, in_idx, in_deg, in_nb, out_deg, iterations=20, epsilon=1e-4, threads=0):
    """Narrow integer pulls: quant=False the W-bit fixed-point forms
    (pageRank.c:1455-1991), quant=True the W-bit quantised forms
    (pageRank.c:2119-2677), width 32, 16 or 8.  Returns dict(ranks,
    iterations, passes, error_total, active)."""
    if width not in (8, 16, 32):
        raise ValueError("width must be 8, 16 or 32")
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    n = len(in_deg)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    ha = np.zeros(max(iterations, 1), np.uint32)
    passes = lib.oracle_pagerank_narrow(1 if quant else 0, width, n, _p(in_idx, u32p), _p(in_deg, u32p),
                                        _p(in_nb, u32p), _p(out_deg, u32p), iterations, epsilon, _p(ranks, f32p),
                                        C.byref(it), C.byref(et), _p(ha, u32p), threads)
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "active": ha[:passes]}


PUSH_FLOAT, PUSH_FIXED64, PUSH_QUANT32 = 0, 1, 2


def pagerank_push(kind, out_idx, out_deg, out_nb, iterations=20, epsilon=1e-4):
    """Push forms, single-thread instance (sources in vertex order): kind
    PUSH_FLOAT (pushpull 1, pageRank.c:1111-1272), PUSH_FIXED64 (pushpull 3,
    :1992-2118) or PUSH_QUANT32 (pushpull 5, :2678-2809).  Returns
    dict(ranks, iterations, passes, error_total, active)."""
    out_idx, out_deg, out_nb = _csr(out_idx, out_deg, out_nb)
    n = len(out_deg)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    ha = np.zeros(max(iterations, 1), np.uint32)
    passes = lib.oracle_pagerank_push(kind, n, _p(out_idx, u32p), _p(out_deg, u32p), _p(out_nb, u32p), iterations,
                                      epsilon, _p(ranks, f32p), C.byref(it), C.byref(et), _p(ha, u32p))
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "active": ha[:passes]}


def pagerank_residual(pull_push, in_idx, in_deg, in_nb, out_idx, out_deg, out_nb, iterations=20, epsilon=1e-4):
    """Residual forms with a worklist, single-thread instance: pull_push=False
    the data-driven push (pushpull 7, pageRank.c:2971-3127), True the
    data-driven pull-push (pushpull 8, :3128-3325).  Returns dict(ranks,
    iterations, passes, error_total, active) (active: activations per
    iteration)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_idx, out_deg, out_nb = _csr(out_idx, out_deg, out_nb)
    n = len(in_deg)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    ha = np.zeros(max(iterations, 1), np.uint32)
    passes = lib.oracle_pagerank_residual(1 if pull_push else 0, n, _p(in_idx, u32p), _p(in_deg, u32p),
                                          _p(in_nb, u32p), _p(out_idx, u32p), _p(out_deg, u32p), _p(out_nb, u32p),
                                          iterations, epsilon, _p(ranks, f32p), C.byref(it), C.byref(et),
                                          _p(ha, u32p))
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "active": ha[:passes]}


def pagerank_dd(in_idx, in_deg, in_nb, out_idx, out_deg, out_nb, iterations=20, epsilon=1e-4, threads=0):
    """Data-driven pull (pageRank.c:2810-2969). Returns dict(ranks,
    iterations, passes, error_total, active)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_idx, out_deg, out_nb = _csr(out_idx, out_deg, out_nb)
    n = len(in_deg)
    ranks = np.zeros(n, np.float32)
    it = C.c_uint32()
    et = C.c_double()
    ha = np.zeros(max(iterations, 1), np.uint32)
    passes = lib.oracle_pagerank_dd(n, _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(out_idx, u32p),
                                    _p(out_deg, u32p), _p(out_nb, u32p), iterations, epsilon, _p(ranks, f32p),
                                    C.byref(it), C.byref(et), _p(ha, u32p), threads)
    return {"ranks": ranks, "iterations": it.value, "passes": passes, "error_total": et.value,
            "active": ha[:passes]}


def pagerank_f64(in_idx, in_deg, in_nb, out_deg, max_iter=1000, tol=1e-13, threads=0):
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    r = np.zeros(len(in_deg), np.float64)
    passes = lib.oracle_pagerank_f64(len(in_deg), _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p),
                                     _p(out_deg, u32p), max_iter, tol, _p(r, f64p), threads)
    return r, passes


def ppr(in_idx, in_deg, in_nb, out_deg, sources, iterations=100, epsilon=1e-6, threads=0):
    """Returns (ranks n x k, iterations, passes)."""
    in_idx, in_deg, in_nb = _csr(in_idx, in_deg, in_nb)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    src = np.ascontiguousarray(sources, np.uint32)
    n, k = len(in_deg), len(src)
    r = np.zeros((n, k), np.float32)
    it = C.c_uint32()
    passes = lib.oracle_ppr(n, _p(in_idx, u32p), _p(in_deg, u32p), _p(in_nb, u32p), _p(out_deg, u32p), k,
                            _p(src, u32p), iterations, epsilon, r.ctypes.data_as(f32p), C.byref(it), threads)
    return r, it.value, passes


def max_threads() -> int:
    return lib.oracle_max_threads()
