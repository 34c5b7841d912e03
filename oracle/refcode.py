"""ctypes binding of the reference's own pull calls, compiled here
(oracle/_ref/libref_pagerank.so; TEST INFRASTRUCTURE ONLY).

`make -C oracle ref` compiles the reference's unmodified
02_capi_graph/src/algorithms/capi/pageRank.c and SPMV.c against stand-ins
for the absent OpenGraph and libcxl headers (oracle/refstubs/) and links
them with a CPU emulation of the accelerator's pull gather
(oracle/refstubs/afu_emulator.c).  pageRankPullGraphCSR and SPMVPullGraphCSR
then run the reference's own host code: its starting ranks, contribution
loop, update, residual, stop test, normalisation, SpMV input vector and
checksum, with the gather done by the emulation (stream-order binary32 sums,
the compute units' semantics).  The library is built where the reference
source is present; elsewhere `available()` is False and the tests that use
it skip.  The GraphCSR and Arguments structures are the ones the reference
headers declare, which this repository's include/ mirrors field for field.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_pagerank.so"
# the reference checkout: $AG_REFERENCE, else `reference` beside this checkout
REF_ROOT = Path(os.environ.get("AG_REFERENCE") or Path(__file__).resolve().parent.parent.parent / "reference")
REF_SOURCE = REF_ROOT / "02_capi_graph/src/algorithms/capi/pageRank.c"


class _PageRankStats(C.Structure):
    _fields_ = [("damp", C.c_float), ("base_pr", C.c_float), ("iterations", C.c_uint32),
                ("num_vertices", C.c_uint32), ("activeVertices", C.c_uint32),
                ("realRanks", C.POINTER(C.c_uint32)), ("pageRanks", C.POINTER(C.c_float)),
                ("time_total", C.c_double), ("error_total", C.c_double)]


class _SPMVStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("arguments", C.c_void_p), ("num_vertices", C.c_uint32),
                ("vector_output", C.POINTER(C.c_float)), ("vector_input", C.POINTER(C.c_float)),
                ("time_total", C.c_double)]


def build() -> bool:
    """Compile the library when the reference source is present and the
    library is missing or older than its recipe; True when it exists."""
    if REF_SOURCE.exists():
        deps = [HERE / "Makefile", HERE / "refstubs" / "afu_emulator.c", HERE / "refstubs" / "exports.map",
                *sorted((HERE / "refstubs").glob("*.h"))]
        if not LIB.exists() or LIB.stat().st_mtime < max(p.stat().st_mtime for p in deps):
            subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)
    return LIB.exists()


_lib = None


def available() -> bool:
    return _load() is not None


def _load():
    global _lib
    if _lib is None and build():
        lib = C.CDLL(str(LIB))
        lib.pageRankPullGraphCSR.restype = C.POINTER(_PageRankStats)
        lib.pageRankPullGraphCSR.argtypes = [C.c_void_p, C.c_void_p]
        lib.pageRankDataDrivenPullGraphCSR.restype = C.POINTER(_PageRankStats)
        lib.pageRankDataDrivenPullGraphCSR.argtypes = [C.c_void_p, C.c_void_p]
        lib.pageRankPullFixedPoint64BitGraphCSR.restype = C.POINTER(_PageRankStats)
        lib.pageRankPullFixedPoint64BitGraphCSR.argtypes = [C.c_void_p, C.c_void_p]
        for name in list(_NARROW.values()) + list(_PUSH.values()) + list(_RESIDUAL.values()):
            getattr(lib, name).restype = C.POINTER(_PageRankStats)
            getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p]
        lib.freePageRankStats.argtypes = [C.POINTER(_PageRankStats)]
        lib.SPMVPullGraphCSR.restype = C.POINTER(_SPMVStats)
        lib.SPMVPullGraphCSR.argtypes = [C.c_void_p, C.c_void_p]
        lib.freeSPMVStats.argtypes = [C.POINTER(_SPMVStats)]
        lib.refemu_set_kernel.argtypes = [C.c_int]
        lib.refemu_gathers.restype = C.c_uint64
        _lib = lib
    return _lib


def pagerank_pull(arguments_ptr, graph_ptr, num_vertices: int):
    """Run the reference's pageRankPullGraphCSR on a GraphCSR (pointer) with
    a struct Arguments (pointer).  Returns ranks (normalised, float32),
    iterations (the reference's stats->iterations), error_total, and the
    number of gathers the emulated accelerator ran."""
    import numpy as np
    lib = _load()
    lib.refemu_set_kernel(0)
    g0 = lib.refemu_gathers()
    st = lib.pageRankPullGraphCSR(C.cast(arguments_ptr, C.c_void_p), C.cast(graph_ptr, C.c_void_p))
    try:
        s = st.contents
        ranks = np.ctypeslib.as_array(s.pageRanks, shape=(num_vertices,)).copy() if num_vertices else \
            np.zeros(0, np.float32)
        out = {"ranks": ranks, "iterations": int(s.iterations), "error_total": float(s.error_total),
               "gathers": int(lib.refemu_gathers() - g0), "damp": float(s.damp), "base_pr": float(s.base_pr)}
    finally:
        lib.freePageRankStats(st)
    return out


def pagerank_dd(arguments_ptr, graph_ptr, num_vertices: int):
    """Run the reference's pageRankDataDrivenPullGraphCSR (its CPU worklist
    pull, pageRank.c:2810-2969, no accelerator involved)."""
    import numpy as np
    lib = _load()
    st = lib.pageRankDataDrivenPullGraphCSR(C.cast(arguments_ptr, C.c_void_p), C.cast(graph_ptr, C.c_void_p))
    try:
        s = st.contents
        ranks = np.ctypeslib.as_array(s.pageRanks, shape=(num_vertices,)).copy() if num_vertices else \
            np.zeros(0, np.float32)
        out = {"ranks": ranks, "iterations": int(s.iterations), "error_total": float(s.error_total)}
    finally:
        lib.freePageRankStats(st)
    return out


def pagerank_fixed64(arguments_ptr, graph_ptr, num_vertices: int):
    """Run the reference's pageRankPullFixedPoint64BitGraphCSR (pushpull 2,
    pageRank.c:1276-1453) with the emulated fixed-point gather and the
    stand-in conversions of oracle/refstubs/fixedPoint.h."""
    import numpy as np
    lib = _load()
    lib.refemu_set_kernel(2)
    g0 = lib.refemu_gathers()
    st = lib.pageRankPullFixedPoint64BitGraphCSR(C.cast(arguments_ptr, C.c_void_p), C.cast(graph_ptr, C.c_void_p))
    try:
        s = st.contents
        ranks = np.ctypeslib.as_array(s.pageRanks, shape=(num_vertices,)).copy() if num_vertices else \
            np.zeros(0, np.float32)
        out = {"ranks": ranks, "iterations": int(s.iterations), "error_total": float(s.error_total),
               "gathers": int(lib.refemu_gathers() - g0)}
    finally:
        lib.freePageRankStats(st)
    return out


_NARROW = {(False, 32): "pageRankPullFixedPoint32BitGraphCSR", (False, 16): "pageRankPullFixedPoint16BitGraphCSR",
           (False, 8): "pageRankPullFixedPoint8BitGraphCSR", (True, 32): "pageRankPullQuant32BitGraphCSR",
           (True, 16): "pageRankPullQuant16BitGraphCSR", (True, 8): "pageRankPullQuant8BitGraphCSR"}


def pagerank_narrow(quant: bool, width: int, arguments_ptr, graph_ptr, num_vertices: int):
    """Run one of the reference's narrow integer pulls: the W-bit fixed-point
    forms (pushpull 9, 10, 11; pageRank.c:1455-1991) or the W-bit quantised
    forms (pushpull 4, 12, 13; pageRank.c:2119-2677), with the emulated
    zero-extending integer gather and the stand-in conversions of
    oracle/refstubs/fixedPoint.h and quantization.h."""
    import numpy as np
    lib = _load()
    lib.refemu_set_kernel({32: 3, 16: 4, 8: 5}[width])
    g0 = lib.refemu_gathers()
    st = getattr(lib, _NARROW[(bool(quant), width)])(C.cast(arguments_ptr, C.c_void_p), C.cast(graph_ptr, C.c_void_p))
    try:
        s = st.contents
        ranks = np.ctypeslib.as_array(s.pageRanks, shape=(num_vertices,)).copy() if num_vertices else \
            np.zeros(0, np.float32)
        out = {"ranks": ranks, "iterations": int(s.iterations), "error_total": float(s.error_total),
               "gathers": int(lib.refemu_gathers() - g0)}
    finally:
        lib.freePageRankStats(st)
    return out


_PUSH = {0: "pageRankPushGraphCSR", 1: "pageRankPushFixedPointGraphCSR", 2: "pageRankPushQuantGraphCSR"}
_RESIDUAL = {False: "pageRankDataDrivenPushGraphCSR", True: "pageRankDataDrivenPullPushGraphCSR"}


def _single_thread(fn):
    """Run fn with OpenMP limited to one thread: the push forms' adds (and
    the residual forms' in-place updates) then happen in vertex order, the
    instance the oracle restates.  The caller also sets
    arguments->ker_numThreads = 1 for the loops that take it."""
    gomp = C.CDLL("libgomp.so.1")
    prev = gomp.omp_get_max_threads()
    gomp.omp_set_num_threads(1)
    try:
        return fn()
    finally:
        gomp.omp_set_num_threads(prev)


def _stats_out(lib, st, num_vertices, g0):
    import numpy as np
    try:
        s = st.contents
        ranks = np.ctypeslib.as_array(s.pageRanks, shape=(num_vertices,)).copy() if num_vertices else \
            np.zeros(0, np.float32)
        return {"ranks": ranks, "iterations": int(s.iterations), "error_total": float(s.error_total),
                "gathers": int(lib.refemu_gathers() - g0)}
    finally:
        lib.freePageRankStats(st)


def pagerank_push(kind: int, arguments_ptr, graph_ptr, num_vertices: int):
    """Run one of the reference's push forms on one thread: kind 0
    pageRankPushGraphCSR (pushpull 1, the emulated push unit), 1
    pageRankPushFixedPointGraphCSR (pushpull 3), 2 pageRankPushQuantGraphCSR
    (pushpull 5, stand-in quantiser with zero point 0).  arguments must carry
    ker_numThreads = 1."""
    lib = _load()
    lib.refemu_set_kernel(6)
    g0 = lib.refemu_gathers()
    st = _single_thread(lambda: getattr(lib, _PUSH[kind])(C.cast(arguments_ptr, C.c_void_p),
                                                         C.cast(graph_ptr, C.c_void_p)))
    return _stats_out(lib, st, num_vertices, g0)


def pagerank_residual(pull_push: bool, arguments_ptr, graph_ptr, num_vertices: int):
    """Run the reference's data-driven push (pushpull 7) or pull-push
    (pushpull 8) on one thread (arguments must carry ker_numThreads = 1)."""
    lib = _load()
    g0 = lib.refemu_gathers()
    st = _single_thread(lambda: getattr(lib, _RESIDUAL[bool(pull_push)])(C.cast(arguments_ptr, C.c_void_p),
                                                                        C.cast(graph_ptr, C.c_void_p)))
    return _stats_out(lib, st, num_vertices, g0)


def spmv_pull(arguments_ptr, graph_ptr, num_vertices: int):
    """Run the reference's SPMVPullGraphCSR: returns its input vector, its
    output vector and its iteration count."""
    import numpy as np
    lib = _load()
    lib.refemu_set_kernel(1)
    st = lib.SPMVPullGraphCSR(C.cast(arguments_ptr, C.c_void_p), C.cast(graph_ptr, C.c_void_p))
    try:
        s = st.contents
        n = num_vertices
        out = {"x": np.ctypeslib.as_array(s.vector_input, shape=(n,)).copy() if n else np.zeros(0, np.float32),
               "y": np.ctypeslib.as_array(s.vector_output, shape=(n,)).copy() if n else np.zeros(0, np.float32),
               "iterations": int(s.iterations)}
    finally:
        lib.freeSPMVStats(st)
    return out
