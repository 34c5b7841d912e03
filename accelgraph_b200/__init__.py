"""accelgraph_b200 -- B200 (sm_100a) pull PageRank / SpMV over inverse CSR.

Python mirror of the C ABI in include/*.h.  The compute path is
libaccelgraph_b200.so (hand-written CUDA for sm_100a behind a C ABI); this
module only binds it with ctypes and offers numpy conveniences.  Importing it
fails loudly when the library has not been built: there is no CPU fallback.

Summation order: the reference entry points and ag_pr_opts_init (the C
defaults) use EXACT order, the reference loop's bits.  The numpy conveniences
here (DeviceGraph.launch / pagerank, MultiGraph.pagerank, make_opts) default
to FAST order, the faster tree sums for rows over 32 in-edges; pass
order=AG_ORDER_EXACT for the reference's bits.

Reference interface mirrored (AccelGraph, 02_capi_graph):
  struct Arguments            include/config/graphConfig.h:11-52
  struct PageRankStats        include/algorithms/capi/pageRank.h:19-30
  struct SPMVStats            include/algorithms/capi/SPMV.h:19-28
  pageRankGraphCSR / pageRankPullGraphCSR   pageRank.h:69-70
  pageRank<form>GraphCSR (13 forms)         pageRank.h:71-86
  SPMVGraphCSR / SPMVPullGraphCSR           SPMV.h:51-52
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libaccelgraph_b200.so"

u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)


class Vertex(C.Structure):
    _fields_ = [("out_degree", u32p), ("in_degree", u32p), ("edges_idx", u32p)]


class EdgeList(C.Structure):
    _fields_ = [
        ("num_edges", C.c_uint32),
        ("num_vertices", C.c_uint32),
        ("avg_degree", C.c_uint32),
        ("max_weight", C.c_float),
        ("edges_array_src", u32p),
        ("edges_array_dest", u32p),
        ("edges_array_weight", f32p),
        ("label_array", u32p),
        ("inverse_label_array", u32p),
    ]


class GraphCSR(C.Structure):
    _fields_ = [
        ("num_edges", C.c_uint32),
        ("num_vertices", C.c_uint32),
        ("avg_degree", C.c_uint32),
        ("max_weight", C.c_float),
        ("vertices", C.POINTER(Vertex)),
        ("inverse_vertices", C.POINTER(Vertex)),
        ("sorted_edges_array", C.POINTER(EdgeList)),
        ("inverse_sorted_edges_array", C.POINTER(EdgeList)),
    ]


class MT19937State(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("mti", C.c_int32)]


class Arguments(C.Structure):
    _fields_ = [
        ("wflag", C.c_int), ("xflag", C.c_int), ("sflag", C.c_int), ("Sflag", C.c_int), ("dflag", C.c_int),
        ("binSize", C.c_uint32), ("verbosity", C.c_uint32), ("iterations", C.c_uint32), ("trials", C.c_uint32),
        ("epsilon", C.c_double), ("source", C.c_int), ("algorithm", C.c_uint32), ("datastructure", C.c_uint32),
        ("pushpull", C.c_uint32), ("sort", C.c_uint32), ("lmode", C.c_uint32), ("lmode_l2", C.c_uint32),
        ("lmode_l3", C.c_uint32), ("mmode", C.c_uint32), ("symmetric", C.c_uint32), ("weighted", C.c_uint32),
        ("delta", C.c_uint32), ("pre_numThreads", C.c_int), ("algo_numThreads", C.c_int),
        ("ker_numThreads", C.c_int), ("fnameb", C.c_char_p), ("fnamel", C.c_char_p),
        ("fnameb_format", C.c_uint32), ("convert_format", C.c_uint32), ("mt19937var", MT19937State),
        ("cache_size", C.c_uint32), ("afu_config", C.c_uint64), ("afu_config_2", C.c_uint64),
        ("cu_config", C.c_uint64), ("cu_config_2", C.c_uint64), ("cu_config_3", C.c_uint64),
        ("cu_config_4", C.c_uint64),
    ]


class PageRankStats(C.Structure):
    _fields_ = [
        ("damp", C.c_float), ("base_pr", C.c_float), ("iterations", C.c_uint32), ("num_vertices", C.c_uint32),
        ("activeVertices", C.c_uint32), ("realRanks", u32p), ("pageRanks", f32p), ("time_total", C.c_double),
        ("error_total", C.c_double),
    ]


class SPMVStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32), ("arguments", C.POINTER(Arguments)), ("num_vertices", C.c_uint32),
        ("vector_output", f32p), ("vector_input", f32p), ("time_total", C.c_double),
    ]


class PROpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("precision", C.c_int32), ("order", C.c_int32), ("quiet", C.c_int32),
        ("switch_residual", C.c_double), ("init_ranks", f32p), ("init_on_device", C.c_int32),
        ("data_driven", C.c_int32), ("direction", C.c_int32), ("keep_graph", C.c_int32),
    ]


class PRResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32), ("passes", C.c_uint32), ("converged", C.c_uint32),
        ("active_last", C.c_uint32), ("switch_pass", C.c_uint32), ("reserved", C.c_uint32),
        ("error_total", C.c_double), ("rank_sum", C.c_double), ("device_ms", C.c_double),
    ]


class TileConfig(C.Structure):
    _fields_ = [("task_edges", C.c_uint32), ("hub_chunk", C.c_uint32), ("hot_entries", C.c_uint32),
                ("warm_entries", C.c_uint32)]


class GraphInfo(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint32), ("num_edges", C.c_uint32), ("num_tasks", C.c_uint32),
        ("num_hub_rows", C.c_uint32), ("grid", C.c_uint32), ("max_in_degree", C.c_uint32),
        ("device_bytes", C.c_uint64),
    ]


# constants of include/accelgraph_b200.h
AG_OK = 0
AG_ERR_INVALID_ARG, AG_ERR_INVALID_GRAPH, AG_ERR_CUDA, AG_ERR_OOM = -1, -2, -3, -4
AG_ERR_TIMEOUT, AG_ERR_NO_DEVICE, AG_ERR_UNSUPPORTED, AG_ERR_DEVICE_WAIT = -5, -6, -7, -8
AG_BUILD_DEDUPE, AG_BUILD_SORT, AG_BUILD_PINNED, AG_BUILD_WEIGHTS, AG_BUILD_SYMMETRIC = 1, 2, 4, 8, 16
AG_FILE_TEXT, AG_FILE_BINARY, AG_FILE_CSR = 0, 1, 2
AG_UPLOAD_WEIGHTS, AG_UPLOAD_VALIDATE, AG_UPLOAD_TRUSTED = 1, 2, 4
AG_UPLOAD_KEEP_ORDER, AG_UPLOAD_NO_SMEM_CACHE = 8, 16
AG_PREC_FP32, AG_PREC_BF16, AG_PREC_FP16, AG_PREC_FIXED64 = 0, 1, 2, 3
AG_PREC_FIXED32, AG_PREC_FIXED16, AG_PREC_FIXED8 = 4, 5, 6
AG_PREC_QUANT32, AG_PREC_QUANT16, AG_PREC_QUANT8 = 7, 8, 9
# pageRankGraphCSR's pushpull code of each integer pull (pageRank.c:874-939)
PUSHPULL_OF_PREC = {AG_PREC_FIXED64: 2, AG_PREC_FIXED32: 9, AG_PREC_FIXED16: 10, AG_PREC_FIXED8: 11,
                    AG_PREC_QUANT32: 4, AG_PREC_QUANT16: 12, AG_PREC_QUANT8: 13}
# (quantised, width in bits) of each narrow integer pull
NARROW_FORM = {AG_PREC_FIXED32: (False, 32), AG_PREC_FIXED16: (False, 16), AG_PREC_FIXED8: (False, 8),
               AG_PREC_QUANT32: (True, 32), AG_PREC_QUANT16: (True, 16), AG_PREC_QUANT8: (True, 8)}
AG_ORDER_FAST, AG_ORDER_EXACT = 0, 1
AG_DIR_PULL, AG_DIR_PUSH, AG_DIR_PULL_PUSH = 0, 1, 2
AG_SPMV_GRAPH_WEIGHTS, AG_SPMV_UNIT, AG_SPMV_EXACT = 0, 1, 2
DAMP = np.float32(0.85)
BASE_PR = np.float32(np.float32(1.0) - DAMP)
REFERENCE_SEED = 27491095  # accel-graph.c:329

GraphP = C.POINTER(GraphCSR)

# (name, restype, argtypes) of every exported symbol declared in include/*.h
SIGNATURES = [
    ("newPageRankStatsGraphCSR", C.POINTER(PageRankStats), [GraphP]),
    ("freePageRankStats", None, [C.POINTER(PageRankStats)]),
    ("pageRankGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPushGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullFixedPoint64BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullFixedPoint32BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullFixedPoint16BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullFixedPoint8BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPushFixedPointGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullQuant32BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullQuant16BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPullQuant8BitGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankPushQuantGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankDataDrivenPullGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankDataDrivenPushGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("pageRankDataDrivenPullPushGraphCSR", C.POINTER(PageRankStats), [C.POINTER(Arguments), GraphP]),
    ("newSPMVStatsGraphCSR", C.POINTER(SPMVStats), [GraphP]),
    ("freeSPMVStats", None, [C.POINTER(SPMVStats)]),
    ("SPMVGraphCSR", C.POINTER(SPMVStats), [C.POINTER(Arguments), GraphP]),
    ("SPMVPullGraphCSR", C.POINTER(SPMVStats), [C.POINTER(Arguments), GraphP]),
    ("ag_status_string", C.c_char_p, [C.c_int32]),
    ("ag_last_error", C.c_char_p, []),
    ("ag_version", C.c_char_p, []),
    ("ag_init", C.c_int32, [C.c_int]),
    ("ag_stream", C.c_void_p, []),
    ("ag_set_stream", C.c_int32, [C.c_void_p]),
    ("ag_synchronize", C.c_int32, [C.c_double]),
    ("ag_num_sms", C.c_int, []),
    ("ag_graph_from_edges", GraphP, [C.c_uint32, C.c_uint64, u32p, u32p, f32p, C.c_uint32]),
    ("ag_graph_rmat", GraphP, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                               C.c_uint32]),
    ("ag_graph_er", GraphP, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32]),
    ("ag_graph_build_csr", GraphP, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    ("ag_graph_build", C.c_int32, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                   C.c_uint32, C.POINTER(C.c_void_p)]),
    ("ag_graph_read_edge_file", GraphP, [C.c_char_p, C.c_int, C.c_uint32]),
    ("ag_graph_read", GraphP, [C.c_char_p, C.c_int, C.c_int, C.c_uint32]),
    ("ag_graph_write", C.c_int32, [GraphP, C.c_char_p, C.c_int]),
    ("ag_graph_free", None, [GraphP]),
    ("ag_fill_uniform", None, [f32p, C.c_uint64, C.c_uint64]),
    ("ag_graph_upload", C.c_int32, [GraphP, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("ag_graph_release", C.c_int32, [C.c_void_p]),
    ("ag_graph_forget", C.c_int32, [GraphP]),
    ("ag_graph_get_info", C.c_int32, [C.c_void_p, C.POINTER(GraphInfo)]),
    ("ag_graph_get_tiles", C.c_int32, [C.c_void_p, C.POINTER(TileConfig)]),
    ("ag_gather_u64", C.c_int32, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("ag_gather_uint", C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64)]),
    ("ag_graph_get_tasks", C.c_int32, [C.c_void_p, C.c_int, u32p, C.c_uint32, C.POINTER(C.c_uint32)]),
    ("ag_graph_set_tiles", C.c_int32, [C.c_void_p, C.POINTER(TileConfig)]),
    ("ag_autotune", C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(TileConfig), f64p]),
    ("ag_pr_opts_init", None, [C.POINTER(PROpts)]),
    ("ag_pagerank_pull_ex", C.c_int32, [C.POINTER(Arguments), GraphP, C.POINTER(PROpts),
                                        C.POINTER(C.POINTER(PageRankStats))]),
    ("ag_pagerank_launch", C.c_int32, [C.c_void_p, C.c_uint32, C.c_double, C.POINTER(PROpts)]),
    ("ag_pagerank_fetch", C.c_int32, [C.c_void_p, f32p, C.POINTER(PRResult), u32p, f64p, f64p, C.c_uint32]),
    ("ag_pagerank_device_ranks", C.c_void_p, [C.c_void_p]),
    ("ag_pagerank_f64", C.c_int32, [C.c_void_p, C.c_uint32, C.c_double, f64p, u32p]),
    ("ag_spmv_pull_device", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    ("ag_spmv_pull", C.c_int32, [C.c_void_p, f32p, f32p, C.c_uint32]),
    ("ag_spmv_pull_ex", C.c_int32, [C.POINTER(Arguments), GraphP, C.c_int, C.POINTER(C.POINTER(SPMVStats))]),
    ("ag_multigraph_upload", C.c_int32, [C.POINTER(GraphP), C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("ag_multigraph_fetch", C.c_int32, [C.c_void_p, f32p, u32p, u32p, u32p, f64p, f64p]),
    ("ag_mlp_num_params", C.c_uint32, []),
    ("ag_mlp_create", C.c_int32, [C.c_uint64, C.POINTER(C.c_void_p)]),
    ("ag_mlp_release", C.c_int32, [C.c_void_p]),
    ("ag_mlp_set_params", C.c_int32, [C.c_void_p, f32p]),
    ("ag_mlp_get_params", C.c_int32, [C.c_void_p, f32p]),
    ("ag_features", C.c_int32, [C.c_void_p, C.c_void_p]),
    ("ag_mlp_forward", C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("ag_mlp_predict", C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("ag_mlp_gradients", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, f32p, f32p]),
    ("ag_mlp_train", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                 f32p]),
    ("ag_mlp_warm_start", C.c_int32, [C.c_void_p, C.c_void_p, f32p]),
    ("ag_mlp_warm_start_device", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ag_graph_upload_rows", C.c_int32, [GraphP, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_void_p)]),
    ("ag_partition_init", C.c_int32, [C.c_void_p, C.c_void_p]),
    ("ag_partition_step", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_void_p,
                                      C.c_void_p]),
    ("ag_partition_close", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ag_partition_pass", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    ("ag_partition_fetch", C.c_int32, [C.c_void_p, f32p]),
    ("ag_ppr_spmm", C.c_int32, [C.c_void_p, u32p, C.c_uint32, C.c_uint32, C.c_double, f32p, C.POINTER(PRResult)]),
    ("ag_spmv_pull_noalloc", C.c_int32, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_uint32, C.c_void_p]),
]


def _ensure_built() -> None:
    """Rebuild the in-tree library when a source is newer than it (the build
    recipe is loaded from its file so that it needs nothing from this
    package)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_accelgraph_b200_build", _PKG / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    if mod._stale():
        mod.build()


def _load() -> C.CDLL:
    if "AG_LIBRARY" not in os.environ:
        _ensure_built()
    path = Path(os.environ.get("AG_LIBRARY", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"accelgraph_b200: {path} is missing; build it with `python -m accelgraph_b200.build` "
            "(the B200 kernels have no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class AGError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = lib.ag_status_string(status).decode()
        detail = lib.ag_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}): {detail}")


def check(status: int, where: str) -> int:
    if status < 0:
        raise AGError(status, where)
    return status


def default_arguments(iterations: int = 20, epsilon: float = 1e-4) -> Arguments:
    """struct Arguments with the reference CLI defaults (accel-graph.c:288-326)."""
    a = Arguments()
    a.binSize = 512
    a.iterations = iterations
    a.trials = 1
    a.epsilon = epsilon
    a.cache_size = 32768
    a.delta = 1
    a.pre_numThreads = a.algo_numThreads = a.ker_numThreads = os.cpu_count() or 1
    a.fnameb_format = a.convert_format = 1
    a.afu_config = a.afu_config_2 = a.cu_config = a.cu_config_2 = a.cu_config_3 = a.cu_config_4 = 1
    return a


def _u32(ptr, n) -> np.ndarray:
    if n == 0 or not ptr:
        return np.zeros(0, np.uint32)
    return np.ctypeslib.as_array(ptr, shape=(n,))


def _f32(ptr, n) -> np.ndarray:
    if n == 0 or not ptr:
        return np.zeros(0, np.float32)
    return np.ctypeslib.as_array(ptr, shape=(n,))


def _edge_ptrs(src, dst, weight):
    """Raw pointers of edge arrays given as numpy arrays (converted to
    contiguous uint32/float32) or CUDA tensors (used in place)."""
    out, keep = [], []
    for a, dt in ((src, np.uint32), (dst, np.uint32), (weight, np.float32)):
        if a is None:
            out.append(None)
            keep.append(None)
        elif hasattr(a, "data_ptr"):
            out.append(a.data_ptr())
            keep.append(a)
        else:
            arr = np.ascontiguousarray(a, dt)
            out.append(arr.ctypes.data)
            keep.append(arr)
    return out, keep


class Graph:
    """A struct GraphCSR plus numpy views of its arrays.

    Either owned (built by the library's host substrate and freed with
    ag_graph_free) or borrowed from numpy arrays kept alive by this object.
    """

    def __init__(self, ptr, owned: bool, keep=None):
        if not ptr:
            raise AGError(AG_ERR_INVALID_ARG, "graph construction")
        self.ptr = ptr
        self.owned = owned
        self._keep = keep

    # -- construction ----------------------------------------------------
    @classmethod
    def rmat(cls, scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed=REFERENCE_SEED,
             flags=AG_BUILD_DEDUPE) -> "Graph":
        return cls(lib.ag_graph_rmat(scale, edge_factor, a, b, c, seed, flags), True)

    @classmethod
    def er(cls, num_vertices: int, avg_degree: int, seed=REFERENCE_SEED, flags=AG_BUILD_DEDUPE) -> "Graph":
        return cls(lib.ag_graph_er(num_vertices, avg_degree, seed, flags), True)

    @classmethod
    def from_edges(cls, num_vertices: int, src, dst, weight=None, flags=0) -> "Graph":
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        w = None if weight is None else np.ascontiguousarray(weight, np.float32)
        ptr = lib.ag_graph_from_edges(num_vertices, len(src), src.ctypes.data_as(u32p), dst.ctypes.data_as(u32p),
                                      None if w is None else w.ctypes.data_as(f32p), flags)
        return cls(ptr, True)

    @classmethod
    def build_gpu(cls, num_vertices: int, src, dst, weight=None, flags=0) -> "Graph":
        """ag_graph_build_csr: the from_edges CSR built on the GPU.  src, dst,
        weight: numpy arrays or CUDA tensors."""
        (ps, pd, pw), keep = _edge_ptrs(src, dst, weight)
        ptr = lib.ag_graph_build_csr(num_vertices, len(keep[0]), ps, pd, pw, flags)
        return cls(ptr, True)

    @classmethod
    def read(cls, path, format=AG_FILE_BINARY, weighted=False, flags=0) -> "Graph":
        """ag_graph_read: text or binary edge list, or a serialised CSR."""
        ptr = lib.ag_graph_read(str(path).encode(), format, int(weighted), flags)
        if not ptr:
            raise AGError(AG_ERR_INVALID_ARG, "ag_graph_read: " + lib.ag_last_error().decode())
        return cls(ptr, True)

    def write(self, path, format=AG_FILE_CSR) -> None:
        check(lib.ag_graph_write(self.ptr, str(path).encode(), format), "ag_graph_write")

    @classmethod
    def read_edge_file(cls, path, weighted=False, flags=0) -> "Graph":
        return cls(lib.ag_graph_read_edge_file(str(path).encode(), int(weighted), flags), True)

    @classmethod
    def from_inverse_csr(cls, num_vertices, in_degree, in_edges_idx, in_neighbours, out_degree,
                         in_weights=None) -> "Graph":
        """Borrow caller arrays: exactly the WED subset the pull path reads
        (capienv.c:845-868).  Forward arrays other than out_degree are left
        NULL; the pull kernels never read them."""
        n = int(num_vertices)
        indeg = np.ascontiguousarray(in_degree, np.uint32)
        idx = np.ascontiguousarray(in_edges_idx, np.uint32)
        nb = np.ascontiguousarray(in_neighbours, np.uint32)
        od = np.ascontiguousarray(out_degree, np.uint32)
        w = None if in_weights is None else np.ascontiguousarray(in_weights, np.float32)
        fv = Vertex(od.ctypes.data_as(u32p), indeg.ctypes.data_as(u32p), None)
        iv = Vertex(indeg.ctypes.data_as(u32p), od.ctypes.data_as(u32p), idx.ctypes.data_as(u32p))
        iel = EdgeList(len(nb), n, 0, 0.0, None, nb.ctypes.data_as(u32p),
                       None if w is None else w.ctypes.data_as(f32p), None, None)
        g = GraphCSR(len(nb), n, (len(nb) // n) if n else 0, 0.0, C.pointer(fv), C.pointer(iv), None,
                     C.pointer(iel))
        keep = (indeg, idx, nb, od, w, fv, iv, iel, g)
        return cls(C.pointer(g), False, keep)

    def free(self) -> None:
        if self.owned and self.ptr:
            lib.ag_graph_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- views -----------------------------------------------------------
    @property
    def g(self) -> GraphCSR:
        return self.ptr.contents

    @property
    def num_vertices(self) -> int:
        return self.g.num_vertices

    @property
    def num_edges(self) -> int:
        return self.g.num_edges

    def out_degree(self) -> np.ndarray:
        return _u32(self.g.vertices.contents.out_degree, self.num_vertices)

    def in_degree(self) -> np.ndarray:
        return _u32(self.g.inverse_vertices.contents.out_degree, self.num_vertices)

    def in_edges_idx(self) -> np.ndarray:
        return _u32(self.g.inverse_vertices.contents.edges_idx, self.num_vertices)

    def in_neighbours(self) -> np.ndarray:
        return _u32(self.g.inverse_sorted_edges_array.contents.edges_array_dest, self.num_edges)

    def in_weights(self):
        w = self.g.inverse_sorted_edges_array.contents.edges_array_weight
        return _f32(w, self.num_edges) if w else None

    def out_edges_idx(self) -> np.ndarray:
        return _u32(self.g.vertices.contents.edges_idx, self.num_vertices)

    def out_neighbours(self) -> np.ndarray:
        return _u32(self.g.sorted_edges_array.contents.edges_array_dest, self.num_edges)

    def out_sources(self) -> np.ndarray:
        return _u32(self.g.sorted_edges_array.contents.edges_array_src, self.num_edges)

    def in_owners(self) -> np.ndarray:
        return _u32(self.g.inverse_sorted_edges_array.contents.edges_array_src, self.num_edges)

    def in_offsets(self) -> np.ndarray:
        """row_off[N+1] of the inverse CSR (contiguous rows)."""
        off = np.zeros(self.num_vertices + 1, np.uint64)
        off[1:] = np.cumsum(self.in_degree(), dtype=np.uint64)
        return off


class DeviceGraph:
    """ag_graph_t: the inverse CSR resident on the GPU."""

    def __init__(self, graph: Graph, weights: bool = False, validate: bool = False, flags: int = 0):
        h = C.c_void_p()
        flags |= (AG_UPLOAD_WEIGHTS if weights else 0) | (AG_UPLOAD_VALIDATE if validate else 0)
        check(lib.ag_graph_upload(graph.ptr, flags, C.byref(h)), "ag_graph_upload")
        self.h = h
        self.num_vertices = graph.num_vertices
        self.num_edges = graph.num_edges

    @classmethod
    def from_edges(cls, num_vertices: int, src, dst, weight=None, build_flags=AG_BUILD_DEDUPE,
                   flags: int = 0) -> "DeviceGraph":
        """ag_graph_build: edge list to device graph, CSR built on the GPU."""
        (ps, pd, pw), keep = _edge_ptrs(src, dst, weight)
        m = len(keep[0]) if keep[0] is not None else 0
        h = C.c_void_p()
        if weight is not None:
            flags |= AG_UPLOAD_WEIGHTS
        check(lib.ag_graph_build(num_vertices, m, ps, pd, pw, build_flags, flags, C.byref(h)), "ag_graph_build")
        self = cls.__new__(cls)
        self.h = h
        self.num_vertices = num_vertices
        inf = self.info()
        self.num_edges = inf.num_edges
        return self

    def info(self) -> GraphInfo:
        inf = GraphInfo()
        check(lib.ag_graph_get_info(self.h, C.byref(inf)), "ag_graph_get_info")
        return inf

    def release(self) -> None:
        if self.h:
            lib.ag_graph_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def tiles(self) -> TileConfig:
        t = TileConfig()
        check(lib.ag_graph_get_tiles(self.h, C.byref(t)), "ag_graph_get_tiles")
        return t

    def tasks(self, exact: bool = False) -> np.ndarray:
        """The pull kernel's work list (items x 4 words, device row numbering)."""
        return _tasks(self.h, exact)

    def set_tiles(self, task_edges=256, hub_chunk=2048, hot_entries=16384, warm_entries=65536) -> None:
        t = TileConfig(task_edges, hub_chunk, hot_entries, warm_entries)
        check(lib.ag_graph_set_tiles(self.h, C.byref(t)), "ag_graph_set_tiles")

    def autotune(self, passes=8):
        t = TileConfig()
        us = C.c_double()
        check(lib.ag_autotune(self.h, passes, C.byref(t), C.byref(us)), "ag_autotune")
        return t, us.value

    def launch(self, iterations=20, epsilon=1e-4, precision=AG_PREC_FP32, order=AG_ORDER_FAST,
               init_ranks=None, switch_residual=1e-4, data_driven=False, direction=AG_DIR_PULL) -> None:
        o = make_opts(precision, order, init_ranks, switch_residual, data_driven=data_driven, direction=direction)
        self._keep_init = init_ranks
        check(lib.ag_pagerank_launch(self.h, iterations, epsilon, C.byref(o)), "ag_pagerank_launch")

    def fetch(self, history: int = 0):
        n = self.num_vertices
        ranks = np.empty(n, np.float32)
        res = PRResult()
        ha = np.zeros(max(history, 1), np.uint32)
        he = np.zeros(max(history, 1), np.float64)
        hs = np.zeros(max(history, 1), np.float64)
        check(lib.ag_pagerank_fetch(self.h, ranks.ctypes.data_as(f32p), C.byref(res), ha.ctypes.data_as(u32p),
                                    he.ctypes.data_as(f64p), hs.ctypes.data_as(f64p), history),
              "ag_pagerank_fetch")
        hist = {"active": ha[:min(history, res.passes)], "error": he[:min(history, res.passes)],
                "seconds": hs[:min(history, res.passes)]}
        return ranks, res, hist

    def pagerank(self, iterations=20, epsilon=1e-4, precision=AG_PREC_FP32, order=AG_ORDER_FAST,
                 init_ranks=None, switch_residual=1e-4, history=0, data_driven=False, direction=AG_DIR_PULL):
        self.launch(iterations, epsilon, precision, order, init_ranks, switch_residual, data_driven, direction)
        return self.fetch(history)

    def pagerank_f64(self, max_iterations=1000, tol=1e-13):
        r = np.empty(self.num_vertices, np.float64)
        passes = C.c_uint32()
        check(lib.ag_pagerank_f64(self.h, max_iterations, tol, r.ctypes.data_as(f64p), C.byref(passes)),
              "ag_pagerank_f64")
        return r, passes.value

    def ppr(self, sources, iterations=100, epsilon=1e-6, want_ranks=True):
        """Batched personalized PageRank (k = len(sources) <= 64); returns
        (ranks N x k or None, PRResult)."""
        src = np.ascontiguousarray(sources, np.uint32)
        k = len(src)
        out = np.empty((self.num_vertices, k), np.float32) if want_ranks else None
        res = PRResult()
        check(lib.ag_ppr_spmm(self.h, src.ctypes.data_as(u32p), k, iterations, epsilon,
                              out.ctypes.data_as(f32p) if want_ranks else None, C.byref(res)), "ag_ppr_spmm")
        return out, res

    def gather_u64(self, x) -> np.ndarray:
        """ag_gather_u64: integer row sums of x modulo 2^64 (caller order)."""
        x = np.ascontiguousarray(x, np.uint64)
        y = np.zeros(self.num_vertices, np.uint64)
        u64p = C.POINTER(C.c_uint64)
        check(lib.ag_gather_u64(self.h, x.ctypes.data_as(u64p), y.ctypes.data_as(u64p)), "ag_gather_u64")
        return y

    def gather_uint(self, x) -> np.ndarray:
        """ag_gather_uint: row sums of x (uint8, uint16, uint32 or uint64),
        each element zero-extended, modulo 2^64 (caller order)."""
        x = np.ascontiguousarray(x)
        if x.dtype not in (np.uint8, np.uint16, np.uint32, np.uint64):
            raise TypeError("gather_uint: x must be uint8, uint16, uint32 or uint64")
        y = np.zeros(self.num_vertices, np.uint64)
        check(lib.ag_gather_uint(self.h, x.ctypes.data_as(C.c_void_p), x.dtype.itemsize,
                                 y.ctypes.data_as(C.POINTER(C.c_uint64))), "ag_gather_uint")
        return y

    def spmv(self, x, mode=AG_SPMV_GRAPH_WEIGHTS) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty(self.num_vertices, np.float32)
        check(lib.ag_spmv_pull(self.h, x.ctypes.data_as(f32p), y.ctypes.data_as(f32p), mode), "ag_spmv_pull")
        return y


def _tasks(h, exact: bool) -> np.ndarray:
    n = C.c_uint32()
    check(lib.ag_graph_get_tasks(h, int(exact), None, 0, C.byref(n)), "ag_graph_get_tasks")
    out = np.zeros((n.value, 4), np.uint32)
    check(lib.ag_graph_get_tasks(h, int(exact), out.ctypes.data_as(u32p), n.value, C.byref(n)),
          "ag_graph_get_tasks")
    return out


class MultiGraph:
    """Many independent graphs solved in one launch (ag_multigraph_*)."""

    def __init__(self, graphs, flags: int = 0):
        arr = (GraphP * len(graphs))(*[g.ptr for g in graphs])
        h = C.c_void_p()
        check(lib.ag_multigraph_upload(arr, len(graphs), flags, C.byref(h)), "ag_multigraph_upload")
        self.h = h
        self.sizes = [g.num_vertices for g in graphs]
        self.edges = [g.num_edges for g in graphs]
        self.count = len(graphs)

    def release(self) -> None:
        if self.h:
            lib.ag_graph_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def autotune(self, passes=8):
        t = TileConfig()
        us = C.c_double()
        check(lib.ag_autotune(self.h, passes, C.byref(t), C.byref(us)), "ag_autotune")
        return t, us.value

    def tasks(self, exact: bool = False) -> np.ndarray:
        """The union's work list (items x 4 words)."""
        return _tasks(self.h, exact)

    def pagerank(self, iterations=100, epsilon=1e-6, order=AG_ORDER_FAST):
        o = make_opts(order=order)
        check(lib.ag_pagerank_launch(self.h, iterations, epsilon, C.byref(o)), "ag_pagerank_launch")
        n = sum(self.sizes)
        ranks = np.empty(n, np.float32)
        it = np.zeros(self.count, np.uint32)
        ps = np.zeros(self.count, np.uint32)
        cv = np.zeros(self.count, np.uint32)
        er = np.zeros(self.count, np.float64)
        ms = C.c_double()
        check(lib.ag_multigraph_fetch(self.h, ranks.ctypes.data_as(f32p), it.ctypes.data_as(u32p),
                                      ps.ctypes.data_as(u32p), cv.ctypes.data_as(u32p), er.ctypes.data_as(f64p),
                                      C.byref(ms)), "ag_multigraph_fetch")
        parts = np.split(ranks, np.cumsum(self.sizes)[:-1])
        return parts, {"iterations": it, "passes": ps, "converged": cv, "error_total": er, "device_ms": ms.value}


def make_opts(precision=AG_PREC_FP32, order=AG_ORDER_FAST, init_ranks=None, switch_residual=1e-4,
              quiet=True, data_driven=False, direction=AG_DIR_PULL) -> PROpts:
    o = PROpts()
    lib.ag_pr_opts_init(C.byref(o))
    o.precision = precision
    o.order = order
    o.data_driven = int(data_driven)
    o.direction = direction
    o.quiet = int(quiet)
    o.switch_residual = switch_residual
    if init_ranks is not None:
        if hasattr(init_ranks, "data_ptr"):  # a device tensor
            o.init_ranks = C.cast(C.c_void_p(init_ranks.data_ptr()), f32p)
            o.init_on_device = 1
            o._keep = init_ranks
        else:
            arr = np.ascontiguousarray(init_ranks, np.float32)
            o.init_ranks = arr.ctypes.data_as(f32p)
            o._keep = arr
    return o


def stats_ranks(stats_ptr) -> np.ndarray:
    st = stats_ptr.contents
    return _f32(st.pageRanks, st.num_vertices).copy()
