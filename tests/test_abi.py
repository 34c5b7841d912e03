"""The C ABI surface: the library loads without a GPU and exports every
function declared in include/*.h."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"#[^\n]*", "", text)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            if name in ("sizeof", "if", "while", "for", "return"):
                continue
            names.add(name)
    return sorted(names)


# every CSR entry point of the reference's pageRank.h:32-86 and SPMV.h:30-52
REFERENCE_CSR_SYMBOLS = (
    "newPageRankStatsGraphCSR", "freePageRankStats", "pageRankGraphCSR", "pageRankPullGraphCSR",
    "pageRankPushGraphCSR", "pageRankPullFixedPoint64BitGraphCSR", "pageRankPullFixedPoint32BitGraphCSR",
    "pageRankPullFixedPoint16BitGraphCSR", "pageRankPullFixedPoint8BitGraphCSR", "pageRankPushFixedPointGraphCSR",
    "pageRankPullQuant32BitGraphCSR", "pageRankPullQuant16BitGraphCSR", "pageRankPullQuant8BitGraphCSR",
    "pageRankPushQuantGraphCSR", "pageRankDataDrivenPullGraphCSR", "pageRankDataDrivenPushGraphCSR",
    "pageRankDataDrivenPullPushGraphCSR",
    "newSPMVStatsGraphCSR", "freeSPMVStats", "SPMVGraphCSR", "SPMVPullGraphCSR",
)


def test_headers_declare_reference_entry_points():
    names = declared_functions()
    missing = [ref for ref in REFERENCE_CSR_SYMBOLS if ref not in names]
    assert not missing, missing


def test_library_exports_every_reference_csr_symbol(ag):
    lib = C.CDLL(str(ag.LIB_PATH))
    missing = [n for n in REFERENCE_CSR_SYMBOLS if not hasattr(lib, n)]
    assert not missing, missing


def test_library_exports_every_declared_symbol(ag):
    lib = C.CDLL(str(ag.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_headers(ag):
    bound = {s[0] for s in ag.SIGNATURES}
    missing = [n for n in declared_functions() if n not in bound]
    assert not missing, missing


def test_struct_layouts(ag, tmp_path):
    """ctypes mirrors match the C compiler's layout of include/*.h."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    checks = {
        "Vertex": ["out_degree", "in_degree", "edges_idx"],
        "EdgeList": ["num_edges", "max_weight", "edges_array_dest", "edges_array_weight", "inverse_label_array"],
        "GraphCSR": ["num_edges", "num_vertices", "avg_degree", "max_weight", "vertices", "inverse_vertices",
                     "sorted_edges_array", "inverse_sorted_edges_array"],
        "Arguments": ["epsilon", "iterations", "pushpull", "ker_numThreads", "fnameb", "mt19937var",
                      "cache_size", "afu_config", "cu_config_4"],
        "PageRankStats": ["damp", "base_pr", "iterations", "activeVertices", "realRanks", "pageRanks",
                          "time_total", "error_total"],
        "SPMVStats": ["iterations", "arguments", "num_vertices", "vector_output", "vector_input", "time_total"],
    }
    typed = {"ag_pr_opts": ("PROpts", ["precision", "switch_residual", "init_ranks"]),
             "ag_pr_result": ("PRResult", ["iterations", "error_total", "device_ms"]),
             "ag_graph_info": ("GraphInfo", ["num_tasks", "device_bytes"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "accelgraph_b200.h"', 'int main(void){']
    for st, fields in checks.items():
        lines.append(f'printf("{st} %zu\\n", sizeof(struct {st}));')
        for f in fields:
            lines.append(f'printf("{st}.{f} %zu\\n", offsetof(struct {st}, {f}));')
    for ct, (py, fields) in typed.items():
        lines.append(f'printf("{py} %zu\\n", sizeof({ct}));')
        for f in fields:
            lines.append(f'printf("{py}.{f} %zu\\n", offsetof({ct}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    pymap = {"Vertex": ag.Vertex, "EdgeList": ag.EdgeList, "GraphCSR": ag.GraphCSR, "Arguments": ag.Arguments,
             "PageRankStats": ag.PageRankStats, "SPMVStats": ag.SPMVStats, "PROpts": ag.PROpts,
             "PRResult": ag.PRResult, "GraphInfo": ag.GraphInfo}
    for line in filter(None, out):
        key, val = line.split()
        if "." in key:
            st, f = key.split(".")
            assert getattr(pymap[st], f).offset == int(val), key
        else:
            assert C.sizeof(pymap[key]) == int(val), key


def test_status_strings(ag):
    assert ag.lib.ag_status_string(ag.AG_ERR_TIMEOUT) == b"timeout"
    assert ag.lib.ag_version().startswith(b"accelgraph-b200")


def test_no_device_is_reported_not_faked(ag):
    """Without a GPU every device entry point reports AG_ERR_NO_DEVICE; there
    is no CPU fallback behind the C ABI."""
    if ag.lib.ag_init(0) == 0:
        pytest.skip("a CUDA device is present")
    g = ag.Graph.rmat(6, 4)
    h = C.c_void_p()
    st = ag.lib.ag_graph_upload(g.ptr, 0, C.byref(h))
    assert st == ag.AG_ERR_NO_DEVICE
    args = ag.default_arguments()
    out = C.POINTER(ag.PageRankStats)()
    assert ag.lib.ag_pagerank_pull_ex(C.byref(args), g.ptr, None, C.byref(out)) == ag.AG_ERR_NO_DEVICE


def test_stats_objects_follow_reference_init(ag):
    g = ag.Graph.rmat(5, 4)
    st = ag.lib.newPageRankStatsGraphCSR(g.ptr)
    s = st.contents
    assert s.num_vertices == 32 and s.damp == pytest.approx(0.85) and s.iterations == 0
    import numpy as np
    ranks = np.ctypeslib.as_array(s.pageRanks, shape=(32,))
    assert np.all(ranks == np.float32(1.0) - np.float32(0.85))
    real = np.ctypeslib.as_array(s.realRanks, shape=(32,))
    assert np.array_equal(real, np.arange(32))
    ag.lib.freePageRankStats(st)
    sp = ag.lib.newSPMVStatsGraphCSR(g.ptr)
    assert sp.contents.num_vertices == 32
    ag.lib.freeSPMVStats(sp)
