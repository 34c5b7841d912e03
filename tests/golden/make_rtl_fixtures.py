"""Generate tests/golden/rtl_fixtures.json from the reference's RTL testbench.

Reads, as text, the reference's independent fixture registry and kernel
testbenches (AccelGraph,
03_capi_integration/accelerator_verification/rtl/unit/algorithms/tb/):
  graph_fixture_pkg.sv   13 hand-authored edge lists (:37-107) and the
                         inverse-row derivation in edge-list order (:128-163)
  pagerank_kernel_tb.sv  contribution classes (:242-265), the run list
                         (:660-720) and the stream-order binary32 golden
                         (:303-314): the accumulator restarts with the first
                         value of a row and adds each following value; for
                         the FixedPoint context the 64-bit contributions
                         (:256-263) and their exact sum modulo 2^64 (:13-16);
                         for the Quantized context the same classes cut to
                         32 bits (DATA_SIZE_READ = 4) and zero-extended into
                         the 64-bit sum (:17-19, :312)
  spmv_kernel_tb.sv      coefficients w/2 (:277-293), product x*w in binary32
                         (:296-301) and the same stream-order sum (:349-359)
and the 19-edge binary edge list 04_test_graphs/TEST/graphbrew/graph.bin.
The goldens are recomputed here with numpy binary32 arithmetic, independently
of the oracle and of the CUDA kernels, exactly as the testbench's DPI model
does in C (models/fp32_reference.cpp:36-49).

Usage (needs the reference checkout; the output is committed):
  python tests/golden/make_rtl_fixtures.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import re
import os
import sys
from pathlib import Path

import numpy as np

# the reference checkout: the first argument, else $AG_REFERENCE, else
# `reference` beside this checkout
REF = Path(sys.argv[1] if len(sys.argv) > 1 else
           (os.environ.get("AG_REFERENCE") or Path(__file__).resolve().parents[3] / "reference"))
TB = REF / "03_capi_integration/accelerator_verification/rtl/unit/algorithms/tb"
OUT = Path(__file__).resolve().parent / "rtl_fixtures.json"

f32 = np.float32
MAXF = np.array([0x7F7FFFFF], np.uint32).view(np.float32)[0]


def bits(x) -> str:
    return "%08x" % int(np.array([x], np.float32).view(np.uint32)[0])


def parse_int_list(block: str) -> list[int]:
    return [int(t) for t in re.findall(r"-?\d+", block)]


def parse_2d(text: str, name: str) -> list[list[int]]:
    m = re.search(name + r"\s*\[[^\]]*\]\s*\[[^\]]*\]\s*=\s*'\{(.*?)\};", text, re.S)
    rows = re.findall(r"'\{([^{}]*)\}", m.group(1))
    return [parse_int_list(re.sub(r"//[^\n]*", "", r)) for r in rows]


def parse_1d(text: str, name: str) -> list[int]:
    m = re.search(name + r"\s*\[[^\]]*\]\s*=\s*'\{(.*?)\};", text, re.S)
    return parse_int_list(re.sub(r"//[^\n]*", "", m.group(1)))


def main() -> None:
    pkg = (TB / "graph_fixture_pkg.sv").read_text()
    names = {}
    for m in re.finditer(r"parameter int (FX_[A-Z0-9_]+)\s*=\s*(\d+)\s*;", pkg):
        if m.group(1) not in ("FX_MAX_VERTICES", "FX_MAX_EDGES"):
            names[m.group(1)] = int(m.group(2))
    count = int(re.search(r"FIXTURE_COUNT\s*=\s*(\d+)", pkg).group(1))
    nv = parse_1d(pkg, "FX_NUM_VERTICES")
    ne = parse_1d(pkg, "FX_NUM_EDGES")
    src = parse_2d(pkg, "FX_EDGE_SRC")
    dst = parse_2d(pkg, "FX_EDGE_DEST")
    wgt = parse_2d(pkg, "FX_EDGE_WEIGHT")
    assert len(nv) == len(ne) == len(src) == len(dst) == len(wgt) == count
    by_id = {v: k for k, v in names.items()}

    fixtures = []
    for fx in range(count):
        n, m = nv[fx], ne[fx]
        s, d, w = src[fx][:m], dst[fx][:m], wgt[fx][:m]
        # inverse rows in edge-list order (graph_fixture_pkg.sv:128-163)
        inv_nb = [[s[e] for e in range(m) if d[e] == v] for v in range(n)]
        inv_w = [[w[e] for e in range(m) if d[e] == v] for v in range(n)]
        out_deg = [sum(1 for e in range(m) if s[e] == v) for v in range(n)]
        fixtures.append({"id": fx, "name": by_id[fx], "num_vertices": n, "src": s, "dst": d, "weight": w,
                         "inverse_neighbours": inv_nb, "inverse_weights": inv_w, "out_degree": out_deg})

    cv = {"CV_SMALL": 0, "CV_ZERO": 1, "CV_MAX": 2, "CV_MIXED": 3}

    def contribution(cls: int, nb: int, k: int):
        if cls == 1:
            return f32(0.0)
        if cls == 2:
            return MAXF
        if cls == 3 and k % 2 == 1:
            return -(f32(k + 1) / f32(7))
        return f32(nb + 1) / f32(3)

    def contribution_fixed(cls: int, nb: int, k: int) -> int:
        """the FixedPoint context's 64-bit contributions (pagerank_kernel_tb.sv:256-263)"""
        if cls == 1:
            return 0
        if cls == 2:
            return (1 << 64) - 1
        if cls == 3:
            return 0xFFFF_FFFF_0000_0001 if k % 2 == 0 else (nb + 1) * 7
        return (nb + 1) * 7 + k

    def contribution_quant(cls: int, nb: int, k: int) -> int:
        """the Quantized context's 32-bit contributions: the same classes at
        DATA_SIZE_READ_BITS = 32 (pagerank_kernel_tb.sv:256-263)"""
        return contribution_fixed(cls, nb, k) & 0xFFFF_FFFF

    def fixed_runs(quant: bool = False):
        text = (TB / "pagerank_kernel_tb.sv").read_text()
        out = []
        value = contribution_quant if quant else contribution_fixed
        digits = 8 if quant else 16
        for m in re.finditer(r"run_fixture\((FX_[A-Z0-9_]+)\s*,\s*(CV_[A-Z]+)\s*,\s*0\s*\)", text):
            fx, cls = names[m.group(1)], cv[m.group(2)]
            fxd = fixtures[fx]
            rows = []
            for v in range(fxd["num_vertices"]):
                nbs = fxd["inverse_neighbours"][v]
                if not nbs:
                    continue
                vals = [value(cls, nb, k) for k, nb in enumerate(nbs)]
                acc = sum(vals) % (1 << 64)  # exact sum, wraps modulo 2^64 (:13-16, :312)
                rows.append({"v": v, "elements": ["%0*x" % (digits, x) for x in vals], "golden": "%016x" % acc})
            out.append({"fixture": fxd["name"], "fixture_id": fx, "class": m.group(2), "rows": rows})
        return out

    def coefficient(cls: int, weight: int):
        if cls == 1:
            return f32(0.0)
        if cls == 2:
            return MAXF
        return f32(weight) / f32(2)

    def runs(tb_name: str, weighted: bool):
        text = (TB / tb_name).read_text()
        out = []
        for m in re.finditer(r"run_fixture\((FX_[A-Z0-9_]+)\s*,\s*(CV_[A-Z]+)\s*,\s*0\s*\)", text):
            fx, cls = names[m.group(1)], cv[m.group(2)]
            fxd = fixtures[fx]
            rows = []
            for v in range(fxd["num_vertices"]):
                nbs = fxd["inverse_neighbours"][v]
                if not nbs:
                    continue  # zero in-degree: never written (cu_vertex_job_filter.sv:105-106)
                vals = []
                acc = None
                with np.errstate(over="ignore", invalid="ignore"):
                    for k, nb in enumerate(nbs):
                        x = contribution(cls, nb, k)
                        if weighted:
                            cw = coefficient(cls, fxd["inverse_weights"][v][k])
                            val = f32(x * cw)
                            vals.append({"x": bits(x), "w": bits(cw), "product": bits(val)})
                        else:
                            val = x
                            vals.append({"x": bits(x)})
                        acc = val if k == 0 else f32(acc + val)
                rows.append({"v": v, "elements": vals, "golden": bits(acc)})
            out.append({"fixture": fxd["name"], "fixture_id": fx, "class": m.group(2), "rows": rows})
        return out

    with np.errstate(over="ignore"):
        exc = [
            {"values": [bits(MAXF), bits(MAXF)], "golden": bits(f32(MAXF + MAXF))},
            {"values": ["00800000", "80800000"],
             "golden": bits(f32(np.array([0x00800000], np.uint32).view(np.float32)[0]
                                + np.array([0x80800000], np.uint32).view(np.float32)[0]))},
        ]

    raw = np.fromfile(REF / "04_test_graphs/TEST/graphbrew/graph.bin", dtype=np.uint32).reshape(-1, 2)
    doc = {
        "generator": "tests/golden/make_rtl_fixtures.py",
        "sources": [
            "03_capi_integration/accelerator_verification/rtl/unit/algorithms/tb/graph_fixture_pkg.sv",
            "03_capi_integration/accelerator_verification/rtl/unit/algorithms/tb/pagerank_kernel_tb.sv",
            "03_capi_integration/accelerator_verification/rtl/unit/algorithms/tb/spmv_kernel_tb.sv",
            "04_test_graphs/TEST/graphbrew/graph.bin",
        ],
        "fixtures": fixtures,
        "pagerank_runs": runs("pagerank_kernel_tb.sv", weighted=False),
        "spmv_runs": runs("spmv_kernel_tb.sv", weighted=True),
        "pagerank_fixed_runs": fixed_runs(),
        "pagerank_quant_runs": fixed_runs(quant=True),
        "fp_exception_rows": exc,
        "graphbrew": {"src": raw[:, 0].tolist(), "dst": raw[:, 1].tolist()},
    }
    OUT.write_text(json.dumps(doc, indent=1) + "\n")
    print(f"wrote {OUT}: {len(fixtures)} fixtures, {len(doc['pagerank_runs'])} pagerank runs, "
          f"{len(doc['pagerank_fixed_runs'])} fixed-point runs, {len(doc['pagerank_quant_runs'])} quantized runs, "
          f"{len(doc['spmv_runs'])} spmv runs, graphbrew {len(raw)} edges")


if __name__ == "__main__":
    main()
