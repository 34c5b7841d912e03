"""Shared fixtures of the test suite.

`-m "not gpu"` tests run anywhere (the oracle against the reference's RTL
goldens, the host graph substrate, the C ABI surface).  `-m gpu` tests need a
CUDA device and call the sm_100a kernels through the C ABI.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def _has_gpu() -> bool:
    import accelgraph_b200 as ag
    return ag.lib.ag_init(int(os.environ.get("AG_DEVICE", "0"))) == 0


@pytest.fixture(scope="session")
def ag():
    import accelgraph_b200  # rebuilds the in-tree library when it is stale
    return accelgraph_b200


@pytest.fixture(scope="session")
def gpu(ag):
    if not _has_gpu():
        pytest.skip("no CUDA device")
    return ag


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def rtl():
    return json.loads((GOLDEN / "rtl_fixtures.json").read_text())


def f32_from_hex(h: str) -> np.float32:
    return np.array([int(h, 16)], np.uint32).view(np.float32)[0]


def hex_of(x) -> str:
    return "%08x" % int(np.array([x], np.float32).view(np.uint32)[0])


def fixture_csr(fx: dict):
    """Inverse CSR of an RTL fixture in the testbench's stream order."""
    n = fx["num_vertices"]
    deg = np.array([len(r) for r in fx["inverse_neighbours"]], np.uint32)
    idx = np.zeros(n, np.uint32)
    if n:
        idx[1:] = np.cumsum(deg)[:-1]
    nb = np.array([u for r in fx["inverse_neighbours"] for u in r], np.uint32)
    w = np.array([x for r in fx["inverse_weights"] for x in r], np.float32)
    od = np.array(fx["out_degree"], np.uint32)
    return n, deg, idx, nb, w, od


def run_inputs(run: dict, fx: dict, weighted: bool):
    """Per-vertex x and per-edge w reproducing one testbench run.

    Classes whose value depends only on the source vertex become x[u]; the
    mixed class (value depends on the stream position) is driven as x = 1 and
    w = the element value, which a binary32 multiply by 1 leaves unchanged."""
    n, deg, idx, nb, wt, od = fixture_csr(fx)
    e = len(nb)
    x = np.ones(max(n, 1), np.float32)[:n]
    w = np.ones(e, np.float32)
    position_dependent = run["class"] == "CV_MIXED"
    for row in run["rows"]:
        v = row["v"]
        for k, el in enumerate(row["elements"]):
            j = idx[v] + k
            u = nb[j]
            if position_dependent:
                w[j] = f32_from_hex(el["product"] if weighted else el["x"])
            else:
                x[u] = f32_from_hex(el["x"])
                if weighted:
                    w[j] = f32_from_hex(el["w"])
    return n, deg, idx, nb, w, od, x, position_dependent


def fixed_inputs(run: dict, fx: dict, dtype=np.uint64):
    """Inputs reproducing one FixedPoint-context (uint64 elements) or
    Quantized-context (uint32 elements) testbench run as a gather.

    The contributions depend on the stream position, so every in-edge is
    given a source vertex of its own (n + j for edge j) carrying its element;
    the rows and their in-degrees are the fixture's."""
    n, deg, idx, nb, wt, od = fixture_csr(fx)
    e = len(nb)
    x = np.zeros(n + e, dtype)
    nb2 = (n + np.arange(e)).astype(np.uint32)
    for row in run["rows"]:
        v = row["v"]
        for k, el in enumerate(row["elements"]):
            x[n + idx[v] + k] = dtype(int(el, 16))
    deg2 = np.concatenate([deg, np.zeros(e, np.uint32)]).astype(np.uint32)
    idx2 = np.concatenate([idx, np.full(e, e, np.uint32)]).astype(np.uint32)
    return n, deg2, idx2, nb2, x
