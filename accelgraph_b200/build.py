"""Build recipe of libaccelgraph_b200.so (host C + sm_100a CUDA, in-tree).

Usage: python -m accelgraph_b200.build [--force]

The host C sources are compiled with gcc (-O3 -fopenmp, the reference's own
flags, 02_capi_graph/Makefile:250), the CUDA sources with nvcc for sm_100a
only, and everything is linked into accelgraph_b200/libaccelgraph_b200.so with
the CUDA runtime linked statically.  Rebuilds only when a source is newer than
the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libaccelgraph_b200.so"

C_SOURCES = ["graph_host.c", "ag_capi.c"]
CU_SOURCES = ["ag_pull.cu", "ag_layout.cu", "ag_runtime.cu", "ag_noalloc.cu", "ag_ppr.cu", "ag_mlp.cu", "ag_plan.cu", "ag_build.cu", "ag_fixed.cu", "ag_push.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the B200 library needs the CUDA toolkit to build")


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}): {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr, flush=True)


def _stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = [CSRC / s for s in C_SOURCES + CU_SOURCES]
    deps += list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False, out: Path | None = None, defines: tuple = ()) -> Path:
    """Compile the library if it is missing or out of date; return its path.

    `defines` (e.g. ("AG_WHUB=1024",)) override the tiling constants of
    csrc/ag_device.h for a tuning build written to `out`."""
    lib = Path(out) if out else LIB
    if not force and not _stale(lib):
        return lib
    nvcc = _nvcc()
    build_dir = BUILD if not out else lib.parent / "_build"
    build_dir.mkdir(parents=True, exist_ok=True)
    dflags = [f"-D{d}" for d in defines]
    inc = ["-I", str(INCLUDE), "-I", str(CSRC)]
    objs = []
    for src in C_SOURCES:
        obj = build_dir / (src + ".o")
        _run(["gcc", "-O3", "-Wall", "-m64", "-fopenmp", "-fPIC", "-std=gnu11", *inc, *dflags, "-c", str(CSRC / src),
              "-o", str(obj)], verbose)
        objs.append(str(obj))
    for src in CU_SOURCES:
        obj = build_dir / (src + ".o")
        _run([nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-Wall,-fopenmp", *inc, *dflags, "-c",
              str(CSRC / src), "-o", str(obj)], verbose)
        objs.append(str(obj))
    tmp = lib.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs, "-Xcompiler", "-fopenmp", "-lgomp",
          "-lpthread", "-lrt"], verbose)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
