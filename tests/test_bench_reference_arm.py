"""The reference arm of bench.py (`--impl reference`) on the CPU: the JSON
line the measurement contract asks for, timed on the oracle alone (the
product library is never loaded), and silence on ranks other than 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

# runs bench.py's main in this process, then reports whether the product
# library was mapped
_RUNNER = (
    "import runpy, sys; sys.argv = ['bench.py'] + sys.argv[1:]; "
    "runpy.run_path('bench.py', run_name='__main__'); "
    "maps = open('/proc/self/maps').read(); "
    "print('PRODUCT_LOADED' if 'libaccelgraph_b200' in maps else 'PRODUCT_NOT_LOADED')"
)


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    res = subprocess.run([sys.executable, "-c", _RUNNER, "--impl", "reference", "--scale", "10", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    return [ln for ln in res.stdout.splitlines() if ln.strip()]


def test_reference_arm_prints_the_contract_line_without_the_product_library():
    lines = _run()
    assert lines[-1] == "PRODUCT_NOT_LOADED"
    rec = json.loads(lines[-2])
    assert rec["impl"] == "reference"
    assert rec["unit"] == "GTEPS" and rec["higher_is_better"] is True
    assert rec["value"] > 0 and rec["steps"] == 2 and rec["warmup"] == 1
    cpu = rec["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == rec["value"] and cpu["sample"]
    assert rec["e2e"] == {"value": rec["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert rec["config"]["workload"].startswith("PageRank pull FP32")


def test_reference_arm_is_silent_on_other_ranks():
    lines = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert lines == ["PRODUCT_NOT_LOADED"]
