"""bench.py --impl reference on the CPU, with the arguments the benchmark
driver gives it (--steps 20 --warmup 5): the reference C (oracle/_ref, built
from the reference's sources as it ships, without the cost pass) timed on a
bounded sample of the 4-D workload, printed as one JSON line with the same
metric, unit and config as our arm. 25 iterations of the cost-on build used to
abort on a rounding-level cost increase; the as-shipped build has no such
check."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not O.ref_available(timing=True), reason="reference build not present")
def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "20",
                        "--warmup", "5"], capture_output=True, text=True, timeout=1200, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "voxel-updates/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["metric"].startswith("time-to-converged cost")
    assert d["config"]["workload"] == "4d_cahn_hilliard_256x256x32_8frames_1024views"
    assert d["steps"] == 20 and d["warmup"] == 5 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert 1 <= cb["busy_threads"] <= cb["cores"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
