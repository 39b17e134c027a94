"""The bench.py JSON contract, checked on CPU through the reference arm.

`bench.py --impl reference` needs no GPU: it times the reference's own CPU
solve (the compiled sources, or the restatement where they are absent) and
prints one JSON line with the same metric, unit and config keys as the GPU
arm, plus its cpu_baseline and a zero-copy e2e.  A small grid keeps it to
about a second.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.usefixtures("oracle_built")


def test_reference_arm_prints_one_contract_line():
    proc = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
         "--shape", "32", "32", "32", "--steps", "1", "--warmup", "0"],
        cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, proc.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    assert d["value"] > 0 and d["vs_baseline"] is None and d["dtype"] == "f64"
    assert d["config"]["shape"] == [32, 32, 32] and "workload" in d["config"]
    cpu = d["cpu_baseline"]
    assert cpu["value"] == d["value"] and cpu["kind"] in ("reference", "port")
    assert cpu["cores"] >= 1 and cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"],
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
