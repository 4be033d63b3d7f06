"""The bench's reference arm runs on the host cores, so its JSON line can be
checked without a GPU: one line, the metric and unit of the GPU arm, the
reference's CPU path described in cpu_baseline, and an e2e entry that moves
no bytes between host and device."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["explicit", "semi"])
def test_reference_arm_line(workload):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", workload,
                        "--steps", "3", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert "unavailable" not in d, d
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["ms_per_step"] > 0 and d["data"] == "synthetic"
    assert d["config"]["particles"] == (70912 if workload == "explicit" else 310912)
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    # the explicit path is the reference's own CPU build where it was compiled
    # from the reference's sources (oracle/_ref)
    if workload == "explicit" and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_expl")):
        assert cb["kind"] == "reference"
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
