"""The committed ncu summaries that bench.py reads.

bench.py takes the measured DRAM traffic of its roofline kernel from a line
``traffic_bytes_per_launch: <stage> <workload> <bytes>`` in ``profiles/``.
These summaries are edited by hand, so check that every such line parses,
that the dominant kernels of the two headline workloads (the PCG of the
semi-implicit dam break, the viscosity stage of the explicit one) have one,
and that every summary gives the ncu command it came from, with the clocks
left alone (``--clock-control none``).
"""
import glob
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")
STAGES = {"visc", "collision", "pnd", "dash", "pressure", "assemble"}
WORKLOADS = {"explicit", "semi", "batch", "large"}


def _summaries():
    return sorted(glob.glob(os.path.join(PROFILES, "*.md")) + glob.glob(os.path.join(PROFILES, "*.txt")))


def test_traffic_lines_parse():
    seen = []
    for f in _summaries():
        for line in open(f):
            if line.startswith("traffic_bytes_per_launch:"):
                parts = line.split()
                assert len(parts) == 4, (f, line)
                assert parts[1] in STAGES and parts[2] in WORKLOADS, (f, line)
                assert int(parts[3]) > 0, (f, line)
                seen.append((parts[1], parts[2]))
    assert len(seen) == len(set(seen)), "a (stage, workload) pair appears twice"


def test_headline_kernels_have_traffic():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._traffic_from_profiles("pressure", "semi") > 0
    assert bench._traffic_from_profiles("visc", "explicit") > 0


def test_every_summary_gives_its_ncu_command():
    files = _summaries()
    assert files
    for f in files:
        text = open(f).read()
        assert "ncu " in text, f
        for line in text.replace("\\\n", " ").splitlines():  # a command continued with backslashes
            if line.strip().startswith("ncu "):
                assert "--clock-control none" in line, (f, line)
