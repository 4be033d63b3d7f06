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
STAGES = {"visc", "collision", "pnd", "dash", "pressure", "pressure_sell", "assemble"}
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


def _ncu_commands(text):
    # a command continued with backslashes is one line
    return [ln.strip() for ln in text.replace("\\\n", " ").splitlines() if ln.strip().startswith("ncu ")]


def test_every_summary_gives_its_ncu_command():
    files = _summaries()
    assert files
    for f in files:
        text = open(f).read()
        assert "ncu " in text, f
        for line in _ncu_commands(text):
            assert "--clock-control none" in line, (f, line)


# metrics that ncu collects in a single pass together (checked on a B200:
# "1 pass" for the three of them on the small tank)
ONE_PASS = {"gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum"}


def test_multi_pass_captures_are_one_kernel_on_a_small_case():
    """A capture that collects more than the one-pass metrics replays each
    launch many times: it must select one kernel (-k without alternatives),
    at most three launches (-c), and a small case (the ~110k-particle tank,
    the 70,912-particle explicit scene, the 8-scene batch, or one scene of
    the training script: about 300k particles, a few hundred MB on the
    device)."""
    import re
    for f in _summaries():
        for line in _ncu_commands(open(f).read()):
            metrics = re.findall(r"--metrics\s+(\S+)", line)
            one_pass = not re.search(r"--set|--section", line) and all(
                set(m.split(",")) <= ONE_PASS for m in metrics)
            if one_pass:
                continue
            k = re.search(r"-k\s+(\S+)", line)
            assert k and "|" not in k.group(1), (f, "one kernel per capture", line)
            c = re.search(r"-c\s+(\d+)", line)
            assert c and int(c.group(1)) <= 3, (f, "at most three launches", line)
            small = ("--size small" in line or "--workload explicit" in line
                     or ("train_precond" in line and re.search(r"--scenes\s+1\b", line)))
            assert small, (f, "a small case", line)
