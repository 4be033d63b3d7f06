"""Parity of the benchmarked semi-implicit dam break over the first 100 steps,
and bit-exact neighbour sets of the PPE stencil.

Reference rules: MPS_CPU_EXPL::step (MPS_CAL_v4.0/MPS_CPU_EXPL.cpp:79-135),
restated by the oracle from MPS_CPU.cpp:573-888 (PND, buildPoisson, CG,
pressCorr, gradient) in double with CG to 1e-12.

* 100-step window.  The 310,912-particle dam break (80,000 fluid, l0 = 0.01
  m, dt = 5e-4 s) runs on the GPU with the benchmark's settings (fast
  arithmetic, PPE to |b - Ax| <= 1e-8 |b| in FP64) next to the FP64 oracle.
  At steps 25, 50 and 100 the test reports, per field, |gpu - oracle| /
  max|oracle| (positions: over the domain extent) as the largest over all
  particles and the median and 99th percentile over the fluid, and asserts
  the stated tolerances below.
* Explicit window.  The explicit step is bit-exact against the reference's
  float build (tests/test_gpu_explicit.py); here its error against the FP64
  oracle over 100 steps of the 70,912-particle dam break is reported and
  bounded, i.e. the error the reference's own float arithmetic carries.
* Neighbour sets.  From the state the GPU assembled its PPE system from
  (mps_ppe_snapshot), the pairs of the stored matrix (mps_ppe_stencil) must
  equal {(i, j): i, j solved rows, j != i, w(r_ij; rlap) != 0} evaluated in
  the reference's float arithmetic (dx = xj - xi, r^2 = (dx dx + dy dy) +
  dz dz, r = sqrt(r^2), w = rlap / r - 1), pair for pair, in both arithmetic
  modes; the solved rows must be exactly those of type != 2 with
  n_i >= beta n0 (FP64 comparison).

Set MPS_PARITY_REPORT to a file path to get the measured errors as JSON.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Stated tolerances over the 100-step window, relative to each field's
# largest magnitude (positions: to the domain extent).  "max" bounds the
# worst particle of all; "p99" bounds the 99th percentile over the fluid
# particles.  The worst particles come from discrete events of the method
# (a pair crossing the collision distance, a free-surface particle crossing
# n = beta n0 into or out of the Dirichlet set) that FP32 and FP64 rounding
# decide differently; they stay local, which the percentile shows.
SEMI_TOL = {"max": {"x": 1e-4, "u": 5e-3, "p": 2e-2, "n": 3e-3},
            "p99": {"x": 1e-6, "u": 5e-4, "p": 2e-3, "n": 5e-5}}
# the explicit pressure is the equation of state rho c^2 (n - n0) / n0, which
# turns the FP32 rounding of n into pressure and velocity differences
# (measured p99 at steps 25-100: u 6.1e-4 - 7.1e-4, p 1.0e-3 - 1.8e-3)
EXPL_TOL = {"max": {"x": 1e-4, "u": 5e-3, "p": 2e-2, "n": 3e-3},
            "p99": {"x": 1e-6, "u": 2e-3, "p": 5e-3, "n": 5e-5}}
CHECK_STEPS = (25, 50, 100)


def _by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def field_errors(gpu, ref):
    """|gpu - ref| / scale per field (particles matched by id): the largest
    over all particles, and the median, 99th percentile and count above
    1e-5 over the fluid particles."""
    a, b = _by_id(gpu), _by_id(ref)
    assert np.array_equal(a["id"], b["id"]) and np.array_equal(a["type"], b["type"])
    fluid = b["type"] == 0
    out = {}
    lo, hi = b["pos"].min(axis=0), b["pos"].max(axis=0)
    ext = float((hi - lo).max())
    for key, f, scale in (("x", "pos", ext), ("u", "vel", None), ("p", "press", None), ("n", "n", None)):
        x = np.asarray(a[f], np.float64)
        y = np.asarray(b[f], np.float64)
        d = np.abs(x - y)
        if d.ndim == 2:
            d = d.max(axis=1)
        s = scale if scale is not None else float(np.abs(y).max())
        s = s if s > 0 else 1.0
        df = d[fluid] / s
        out[key] = {"max": float(d.max() / s), "median": float(np.median(df)),
                    "p99": float(np.percentile(df, 99)), "above_1e-5": int((df > 1e-5).sum())}
    return out


def _assert_within(rep, tol):
    for k in CHECK_STEPS:
        for kind in ("max", "p99"):
            for f, t in tol[kind].items():
                assert rep[str(k)][f][kind] < t, (k, f, kind, rep[str(k)][f])


def _report(name, data):
    path = os.environ.get("MPS_PARITY_REPORT")
    print(f"\n{name}: {json.dumps(data)}")
    if not path:
        return
    allr = {}
    if os.path.exists(path):
        with open(path) as fh:
            allr = json.load(fh)
    allr[name] = data
    with open(path, "w") as fh:
        json.dump(allr, fh, indent=1)


def _input_values(case_dir):
    """The 16 values of input.dat as float32 (the reference parses them with
    %f), r0 / rlap / col_dis scaled by dp in float as MPS::loadCase does."""
    with open(os.path.join(case_dir, "input.dat")) as fh:
        lines = [ln.strip() for ln in fh if ln.strip()]
    vals = [np.float32(float(lines[2 * k + 1])) for k in range(16)]
    dp = vals[3]
    return {"dp": dp, "rzero": np.float32(vals[4] * dp), "rlap": np.float32(vals[5] * dp), "beta": vals[6]}


def reference_ppe_pairs(pos4, n, n0, beta, rlap):
    """Rows and off-diagonal pairs of buildPoisson (MPS_CAL_v4.0/MPS_CPU.cpp:
    651-698) from float positions, in the reference's float arithmetic.
    Returns (is_row bool array, sorted int64 codes i * np + j)."""
    from scipy.spatial import cKDTree
    npart = len(pos4)
    typ = pos4[:, 3].view(np.uint32)
    is_row = (typ != 2) & ~(n.astype(np.float64) < float(beta) * float(n0))
    rows = np.nonzero(is_row)[0]
    p = pos4[rows, :3]
    tree = cKDTree(p.astype(np.float64))
    cand = tree.query_pairs(float(rlap) * (1 + 1e-5), output_type="ndarray")
    a, b = rows[cand[:, 0]], rows[cand[:, 1]]
    d = pos4[b, :3] - pos4[a, :3]  # float32 subtractions
    rr = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    r = np.sqrt(rr.astype(np.float64)).astype(np.float32)
    with np.errstate(divide="ignore"):
        w = np.where(r < rlap, (rlap / r).astype(np.float32) - np.float32(1.0), np.float32(0.0))
    keep = w != 0
    a, b = a[keep].astype(np.int64), b[keep].astype(np.int64)
    codes = np.concatenate([a * npart + b, b * npart + a])
    codes.sort()
    return is_row, codes


def gpu_ppe_pairs(sim):
    st = sim.ppe_stencil()
    npart = len(st["row_start"]) - 1
    cnt = np.diff(st["row_start"].astype(np.int64))
    i = np.repeat(np.arange(npart, dtype=np.int64), cnt)
    codes = i * npart + st["cols"].astype(np.int64)
    codes.sort()
    return codes, st


def _check_pairs(sim, case_dir, tag):
    snap = sim.ppe_snapshot()
    iv = _input_values(case_dir)
    n0 = sim.scalars()["nzero"]
    is_row, want = reference_ppe_pairs(snap["pos4"], snap["n"], n0, iv["beta"], iv["rlap"])
    got, st = gpu_ppe_pairs(sim)
    gpu_rows = snap["is_row"].astype(bool)
    assert np.array_equal(gpu_rows, is_row), f"{tag}: solved rows differ at {np.nonzero(gpu_rows != is_row)[0][:10]}"
    extra = np.setdiff1d(got, want)
    missing = np.setdiff1d(want, got)
    _report(f"ppe_pairs_{tag}", {"rows": int(is_row.sum()), "pairs": int(len(want)), "extra": int(len(extra)),
                                 "missing": int(len(missing))})
    assert len(extra) == 0 and len(missing) == 0, (tag, len(extra), len(missing), extra[:5], missing[:5])
    assert np.array_equal(got, want)
    # every row's columns ascend (the reference's summation order)
    rs = st["row_start"].astype(np.int64)
    c = st["cols"].astype(np.int64)
    inner = np.ones(len(c), bool)
    inner[rs[:-1][rs[:-1] < len(c)]] = False
    assert np.all(np.diff(c)[inner[1:]] > 0)


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_ppe_neighbour_sets_bit_exact_golden(capi, tmp_path, arith):
    from helpers import load_golden, write_golden_case
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    mode = capi.ARITH_EXACT if arith == "exact" else capi.ARITH_FAST
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=mode) as s:
        for k in range(3):
            s.step(2)
            _check_pairs(s, d, f"golden_{arith}_step{2 * k + 2}")


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_ppe_neighbour_sets_bit_exact_full_size(capi, tmp_path, arith):
    """The benchmark's 310,912-particle scene after 1 and 20 steps."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "c2")
    scene.write_case(d, scene.dam_break_semi())
    mode = capi.ARITH_EXACT if arith == "exact" else capi.ARITH_FAST
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=mode) as s:
        s.step(1)
        _check_pairs(s, d, f"c2_{arith}_step1")
        s.step(19)
        _check_pairs(s, d, f"c2_{arith}_step20")


def test_semi_dam_break_100_steps_vs_fp64_oracle(capi, oracle_mod, tmp_path):
    """The benchmark's workload, as benchmarked (fast arithmetic, PPE to 1e-8
    FP64 relative residual), against the FP64 oracle (CG to 1e-12) over the
    first 100 steps; errors reported at steps 25, 50 and 100."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "c2")
    scene.write_case(d, scene.dam_break_semi())
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    rep = {}
    iters = []
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=capi.ARITH_FAST) as s:
        done = 0
        for k in CHECK_STEPS:
            while done < k:
                st = s.step(1)
                orc.step(1)
                assert st.cg_relres <= 1e-8 and st.status == 0
                iters.append((st.cg_iters, orc.cg_iters()))
                done += 1
            rep[str(k)] = field_errors(s.state(), orc.state())
    rep["cg_iters_gpu_mean"] = float(np.mean([a for a, _ in iters]))
    rep["cg_iters_oracle_mean"] = float(np.mean([b for _, b in iters]))
    rep["tolerance"] = SEMI_TOL
    _report("semi_c2_100_steps", rep)
    _assert_within(rep, SEMI_TOL)


def test_explicit_dam_break_100_steps_fp64_error(capi, oracle_mod, tmp_path):
    """The explicit 70,912-particle dam break: the GPU equals the reference's
    float build bit for bit (tests/test_gpu_explicit.py); its distance to an
    FP64 run of the same rules over 100 steps is reported and bounded."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "c1")
    scene.write_case(d, scene.dam_break_explicit())
    orc64 = oracle_mod.Oracle(d, oracle_mod.EXPL, 64)
    rep = {}
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        done = 0
        for k in CHECK_STEPS:
            s.step(k - done)
            orc64.step(k - done)
            done = k
            rep[str(k)] = field_errors(s.state(), orc64.state())
    rep["tolerance"] = EXPL_TOL
    _report("explicit_c1_100_steps_vs_fp64", rep)
    _assert_within(rep, EXPL_TOL)
