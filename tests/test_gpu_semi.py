"""Semi-implicit step (PPE + CG) on the GPU through the C ABI.

The GPU keeps particles in float (FP32 sums and SpMV) and solves the PPE to
|b - Ax| <= 1e-8 |b| measured in FP64 (defect correction); the oracle runs
the same two-phase rules in double with CG to 1e-12.  Stated tolerances,
relative to each field's largest magnitude after 8 steps: pressure 2e-3,
velocity 1e-3, positions 1e-6 of the domain size.
"""
import numpy as np
import pytest

from helpers import load_golden, rel_err, write_golden_case

pytestmark = pytest.mark.gpu

P_TOL, U_TOL, X_TOL = 2e-3, 1e-3, 1e-6


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def compare(a, b):
    a, b = by_id(a), by_id(b)
    assert np.array_equal(a["id"], b["id"])
    assert np.array_equal(a["type"], b["type"])
    ext = np.abs(b["pos"]).max()
    ex = np.abs(a["pos"] - b["pos"]).max() / ext
    ep = rel_err(a["press"], b["press"])
    eu = rel_err(a["vel"], b["vel"])
    return ex, eu, ep


def test_semi_steps_vs_fp64_oracle(capi, oracle_mod, tmp_path):
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        for k in range(8):
            st = s.step(1)
            orc.step(1)
            assert st.cg_relres <= 1e-8 and st.cg_iters > 0
        ex, eu, ep = compare(s.state(), orc.state())
        assert orc.state()["press"].max() > 100.0
    assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)


def test_semi_steps_vs_reference_golden(capi, tmp_path):
    """Against the reference's own sequential build (MPS_CAL_v4.0, double,
    dense CG): the two-phase form differs from it by ~2e-5 in velocity (see
    tests/test_oracle_golden.py), within the same stated tolerances."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        s.step(8)
        a = s.state()
    ref = {f: g[f"s8_{f}"] for f in ("id", "type", "pos", "vel", "press", "n")}
    ex, eu, ep = compare(a, ref)
    assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)


def test_ppe_solution_meets_fp64_tolerance_and_is_reproducible(capi, tmp_path):
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    out = []
    for _ in range(2):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, cg_tol=1e-10) as s:
            st = s.step(6)
            assert st.cg_relres <= 1e-10
            out.append(s.state())
    for f in ("pos", "vel", "press"):
        assert np.array_equal(out[0][f], out[1][f]), f


def test_cg_not_converged_is_reported(capi, tmp_path):
    """An iteration limit too small for the tolerance returns
    MPS_ERR_CG_NOT_CONVERGED instead of a silent result."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, cg_max_iter=2) as s:
        s.step(5, check=False)
        st = s.step(1, check=False)
        assert st.status == 5


def test_full_size_semi_dam_break(capi, oracle_mod, tmp_path):
    """310,912-particle semi-implicit dam break: 2 steps against the FP64
    oracle (same tolerances), then 20 more steps converging every PPE."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "c2")
    scene.write_case(d, scene.dam_break_semi())
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        for _ in range(2):
            st = s.step(1)
            orc.step(1)
            assert st.cg_relres <= 1e-8
        ex, eu, ep = compare(s.state(), orc.state())
        assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)
        for _ in range(20):
            st = s.step(1)
            assert st.cg_relres <= 1e-8 and st.status == 0
        a = s.state()
        assert np.isfinite(a["press"]).all() and a["press"].min() >= 0.0


def test_semi_graph_replay_equals_direct_launches(capi, tmp_path):
    """The semi-implicit step (with its cooperative PPE launch) replays as a
    captured CUDA graph, with the same results as direct launches."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    out = []
    for use_graph in (1, 0):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, use_graph=use_graph) as s:
            s.step(6)
            assert s.scalars()["graph"] == use_graph
            out.append(s.state())
    for f in ("pos", "vel", "press"):
        assert np.array_equal(out[0][f], out[1][f]), f


def test_fast_arith_is_reproducible_run_to_run(capi, tmp_path):
    """Fast arithmetic (refined cells, two fluid particles a warp in the
    viscosity) gives the same bits in every run, with and without the CUDA
    graph: the gathers' list order varies from run to run, but the pairs the
    viscosity forms do not (each gather warp's fluid run is padded to an
    even length).  A 70-step window of the 310,912-particle dam break
    measured the same on the GPU."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "t")
    scene.write_case(d, scene.small_tank(seed=5, interior=(40, 16, 30), fluid=(16, 12, 20), l0=0.01, dt=5e-4))
    out = []
    for use_graph in (1, 1, 0):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=capi.ARITH_FAST,
                             use_graph=use_graph) as s:
            s.step(12)
            out.append(s.state(capi.ORDER_BY_ID))
    for o in out[1:]:
        for f in ("pos", "vel", "press", "n"):
            assert np.array_equal(out[0][f], o[f]), f


def test_pipelined_pcg_matches_fp64_oracle(capi, oracle_mod, tmp_path):
    """The single-reduction pipelined PCG reaches the same FP64 tolerance and
    the same state as the standard form, within the stated tolerances."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, ppe_pipelined=1) as s:
        for k in range(8):
            st = s.step(1)
            orc.step(1)
            assert st.cg_relres <= 1e-8 and st.cg_iters > 0
        ex, eu, ep = compare(s.state(), orc.state())
    assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)


def test_l2_residency_hints_change_no_result(capi, tmp_path):
    """The stencil's L2 policy (evict_last head, evict_first tail, or plain
    loads) only moves data between cache and DRAM: states agree bit for bit."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    out = []
    for keep in (0, -1, 1):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, ppe_l2_keep_mb=keep) as s:
            assert s.step(6).cg_relres <= 1e-8
            out.append(s.state())
    for o in out[1:]:
        for f in ("pos", "vel", "press", "n"):
            assert np.array_equal(out[0][f], o[f]), f


def test_semi_fast_arith_vs_fp64_oracle(capi, oracle_mod, tmp_path):
    """The fast arithmetic the benchmark runs (FMA contraction, two fluid
    particles per warp in the viscosity stage) within the same tolerances of
    the FP64 oracle as the exact kernels."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=capi.ARITH_FAST) as s:
        for k in range(8):
            st = s.step(1)
            orc.step(1)
            assert st.cg_relres <= 1e-8 and st.cg_iters > 0
        ex, eu, ep = compare(s.state(), orc.state())
    assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)


def test_device_wait_timeout_is_reported_and_handle_survives(capi, tmp_path):
    """A grid-wide wait limit of 1 ns makes the persistent PPE solver's
    barriers give up before the other blocks arrive: every block returns, the
    step reports MPS_ERR_DEVICE_TIMEOUT (6) instead of hanging or faulting,
    the handle still answers its getters and is destroyed cleanly, and a new
    handle on the same device solves normally."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    s = capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT)
    assert s.step(2).status == 0
    s.set_device_wait_limit(1)
    st = s.step(1, check=False)
    assert st.status == 6
    with pytest.raises(capi.MPSError):
        s.step(1)
    c = s.counts()
    assert c["np"] > 0
    a = s.state()
    assert len(a["id"]) == c["np"]
    s.set_device_wait_limit(0)
    s.close()
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s2:
        st = s2.step(3)
        assert st.status == 0 and st.cg_relres <= 1e-8
