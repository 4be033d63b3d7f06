"""Crank-Nicolson viscosity (the reference's MPS_CPU_IMPL step) on the GPU
against the FP64 CPU oracle: three persistent-PCG solves per step, one per
velocity component, then the semi-implicit pressure step."""
import numpy as np
import pytest

from helpers import assert_bitwise, rel_err

pytestmark = pytest.mark.gpu


def case(tmp_path, niu, dt=5e-4):
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=1, dt=dt)
    sc.params.niu = niu
    d = str(tmp_path / f"tank_{niu}")
    scene.write_case(d, sc)
    return d


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


@pytest.mark.parametrize("niu", [1e-2, 1.0])
def test_cn_vs_fp64_oracle(capi, oracle_mod, tmp_path, niu):
    d = case(tmp_path, niu)
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    orc.set_visc_implicit(True)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, visc_implicit=1) as s:
        for _ in range(8):
            st = s.step(1)
            assert st.status == 0 and st.cg_relres <= 1e-8
            assert orc.step(1) == 0
        a, b = by_id(s.state()), by_id(orc.state())
    ext = np.abs(b["pos"]).max()
    assert np.abs(a["pos"] - b["pos"]).max() / ext < 1e-6
    assert rel_err(a["vel"], b["vel"]) < 1e-3
    assert rel_err(a["press"], b["press"]) < 2e-3
    if niu >= 1.0:  # far past the explicit form's stability limit, and calm
        assert np.abs(a["vel"][a["type"] == 0]).max() < 0.01


def test_cn_graph_replay_bitwise(capi, tmp_path):
    d = case(tmp_path, 1e-2)
    out = []
    for g in (1, 0):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, visc_implicit=1, use_graph=g) as s:
            s.step(6)
            out.append(by_id(s.state()))
    for f in ("pos", "vel", "press", "n"):
        assert_bitwise(out[0][f], out[1][f], f)


def test_cn_differs_from_explicit_only_by_viscosity(capi, tmp_path):
    d = case(tmp_path, 1e-6)
    res = []
    for v in (1, 0):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, visc_implicit=v) as s:
            s.step(6)
            res.append(by_id(s.state()))
    f = res[0]["type"] == 0
    assert rel_err(res[0]["vel"][f], res[1]["vel"][f]) < 1e-3


def test_cn_needs_semi_single_scene(capi, tmp_path):
    d = case(tmp_path, 1e-2)
    with pytest.raises(capi.MPSError):
        capi.Simulation(d, method=capi.METHOD_EXPLICIT, visc_implicit=1)
    with pytest.raises(capi.MPSError):
        capi.Simulation.batch([d, d], method=capi.METHOD_SEMI_IMPLICIT, visc_implicit=1)


def test_cn_vs_reference_golden(capi, tmp_path):
    """Against the reference's own MPS_CPU_IMPL build (MPS_CAL_v4.0, double,
    dense CG, sequential collision), 6 steps at niu = 0.01, within the
    semi-implicit tolerances."""
    from helpers import load_golden, write_golden_case
    g = load_golden("impl_tank")
    d = write_golden_case(g, str(tmp_path / "impl"))
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, visc_implicit=1) as s:
        s.step(6)
        a = by_id(s.state())
    b = by_id({f: g[f"s6_{f}"] for f in ("id", "type", "pos", "vel", "press", "n")})
    assert np.array_equal(a["id"], b["id"]) and np.array_equal(a["type"], b["type"])
    ext = np.abs(b["pos"]).max()
    assert np.abs(a["pos"] - b["pos"]).max() / ext < 1e-6
    assert rel_err(a["vel"], b["vel"]) < 1e-3
    assert rel_err(a["press"], b["press"]) < 2e-3
