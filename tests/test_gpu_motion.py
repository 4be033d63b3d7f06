"""Prescribed boundary motion on the GPU against the CPU oracle.

A piston (the x-min wall and dummy layers) oscillates and drifts while the
fluid responds:

* explicit, exact arithmetic: bit for bit against the float oracle, with and
  without CUDA graphs, across a stop (mps_clear_wall_motion);
* semi-implicit: within the stated tolerances of the FP64 oracle.
"""
import numpy as np
import pytest

from helpers import assert_bitwise, rel_err

pytestmark = pytest.mark.gpu

VEL, AMP, FREQ, PHASE = (0.01, 0.0, 0.0), (0.004, 0.0, 0.002), 5.0, 0.3


def case(tmp_path, dt):
    from mps_solvers_b200 import scene
    d = str(tmp_path / "tank")
    scene.write_case(d, scene.small_tank(seed=1, dt=dt))
    return d


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def piston_box(st):
    xf = st["pos"][st["type"] == 0][:, 0].min()
    return (-1.0, -1.0, -1.0), (float(xf) - 0.05, 10.0, 10.0)


@pytest.mark.parametrize("use_graph", [1, 0])
def test_explicit_motion_bitwise_vs_oracle(capi, oracle_mod, tmp_path, use_graph):
    d = case(tmp_path, 1e-4)
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT, use_graph=use_graph) as s:
        s.step(5)
        assert orc.step(5) == 0
        lo, hi = piston_box(by_id(s.state()))
        n = s.add_wall_motion(lo, hi, VEL, AMP, FREQ, PHASE)
        assert n == orc.add_wall_motion(lo, hi, VEL, AMP, FREQ, PHASE) > 0
        s.step(40)
        assert orc.step(40) == 0
        got, want = by_id(s.state()), by_id(orc.state())
        for f in ("id", "type", "pos", "vel", "press", "n"):
            assert_bitwise(got[f], want[f], f)
        s.clear_wall_motion()
        orc.clear_wall_motion()
        s.step(10)
        assert orc.step(10) == 0
        got, want = by_id(s.state()), by_id(orc.state())
        for f in ("id", "type", "pos", "vel", "press", "n"):
            assert_bitwise(got[f], want[f], f"after stop: {f}")
    # the motion acts: without it the fluid differs
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT, use_graph=use_graph) as s:
        s.step(55)
        plain = by_id(s.state())
    assert not np.array_equal(plain["vel"][plain["type"] == 0], got["vel"][got["type"] == 0])


def test_semi_motion_vs_fp64_oracle(capi, oracle_mod, tmp_path):
    d = case(tmp_path, 5e-4)
    orc = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        lo, hi = piston_box(by_id(s.state()))
        assert s.add_wall_motion(lo, hi, VEL, AMP, FREQ, PHASE) == orc.add_wall_motion(lo, hi, VEL, AMP, FREQ,
                                                                                       PHASE)
        for _ in range(8):
            assert s.step(1).cg_relres <= 1e-8
            assert orc.step(1) == 0
        a, b = by_id(s.state()), by_id(orc.state())
    ext = np.abs(b["pos"]).max()
    assert np.abs(a["pos"] - b["pos"]).max() / ext < 1e-6
    assert rel_err(a["vel"], b["vel"]) < 1e-3
    assert rel_err(a["press"], b["press"]) < 2e-3


def test_motion_limits(capi, tmp_path):
    d = case(tmp_path, 1e-4)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        box = ((-1.0, -1.0, -1.0), (10.0, 10.0, 10.0))
        assert s.add_wall_motion(*box) > 0          # every boundary particle, at rest
        for _ in range(7):
            assert s.add_wall_motion(*box) == 0     # nobody left to take
        with pytest.raises(capi.MPSError):
            s.add_wall_motion(*box)                 # the ninth motion
