"""Crank-Nicolson viscosity in the CPU oracle (the checker of the GPU path):
it agrees with the explicit viscosity where viscosity is weak and stays
stable where the explicit form blows up."""
import numpy as np

from mps_solvers_b200 import scene


def run(oracle_mod, tmp_path, niu, cn, steps=10):
    sc = scene.small_tank(seed=1, dt=5e-4)
    sc.params.niu = niu
    d = str(tmp_path / f"tank_{niu}_{int(cn)}")
    scene.write_case(d, sc)
    o = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    o.set_cg(True, 1e-12, 100000)
    o.set_visc_implicit(cn)
    st = o.step(steps)
    s = o.state()
    k = np.argsort(s["id"], kind="stable")
    return st, {f: v[k] for f, v in s.items()}


def test_weak_viscosity_matches_explicit(oracle_mod, tmp_path):
    sa, a = run(oracle_mod, tmp_path, 1e-6, True)
    sb, b = run(oracle_mod, tmp_path, 1e-6, False)
    assert sa == 0 and sb == 0
    f = a["type"] == 0
    scale = np.abs(b["vel"][f]).max()
    assert np.abs(a["vel"][f] - b["vel"][f]).max() < 1e-4 * scale
    assert np.abs(a["pos"][f] - b["pos"][f]).max() < 1e-8


def test_strong_viscosity_stays_stable(oracle_mod, tmp_path):
    st, a = run(oracle_mod, tmp_path, 1.0, True)
    assert st == 0
    f = a["type"] == 0
    assert np.isfinite(a["vel"]).all() and np.abs(a["vel"][f]).max() < 0.01
    # the explicit form is past its stability limit here (niu dt / l0^2 > 1)
    st_e, b = run(oracle_mod, tmp_path, 1.0, False)
    assert st_e != 0 or np.abs(b["vel"][f]).max() > 1.0
