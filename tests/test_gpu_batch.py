"""Batches of scenes and the tank-acceleration body force on the GPU.

A batch steps several scenes of different sizes as one particle set; each
scene must evolve exactly as it does in its own handle:

* explicit, exact arithmetic: bit for bit, per scene, against single-scene
  handles -- and a single-scene handle with a body force bit for bit against
  the float oracle with the same body force (so the batch is pinned to the
  oracle through it);
* semi-implicit: within the FP64-CG tolerance of single-scene handles (each
  scene runs its own PCG inside one persistent launch), and a single-scene
  handle with a body force within the stated tolerances of the FP64 oracle.
"""
import numpy as np
import pytest

from helpers import assert_bitwise, rel_err

pytestmark = pytest.mark.gpu

# scenes of different sizes, shapes and tank accelerations (m/s^2, Hz)
SCENES = [dict(seed=1, interior=(14, 6, 12), fluid=(5, 4, 8)),
          dict(seed=2, interior=(10, 5, 10), fluid=(4, 3, 6)),
          dict(seed=3, interior=(18, 6, 10), fluid=(7, 4, 5))]
ACCEL = [(0.0, 0.0), (1.5, 1.0), (2.0, 2.0)]


def write_scenes(tmp_path, dt):
    from mps_solvers_b200 import scene
    dirs = []
    for k, kw in enumerate(SCENES):
        d = str(tmp_path / f"scene{k}")
        scene.write_case(d, scene.small_tank(dt=dt, **kw))
        dirs.append(d)
    return dirs


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def scene_slice(state, info):
    """The by-id rows of one scene of a batch, ids made scene-local."""
    sl = slice(info.id_base, info.id_base + info.np0)
    out = {k: v[sl] for k, v in state.items()}
    out["id"] = out["id"] - info.id_base
    return out


def test_explicit_batch_equals_single_scenes_bitwise(capi, tmp_path):
    dirs = write_scenes(tmp_path, 1e-4)
    steps = 40
    with capi.Simulation.batch(dirs, accel=ACCEL, method=capi.METHOD_EXPLICIT) as b:
        b.step(steps)
        whole = b.state(capi.ORDER_BY_ID)
        infos = [b.scene_info(s) for s in range(len(dirs))]
    for s, d in enumerate(dirs):
        with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as one:
            one.set_body_force(*ACCEL[s])
            one.step(steps)
            want = one.state(capi.ORDER_BY_ID)
            want_info = one.scene_info(0)
        got = scene_slice(whole, infos[s])
        for f in ("id", "type", "pos", "vel", "press", "n"):
            assert_bitwise(got[f], want[f], f"scene {s} {f}")
        assert np.float32(infos[s].time) == np.float32(want_info.time)
        assert np.float32(infos[s].nzero) == np.float32(want_info.nzero)


def test_body_force_bitwise_vs_oracle(capi, oracle_mod, tmp_path):
    dirs = write_scenes(tmp_path, 1e-4)
    amp, freq = 2.0, 2.0
    with capi.Simulation(dirs[2], method=capi.METHOD_EXPLICIT) as s:
        s.set_body_force(amp, freq)
        s.step(40)
        got = by_id(s.state())
    orc = oracle_mod.Oracle(dirs[2], oracle_mod.EXPL, 32)
    orc.set_body_force(amp, freq)
    assert orc.step(40) == 0
    want = by_id(orc.state())
    for f in ("id", "type", "pos", "vel", "press", "n"):
        assert_bitwise(got[f], want[f], f)
    # and the term acts: without it the state differs
    with capi.Simulation(dirs[2], method=capi.METHOD_EXPLICIT) as s:
        s.step(40)
        plain = by_id(s.state())
    assert not np.array_equal(plain["vel"], got["vel"])


def test_semi_batch_matches_single_scenes(capi, tmp_path):
    dirs = write_scenes(tmp_path, 5e-4)
    steps = 8
    with capi.Simulation.batch(dirs, accel=ACCEL, method=capi.METHOD_SEMI_IMPLICIT) as b:
        for _ in range(steps):
            st = b.step(1)
            assert st.status == 0 and st.cg_relres <= 1e-8
            for s in range(len(dirs)):
                info = b.scene_info(s)
                assert info.cg_relres <= 1e-8 and info.cg_iters > 0
        whole = b.state(capi.ORDER_BY_ID)
        infos = [b.scene_info(s) for s in range(len(dirs))]
    for s, d in enumerate(dirs):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as one:
            one.set_body_force(*ACCEL[s])
            one.step(steps)
            want = one.state(capi.ORDER_BY_ID)
        got = scene_slice(whole, infos[s])
        assert np.array_equal(got["id"], want["id"]) and np.array_equal(got["type"], want["type"])
        ext = np.abs(want["pos"]).max()
        assert np.abs(got["pos"] - want["pos"]).max() / ext < 1e-7
        assert rel_err(got["vel"], want["vel"]) < 1e-5
        assert rel_err(got["press"], want["press"]) < 1e-5


def test_semi_body_force_vs_fp64_oracle(capi, oracle_mod, tmp_path):
    dirs = write_scenes(tmp_path, 5e-4)
    amp, freq = 2.0, 2.0
    orc = oracle_mod.Oracle(dirs[0], oracle_mod.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-12, 100000)
    orc.set_body_force(amp, freq)
    with capi.Simulation(dirs[0], method=capi.METHOD_SEMI_IMPLICIT) as s:
        s.set_body_force(amp, freq)
        for _ in range(8):
            assert s.step(1).cg_relres <= 1e-8
            assert orc.step(1) == 0
        a, b = by_id(s.state()), by_id(orc.state())
    ext = np.abs(b["pos"]).max()
    assert np.abs(a["pos"] - b["pos"]).max() / ext < 1e-6
    assert rel_err(a["vel"], b["vel"]) < 1e-3
    assert rel_err(a["press"], b["press"]) < 2e-3


def test_batch_scene_table(capi, tmp_path):
    dirs = write_scenes(tmp_path, 1e-4)
    with capi.Simulation.batch(dirs, method=capi.METHOD_EXPLICIT) as b:
        base = 0
        for s, d in enumerate(dirs):
            info = b.scene_info(s)
            with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as one:
                c = one.counts()
            assert info.id_base == base and info.np0 == c["np"]
            assert info.nb2 == c["nb2"] and info.nb1 == c["nb1"]
            base += info.np0
        assert b.counts()["np"] == base
        with pytest.raises(capi.MPSError):
            b.scene_info(len(dirs))
        with pytest.raises(capi.MPSError):
            b.run(None)


def test_learned_batch_matches_single_scenes(capi, tmp_path):
    """The learned S' inside the batched PCG (particle columns, one product
    fused into the residual update, each scene's own alpha): every scene
    converges to 1e-8 in fewer iterations than with diagonal scaling and
    evolves within the solve tolerance of its own learned single-scene
    handle."""
    from mps_solvers_b200 import precond_weights
    wts = precond_weights.load()
    dirs = write_scenes(tmp_path, 5e-4)
    steps = 4
    iters = {}
    for pc in (capi.PRECOND_DIAGONAL, capi.PRECOND_LEARNED):
        with capi.Simulation.batch(dirs, accel=ACCEL, method=capi.METHOD_SEMI_IMPLICIT, precond=pc) as b:
            if pc == capi.PRECOND_LEARNED:
                b.set_precond_params(wts)
            its = np.zeros(len(dirs))
            for _ in range(steps):
                st = b.step(1)
                assert st.status == 0 and st.cg_relres <= 1e-8
                for s in range(len(dirs)):
                    info = b.scene_info(s)
                    assert info.cg_relres <= 1e-8 and info.cg_iters > 0
                    its[s] += info.cg_iters
            iters[pc] = its
            if pc == capi.PRECOND_LEARNED:
                whole = b.state(capi.ORDER_BY_ID)
                infos = [b.scene_info(s) for s in range(len(dirs))]
    assert np.all(iters[capi.PRECOND_LEARNED] < iters[capi.PRECOND_DIAGONAL]), iters
    for s, d in enumerate(dirs):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, precond=capi.PRECOND_LEARNED) as one:
            one.set_precond_params(wts)
            one.set_body_force(*ACCEL[s])
            one.step(steps)
            want = one.state(capi.ORDER_BY_ID)
        got = scene_slice(whole, infos[s])
        ext = np.abs(want["pos"]).max()
        assert np.abs(got["pos"] - want["pos"]).max() / ext < 1e-7
        assert rel_err(got["vel"], want["vel"]) < 1e-5
        assert rel_err(got["press"], want["press"]) < 1e-5
