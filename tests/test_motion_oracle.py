"""Prescribed boundary motion in the CPU oracle (the checker of the GPU
path): the motion law, the selection and the stop, on a small tank."""
import numpy as np

from mps_solvers_b200 import scene


def case(tmp_path, dt=1e-4):
    d = str(tmp_path / "tank")
    scene.write_case(d, scene.small_tank(seed=1, dt=dt))
    return d


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def piston_box(st):
    """The x-min wall and dummy layers (everything left of the fluid)."""
    xf = st["pos"][st["type"] == 0][:, 0].min()
    return (-1.0, -1.0, -1.0), (xf - 0.05, 10.0, 10.0)


def test_motion_law_and_selection(oracle_mod, tmp_path):
    o = oracle_mod.Oracle(case(tmp_path), oracle_mod.EXPL, 32)
    s0 = by_id(o.state())
    lo, hi = piston_box(s0)
    inside = np.all((s0["pos"] >= np.float32(lo)) & (s0["pos"] <= np.float32(hi)), axis=1)
    want_sel = inside & ((s0["type"] == 1) | (s0["type"] == 2))
    vel, amp, freq, phase = (0.01, 0.0, 0.0), (0.004, 0.0, 0.002), 5.0, 0.3
    assert o.add_wall_motion(lo, hi, vel, amp, freq, phase) == int(want_sel.sum()) > 0
    # a second motion over the same box takes nobody
    assert o.add_wall_motion(lo, hi, amp=(0.0, 0.0, 0.001), freq=1.0) == 0
    steps = 25
    assert o.step(steps) == 0
    # the law holds at the start of the last step (time before its dt was added)
    t_last = float(o.scalars()["time"]) - float(o.scalars()["dt"])
    s1 = by_id(o.state())
    tau = float(np.float32(t_last))
    v32, a32 = np.float32(vel).astype(np.float64), np.float32(amp).astype(np.float64)
    om, ph = 2 * np.pi * float(np.float32(freq)), float(np.float32(phase))
    x = (s0["pos"][want_sel].astype(np.float64) + v32 * tau + a32 * (np.sin(om * tau + ph) - np.sin(ph)))
    u = v32 + a32 * om * np.cos(om * tau + ph)
    assert np.array_equal(s1["pos"][want_sel], x.astype(np.float32))
    assert np.array_equal(s1["vel"][want_sel], np.broadcast_to(u.astype(np.float32), x.shape))
    # walls outside the box stay put
    still = (s0["type"] != 0) & ~want_sel
    assert np.array_equal(s1["pos"][still], s0["pos"][still])


def test_clear_stops_and_rests(oracle_mod, tmp_path):
    o = oracle_mod.Oracle(case(tmp_path), oracle_mod.EXPL, 32)
    s0 = by_id(o.state())
    lo, hi = piston_box(s0)
    o.add_wall_motion(lo, hi, amp=(0.004, 0.0, 0.0), freq=5.0)
    assert o.step(10) == 0
    o.clear_wall_motion()
    s1 = by_id(o.state())
    assert o.step(5) == 0
    s2 = by_id(o.state())
    walls = s0["type"] != 0
    assert np.array_equal(s2["pos"][walls], s1["pos"][walls])
    assert not np.array_equal(s1["pos"][walls], s0["pos"][walls])
    assert np.all(s2["vel"][walls] == 0)
