"""Explicit (EOS) step on the GPU through the C ABI, against the reference.

Exact arithmetic must reproduce the reference's float results bit for bit:
the golden fixtures come from the reference's own CPU build, and every other
case is checked against the oracle, which is itself pinned to that build.
"""
import os

import numpy as np
import pytest

from helpers import assert_bitwise, load_golden, rel_err, write_golden_case

pytestmark = pytest.mark.gpu

FIELDS = ("id", "type", "pos", "vel", "press", "n")


def sim_from(capi, d, **kw):
    return capi.Simulation(d, method=capi.METHOD_EXPLICIT, **kw)


def test_initial_state_matches_reference(capi, oracle_mod, tmp_path):
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    with sim_from(capi, d) as s:
        sc = s.scalars()
        assert np.float32(sc["nzero"]) == np.float32(g["nzero"])
        assert np.float32(sc["lambda"]) == np.float32(g["lambda_"])
        cell_of, start, end = s.cell_tables()
        assert_bitwise(cell_of, g["cell_of"], "cell_of")
        assert_bitwise(start, g["cell_start"], "cell_start")
        assert_bitwise(end, g["cell_end"], "cell_end")
        st = s.state()
        for f in FIELDS:
            if f in ("n",):
                continue  # the reference stores n0's scan in n; compared below
            assert_bitwise(st[f], g[f"s0_{f}"], f"initial {f}")
        assert_bitwise(st["n"], g["s0_n"], "initial n")
        # dummy-to-wall map: oracle's i_normal (sorted indices) as GEO indices
        orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
        ost = orc.state()
        onorm = orc.normal()
        ids = ost["id"]
        want = ids.copy()
        t2 = ost["type"] == 2
        want[t2] = ids[onorm[t2]]
        got = s.normal_ids()[ids]
        assert np.array_equal(got, want)


@pytest.mark.parametrize("use_graph", [1, 0])
def test_steps_bit_exact_vs_reference_golden(capi, tmp_path, use_graph):
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    with sim_from(capi, d, use_graph=use_graph) as s:
        done = 0
        for k in g["steps"][1:]:
            stats = s.step(int(k) - done)
            done = int(k)
            st = s.state()
            for f in FIELDS:
                assert_bitwise(st[f], g[f"s{k}_{f}"], f"step {k} {f}")
            assert np.float32(stats.dt) == np.float32(g[f"s{k}_dt"])
            assert np.float32(stats.time) == np.float32(g[f"s{k}_time"])


def test_stagewise_bit_exact_vs_oracle(capi, oracle_mod, tmp_path):
    """Each stage alone from the same state: visc, divideCell, collision,
    cal_n, EOS, gradient."""
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    with sim_from(capi, d) as s:
        s.step(25)
        orc.step(25)
        seq = ["update_dt", "visc", "divide_cell", "collision", "divide_cell", "cal_n", "pres_expl",
               "dash", "divide_cell"]
        for ph in seq:
            s.phase(ph)
            orc.phase(ph)
            if ph in ("visc", "collision", "dash"):
                continue  # pending update: compared after the divideCell that applies it
            a, b = s.state(), orc.state()
            for f in FIELDS:
                assert_bitwise(a[f], b[f], f"after {ph}: {f}")
            c1, s1, e1 = s.cell_tables()
            c2, s2, e2 = orc.cells()
            assert_bitwise(c1, c2, f"after {ph}: cell_of")
            assert_bitwise(s1, s2, f"after {ph}: start")
            assert_bitwise(e1, e2, f"after {ph}: end")


def test_full_size_dam_break_bit_exact(capi, oracle_mod, tmp_path):
    """The 70,912-particle explicit dam break, 100 steps, against the oracle."""
    from mps_solvers_b200 import scene
    d = str(tmp_path / "c1")
    scene.write_case(d, scene.dam_break_explicit())
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    with sim_from(capi, d) as s:
        for k in (50, 50):
            s.step(k)
            orc.step(k)
            a, b = s.state(), orc.state()
            for f in FIELDS:
                assert_bitwise(a[f], b[f], f"full size {f}")
        assert a["press"].max() > 0


def test_fast_arithmetic_within_tolerance(capi, oracle_mod, tmp_path):
    """MPS_ARITH_FAST (FMA, rsqrt weight) after 100 steps: relative to each
    field's largest magnitude, n within 1e-5, x within 1e-6, u and p within
    2e-2 (the EOS multiplies n's rounding by rho c^2 / n0)."""
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    with sim_from(capi, d, arith=capi.ARITH_FAST) as s:
        s.step(100)
        orc.step(100)
        a, b = s.state(), orc.state()
    ia, ib = np.argsort(a["id"]), np.argsort(b["id"])
    assert np.array_equal(a["id"][ia], b["id"][ib])
    assert rel_err(a["n"][ia], b["n"][ib]) < 1e-5
    assert rel_err(a["pos"][ia], b["pos"][ib]) < 1e-6
    assert rel_err(a["vel"][ia], b["vel"][ib]) < 2e-2
    assert rel_err(a["press"][ia], b["press"][ib]) < 2e-2


def test_particle_leaving_grid_is_dropped(capi, oracle_mod, tmp_path):
    """A fluid particle placed outside the grid becomes type 3 and leaves the
    active range at the next divideCell, as MPS_GPU::divideCell does.  (A
    velocity large enough to leave in one step would instead trip the
    dt < dt_min check of update_dt first.)"""
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    with sim_from(capi, d) as s:
        st = s.state()
        fluid = np.nonzero(st["type"] == 0)[0]
        k = fluid[len(fluid) // 2]
        pos = st["pos"].copy()
        pos[k, 2] = 50.0  # far above the grid
        s.set_state(pos=pos)
        orc.set_state(pos=pos)
        s.step(1)
        orc.step(1)
        c = s.counts()
        oc = orc.counts()
        assert c["nexcl"] == oc["nexcl"] >= 1 and c["np"] == oc["np"]
        a, b = s.state(), orc.state()
        for f in FIELDS:
            assert_bitwise(a[f], b[f], f"after exclusion {f}")


def test_by_id_order_and_write_case(capi, tmp_path):
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "c"))
    with sim_from(capi, d) as s:
        s.step(30)
        a = s.state(capi.ORDER_SORTED)
        b = s.state(capi.ORDER_BY_ID)
        assert np.array_equal(b["id"], np.arange(len(b["id"])))
        assert np.array_equal(b["pos"][a["id"]], a["pos"])
        path = str(tmp_path / "0000.out")
        s.write_case(path, 0)
        tok = open(path).read().split()
        assert len(tok) == 9 * len(a["id"])
        assert int(tok[0]) == a["id"][0] and int(tok[1]) == a["type"][0]


def test_mps_cal_run_writes_reference_outputs(capi, tmp_path):
    """mps_run: steps until tt with an output file every tout (mps_cal)."""
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=5)
    sc.params.tt = 20 * 1e-4
    sc.params.tout = 5 * 1e-4
    d = str(tmp_path / "c")
    scene.write_case(d, sc)
    m = capi.MPS_GPU_EXPL()
    m.mps_cal(d)
    outs = sorted(os.listdir(os.path.join(d, "out")))
    assert outs[0] == "0000.out" and len(outs) >= 4
    assert m.getNp() == len(m.getId()) and m.getPos().shape == (m.getNp(), 3)


def test_cell_sort_primitive_matches_stable_argsort(capi):
    import ctypes as C
    import torch
    rng = np.random.default_rng(0)
    n = 50000
    g = capi.mps_grid(left=0.0, back=0.0, bottom=0.0, cell_size=0.1, cdx=20, cdy=10, cdz=15,
                      ncells=3000, dim=3)
    pos = rng.uniform(-0.05, 2.05, size=(n, 4)).astype(np.float32)
    pos[:, 1] *= 0.5
    pos[:, 2] *= 0.75
    x = torch.from_numpy(pos).cuda()
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    cell = torch.empty(n, dtype=torch.int32, device="cuda")
    start = torch.empty(3000, dtype=torch.int32, device="cuda")
    end = torch.empty(3000, dtype=torch.int32, device="cuda")
    nin = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = capi.lib().mps_cell_sort_dev(C.c_void_p(x.data_ptr()), n, C.byref(g),
                                      C.c_void_p(perm.data_ptr()), C.c_void_p(cell.data_ptr()),
                                      C.c_void_p(start.data_ptr()), C.c_void_p(end.data_ptr()),
                                      C.c_void_p(nin.data_ptr()), None)
    assert st == 0
    # host reference of the same keys, stable order
    p = pos.astype(np.float32)
    cx = np.trunc((p[:, 0] - np.float32(0)) / np.float32(0.1)).astype(np.int64)
    cy = np.trunc((p[:, 1] - np.float32(0)) / np.float32(0.1)).astype(np.int64)
    cz = np.trunc((p[:, 2] - np.float32(0)) / np.float32(0.1)).astype(np.int64)
    out = (cx < 0) | (cy < 0) | (cz < 0) | (cx >= 20) | (cy >= 10) | (cz >= 15)
    key = np.where(out, 3000, cz * 200 + cy * 20 + cx)
    # truncation toward zero maps (-1, 0) to cell 0 like the reference
    key = np.where((cx >= 0) & (cy >= 0) & (cz >= 0) & ~out, key, key)
    order = np.argsort(key, kind="stable")
    assert np.array_equal(perm.cpu().numpy().astype(np.int64), order)
    assert np.array_equal(cell.cpu().numpy().astype(np.int64), key[order])
    counts = np.bincount(key[key < 3000], minlength=3000)
    st0 = np.concatenate([[0], np.cumsum(counts)[:-1]])
    assert np.array_equal(start.cpu().numpy(), st0)
    assert np.array_equal(end.cpu().numpy(), st0 + counts)
    assert int(nin.item()) == int((key < 3000).sum())
