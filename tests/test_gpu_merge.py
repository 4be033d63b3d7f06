"""The merge rebuild against the full radix sort.

Between two cell rebuilds only the particles whose cell changed move in the
stably sorted order, so the new order is the unchanged particles merged with
the changed ones sorted by (new cell, previous position).  With
``rebuild_merge=0`` a handle whose fluid (plus moving walls) fits the merge's
one-block sort takes that path; ``rebuild_merge=-1`` always sorts.  Both must
give the same particle order, cell tables and states bit for bit:

* explicit, exact arithmetic, with and without CUDA graphs;
* semi-implicit with a moving piston (walls change cells too);
* a state set from the host that moves 3,000 particles one cell along x
  (the sort's shared-memory bitonic case; fewer take its rank sort), or
  every particle, so that more change cell than shared memory takes (its
  global-memory case) and some leave the grid.
"""
import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu

TANK = dict(interior=(40, 20, 24), fluid=(20, 20, 16))  # 30,208 particles, 6,400 fluid


def case(tmp_path, name, **kw):
    from mps_solvers_b200 import scene
    d = str(tmp_path / name)
    scene.write_case(d, scene.small_tank(seed=3, **kw))
    return d


def snapshot(s):
    return s.state(), s.cell_tables(), s.counts()


def assert_same(a, b):
    sa, ca, na = a
    sb, cb, nb = b
    assert na == nb, (na, nb)
    for f in ("id", "type", "pos", "vel", "press", "n"):
        assert_bitwise(sa[f], sb[f], f)
    for x, y, what in zip(ca, cb, ("cell_of", "start", "end")):
        assert np.array_equal(x, y), what


@pytest.mark.parametrize("use_graph", [1, 0])
def test_explicit_merge_equals_full_sort(capi, tmp_path, use_graph):
    d = case(tmp_path, "t", **TANK)
    out = []
    for merge in (0, -1):
        with capi.Simulation(d, method=capi.METHOD_EXPLICIT, rebuild_merge=merge, use_graph=use_graph) as s:
            st = s.step(30)
            assert st.status == 0
            out.append(snapshot(s))
    assert_same(out[0], out[1])


def test_semi_merge_with_moving_piston_equals_full_sort(capi, tmp_path):
    d = case(tmp_path, "t", dt=5e-4)
    out = []
    for merge in (0, -1):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, rebuild_merge=merge) as s:
            st0 = s.state()
            xf = float(st0["pos"][st0["type"] == 0][:, 0].min())
            assert s.add_wall_motion((-1.0, -1.0, -1.0), (xf - 0.05, 10.0, 10.0), vel=(0.2, 0.0, 0.0)) > 0
            st = s.step(8)
            assert st.status == 0 and st.cg_relres <= 1e-8
            out.append(snapshot(s))
    assert_same(out[0], out[1])


@pytest.mark.parametrize("moved", [3000, None])
def test_merge_after_host_state_moves_particles(capi, tmp_path, moved):
    d = case(tmp_path, "t", **TANK)
    out = []
    for merge in (0, -1):
        with capi.Simulation(d, method=capi.METHOD_EXPLICIT, rebuild_merge=merge) as s:
            s.step(2)
            g = s.grid()
            st = s.state()
            pos = st["pos"].copy()
            sel = slice(None) if moved is None else slice(0, moved)
            pos[sel, 0] += np.float32(g.cell_size)  # one cell along x; the last layer leaves
            s.set_state(pos=pos)
            try:
                s.step(1)
            except capi.MPSError:
                pass  # the shifted tank may be flagged; both paths must flag it alike
            c = s.counts()
            assert c["nexcl"] > 0
            out.append(snapshot(s))
    assert_same(out[0], out[1])
