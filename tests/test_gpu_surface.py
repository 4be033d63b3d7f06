"""Free-surface extraction (marching cubes) on the GPU against the CPU
restatement in oracle/mc_oracle.py: the iso level, the vertex values, and
the triangles (count and positions), after some explicit steps."""
import os

import numpy as np
import pytest
from scipy.spatial import cKDTree

import mc_oracle as mo

pytestmark = pytest.mark.gpu


def _case(tmp_path):
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=5, interior=(20, 8, 16), fluid=(8, 8, 12), l0=0.02, dt=1e-4)
    d = str(tmp_path / "c")
    scene.write_case(d, sc)
    return sc, d


def test_surface_matches_cpu_oracle(capi, tmp_path):
    from mps_solvers_b200 import scene
    sc, d = _case(tmp_path)
    shape = (33, 14, 27)
    origin, spacing = scene.surface_grid(sc, shape)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        st0 = s.state()
        s.surface_setup(shape, origin, spacing, 200000)
        s.step(30)
        n = s.surface_extract()
        pos, nrm = s.surface_triangles()
        values, iso = s.surface_vertex_values()
        st = s.state()
        stl = str(tmp_path / "surface.stl")
        s.surface_write_stl(stl)
    r0 = np.float32(np.float32(2.1) * np.float32(sc.l0))
    iso_cpu = mo.iso_level(st0["pos"].astype(np.float64), float(r0))
    assert abs(iso - iso_cpu) <= 1e-5 * iso_cpu
    fluid = st["pos"][st["type"] == 0].astype(np.float64)
    v_cpu = mo.vertex_values(fluid, float(r0), shape, origin, spacing)
    assert np.abs(values - v_cpu).max() <= 1e-5 * v_cpu.max()
    # triangles from the GPU's own vertex values: the same cubes and points
    table = [list(t) for t in mo.build_table()]
    tri_cpu = mo.triangles(values.astype(np.float64), iso, origin, spacing, table)
    assert n == len(tri_cpu) and n > 100
    tree = cKDTree(tri_cpu.mean(1))
    dist, idx = tree.query(pos.astype(np.float64).mean(1))
    assert dist.max() < 1e-5
    assert np.abs(pos - tri_cpu[idx]).max() < 1e-5
    # normals are unit and point away from the fluid (towards lower n)
    ln = np.linalg.norm(nrm, axis=2)
    assert np.all(np.abs(ln - 1) < 1e-3)
    # winding agrees with the normals
    fn = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0])
    agree = (fn * nrm.mean(1)).sum(1) > 0
    assert agree.mean() > 0.95
    assert os.path.getsize(stl) == 84 + 50 * n


def test_surface_capacity_is_reported(capi, tmp_path):
    from mps_solvers_b200 import scene
    sc, d = _case(tmp_path)
    shape = (33, 14, 27)
    origin, spacing = scene.surface_grid(sc, shape)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        s.surface_setup(shape, origin, spacing, 10)
        with pytest.raises(capi.MPSError) as e:
            s.surface_extract()
        assert e.value.status == 10
