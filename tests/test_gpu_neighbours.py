"""Neighbour-completeness check of the reference's MPS_GPU::check
(MPS_CAL_/MPS_GPU.cpp:1833-1927), on the GPU's own cell tables: every pair
closer than the search radius lies in linked cells (the 27 cells of
MPS_GPU::makeLink around the particle's cell, with its unsigned
wrap-around), every particle sits in the cell its position maps to, and the
cell table lists each cell's particles as one contiguous run in sorted
order.  Run after steps of both methods, for r0 (explicit) and rlap
(semi-implicit, the largest stencil)."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

pytestmark = pytest.mark.gpu


def linked(c, g):
    """The 27 cell ids of makeLink for cell c (uint32 arithmetic)."""
    c = np.asarray(c, np.int64)
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                out.append((c + dz * g.cdx * g.cdy + dy * g.cdx + dx) & 0xFFFFFFFF)
    return np.stack(out, 1)


def check(s, radius):
    st = s.state()  # sorted order
    cell_of, start, end = s.cell_tables()
    g = s.grid()
    pos = st["pos"].astype(np.float64)
    n = len(pos)
    # cells: contiguous runs in sorted order, consistent with cell_of
    assert np.all(np.diff(cell_of.astype(np.int64)) >= 0)
    for c in np.unique(cell_of):
        idx = np.nonzero(cell_of == c)[0]
        assert start[c] == idx[0] and end[c] == idx[-1] + 1
    # each particle in the cell of its position (the reference's float
    # expression; a particle within rounding of a face may sit on either side)
    ix = np.floor((pos[:, 0] - g.left) / g.cell_size)
    iy = np.floor((pos[:, 1] - g.back) / g.cell_size)
    iz = np.floor((pos[:, 2] - g.bottom) / g.cell_size)
    want = (iz * g.cdx * g.cdy + iy * g.cdx + ix).astype(np.int64)
    off = want != cell_of.astype(np.int64)
    assert off.mean() < 1e-3
    # completeness: every pair within `radius` is in linked cells
    pairs = cKDTree(pos).query_pairs(radius, output_type="ndarray")
    assert len(pairs) > 0
    lk = linked(cell_of.astype(np.int64)[pairs[:, 0]], g)
    ok = np.any(lk == cell_of.astype(np.int64)[pairs[:, 1], None], axis=1)
    assert ok.all(), f"{(~ok).sum()} of {len(pairs)} pairs outside the linked cells"


def test_neighbour_completeness_explicit(capi, tmp_path):
    from mps_solvers_b200 import scene
    d = str(tmp_path / "e")
    sc = scene.small_tank(seed=3, interior=(20, 8, 16), fluid=(8, 6, 12))
    scene.write_case(d, sc)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        for _ in range(3):
            s.step(40)
            check(s, sc.params.r0 * sc.params.dp)


def test_neighbour_completeness_semi(capi, tmp_path):
    from mps_solvers_b200 import scene
    d = str(tmp_path / "s")
    sc = scene.small_tank(seed=4, interior=(20, 8, 16), fluid=(8, 6, 12), dt=5e-4)
    scene.write_case(d, sc)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        for _ in range(3):
            s.step(5)
            check(s, sc.params.rlap * sc.params.dp)
