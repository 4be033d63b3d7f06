"""The compact PPE layout (mps_solvers_b200/csrc/ppe_compact.cu) against the
8-byte sliced layout of the same matrix.

Both layouts store the matrix buildPoisson defines
(MPS_CAL_v4.0/MPS_CPU.cpp:619-710) and solve it to the same FP64 relative
residual (1e-8); they add the row products in different orders, so states
agree within the semi-implicit tolerances of tests/test_gpu_semi.py, not bit
for bit.  The stored pair sets are identical (the same neighbour set), and a
wide, shallow pool whose rows couple to rows more than 32,767 rows away in
the compact numbering exercises the escaped entries.
"""
import numpy as np
import pytest

from helpers import load_golden, rel_err, write_golden_case

pytestmark = pytest.mark.gpu

P_TOL, U_TOL, X_TOL = 2e-3, 1e-3, 1e-6


def _by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: v[o] for k, v in st.items()}


def _close(a, b):
    a, b = _by_id(a), _by_id(b)
    assert np.array_equal(a["id"], b["id"])
    ex = np.abs(a["pos"] - b["pos"]).max() / np.abs(b["pos"]).max()
    return ex, rel_err(a["vel"], b["vel"]), rel_err(a["press"], b["press"])


def _pairs(sim):
    st = sim.ppe_stencil()
    n = len(st["row_start"]) - 1
    i = np.repeat(np.arange(n, dtype=np.int64), np.diff(st["row_start"].astype(np.int64)))
    return np.sort(i * n + st["cols"].astype(np.int64)), st["weights"]


def _compare_layouts(capi, d, steps, arith, expect_escapes):
    out = {}
    for layout in (0, -1):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, arith=arith, ppe_layout=layout) as s:
            for _ in range(steps):
                st = s.step(1)
                assert st.cg_relres <= 1e-8 and st.status == 0
            esc = s.scalars()["ppe_escaped"]
            if layout == 0:
                assert (esc > 0) == expect_escapes, esc
            else:
                assert esc == -1
            out[layout] = (s.state(), _pairs(s))
    (sa, (pa, wa)), (sb, (pb, wb)) = out[0], out[-1]
    assert np.array_equal(pa, pb)
    ex, eu, ep = _close(sa, sb)
    assert ex < X_TOL and eu < U_TOL and ep < P_TOL, (ex, eu, ep)


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_compact_layout_matches_8_byte_layout(capi, tmp_path, arith):
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    mode = capi.ARITH_EXACT if arith == "exact" else capi.ARITH_FAST
    _compare_layouts(capi, d, 8, mode, expect_escapes=False)


def test_compact_layout_escaped_entries(capi, tmp_path):
    """A 200 x 100 x 8 pool (160,000 fluid particles, l0 = 0.01 m): a cell
    layer holds more rows than a 16-bit code can reach, so many entries are
    escaped; the solve still matches the 8-byte layout."""
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=2, interior=(204, 104, 14), fluid=(200, 100, 8), l0=0.01, dt=5e-4)
    d = str(tmp_path / "pool")
    scene.write_case(d, sc)
    _compare_layouts(capi, d, 3, capi.ARITH_FAST, expect_escapes=True)


def test_compact_layout_without_shared_memory_chunks(capi, tmp_path):
    """Keeping no matrix chunks in shared memory reads every chunk from
    global memory: the same products in the same order, so the states are
    identical bit for bit."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    out = []
    for chunks in (0, -1, 3):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, ppe_smem_chunks=chunks) as s:
            s.step(6)
            out.append(s.state())
    for o in out[1:]:
        for f in ("pos", "vel", "press"):
            assert np.array_equal(out[0][f], o[f]), f



def test_8_byte_layout_shared_memory_chunks(capi, tmp_path):
    """The 8-byte layout's solver also keeps each warp's last chunks in
    shared memory (stored weights): the same products in the same order
    with any number of them, so the states are identical bit for bit."""
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    out = []
    for chunks in (0, -1, 3):
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, ppe_layout=-1, ppe_smem_chunks=chunks) as s:
            s.step(6)
            out.append(s.state())
    for o in out[1:]:
        for f in ("pos", "vel", "press"):
            assert np.array_equal(out[0][f], o[f]), f
