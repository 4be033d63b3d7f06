"""The autotuner: it picks among valid launch shapes, and the shapes it
chooses between do not change results (bit for bit in the explicit exact
path, within the solve tolerance in the semi-implicit one)."""
import numpy as np
import pytest

from helpers import assert_bitwise, load_golden, rel_err, write_golden_case

pytestmark = pytest.mark.gpu


def test_autotune_explicit_keeps_bitwise_results(capi, tmp_path):
    g = load_golden("expl_tank")
    d = write_golden_case(g, str(tmp_path / "e"))
    steps = 2
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        rep = s.autotune(steps)
        assert rep["stage_threads"] in (64, 128, 256)
        assert all(t > 0 for t in rep["stage_ms"])
        s.step(10)
        tuned = s.state(capi.ORDER_BY_ID)
    with capi.Simulation(d, method=capi.METHOD_EXPLICIT) as s:
        s.step(3 * steps + 10)   # the tuner took 3 candidates x steps
        plain = s.state(capi.ORDER_BY_ID)
    for f in ("pos", "vel", "press", "n"):
        assert_bitwise(tuned[f], plain[f], f)


def test_autotune_semi_shapes(capi, tmp_path):
    g = load_golden("semi_tank")
    d = write_golden_case(g, str(tmp_path / "s"))
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        rep = s.autotune(2)
        assert rep["ppe_threads"] in (256, 512, 1024)
        assert rep["ppe_ms"][0] > 0 and rep["ppe_ms"][3] > 0 and rep["ppe_ms"][6] > 0  # 1024 threads
        assert rep["ppe_stored_weights"] in (0, 1) and rep["ppe_pipelined"] in (0, 1)
        for _ in range(3):
            st = s.step(1)
            assert st.status == 0 and st.cg_relres <= 1e-8
        tuned = s.state(capi.ORDER_BY_ID)
    with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT) as s:
        held = sum(1 for t in list(rep["ppe_ms"]) + list(rep["ppe_compact_ms"]) if t > 0)
        s.step(3 * 2 + held * 2 + 3)   # the steps the tuner took, then the same 3
        plain = s.state(capi.ORDER_BY_ID)
    assert rel_err(tuned["press"], plain["press"]) < 1e-4
    assert np.abs(tuned["pos"] - plain["pos"]).max() < 1e-7
