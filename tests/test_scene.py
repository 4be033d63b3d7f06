"""Scene generator: counts of the named workloads and exact float round trip."""
import numpy as np

from mps_solvers_b200 import scene


def test_dam_break_explicit_counts():
    pos, nb2, nb1 = scene.build(scene.dam_break_explicit())
    nfluid = len(pos) - nb2 - nb1
    assert len(pos) == 70912 and nfluid == 8000
    # 80 x 20 x 50 interior, 2 wall + 2 dummy layers: 88 x 28 x 58 sites
    assert nb2 + nb1 == 88 * 28 * 58 - 80 * 20 * 50


def test_dam_break_semi_counts():
    sc = scene.dam_break_semi()
    x, y, z, t = scene._site_types(sc)
    assert (t == 0).sum() == 80000
    assert (t >= 0).sum() == 310912


def test_jitter_bounds_and_determinism():
    sc = scene.small_tank(seed=3)
    a, _, _ = scene.build(sc)
    b, _, _ = scene.build(sc)
    assert np.array_equal(a, b)
    sc0 = scene.small_tank(seed=3)
    sc0.jitter = 0.0
    lat, _, _ = scene.build(sc0)
    d = np.abs(a.astype(np.float64) - lat.astype(np.float64))
    assert d.max() <= 1.0001e-4 * sc.l0 + 1e-7 and d.max() > 0


def test_geo_text_round_trip(tmp_path):
    sc = scene.small_tank(seed=4)
    pos, nb2, nb1 = scene.write_case(str(tmp_path), sc)
    txt = open(tmp_path / "GEO.dat").read().split()
    n = int(txt[0])
    vals = np.array(txt[3:3 + 3 * n], dtype=np.float64)
    assert np.array_equal(vals.astype(np.float32), pos.ravel())
    assert np.array_equal(vals, pos.ravel().astype(np.float64))
