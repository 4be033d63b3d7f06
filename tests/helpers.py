"""Shared helpers for the parity tests."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def write_golden_case(g, d):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.dat"), "wb") as f:
        f.write(g["input_dat"].tobytes())
    with open(os.path.join(d, "GEO.dat"), "wb") as f:
        f.write(g["geo_dat"].tobytes())
    return d


def bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.float32:
        return a.view(np.uint32)
    if a.dtype == np.float64:
        return a.view(np.uint64)
    return a


def assert_bitwise(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    ba, bb = bits(a), bits(b)
    bad = np.nonzero(ba != bb)
    if len(bad[0]):
        k = tuple(x[0] for x in bad)
        raise AssertionError(f"{what}: {len(bad[0])} entries differ; first at {k}: {a[k]!r} vs {b[k]!r}")


def rel_err(a, b):
    """max |a-b| / max |b| (0 when both are 0)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = np.abs(b).max()
    num = np.abs(a - b).max()
    return 0.0 if num == 0 else num / (den if den > 0 else 1.0)


def by_id(state, np0):
    """Reorder a sorted-order state dict by particle id."""
    order = np.argsort(state["id"], kind="stable")
    return {k: v[order] for k, v in state.items()}
