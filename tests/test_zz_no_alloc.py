"""mps_cell_sort_dev_noalloc, the allocation-free cell sort, against
mps_cell_sort_dev.

The allocation-free entry point is for callers that must not allocate device
memory (a host whose pool allocator owns all GPU memory, or a latency-critical
loop that cannot afford the device synchronisation of cudaMalloc/cudaFree).
It keeps its scratch in one fixed array inside the library, so two calls in a
row must give the same results as the allocating entry point even though the
second call finds the first call's leftovers in that array.  The results are
integer permutations and tables, so they must be identical.  This file is
named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grid(capi, ncells_xyz=(20, 10, 15), cell=0.1):
    cdx, cdy, cdz = ncells_xyz
    return capi.mps_grid(left=0.0, back=0.0, bottom=0.0, cell_size=cell, cdx=cdx, cdy=cdy, cdz=cdz,
                         ncells=cdx * cdy * cdz, dim=3)


def _positions(n, seed, extent):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    for a in range(3):
        pos[:, a] = rng.uniform(-0.05, extent[a] + 0.05, size=n)
    return pos


def _run(capi, fn, pos, g):
    import torch
    n = len(pos)
    x = torch.from_numpy(pos).cuda()
    out = dict(perm=torch.full((max(n, 1),), 7, dtype=torch.int32, device="cuda"),
               cell=torch.full((max(n, 1),), 7, dtype=torch.int32, device="cuda"),
               start=torch.full((g.ncells,), 7, dtype=torch.int32, device="cuda"),
               end=torch.full((g.ncells,), 7, dtype=torch.int32, device="cuda"),
               nin=torch.full((1,), 7, dtype=torch.int32, device="cuda"))
    st = fn(C.c_void_p(x.data_ptr()), n, C.byref(g), C.c_void_p(out["perm"].data_ptr()),
            C.c_void_p(out["cell"].data_ptr()), C.c_void_p(out["start"].data_ptr()),
            C.c_void_p(out["end"].data_ptr()), C.c_void_p(out["nin"].data_ptr()), None)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy()[:n] if k in ("perm", "cell") else v.cpu().numpy() for k, v in out.items()}
    return st, res


def test_noalloc_matches_allocating_entry_point_twice(capi):
    L = capi.lib()
    g = _grid(capi)
    # two calls in a row with different inputs; the second starts from the
    # first call's leftovers in the shared scratch array
    for seed, n in ((1, 60000), (2, 23456)):
        pos = _positions(n, seed, (2.0, 1.0, 1.5))
        st_a, a = _run(capi, L.mps_cell_sort_dev, pos, g)
        st_b, b = _run(capi, L.mps_cell_sort_dev_noalloc, pos, g)
        assert st_a == 0 and st_b == 0
        for k in a:
            assert np.array_equal(a[k], b[k]), (seed, k)
        # and the tables describe a stable sort by cell
        key = b["cell"].astype(np.int64)
        assert np.all(np.diff(key) >= 0)
        assert int(b["nin"][0]) == int((key < g.ncells).sum())


def test_noalloc_edges_of_its_fixed_regions(capi):
    """The edges of the fixed scratch regions, each against the allocating
    entry point bit for bit: no particles (only the cell table is written),
    exactly MPS_NOALLOC_MAX_PARTICLES particles (every histogram tile in
    use), and a grid of exactly MPS_NOALLOC_MAX_CELLS cells (the whole
    cell-table region, and a third radix pass for the larger cell ids)."""
    L = capi.lib()
    cases = [
        (_grid(capi), 0, 3),
        (_grid(capi), capi.NOALLOC_MAX_PARTICLES, 4),
        (_grid(capi, ncells_xyz=(128, 64, 64), cell=0.02), 200000, 5),
    ]
    assert cases[2][0].ncells == capi.NOALLOC_MAX_CELLS
    for g, n, seed in cases:
        ext = (g.cdx * g.cell_size, g.cdy * g.cell_size, g.cdz * g.cell_size)
        pos = _positions(n, seed, ext)
        st_a, a = _run(capi, L.mps_cell_sort_dev, pos, g)
        st_b, b = _run(capi, L.mps_cell_sort_dev_noalloc, pos, g)
        assert st_a == 0 and st_b == 0, (n, st_a, st_b)
        for k in a:
            assert np.array_equal(a[k], b[k]), (n, g.ncells, k)
        assert int(b["nin"][0]) == int((b["cell"].astype(np.int64) < g.ncells).sum())
        if n == 0:
            assert not b["start"].any() and not b["end"].any()


def test_noalloc_rejects_sizes_beyond_its_limits(capi):
    L = capi.lib()
    g = _grid(capi)
    n = capi.NOALLOC_MAX_PARTICLES + 1
    st = L.mps_cell_sort_dev_noalloc(C.c_void_p(16), n, C.byref(g), C.c_void_p(16), C.c_void_p(16),
                                     C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None)
    assert st == 10  # MPS_ERR_CAPACITY, refused before any GPU work
    big = _grid(capi, ncells_xyz=(100, 100, 100))
    st = L.mps_cell_sort_dev_noalloc(C.c_void_p(16), 10, C.byref(big), C.c_void_p(16), C.c_void_p(16),
                                     C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None)
    assert st == 10
