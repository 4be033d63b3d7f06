"""The marching-cubes case table (no GPU: the library generates it on the
host): the C++ generator against the oracle's independent generator, the
cut edges of every case, a closed and consistently oriented surface on
random fields, and the reference's own table where it is readable."""
import os
import re

import numpy as np
import pytest

import mc_oracle as mo


@pytest.fixture(scope="module")
def lib_table():
    from mps_solvers_b200 import capi
    return capi.surface_case_table()


def test_library_table_equals_oracle_generator(lib_table):
    assert lib_table == [list(t) for t in mo.build_table()]


def test_every_case_cuts_exactly_its_crossing_edges(lib_table):
    for c in range(256):
        inside = [(c >> k) & 1 for k in range(8)]
        want = {e for e, (a, b) in enumerate(mo.EDGE) if inside[a] != inside[b]}
        got = {e for tri in lib_table[c] for e in tri}
        assert got == want, c
        assert len(lib_table[c]) <= 5


def _mesh_edges(values, iso, table):
    """Directed mesh edges between cut points, each cut point keyed by its
    grid edge (the two global vertex ids), over the whole grid."""
    nz, ny, nx = values.shape
    gid = lambda x, y, z: (z * ny + y) * nx + x
    edges = []
    for iz in range(nz - 1):
        for iy in range(ny - 1):
            for ix in range(nx - 1):
                case = sum(1 << k for k, c in enumerate(mo.CORNER)
                           if values[iz + c[2], iy + c[1], ix + c[0]] > iso)
                for tri in table[case]:
                    key = []
                    for e in tri:
                        a, b = mo.EDGE[e]
                        ca, cb = mo.CORNER[a], mo.CORNER[b]
                        ka = gid(ix + ca[0], iy + ca[1], iz + ca[2])
                        kb = gid(ix + cb[0], iy + cb[1], iz + cb[2])
                        key.append((min(ka, kb), max(ka, kb)))
                    for t in range(3):
                        edges.append((key[t], key[(t + 1) % 3]))
    return edges


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_surface_is_closed_and_oriented(lib_table, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(0.0, 1.0, (9, 9, 9))
    v[0, :, :] = v[-1, :, :] = v[:, 0, :] = v[:, -1, :] = v[:, :, 0] = v[:, :, -1] = 0.0
    edges = _mesh_edges(v, 0.5, lib_table)
    assert edges
    from collections import Counter
    directed = Counter(edges)
    undirected = Counter(frozenset(e) for e in edges)
    # every mesh edge is shared by exactly two triangles, traversed once each way
    assert all(n == 2 for n in undirected.values())
    assert all(n == 1 for n in directed.values())


def _reference_table():
    import oracle
    ref = oracle.reference_dir()
    path = os.path.join(ref, "MPS_CAL_", "marchingCube_table.h") if ref else ""
    if not path or not os.path.exists(path):
        pytest.skip("the reference sources are not present")
    text = open(path).read()
    body = text[text.index("triTable"):]
    body = body[body.index("{") + 1:]
    # entries are edge numbers, X (255) for unused slots
    nums = [-1 if x == "X" else int(x) for x in re.findall(r"\bX\b|\d+", body[:body.index("};")])]
    assert len(nums) == 256 * 16
    return [[tuple(nums[16 * c + 3 * k:16 * c + 3 * k + 3]) for k in range(5)
             if nums[16 * c + 3 * k] != -1] for c in range(256)]


def _loops(tris):
    """The cut-edge sets of the connected pieces of a case's triangles."""
    groups = []
    for t in tris:
        s = set(t)
        hit = [g for g in groups if g & s]
        for g in hit:
            groups.remove(g)
            s |= g
        groups.append(s)
    return sorted(sorted(g) for g in groups)


def test_against_the_reference_table(lib_table):
    ref = _reference_table()
    ambiguous = 0
    for c in range(256):
        assert {e for t in ref[c] for e in t} == {e for t in lib_table[c] for e in t}, c
        inside = [(c >> k) & 1 for k in range(8)]
        amb = any(sum(inside[v] for v in q) == 2 and inside[q[0]] == inside[q[2]] for q in mo.FACE)
        if amb:
            ambiguous += 1
            continue
        assert _loops(ref[c]) == _loops(lib_table[c]), c
        assert len(ref[c]) == len(lib_table[c]), c
    assert ambiguous < 256
