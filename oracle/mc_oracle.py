"""TEST INFRASTRUCTURE ONLY: CPU restatement of the free-surface extraction
(marching cubes) the library runs on the GPU.

Follows the reference's iso-surface pipeline of MPS_CAL_expl_gl_v3.1:
* iso = 0.8 * max_i sum_{j != i} w(r_ij; r0), the cubic spline of
  MPS_GPU::r_cubic_weight (MPS_CAL_/MPS_GPU.cpp:54-62), in MPS_GPU::calOnce
  (MPS_CAL_/MPS_GPU.cpp:222-272, ISO = 0.8 in marchingCube_define.h);
* vertex value = sum of w over the fluid particles (kerCalVertex_n,
  gpu_kernel/renderer_gpu_cudaker.cu:136-226);
* a corner is inside when its value exceeds iso and edge points follow
  vertexInterp (renderer_gpu_cudaker.cu:72-87) (kerCalTriangle, :226-340).

The case table is generated by the rule the library documents (crossing
edges paired around each run of inside corners on every face, segments
linked into loops, loops oriented inside -> outside and fanned), written
here independently of the library's C++ generator so the two can be
compared.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

CORNER = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGE = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
FACE = [(0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
EDGE_OF = {frozenset(e): k for k, e in enumerate(EDGE)}


def build_table():
    """[case] -> list of triangles (edge triples)."""
    table = []
    for c in range(256):
        inside = [(c >> k) & 1 for k in range(8)]
        links = {e: [] for e in range(12)}
        for q in FACE:
            ins = [inside[v] for v in q]
            if sum(ins) in (0, 4):
                continue
            for k in range(4):
                if not ins[k] or ins[k - 1]:
                    continue
                end = k
                while ins[(end + 1) % 4]:
                    end = (end + 1) % 4
                ea = EDGE_OF[frozenset((q[k - 1], q[k]))]
                eb = EDGE_OF[frozenset((q[end], q[(end + 1) % 4]))]
                links[ea].append(eb)
                links[eb].append(ea)
        seen, tris = set(), []
        for e0 in range(12):
            if len(links[e0]) != 2 or e0 in seen:
                continue
            loop, prev, cur = [], None, e0
            while True:
                loop.append(cur)
                seen.add(cur)
                a, b = links[cur]
                nxt = a if a != prev else b
                prev, cur = cur, nxt
                if cur == e0:
                    break
            mid = np.array([[0.5 * (CORNER[EDGE[e][0]][d] + CORNER[EDGE[e][1]][d]) for d in range(3)]
                            for e in loop])
            out = np.zeros(3)
            for e in loop:
                a, b = EDGE[e]
                ci, co = (a, b) if inside[a] else (b, a)
                out += np.subtract(CORNER[co], CORNER[ci])
            nrm = np.zeros(3)
            for t in range(len(loop)):
                p, r = mid[t], mid[(t + 1) % len(loop)]
                nrm += [(p[1] - r[1]) * (p[2] + r[2]), (p[2] - r[2]) * (p[0] + r[0]),
                        (p[0] - r[0]) * (p[1] + r[1])]
            if nrm @ out < 0:
                loop = loop[::-1]
            tris += [(loop[0], loop[t], loop[t + 1]) for t in range(1, len(loop) - 1)]
        table.append(tris)
    return table


def cubic_w(r0, r):
    q = np.asarray(r, np.float64) / r0
    w = np.where(q <= 0.5, 8.0 / np.pi * (1 - 6 * q * q + 6 * q ** 3),
                 np.where(q <= 1.0, 16.0 / np.pi * (1 - q) ** 3, 0.0))
    return w


def iso_level(pos, r0):
    tree = cKDTree(pos)
    pairs = tree.query_pairs(r0, output_type="ndarray")
    r = np.sqrt(((pos[pairs[:, 0]] - pos[pairs[:, 1]]) ** 2).sum(1))
    s = np.zeros(len(pos))
    w = cubic_w(r0, r)
    np.add.at(s, pairs[:, 0], w)
    np.add.at(s, pairs[:, 1], w)
    return 0.8 * s.max()


def vertex_values(pos_fluid, r0, shape, origin, spacing):
    nx, ny, nz = shape
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    verts = np.stack([origin[0] + spacing[0] * ix, origin[1] + spacing[1] * iy,
                      origin[2] + spacing[2] * iz], -1).reshape(-1, 3)
    tree = cKDTree(pos_fluid)
    out = np.zeros(len(verts))
    for v, nb in enumerate(tree.query_ball_point(verts, r0)):
        if nb:
            out[v] = cubic_w(r0, np.sqrt(((pos_fluid[nb] - verts[v]) ** 2).sum(1))).sum()
    # x fastest
    return out.reshape(nx, ny, nz).transpose(2, 1, 0).copy()


def triangles(values, iso, origin, spacing, table):
    """values[z, y, x]; returns (T, 3, 3) vertex positions."""
    nz, ny, nx = values.shape
    out = []
    for iz in range(nz - 1):
        for iy in range(ny - 1):
            for ix in range(nx - 1):
                val = [values[iz + c[2], iy + c[1], ix + c[0]] for c in CORNER]
                case = sum(1 << k for k in range(8) if val[k] > iso)
                for tri in table[case]:
                    pts = []
                    for e in tri:
                        a, b = EDGE[e]
                        n1, n2 = np.float32(val[a]), np.float32(val[b])
                        pa = np.array([origin[d] + spacing[d] * ((ix, iy, iz)[d] + CORNER[a][d])
                                       for d in range(3)], np.float32)
                        pb = np.array([origin[d] + spacing[d] * ((ix, iy, iz)[d] + CORNER[b][d])
                                       for d in range(3)], np.float32)
                        pts.append((iso * (pb - pa) + pa * n2 - pb * n1) / (n2 - n1))
                    out.append(pts)
    return np.array(out, np.float64).reshape(-1, 3, 3)


def canonical(tris, decimals=5):
    """Triangles sorted by rounded centroid, for order-free comparison."""
    c = np.round(tris.mean(1), decimals)
    o = np.lexsort((c[:, 2], c[:, 1], c[:, 0]))
    return tris[o]
