"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the learned PPE
preconditioner's network and training loss (mps_solvers_b200/csrc/learned.cu).

The reference has no such component; this oracle checks the GPU's
hand-written forward and backward kernels.  Given the state a PPE system was
assembled from (positions, n, ids, which rows are solved, the diagonal of
A), it rebuilds:

* the stencil: solved rows j != i with |x_j - x_i|^2 < r0^2;
* edge features (dx, dy, dz, |r| over r0, r0/r - 1, n_i / n0, [j wall]);
* the two message-passing rounds, the readout of G (lower triangle in
  particle index order, softplus diagonal + 1e-3);
* Ahat = D^-1/2 (-A) D^-1/2 on the solved rows from the rlap weights;
* the probe z (the GPU's hash of seed and particle id) and the loss
  log(T / n) - (2 / n) sum_i log G_ii with T = v1 . Ahat v1, v1 = G^T z
  (Kaporin's condition number of G Ahat G^T up to a constant, with
  Hutchinson's trace estimate).

Gradients are taken by central finite differences of this float64 loss.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

H, F = 64, 7
GMIN = 1e-3

# parameter layout, in the order of learned.cuh
LAYOUT = [("W1e", (H, F)), ("b1", (H,)), ("V1", (H, H)), ("c1", (H,)), ("W2e", (H, F)), ("U2", (H, H)),
          ("b2", (H,)), ("V2", (H, H)), ("c2", (H,)), ("Re", (H, F)), ("Ra", (H, H)), ("Rb", (H, H)),
          ("br", (H,)), ("om", (H,)), ("dl", (H,)), ("bd", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in LAYOUT)


def unpack(w):
    out, k = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = np.asarray(w[k:k + n], np.float64).reshape(shape)
        k += n
    return out


def to_bf16(w):
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def softplus(x):
    return np.where(x > 20, x, np.log1p(np.exp(np.minimum(x, 20))))


def probe(seed, ids):
    with np.errstate(over="ignore"):
        h = (np.uint64(seed) << np.uint64(32)) + ids.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        h = (h ^ (h >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        h = (h ^ (h >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        h = h ^ (h >> np.uint64(31))
    return np.where((h >> np.uint64(63)) == 1, 1.0, -1.0)


class System:
    """The PPE system of a snapshot, on its solved rows."""

    def __init__(self, snap, r0, rlap, n0_inv):
        pos4 = snap["pos4"]
        self.rows = np.nonzero(snap["is_row"])[0]           # ascending particle index
        x = pos4[self.rows, :3].astype(np.float64)
        self.x = x
        self.n = snap["n"][self.rows].astype(np.float64)
        self.ids = snap["id"][self.rows]
        typ = pos4[self.rows, 3].view(np.uint32)
        self.wall = (typ == 1).astype(np.float64)
        self.d = -snap["diag"][self.rows]                     # positive
        self.r0, self.rlap, self.n0_inv = r0, rlap, n0_inv
        tree = cKDTree(x)
        m = len(self.rows)
        # stencil within r0 (pairs both directions), row-local indices
        pairs = tree.query_pairs(r0, output_type="ndarray")
        d2 = ((x[pairs[:, 0]] - x[pairs[:, 1]]) ** 2).sum(1)
        pairs = pairs[d2 < r0 * r0]
        src = np.concatenate([pairs[:, 0], pairs[:, 1]])
        dst = np.concatenate([pairs[:, 1], pairs[:, 0]])
        self.ei, self.ej = src, dst                            # edge (i, j): row i, neighbour j
        self.cnt = np.bincount(self.ei, minlength=m).astype(np.float64)
        # edge features
        dx = x[self.ej] - x[self.ei]
        r = np.sqrt((dx ** 2).sum(1))
        self.feat = np.stack([dx[:, 0] / r0, dx[:, 1] / r0, dx[:, 2] / r0, r / r0, r0 / r - 1.0,
                              self.n[self.ei] * n0_inv, self.wall[self.ej]], axis=1)
        self.low = self.ej < self.ei   # particle index order equals row order
        # Ahat on the solved rows
        # the solver's own test: float32 differences and squared length,
        # sqrt(rr) < rlap in float32 (pairs at the lattice distance 4 l0 sit
        # on that edge)
        lp = tree.query_pairs(rlap * (1 + 1e-5), output_type="ndarray")
        x32 = pos4[self.rows, :3]
        d32 = x32[lp[:, 1]] - x32[lp[:, 0]]
        rr32 = (d32[:, 0] * d32[:, 0] + d32[:, 1] * d32[:, 1]) + d32[:, 2] * d32[:, 2]
        keep = np.sqrt(rr32) < np.float32(rlap)
        lp = lp[keep]
        dl = np.sqrt(rr32[keep].astype(np.float64))
        w = rlap / dl - 1.0
        self.ai = np.concatenate([lp[:, 0], lp[:, 1]])
        self.aj = np.concatenate([lp[:, 1], lp[:, 0]])
        self.aw = -np.concatenate([w, w]) / np.sqrt(self.d[self.ai] * self.d[self.aj])
        self.m = m

    def ahat(self, v):
        out = v.copy()
        np.add.at(out, self.ai, self.aw * v[self.aj])
        return out

    def mean_edges(self, vals):
        out = np.zeros((self.m, vals.shape[1]))
        np.add.at(out, self.ei, vals)
        inv = np.where(self.cnt > 0, 1.0 / np.maximum(self.cnt, 1), 0.0)
        return out * inv[:, None]

    def factor(self, w):
        """G's lower entries (edge mask self.low) and its diagonal."""
        P = unpack(w)
        e = self.feat
        a1 = self.mean_edges(gelu(e @ P["W1e"].T + P["b1"]))
        h1 = gelu(a1 @ P["V1"].T + P["c1"])
        uh1 = h1 @ P["U2"].T
        a2 = self.mean_edges(gelu(e @ P["W2e"].T + uh1[self.ej] + P["b2"]))
        h2 = gelu(a2 @ P["V2"].T + P["c2"]) + h1
        ra, rb = h2 @ P["Ra"].T, h2 @ P["Rb"].T
        li, lj = self.ei[self.low], self.ej[self.low]
        t = e[self.low] @ P["Re"].T + ra[li] + rb[lj] + P["br"]
        g = gelu(t) @ P["om"]
        gd = softplus(h2 @ P["dl"] + P["bd"][0]) + GMIN
        return li, lj, g, gd

    def loss(self, w, seed):
        li, lj, g, gd = self.factor(w)
        z = probe(seed, self.ids)
        v1 = gd * z                                   # G^T z
        np.add.at(v1, lj, g * z[li])
        v2 = self.ahat(v1)
        n = float(self.m)
        return float(np.log((v1 @ v2) / n) - 2.0 * np.log(gd).sum() / n)


def directional_fd(system, w, v, seed, h=1e-3):
    w = np.asarray(w, np.float64)
    return (system.loss(w + h * v, seed) - system.loss(w - h * v, seed)) / (2 * h)
