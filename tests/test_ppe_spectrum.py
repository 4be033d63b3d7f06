"""Why a local sparse factor cannot cut the PPE's CG iterations by much
(CPU, from the oracle's state): with A = diag(sum w + Aii) - W, the Jacobi
scaled matrix D^-1/2 (-A) D^-1/2 = I - N has its spectrum in
[~Aii/d, ~1.1]; the compressibility term Aii sets the low end, so its
condition number stays near 1/(Aii/d) whatever the scene size.  The
factorized sparse approximate inverse (FSAI), the optimum of the learned
factor's loss over the same r0 pattern, removes only a fraction of the
diagonally scaled CG iterations."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla
from scipy.spatial import cKDTree


def ppe_system(oracle_mod, tmp_path):
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=4, interior=(24, 8, 20), fluid=(10, 8, 16), l0=0.01, dt=5e-4)
    d = str(tmp_path / "p")
    scene.write_case(d, sc)
    o = oracle_mod.Oracle(d, oracle_mod.SEMI_JACOBI, 64)
    o.set_cg(True, 1e-8, 0)
    assert o.step(5) == 0
    st, S = o.state(), o.scalars()
    pos, n, typ = st["pos"], st["n"], st["type"]
    p = sc.params
    rlap = p.rlap * p.dp
    n0, lam, alpha, dt = S["nzero"], S["lambda"], S["alpha"], S["dt"]
    rows = np.nonzero((typ != 2) & (n >= p.beta * n0))[0]
    idx = -np.ones(len(pos), int)
    idx[rows] = np.arange(len(rows))
    pairs = cKDTree(pos).query_pairs(rlap, output_type="ndarray")
    r = np.sqrt(((pos[pairs[:, 0]] - pos[pairs[:, 1]]) ** 2).sum(1))
    keep = (typ[pairs[:, 0]] != 2) & (typ[pairs[:, 1]] != 2) & (r < rlap)
    pairs, w = pairs[keep], rlap / r[keep] - 1
    diag = np.zeros(len(pos))
    np.add.at(diag, pairs[:, 0], w)
    np.add.at(diag, pairs[:, 1], w)
    aii = p.rho * lam * alpha * n0 / (2 * 3 * dt * dt)
    both = (idx[pairs[:, 0]] >= 0) & (idx[pairs[:, 1]] >= 0)
    i, j, ww = idx[pairs[both, 0]], idx[pairs[both, 1]], w[both]
    m = len(rows)
    W = sp.coo_matrix((np.r_[ww, ww], (np.r_[i, j], np.r_[j, i])), shape=(m, m)).tocsr()
    d = diag[rows] + aii
    K = (sp.diags(d) - W).tocsr()
    b = -(n0 - n[rows])
    return K, d, aii, b, pos[rows], p.r0 * p.dp


def cg_iters(K, b, apply_m, tol=1e-8):
    x = np.zeros_like(b); r = b.copy(); z = apply_m(r); q = z.copy(); rz = r @ z
    nb = np.linalg.norm(b)
    for it in range(10000):
        Aq = K @ q
        a = rz / (q @ Aq)
        x += a * q
        r -= a * Aq
        if np.linalg.norm(r) <= tol * nb:
            return it + 1
        z = apply_m(r)
        rz2 = r @ z
        q = z + rz2 / rz * q
        rz = rz2
    return 10000


def test_spectrum_floor_and_fsai_gain(oracle_mod, tmp_path):
    K, d, aii, b, x, r0 = ppe_system(oracle_mod, tmp_path)
    dh = 1 / np.sqrt(d)
    Ah = sp.diags(dh) @ K @ sp.diags(dh)
    lo = sla.eigsh(Ah, k=1, sigma=0, which="LM", return_eigenvectors=False)[0]
    hi = sla.eigsh(Ah, k=1, which="LA", return_eigenvectors=False)[0]
    floor = (aii / d).min()
    assert lo >= 0.9 * floor          # the compressibility term bounds the low end
    assert hi < 1.3
    assert hi / lo < 1.3 / (0.9 * floor)
    ds = cg_iters(K, b, lambda r: r / d)
    # FSAI on the lower r0 pattern (the learned factor's pattern)
    m = len(d)
    nb = cKDTree(x).query_ball_point(x, r0)
    Gi, Gj, Gv = [], [], []
    for i in range(m):
        P = sorted(j for j in nb[i] if j <= i)
        e = np.zeros(len(P)); e[-1] = 1.0
        g = np.linalg.solve(K[P][:, P].toarray(), e)
        g /= np.sqrt(g[-1])
        Gi += [i] * len(P); Gj += P; Gv += list(g)
    G = sp.csr_matrix((Gv, (Gi, Gj)), shape=(m, m))
    GT = G.T.tocsr()
    fsai = cg_iters(K, b, lambda r: GT @ (G @ r))
    assert fsai < ds                  # the pattern helps ...
    assert fsai > 0.6 * ds            # ... by well under 2x
