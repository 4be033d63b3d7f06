"""Synthetic dam-break scenes written as the reference's input files.

The reference reads two text files from the working directory:

* ``input.dat``: 16 "label line / value line" pairs in a fixed order
  (``MPS_CAL_expl_v1.0/MPS.cpp:173-331``);
* ``GEO.dat``: ``np nb2 nb1`` then np positions, np velocities and np
  pressures, particles ordered dummy (type 2), wall (type 1), fluid (type 0)
  (``MPS_CAL_expl_v1.0/MPS.cpp:336-407``), as the reference's generator
  ``MPS_INI/main.cpp:13-196`` writes them.

The generator here builds closed tanks on a cubic lattice of spacing ``l0``:
``wall_layers`` layers of type-1 particles around the interior and
``dummy_layers`` layers of type-2 particles outside them on all six faces,
fluid blocks inside, optional box obstacles (wall + dummy shells), and a
uniform jitter of +-``jitter`` * l0 per coordinate drawn from splitmix64 of
(seed, particle, axis).  Axes: x = length, y = depth, z = height (gravity is
-z in the reference, ``common.h:44``).

Every coordinate is rounded to float32 and printed with a decimal that parses
back to exactly that float32 value both as ``%f`` (float) and ``%lf``
(double), so the float and double builds of the reference see identical
particles.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Sequence, Tuple

import numpy as np

# input.dat labels in the reference's order (MPS_CAL_expl_v1.0/input.dat)
INPUT_LABELS = (
    "DIMENTION",
    "FLUID RHO",
    "FLUID DYNAMICS VISCOSITY",
    "INITIAL PARTICLE DISTANCE(DP)",
    "R0(times of DP)",
    "RLAP(times of DP)",
    "BETA",
    "NUMERICAL SPEED OF SOUND",
    "CFL NUMBER",
    "COLLISION DISTANCE(times of DP)",
    "COLLISION RATE",
    "MAX TIME STEP",
    "MIN TIME STEP(times of MAX)",
    "TT TOTAL CALCULATION TIME",
    "TOUT TIME STEP OF OUTPUT",
    "MAXIMUM DISPLACEMENT OF THE GEOMETRY",
)


@dataclasses.dataclass
class Params:
    """The 16 values of input.dat, unscaled (r0, rlap, col_dis in units of dp)."""

    dim: int = 3
    rho: float = 1000.0
    niu: float = 1e-6
    dp: float = 0.02
    r0: float = 2.1
    rlap: float = 4.0
    beta: float = 0.97
    cs: float = 20.0
    cfl: float = 0.2
    col_dis: float = 0.8
    col_rate: float = 2.0
    dt_max: float = 1e-4
    dt_min: float = 1e-3
    tt: float = 0.05
    tout: float = 1.0e9
    max_dis: float = 0.02

    def values(self) -> Tuple:
        return (self.dim, self.rho, self.niu, self.dp, self.r0, self.rlap, self.beta, self.cs,
                self.cfl, self.col_dis, self.col_rate, self.dt_max, self.dt_min, self.tt,
                self.tout, self.max_dis)


@dataclasses.dataclass
class Box:
    """Axis-aligned block of lattice sites [x0, x0+nx) x [y0, y0+ny) x [z0, z0+nz)
    in interior-site coordinates (the interior starts at site 0)."""

    x0: int
    y0: int
    z0: int
    nx: int
    ny: int
    nz: int


@dataclasses.dataclass
class Scene:
    l0: float
    interior: Tuple[int, int, int]  # (nx, ny, nz) interior sites
    fluid: List[Box]
    obstacles: List[Box] = dataclasses.field(default_factory=list)
    wall_layers: int = 2
    dummy_layers: int = 2
    jitter: float = 1e-4
    seed: int = 0
    params: Params = dataclasses.field(default_factory=Params)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser over a uint64 array (Steele, Lea & Flood 2014)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def jitter_values(seed: int, count: int) -> np.ndarray:
    """count uniform values in [-1, 1) from splitmix64(seed * 2^40 + k)."""
    k = np.arange(count, dtype=np.uint64) + np.uint64((seed & 0xFFFFFF) << 40)
    u = (splitmix64(k) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def _site_types(scene: Scene):
    """Lattice sites and their type: 2 dummy, 1 wall, 0 fluid, -1 empty."""
    nx, ny, nz = scene.interior
    S = scene.wall_layers + scene.dummy_layers
    X, Y, Z = nx + 2 * S, ny + 2 * S, nz + 2 * S
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    ix, iy, iz = x - S, y - S, z - S  # interior-site coordinates

    def outside(v, n):
        return np.where(v < 0, -v, np.where(v >= n, v - n + 1, 0))

    d = np.maximum(np.maximum(outside(ix, nx), outside(iy, ny)), outside(iz, nz))
    t = np.full(d.shape, -1, dtype=np.int8)
    t[(d >= 1) & (d <= scene.wall_layers)] = 1
    t[d > scene.wall_layers] = 2
    for b in scene.fluid:
        m = ((ix >= b.x0) & (ix < b.x0 + b.nx) & (iy >= b.y0) & (iy < b.y0 + b.ny)
             & (iz >= b.z0) & (iz < b.z0 + b.nz) & (d == 0))
        t[m] = 0
    for b in scene.obstacles:
        # solid box: its outer wall_layers shell is type 1, everything inside type 2
        def inside(v, a, n):
            return (v >= a) & (v < a + n)

        m = inside(ix, b.x0, b.nx) & inside(iy, b.y0, b.ny) & inside(iz, b.z0, b.nz) & (d == 0)
        dx = np.minimum(ix - b.x0, b.x0 + b.nx - 1 - ix)
        dy = np.minimum(iy - b.y0, b.y0 + b.ny - 1 - iy)
        dz = np.minimum(iz - b.z0, b.z0 + b.nz - 1 - iz)
        depth = np.minimum(np.minimum(dx, dy), dz)
        t[m & (depth < scene.wall_layers)] = 1
        t[m & (depth >= scene.wall_layers)] = 2
    return x.ravel(), y.ravel(), z.ravel(), t.ravel()


def build(scene: Scene):
    """Return (pos float32 [np,3], nb2, nb1) in the GEO.dat order b2, b1, fluid;
    each type in lattice order z outer, y, x inner (as MPS_INI writes it)."""
    x, y, z, t = _site_types(scene)
    parts = []
    for ty in (2, 1, 0):
        m = t == ty
        parts.append(np.stack([x[m], y[m], z[m]], axis=1))
    nb2, nb1 = len(parts[0]), len(parts[1])
    sites = np.concatenate(parts).astype(np.float64)
    pos = sites * scene.l0
    if scene.jitter:
        j = jitter_values(scene.seed, pos.size).reshape(pos.shape)
        pos = pos + j * (scene.jitter * scene.l0)
    return pos.astype(np.float32), nb2, nb1


def _fmt(a: np.ndarray) -> str:
    # repr of the float32 value as a Python float: shortest decimal that parses
    # back to that exact value as double, hence also as float.
    return " ".join(repr(v) for v in a.astype(np.float64).tolist())


def write_input_dat(path: str, p: Params) -> None:
    lines = []
    for label, v in zip(INPUT_LABELS, p.values()):
        lines.append(label)
        lines.append(str(int(v)) if label == "DIMENTION" else repr(float(v)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_geo_dat(path: str, pos: np.ndarray, nb2: int, nb1: int,
                  vel: np.ndarray | None = None, press: np.ndarray | None = None) -> None:
    n = len(pos)
    vel = np.zeros((n, 3), np.float32) if vel is None else vel
    press = np.zeros(n, np.float32) if press is None else press
    with open(path, "w") as f:
        f.write(f"{n} {nb2} {nb1}\n")
        f.write(_fmt(pos.ravel()) + " \n")
        f.write(_fmt(vel.ravel()) + " \n")
        f.write(_fmt(press.ravel()) + " \n")


def write_case(directory: str, scene: Scene):
    """Write input.dat and GEO.dat for ``scene`` into ``directory``."""
    os.makedirs(directory, exist_ok=True)
    pos, nb2, nb1 = build(scene)
    write_input_dat(os.path.join(directory, "input.dat"), scene.params)
    write_geo_dat(os.path.join(directory, "GEO.dat"), pos, nb2, nb1)
    return pos, nb2, nb1


# ---- the workloads ------------------------------------------------------------


def dam_break_explicit(seed: int = 0, steps: int = 500) -> Scene:
    """Explicit EOS dam break: l0 = 0.02 m, tank interior 1.6 x 0.4 x 1.0 m
    (80 x 20 x 50 sites, x length, y depth, z height), 2 wall + 2 dummy
    layers, water column 0.4 x 0.2 x 0.8 m (20 x 10 x 40 = 8,000 fluid
    particles) in the corner; N = 70,912.  r0 = 2.1 l0, rlap = 4.0 l0,
    c0 = 20 m/s, dt = 1e-4 s."""
    p = Params(dim=3, dp=0.02, r0=2.1, rlap=4.0, cs=20.0, dt_max=1e-4, tt=steps * 1e-4,
               max_dis=0.02)
    return Scene(l0=0.02, interior=(80, 20, 50), fluid=[Box(0, 0, 0, 20, 10, 40)], seed=seed,
                 params=p)


def dam_break_semi(seed: int = 0, steps: int = 1000) -> Scene:
    """Semi-implicit dam break: the same tank at l0 = 0.01 m (160 x 40 x 100
    interior sites), water column 0.4 x 0.25 x 0.8 m (40 x 25 x 80 = 80,000
    fluid particles); N = 310,912.  dt = 5e-4 s."""
    p = Params(dim=3, dp=0.01, r0=2.1, rlap=4.0, cs=20.0, dt_max=5e-4, tt=steps * 5e-4,
               max_dis=0.01)
    return Scene(l0=0.01, interior=(160, 40, 100), fluid=[Box(0, 0, 0, 40, 25, 80)], seed=seed,
                 params=p)


def batch_scenes(n: int = 64, seed: int = 0):
    """Batched workload: n dam-break tanks at l0 = 0.01 m whose fluid counts
    are log-uniform in [5,000, 60,000].  Per tank (from a generator seeded by
    `seed`): fluid depth 10-20 sites, column height/width 1-2, tank interior
    3x the column width, the column's depth, 1.2x its height plus 2 sites;
    tank acceleration amplitude uniform in [0, 2] m/s^2 and frequency in
    [0.5, 2] Hz.  Returns [(Scene, accel_amp, accel_freq)]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nf = float(np.exp(rng.uniform(np.log(5000.0), np.log(60000.0))))
        ny = int(rng.integers(10, 21))
        aspect = float(rng.uniform(1.0, 2.0))
        nx = max(4, int(round(np.sqrt(nf / (ny * aspect)))))
        nz = max(4, int(round(nf / (ny * nx))))
        interior = (3 * nx, ny, int(np.ceil(1.2 * nz)) + 2)
        p = Params(dim=3, dp=0.01, r0=2.1, rlap=4.0, cs=20.0, dt_max=5e-4, tt=1.0, max_dis=0.01)
        sc = Scene(l0=0.01, interior=interior, fluid=[Box(0, 0, 0, nx, ny, nz)], seed=seed * 1000 + k,
                   params=p)
        out.append((sc, float(rng.uniform(0.0, 2.0)), float(rng.uniform(0.5, 2.0))))
    return out


def surface_grid(scene: Scene, shape):
    """Origin and spacing of a marching-cubes vertex grid of `shape`
    (vertices per axis) spanning the tank interior's lattice sites."""
    S = scene.wall_layers + scene.dummy_layers
    origin = tuple(S * scene.l0 for _ in range(3))
    spacing = tuple((n - 1) * scene.l0 / (m - 1) for n, m in zip(scene.interior, shape))
    return origin, spacing


def small_tank(seed: int = 0, interior=(14, 6, 12), fluid=(5, 4, 8), l0: float = 0.02,
               rlap: float = 4.0, dt: float = 1e-4, cs: float = 20.0) -> Scene:
    """A few-thousand-particle tank for parity tests."""
    p = Params(dim=3, dp=l0, r0=2.1, rlap=rlap, cs=cs, dt_max=dt, tt=1.0, max_dis=l0)
    return Scene(l0=l0, interior=tuple(interior), fluid=[Box(0, 0, 0, *fluid)], seed=seed,
                 params=p)


def large_obstacle(seed: int = 0) -> Scene:
    """2,000,000-fluid-particle dam break with a 0.15 x 0.15 x 0.3 m box
    obstacle at x = 1.0 m in a 2.4 x 1.2 x 0.6 m tank, l0 = 0.005 m."""
    p = Params(dim=3, dp=0.005, r0=2.1, rlap=4.0, cs=20.0, dt_max=2.5e-4, tt=2000 * 2.5e-4,
               max_dis=0.005)
    # interior 480 (x) x 120 (y) x 240 (z); fluid column 0.5 x 0.6 x 0.333 m
    fluid = [Box(0, 0, 0, 100, 120, 167)]
    obstacle = [Box(200, 45, 0, 30, 30, 60)]
    return Scene(l0=0.005, interior=(480, 120, 240), fluid=fluid, obstacles=obstacle, seed=seed,
                 params=p)
