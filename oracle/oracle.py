"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

* :class:`Oracle` wraps ``oracle/liboracle.so`` (the project's C restatement of
  the reference's CPU step, ``oracle/mps_oracle_impl.inc``).
* :func:`run_reference` runs the reference's own CPU step classes built by
  ``oracle/Makefile`` (``oracle/_ref/ref_expl``, ``oracle/_ref/ref_semi``) and
  :func:`read_dump` parses their state dumps.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

EXPL, SEMI_SEQ, SEMI_JACOBI = 0, 1, 2
PHASE = dict(update_dt=0, visc=1, divide_cell=2, collision=3, cal_n=4, pres_expl=5, dash=6, ppe=7)

_lib = None


def reference_dir() -> Optional[str]:
    """The reference source tree that oracle/Makefile reads (its REF: the
    environment variable MPS_REFERENCE_DIR, else the recipe's default), or
    None when that directory is absent (as on a machine without the
    reference, where only the committed fixtures are used)."""
    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = r.stdout.strip().splitlines()[-1].strip() if r.stdout.strip() else ""
    return path if path and os.path.isdir(path) else None


def build(ref: Optional[str] = None, quiet: bool = True) -> None:
    """Build liboracle.so (and the reference binaries when the reference tree
    is present)."""
    cmd = ["make", "-C", HERE]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for s, rt in (("f32", C.c_float), ("f64", C.c_double)):
            P = C.POINTER(rt)
            U = C.POINTER(C.c_uint32)
            getattr(L, f"orc_create_{s}").restype = C.c_void_p
            getattr(L, f"orc_create_{s}").argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_int)]
            getattr(L, f"orc_destroy_{s}").argtypes = [C.c_void_p]
            getattr(L, f"orc_step_{s}").argtypes = [C.c_void_p]
            getattr(L, f"orc_step_{s}").restype = C.c_int
            getattr(L, f"orc_set_cg_{s}").argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
            getattr(L, f"orc_set_body_force_{s}").argtypes = [C.c_void_p, C.c_double, C.c_double]
            D3 = C.c_double * 3
            getattr(L, f"orc_add_wall_motion_{s}").argtypes = [C.c_void_p, D3, D3, D3, D3, C.c_double, C.c_double]
            getattr(L, f"orc_add_wall_motion_{s}").restype = C.c_int
            getattr(L, f"orc_clear_wall_motion_{s}").argtypes = [C.c_void_p]
            getattr(L, f"orc_set_visc_implicit_{s}").argtypes = [C.c_void_p, C.c_int]
            getattr(L, f"orc_counts_{s}").argtypes = [C.c_void_p] + [U] * 5
            getattr(L, f"orc_scalars_{s}").argtypes = [C.c_void_p, C.POINTER(C.c_double)]
            getattr(L, f"orc_get_state_{s}").argtypes = [C.c_void_p, U, U, P, P, P, P]
            getattr(L, f"orc_set_state_{s}").argtypes = [C.c_void_p, P, P, P, P]
            getattr(L, f"orc_get_cells_{s}").argtypes = [C.c_void_p, U, U, U]
            getattr(L, f"orc_get_normal_{s}").argtypes = [C.c_void_p, U]
            getattr(L, f"orc_divide_cell_{s}").argtypes = [C.c_void_p]
            getattr(L, f"orc_divide_cell_{s}").restype = C.c_int
            getattr(L, f"orc_phase_{s}").argtypes = [C.c_void_p, C.c_int]
            getattr(L, f"orc_cg_iters_{s}").argtypes = [C.c_void_p]
            getattr(L, f"orc_cg_iters_{s}").restype = C.c_int
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Oracle:
    """One scene on the CPU oracle (float32 or float64)."""

    def __init__(self, case_dir: str, variant: int = EXPL, precision: int = 32):
        self.s = "f32" if precision == 32 else "f64"
        self.dtype = np.float32 if precision == 32 else np.float64
        self.ct = C.c_float if precision == 32 else C.c_double
        L = lib()
        st = C.c_int(0)
        self.h = getattr(L, f"orc_create_{self.s}")(
            os.path.join(case_dir, "input.dat").encode(), os.path.join(case_dir, "GEO.dat").encode(),
            variant, C.byref(st))
        self.status = st.value
        if self.status != 0:
            raise RuntimeError(f"oracle create failed with status {self.status}")

    def _f(self, name):
        return getattr(lib(), f"orc_{name}_{self.s}")

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_cg(self, relative: bool, tol: float = 1e-8, max_iter: int = 0):
        self._f("set_cg")(self.h, int(relative), tol, max_iter)

    def set_body_force(self, amp: float, freq: float):
        """Tank acceleration amp*sin(2*pi*freq*t) along x (amp and freq are
        taken as float32 values, as the GPU API takes them)."""
        self._f("set_body_force")(self.h, C.c_double(float(np.float32(amp))),
                                  C.c_double(float(np.float32(freq))))

    def add_wall_motion(self, lo, hi, vel=(0.0, 0.0, 0.0), amp=(0.0, 0.0, 0.0), freq: float = 0.0,
                        phase: float = 0.0) -> int:
        """Prescribed motion of the wall and dummy particles inside [lo, hi]
        (all values taken as float32, as the GPU API takes them); returns the
        number selected."""
        D3 = C.c_double * 3
        f = lambda v: D3(*[float(np.float32(x)) for x in v])
        n = self._f("add_wall_motion")(self.h, f(lo), f(hi), f(vel), f(amp), float(np.float32(freq)),
                                       float(np.float32(phase)))
        if n < 0:
            raise RuntimeError("too many wall motions")
        return n

    def set_visc_implicit(self, on: bool = True):
        """Viscosity by Crank-Nicolson (the reference's MPS_CPU_IMPL step)."""
        self._f("set_visc_implicit")(self.h, int(on))

    def clear_wall_motion(self):
        self._f("clear_wall_motion")(self.h)

    def step(self, n: int = 1) -> int:
        st = 0
        for _ in range(n):
            st = self._f("step")(self.h)
            if st:
                break
        return st

    def phase(self, name: str):
        self._f("phase")(self.h, PHASE[name])

    def counts(self) -> Dict[str, int]:
        v = [C.c_uint32() for _ in range(5)]
        self._f("counts")(self.h, *[C.byref(x) for x in v])
        return dict(zip(("np", "nb2", "nb1", "nexcl", "ncells"), [x.value for x in v]))

    def scalars(self) -> Dict[str, float]:
        o = (C.c_double * 16)()
        self._f("scalars")(self.h, o)
        names = ("nzero", "lambda", "dt", "time", "cell_size", "left", "back", "bottom", "c_lap",
                 "one_over_alpha", "alpha", "cg_iters", "cg_relres", "step", "status", "dims")
        return dict(zip(names, list(o)))

    def state(self) -> Dict[str, np.ndarray]:
        n = self.counts()["np"]
        out = dict(id=np.empty(n, np.uint32), type=np.empty(n, np.uint32),
                   pos=np.empty((n, 3), self.dtype), vel=np.empty((n, 3), self.dtype),
                   press=np.empty(n, self.dtype), n=np.empty(n, self.dtype))
        self._f("get_state")(self.h, _ptr(out["id"], C.c_uint32), _ptr(out["type"], C.c_uint32),
                             _ptr(out["pos"], self.ct), _ptr(out["vel"], self.ct),
                             _ptr(out["press"], self.ct), _ptr(out["n"], self.ct))
        return out

    def set_state(self, pos=None, vel=None, press=None, n=None):
        def c(a):
            return None if a is None else np.ascontiguousarray(a, self.dtype)
        pos, vel, press, n = c(pos), c(vel), c(press), c(n)
        self._f("set_state")(self.h, _ptr(pos, self.ct), _ptr(vel, self.ct), _ptr(press, self.ct),
                             _ptr(n, self.ct))

    def cells(self):
        c = self.counts()
        cell_of = np.empty(c["np"], np.uint32)
        start = np.empty(c["ncells"], np.uint32)
        end = np.empty(c["ncells"], np.uint32)
        self._f("get_cells")(self.h, _ptr(cell_of, C.c_uint32), _ptr(start, C.c_uint32),
                             _ptr(end, C.c_uint32))
        return cell_of, start, end

    def normal(self):
        out = np.empty(self.counts()["np"], np.uint32)
        self._f("get_normal")(self.h, _ptr(out, C.c_uint32))
        return out

    def cg_iters(self) -> int:
        return self._f("cg_iters")(self.h)


# ---- the reference's own build -------------------------------------------------

def have_reference_build() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_expl")) and os.path.exists(
        os.path.join(REF_DIR, "ref_semi"))


def run_reference(kind: str, case_dir: str, nsteps: int, dump_every: int, out_path: str,
                  threads: int = 1, timeout: float = 600.0, untimed: int = 0) -> dict:
    """Run oracle/_ref/ref_{expl,semi} on case_dir; returns its timing JSON
    (steps_s covers the steps after the first `untimed` ones)."""
    exe = os.path.join(REF_DIR, f"ref_{kind}")
    r = subprocess.run([exe, case_dir, str(nsteps), str(dump_every), out_path, str(threads), str(untimed)],
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{exe} failed ({r.returncode}): {r.stderr[-2000:]}")
    return json.loads(r.stderr.strip().splitlines()[-1])


def read_dump(path: str) -> dict:
    """Parse a dump written by oracle/ref_harness.cpp."""
    with open(path, "rb") as f:
        buf = f.read()
    off = 0

    def take(dt, count):
        nonlocal off
        a = np.frombuffer(buf, dtype=dt, count=count, offset=off)
        off += a.nbytes
        return a

    assert buf[:4] == b"MPSD"
    off = 4
    ver, rsize, np_, nb2, nb1 = take(np.uint32, 5)
    rdt = np.float32 if rsize == 4 else np.float64
    nzero, lam, cell_size, left, back, bottom = take(np.float64, 6)
    cdx, cdy, cdz, ncells = take(np.uint32, 4)
    hdr = dict(np=int(np_), nb2=int(nb2), nb1=int(nb1), nzero=nzero, lambda_=lam,
               cell_size=cell_size, left=left, back=back, bottom=bottom, cdx=int(cdx),
               cdy=int(cdy), cdz=int(cdz), ncells=int(ncells))
    hdr["cell_of"] = take(np.uint32, np_).copy()
    hdr["cell_start"] = take(np.uint32, ncells).copy()
    hdr["cell_end"] = take(np.uint32, ncells).copy()
    hdr["normal"] = take(np.uint32, np_).copy()
    steps: List[dict] = []
    while off < len(buf):
        magic, step, n = take(np.uint32, 3)
        assert magic == 0x53544550
        dt, t = take(np.float64, 2)
        rec = dict(step=int(step), np=int(n), dt=float(dt), time=float(t))
        rec["id"] = take(np.uint32, n).copy()
        rec["type"] = take(np.uint32, n).copy()
        rec["pos"] = take(rdt, 3 * n).reshape(n, 3).copy()
        rec["vel"] = take(rdt, 3 * n).reshape(n, 3).copy()
        rec["press"] = take(rdt, n).copy()
        rec["n"] = take(rdt, n).copy()
        steps.append(rec)
    hdr["steps"] = steps
    return hdr
