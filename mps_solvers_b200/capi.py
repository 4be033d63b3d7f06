"""ctypes binding of libmps_b200.so (include/mps_capi.h) and a Python mirror
of the reference's step-class interface.

:class:`MPS_GPU_EXPL` has the members a caller of the reference's
``MPS_GPU_EXPL`` / ``MPS_GPU`` uses (``Initial``, ``step``, ``mps_cal`` and the
getters of ``MPS_CAL_/MPS_GPU.h:157-166``); every call goes through the C ABI.
The library is the only compute path: when it is missing this module raises
instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmps_b200.so")

METHOD_EXPLICIT, METHOD_SEMI_IMPLICIT = 0, 1
ARITH_EXACT, ARITH_FAST = 0, 1
PRECOND_DIAGONAL, PRECOND_LEARNED = 0, 1
ORDER_SORTED, ORDER_BY_ID = 0, 1
PHASE = dict(update_dt=0, visc=1, divide_cell=2, collision=3, cal_n=4, pres_expl=5, dash=6, ppe=7)

NOALLOC_MAX_PARTICLES = 524288
NOALLOC_MAX_CELLS = 524288

STATUS = {0: "MPS_OK", 1: "MPS_ERR_IO", 2: "MPS_ERR_CELLS_TOO_THIN", 3: "MPS_ERR_DT_TOO_SMALL",
          4: "MPS_ERR_PARTICLE_OUT", 5: "MPS_ERR_CG_NOT_CONVERGED", 6: "MPS_ERR_DEVICE_TIMEOUT",
          7: "MPS_ERR_CUDA", 8: "MPS_ERR_NAN", 9: "MPS_ERR_INVALID", 10: "MPS_ERR_CAPACITY"}

# every function include/mps_capi.h declares
EXPORTS = ("mps_status_string", "mps_default_options", "mps_create", "mps_create_from_arrays",
           "mps_destroy", "mps_step", "mps_step_async", "mps_run", "mps_get_counts", "mps_get_state", "mps_set_state",
           "mps_get_cell_tables", "mps_get_grid", "mps_get_scalars", "mps_get_normal_ids",
           "mps_phase", "mps_get_stream", "mps_write_case", "mps_last_error", "mps_cell_sort_dev",
           "mps_profile_steps", "mps_stage_name", "mps_cell_sort_dev_noalloc",
           "mps_precond_num_params", "mps_precond_get_params", "mps_precond_set_params",
           "mps_precond_loss_grad", "mps_precond_train", "mps_ppe_snapshot",
           "mps_batch_create", "mps_batch_step", "mps_batch_scene_info", "mps_set_body_force",
           "mps_autotune", "mps_surface_setup", "mps_surface_extract_async", "mps_surface_extract",
           "mps_surface_get", "mps_surface_vertex_values", "mps_surface_write_stl",
           "mps_surface_case_table", "mps_precond_tensor_cores", "mps_add_wall_motion",
           "mps_clear_wall_motion", "mps_set_device_wait_limit", "mps_ppe_stencil", "mps_apply_tuning",
           "mps_precond_train_tensor_cores")


class mps_options(C.Structure):
    _fields_ = [("method", C.c_int), ("arith", C.c_int), ("device", C.c_int),
                ("use_graph", C.c_int), ("cg_tol", C.c_double), ("cg_max_iter", C.c_int),
                ("cg_check_every", C.c_int), ("precond", C.c_int), ("capacity", C.c_uint32),
                ("cg_inner_digits", C.c_int), ("ppe_pipelined", C.c_int), ("ppe_l2_keep_mb", C.c_int),
                ("visc_implicit", C.c_int), ("rebuild_merge", C.c_int), ("ppe_layout", C.c_int),
                ("ppe_smem_chunks", C.c_int), ("precond_every", C.c_int)]


class mps_params(C.Structure):
    _fields_ = [("dim", C.c_int)] + [(n, C.c_float) for n in (
        "rho", "niu", "dp", "rzero", "rlap", "beta", "cs", "cfl", "col_dis", "col_rate", "dt_max",
        "dt_min", "tt", "tout", "max_dis")]


class mps_step_stats(C.Structure):
    _fields_ = [("np", C.c_uint32), ("nexcl", C.c_uint32), ("step", C.c_int), ("time", C.c_float),
                ("dt", C.c_float), ("cg_iters", C.c_int), ("cg_relres", C.c_double),
                ("status", C.c_int), ("ms", C.c_float), ("cg_outer", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class mps_grid(C.Structure):
    _fields_ = [("left", C.c_float), ("back", C.c_float), ("bottom", C.c_float),
                ("cell_size", C.c_float), ("cdx", C.c_uint32), ("cdy", C.c_uint32),
                ("cdz", C.c_uint32), ("ncells", C.c_uint32), ("dim", C.c_int), ("cell_yz", C.c_float)]


class mps_scene_spec(C.Structure):
    _fields_ = [("input_dat", C.c_char_p), ("geo_dat", C.c_char_p), ("accel_amp", C.c_float),
                ("accel_freq", C.c_float), ("reserved", C.c_uint32 * 4)]


class mps_scene_info(C.Structure):
    _fields_ = [("id_base", C.c_uint32), ("np0", C.c_uint32), ("nb2", C.c_uint32), ("nb1", C.c_uint32),
                ("time", C.c_float), ("dt", C.c_float), ("nzero", C.c_float), ("pad", C.c_float),
                ("cg_iters", C.c_int), ("cg_outer", C.c_int), ("cg_relres", C.c_double),
                ("reserved", C.c_uint32 * 4)]


class mps_tune_report(C.Structure):
    _fields_ = [("stage_threads", C.c_int), ("ppe_threads", C.c_int), ("ppe_stored_weights", C.c_int),
                ("ppe_pipelined", C.c_int), ("stage_ms", C.c_float * 3), ("ppe_ms", C.c_float * 9),
                ("ppe_compact", C.c_int), ("ppe_compact_ms", C.c_float * 3)]


class mps_surface_grid(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("pad", C.c_uint32),
                ("origin", C.c_float * 3), ("spacing", C.c_float * 3), ("reserved", C.c_uint32 * 4)]


class MPSError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """Load libmps_b200.so; raise when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -m mps_solvers_b200.build` (no other compute path exists)")
        L = C.CDLL(LIB_PATH)
        H = C.c_void_p
        U = C.POINTER(C.c_uint32)
        Fp = C.POINTER(C.c_float)
        sig = {
            "mps_status_string": (C.c_char_p, [C.c_int]),
            "mps_default_options": (None, [C.POINTER(mps_options)]),
            "mps_create": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(mps_options), C.POINTER(H)]),
            "mps_create_from_arrays": (C.c_int, [C.POINTER(mps_params), C.c_uint32, C.c_uint32,
                                                 C.c_uint32, Fp, Fp, Fp, C.POINTER(mps_options),
                                                 C.POINTER(H)]),
            "mps_destroy": (None, [H]),
            "mps_step": (C.c_int, [H, C.c_int, C.POINTER(mps_step_stats)]),
            "mps_run": (C.c_int, [H, C.c_char_p]),
            "mps_step_async": (C.c_int, [H, C.c_int]),
            "mps_get_counts": (C.c_int, [H, U, U, U, U]),
            "mps_get_state": (C.c_int, [H, U, U, Fp, Fp, Fp, Fp, C.c_int]),
            "mps_set_state": (C.c_int, [H, Fp, Fp, Fp, Fp]),
            "mps_get_cell_tables": (C.c_int, [H, U, U, U]),
            "mps_get_grid": (C.c_int, [H, C.POINTER(mps_grid)]),
            "mps_get_scalars": (C.c_int, [H, C.POINTER(C.c_double)]),
            "mps_get_normal_ids": (C.c_int, [H, U]),
            "mps_phase": (C.c_int, [H, C.c_int]),
            "mps_get_stream": (C.c_int, [H, C.POINTER(C.c_void_p)]),
            "mps_write_case": (C.c_int, [H, C.c_char_p, C.c_int]),
            "mps_last_error": (C.c_char_p, [H]),
            "mps_profile_steps": (C.c_int, [H, C.c_int, C.POINTER(C.c_double), C.c_int,
                                            C.POINTER(C.c_int)]),
            "mps_stage_name": (C.c_char_p, [C.c_int]),
            "mps_precond_num_params": (C.c_uint32, []),
            "mps_precond_get_params": (C.c_int, [H, Fp, C.c_uint32]),
            "mps_precond_set_params": (C.c_int, [H, Fp, C.c_uint32]),
            "mps_precond_loss_grad": (C.c_int, [H, C.c_uint64, C.POINTER(C.c_double), Fp]),
            "mps_precond_train": (C.c_int, [H, C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
            "mps_ppe_snapshot": (C.c_int, [H, Fp, Fp, U, U, C.POINTER(C.c_double), U]),
            "mps_cell_sort_dev": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(mps_grid), C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
            "mps_cell_sort_dev_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(mps_grid),
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p]),
            "mps_batch_create": (C.c_int, [C.POINTER(mps_scene_spec), C.c_uint32, C.POINTER(mps_options),
                                           C.POINTER(H)]),
            "mps_batch_step": (C.c_int, [H, C.c_int, C.POINTER(mps_step_stats)]),
            "mps_batch_scene_info": (C.c_int, [H, C.c_uint32, C.POINTER(mps_scene_info)]),
            "mps_set_body_force": (C.c_int, [H, C.c_uint32, C.c_float, C.c_float]),
            "mps_add_wall_motion": (C.c_int, [H, Fp, Fp, Fp, Fp, C.c_float, C.c_float, U]),
            "mps_clear_wall_motion": (C.c_int, [H]),
            "mps_set_device_wait_limit": (C.c_int, [H, C.c_uint64]),
            "mps_ppe_stencil": (C.c_int, [H, U, U, Fp, C.c_uint64, C.POINTER(C.c_uint64)]),
            "mps_autotune": (C.c_int, [H, C.c_int, C.POINTER(mps_tune_report)]),
            "mps_apply_tuning": (C.c_int, [H, C.POINTER(mps_tune_report)]),
            "mps_surface_setup": (C.c_int, [H, C.POINTER(mps_surface_grid), C.c_uint32]),
            "mps_surface_extract_async": (C.c_int, [H]),
            "mps_surface_extract": (C.c_int, [H, U]),
            "mps_surface_get": (C.c_int, [H, Fp, Fp, C.c_uint32, U]),
            "mps_surface_vertex_values": (C.c_int, [H, Fp, Fp]),
            "mps_surface_write_stl": (C.c_int, [H, C.c_char_p]),
            "mps_surface_case_table": (C.c_int, [C.POINTER(C.c_uint8), C.POINTER(C.c_int8)]),
            "mps_precond_tensor_cores": (C.c_int, [H, C.c_int, C.POINTER(C.c_double)]),
            "mps_precond_train_tensor_cores": (C.c_int, [H, C.c_int]),
        }
        for name, (rt, args) in sig.items():
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = args
        _lib = L
    return _lib


def default_options(**kw) -> mps_options:
    o = mps_options()
    lib().mps_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _p(a, t=C.c_float):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def surface_case_table():
    """The library's generated marching-cubes table: list of triangles
    (edge triples) per case."""
    n = (C.c_uint8 * 256)()
    t = (C.c_int8 * (256 * 16))()
    st = lib().mps_surface_case_table(n, t)
    if st != 0:
        raise MPSError(st, "case table")
    return [[tuple(t[16 * c + 3 * k + j] for j in range(3)) for k in range(n[c])] for c in range(256)]


class Simulation:
    """One scene on one GPU through the C ABI."""

    def __init__(self, case_dir: Optional[str] = None, *, input_dat: Optional[str] = None,
                 geo_dat: Optional[str] = None, options: Optional[mps_options] = None, **opt):
        L = lib()
        if options is None:
            options = default_options(**opt)
        self.options = options
        if case_dir is not None:
            input_dat = os.path.join(case_dir, "input.dat")
            geo_dat = os.path.join(case_dir, "GEO.dat")
        h = C.c_void_p()
        st = L.mps_create(input_dat.encode(), geo_dat.encode(), C.byref(options), C.byref(h))
        self.h = h
        if st != 0:
            msg = L.mps_last_error(h).decode() if h else ""
            self.close()
            raise MPSError(st, msg)

    @classmethod
    def from_arrays(cls, params: mps_params, pos: np.ndarray, nb2: int, nb1: int,
                    vel: Optional[np.ndarray] = None, press: Optional[np.ndarray] = None,
                    options: Optional[mps_options] = None, **opt) -> "Simulation":
        self = cls.__new__(cls)
        L = lib()
        self.options = options if options is not None else default_options(**opt)
        pos = np.ascontiguousarray(pos, np.float32)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32)
        press = None if press is None else np.ascontiguousarray(press, np.float32)
        h = C.c_void_p()
        st = L.mps_create_from_arrays(C.byref(params), len(pos), nb2, nb1, _p(pos), _p(vel),
                                      _p(press), C.byref(self.options), C.byref(h))
        self.h = h
        if st != 0:
            msg = L.mps_last_error(h).decode() if h else ""
            self.close()
            raise MPSError(st, msg)
        return self

    @classmethod
    def batch(cls, case_dirs, accel=None, options: Optional[mps_options] = None, **opt) -> "Simulation":
        """A batch handle over the scenes in `case_dirs` (each with input.dat
        and GEO.dat); accel[s] = (amplitude m/s^2, frequency Hz) of scene s's
        tank acceleration."""
        self = cls.__new__(cls)
        L = lib()
        self.options = options if options is not None else default_options(**opt)
        n = len(case_dirs)
        specs = (mps_scene_spec * n)()
        keep = []
        for s, d in enumerate(case_dirs):
            a = os.path.join(d, "input.dat").encode()
            g = os.path.join(d, "GEO.dat").encode()
            keep += [a, g]
            specs[s].input_dat = a
            specs[s].geo_dat = g
            amp, freq = accel[s] if accel is not None else (0.0, 0.0)
            specs[s].accel_amp = amp
            specs[s].accel_freq = freq
        h = C.c_void_p()
        st = L.mps_batch_create(specs, n, C.byref(self.options), C.byref(h))
        self.h = h
        if st != 0:
            msg = L.mps_last_error(h).decode() if h else ""
            self.close()
            raise MPSError(st, msg)
        self.nscenes = n
        return self

    def _check(self, st: int):
        if st != 0:
            raise MPSError(st, lib().mps_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().mps_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, n: int = 1, check: bool = True) -> mps_step_stats:
        s = mps_step_stats()
        st = lib().mps_step(self.h, n, C.byref(s))
        if check:
            self._check(st)
        return s

    def step_async(self, n: int = 1):
        self._check(lib().mps_step_async(self.h, n))

    def get_state_into(self, pos=None, vel=None, press=None, order: int = ORDER_SORTED):
        """Copy the current state into caller-provided float32 host arrays
        (pinned memory makes the copies direct DMA)."""
        self._check(lib().mps_get_state(self.h, None, None, _p(pos), _p(vel), _p(press), None, order))

    def phase(self, name: str):
        self._check(lib().mps_phase(self.h, PHASE[name]))

    def run(self, out_dir: Optional[str] = None):
        self._check(lib().mps_run(self.h, out_dir.encode() if out_dir else None))

    def counts(self) -> Dict[str, int]:
        v = [C.c_uint32() for _ in range(4)]
        self._check(lib().mps_get_counts(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("np", "nb2", "nb1", "nexcl"), [x.value for x in v]))

    def state(self, order: int = ORDER_SORTED) -> Dict[str, np.ndarray]:
        c = self.counts()
        n = c["np"] if order == ORDER_SORTED else self._np0
        out = dict(id=np.empty(n, np.uint32), type=np.empty(n, np.uint32),
                   pos=np.empty((n, 3), np.float32), vel=np.empty((n, 3), np.float32),
                   press=np.empty(n, np.float32), n=np.empty(n, np.float32))
        self._check(lib().mps_get_state(self.h, _p(out["id"], C.c_uint32),
                                        _p(out["type"], C.c_uint32), _p(out["pos"]),
                                        _p(out["vel"]), _p(out["press"]), _p(out["n"]), order))
        return out

    @property
    def _np0(self) -> int:
        if not hasattr(self, "_np0_cache"):
            self._np0_cache = self.counts()["np"] + self.counts()["nexcl"]
        return self._np0_cache

    def set_state(self, pos=None, vel=None, press=None, n=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        pos, vel, press, n = f(pos), f(vel), f(press), f(n)
        self._check(lib().mps_set_state(self.h, _p(pos), _p(vel), _p(press), _p(n)))

    def grid(self) -> mps_grid:
        g = mps_grid()
        self._check(lib().mps_get_grid(self.h, C.byref(g)))
        return g

    def cell_tables(self):
        g = self.grid()
        n = self.counts()["np"]
        cell_of = np.empty(n, np.uint32)
        start = np.empty(g.ncells, np.uint32)
        end = np.empty(g.ncells, np.uint32)
        self._check(lib().mps_get_cell_tables(self.h, _p(cell_of, C.c_uint32),
                                              _p(start, C.c_uint32), _p(end, C.c_uint32)))
        return cell_of, start, end

    def scalars(self) -> Dict[str, float]:
        o = (C.c_double * 16)()
        self._check(lib().mps_get_scalars(self.h, o))
        names = ("nzero", "lambda", "dt", "time", "c_lap", "one_over_alpha", "alpha", "cg_iters",
                 "cg_relres", "step", "status", "ncells", "launches_per_step", "cg_outer", "graph",
                 "ppe_escaped")
        return dict(zip(names, list(o)))

    def normal_ids(self) -> np.ndarray:
        out = np.empty(self._np0, np.uint32)
        self._check(lib().mps_get_normal_ids(self.h, _p(out, C.c_uint32)))
        return out

    def profile(self, nsteps: int) -> Dict[str, float]:
        """Per-stage device milliseconds summed over nsteps steps."""
        buf = (C.c_double * 32)()
        ns = C.c_int()
        self._check(lib().mps_profile_steps(self.h, nsteps, buf, 32, C.byref(ns)))
        return {lib().mps_stage_name(k).decode(): buf[k] for k in range(ns.value)}

    # ---- learned PPE preconditioner
    def precond_params(self) -> np.ndarray:
        n = lib().mps_precond_num_params()
        w = np.empty(n, np.float32)
        self._check(lib().mps_precond_get_params(self.h, _p(w), n))
        return w

    def set_precond_params(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        self._check(lib().mps_precond_set_params(self.h, _p(w), len(w)))

    def precond_loss_grad(self, seed: int):
        n = lib().mps_precond_num_params()
        g = np.empty(n, np.float32)
        loss = C.c_double()
        self._check(lib().mps_precond_loss_grad(self.h, seed, C.byref(loss), _p(g)))
        return loss.value, g

    def precond_train(self, iters: int, lr: float, seed: int):
        a, b = C.c_double(), C.c_double()
        self._check(lib().mps_precond_train(self.h, iters, lr, seed, C.byref(a), C.byref(b)))
        return a.value, b.value

    def precond_tensor_cores(self, enable: bool = True) -> float:
        """Compare the tensor-core forward with the FP32 one on the last
        system (max relative difference of G) and use it when enabled."""
        d = C.c_double()
        self._check(lib().mps_precond_tensor_cores(self.h, int(enable), C.byref(d)))
        return d.value

    def precond_train_tensor_cores(self, enable: bool = True):
        """Train with the network's 64 -> 64 layers (forward, dx and dW) on
        the tensor cores, BF16 operands and FP32 accumulation; off: FP32 on
        the CUDA cores."""
        self._check(lib().mps_precond_train_tensor_cores(self.h, int(enable)))

    def ppe_snapshot(self) -> Dict[str, np.ndarray]:
        n = self.counts()["np"]
        out = dict(pos4=np.empty((n, 4), np.float32), n=np.empty(n, np.float32),
                   id=np.empty(n, np.uint32), is_row=np.empty(n, np.uint32),
                   diag=np.empty(n, np.float64))
        cnt = C.c_uint32()
        self._check(lib().mps_ppe_snapshot(self.h, _p(out["pos4"]), _p(out["n"]),
                                           _p(out["id"], C.c_uint32), _p(out["is_row"], C.c_uint32),
                                           out["diag"].ctypes.data_as(C.POINTER(C.c_double)),
                                           C.byref(cnt)))
        return out

    def ppe_stencil(self) -> Dict[str, np.ndarray]:
        """The last assembled PPE matrix's off-diagonal entries as the solver
        stores them: row_start (np + 1, sorted order), cols, weights."""
        n = self.counts()["np"]
        row_start = np.empty(n + 1, np.uint32)
        nnz = C.c_uint64()
        self._check(lib().mps_ppe_stencil(self.h, _p(row_start, C.c_uint32), None, None, 0, C.byref(nnz)))
        cols = np.empty(max(nnz.value, 1), np.uint32)
        w = np.empty(max(nnz.value, 1), np.float32)
        self._check(lib().mps_ppe_stencil(self.h, _p(row_start, C.c_uint32), _p(cols, C.c_uint32), _p(w),
                                          nnz.value, C.byref(nnz)))
        return dict(row_start=row_start, cols=cols[:nnz.value], weights=w[:nnz.value])

    def set_device_wait_limit(self, ns: int):
        """Longest spin (ns) of one grid-wide wait in the PPE solvers before it
        gives up with MPS_ERR_DEVICE_TIMEOUT (0: the default, 1 s)."""
        self._check(lib().mps_set_device_wait_limit(self.h, int(ns)))

    def set_body_force(self, accel_amp: float, accel_freq: float, scene: int = 0):
        """Tank acceleration accel_amp*sin(2*pi*accel_freq*t) along x."""
        self._check(lib().mps_set_body_force(self.h, scene, accel_amp, accel_freq))

    def add_wall_motion(self, lo, hi, vel=(0.0, 0.0, 0.0), amp=(0.0, 0.0, 0.0), freq: float = 0.0,
                        phase: float = 0.0) -> int:
        """Move the wall and dummy particles inside the box [lo, hi] rigidly
        from now on: x = x0 + vel*tau + amp*(sin(2*pi*freq*tau + phase) -
        sin(phase)), tau = time since this call.  Returns how many were taken."""
        f3 = lambda v: (C.c_float * 3)(*[float(x) for x in v])
        n = C.c_uint32()
        self._check(lib().mps_add_wall_motion(self.h, f3(lo), f3(hi), f3(vel), f3(amp), freq, phase,
                                              C.byref(n)))
        return n.value

    def clear_wall_motion(self):
        """Stop every wall motion (the moved particles stay, at rest)."""
        self._check(lib().mps_clear_wall_motion(self.h))

    def scene_info(self, scene: int = 0) -> mps_scene_info:
        info = mps_scene_info()
        self._check(lib().mps_batch_scene_info(self.h, scene, C.byref(info)))
        return info

    def autotune(self, steps: int = 3) -> Dict[str, object]:
        """Pick the stage block size and the PPE grid shape by timing them."""
        r = mps_tune_report()
        self._check(lib().mps_autotune(self.h, steps, C.byref(r)))
        return {"stage_threads": r.stage_threads, "ppe_threads": r.ppe_threads,
                "ppe_stored_weights": r.ppe_stored_weights, "ppe_pipelined": r.ppe_pipelined,
                "stage_ms": list(r.stage_ms), "ppe_ms": list(r.ppe_ms), "ppe_compact": r.ppe_compact,
                "ppe_compact_ms": list(r.ppe_compact_ms)}

    def apply_tuning(self, tune: Dict[str, object]):
        """Apply an autotune() result (from this or another handle of the same
        scene) without stepping."""
        r = mps_tune_report()
        for k in ("stage_threads", "ppe_threads", "ppe_stored_weights", "ppe_pipelined", "ppe_compact"):
            setattr(r, k, int(tune[k]))
        self._check(lib().mps_apply_tuning(self.h, C.byref(r)))

    # ---- free surface (marching cubes)
    def surface_setup(self, shape, origin, spacing, max_triangles: int):
        g = mps_surface_grid()
        g.nx, g.ny, g.nz = (int(v) for v in shape)
        for d in range(3):
            g.origin[d] = origin[d]
            g.spacing[d] = spacing[d]
        self._check(lib().mps_surface_setup(self.h, C.byref(g), max_triangles))
        self._surf_shape = tuple(int(v) for v in shape)
        self._surf_cap = max_triangles

    def surface_extract(self, wait: bool = True) -> int:
        if not wait:
            self._check(lib().mps_surface_extract_async(self.h))
            return -1
        n = C.c_uint32()
        self._check(lib().mps_surface_extract(self.h, C.byref(n)))
        return n.value

    def surface_triangles(self):
        n = C.c_uint32()
        self._check(lib().mps_surface_get(self.h, None, None, 0, C.byref(n)))
        m = min(n.value, self._surf_cap)
        pos = np.empty((m, 3, 3), np.float32)
        nrm = np.empty((m, 3, 3), np.float32)
        self._check(lib().mps_surface_get(self.h, _p(pos), _p(nrm), m, C.byref(n)))
        return pos, nrm

    def surface_vertex_values(self):
        nx, ny, nz = self._surf_shape
        out = np.empty((nz, ny, nx), np.float32)
        iso = C.c_float()
        self._check(lib().mps_surface_vertex_values(self.h, _p(out), C.byref(iso)))
        return out, iso.value

    def surface_write_stl(self, path: str):
        self._check(lib().mps_surface_write_stl(self.h, path.encode()))

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(lib().mps_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def write_case(self, path: str, fmt: int = 0):
        self._check(lib().mps_write_case(self.h, path.encode(), fmt))


class MPS_GPU_EXPL:
    """The reference's ``MPS_GPU_EXPL`` driven through the C ABI.

    ``Initial()`` reads ``input.dat`` and ``GEO.dat`` from the working
    directory like ``MPS_GPU::Initial`` (MPS_CAL_expl_v1.0/MPS_GPU.cpp:63-115);
    ``step()`` is one ``MPS_GPU_EXPL::step``; ``mps_cal()`` is the full run
    with ``./out/NNNN.out`` dumps (MPS_GPU_EXPL.cpp:216-272).  The getters
    return host copies of the current (cell-sorted) particle arrays, refreshed
    after every step, as the reference's getters alias its host arrays.
    """

    method = METHOD_EXPLICIT

    def __init__(self, **options):
        self._opt = options
        self.sim: Optional[Simulation] = None
        self._cache = None

    def Initial(self, case_dir: str = "."):
        self.sim = Simulation(case_dir, method=self.method, **self._opt)
        self._cache = None

    def step(self):
        if self.sim is None:
            self.Initial()
        self.sim.step(1)
        self._cache = None

    def mps_cal(self, case_dir: str = "."):
        out = os.path.join(case_dir, "out")
        os.makedirs(out, exist_ok=True)
        self.Initial(case_dir)
        self.sim.run(out)
        self._cache = None

    def _state(self):
        if self._cache is None:
            self._cache = self.sim.state()
        return self._cache

    def getNp(self) -> int:
        return self.sim.counts()["np"]

    def getNb2(self) -> int:
        return self.sim.counts()["nb2"]

    def getNb1(self) -> int:
        return self.sim.counts()["nb1"]

    def getId(self):
        return self._state()["id"]

    def getType(self):
        return self._state()["type"]

    def getPos(self):
        return self._state()["pos"]

    def getVel(self):
        return self._state()["vel"]

    def getPres(self):
        return self._state()["press"]


class MPS_CPU_EXPL(MPS_GPU_EXPL):
    """The semi-implicit step class of the reference (MPS_CAL_v4.0/MPS_CPU_EXPL.h),
    same interface, on the GPU."""

    method = METHOD_SEMI_IMPLICIT
