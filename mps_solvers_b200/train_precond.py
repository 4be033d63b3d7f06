"""Train the learned PPE preconditioner on systems the semi-implicit solver
generates, then compare it with diagonal scaling on a held-out scene.

Scenes: the semi-implicit dam-break tank (l0 = 0.01 m, 160 x 40 x 100
interior sites) with a water column of seeded width 0.2-0.6 m and height
0.4-0.9 m, 0.25 m deep as in the benchmark scene.  Each scene is stepped with the diagonally
scaled CG (so every snapshot comes from the solver's own trajectory); after
every step the network takes `--iters-per-step` Adam steps on that step's
PPE system, each with a new Rademacher probe.  Defaults: 50 scenes x 400
steps = 20,000 PPE systems.

    python -m mps_solvers_b200.train_precond [--scenes 50] [--steps 400] [--tensor-cores]

--tensor-cores trains with the network's 64 -> 64 layers (forward, input
and weight gradients) on the tensor cores, BF16 operands and FP32
accumulation; without it training runs in FP32 on the CUDA cores.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import capi, precond_weights, scene

HELD_OUT = 1000  # scene index of the evaluation scene (not in the training range)


def training_scene(k: int) -> scene.Scene:
    """Scene k: column width and height drawn from a generator seeded by k."""
    rng = np.random.default_rng(1000 + k)
    width = rng.uniform(0.2, 0.6)
    height = rng.uniform(0.4, 0.9)
    sc = scene.dam_break_semi(seed=100 + k)
    depth = sc.fluid[0].ny
    sc.fluid = [scene.Box(0, 0, 0, int(round(width / sc.l0)), depth, int(round(height / sc.l0)))]
    return sc


def evaluate(w: np.ndarray, k: int = HELD_OUT, warm: int = 50, steps: int = 20) -> dict:
    """PCG iterations and PPE solve milliseconds per step, diagonal scaling
    against the learned preconditioner, on scene k after `warm` steps."""
    out = {}
    with tempfile.TemporaryDirectory() as d:
        scene.write_case(d, training_scene(k))
        for name, pc in (("diagonal", capi.PRECOND_DIAGONAL), ("learned", capi.PRECOND_LEARNED)):
            with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, precond=pc,
                                 arith=capi.ARITH_FAST) as s:
                if pc == capi.PRECOND_LEARNED:
                    s.set_precond_params(w)
                s.step(warm)
                iters, relres = [], []
                for _ in range(steps):
                    st = s.step(1)
                    iters.append(st.cg_iters)
                    relres.append(st.cg_relres)
                prof = s.profile(steps)
                out[name] = dict(cg_iters=float(np.mean(iters)), max_relres=float(np.max(relres)),
                                 ppe_solve_ms=prof["ppe_solve"] / steps)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=50)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--iters-per-step", type=int, default=1)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=precond_weights.PATH)
    ap.add_argument("--log", default=None)
    ap.add_argument("--init", default=None, help="start from these weights (.npy)")
    ap.add_argument("--eval-only", action="store_true", help="only compare --init with diagonal scaling")
    ap.add_argument("--tensor-cores", action="store_true", help="train the 64 -> 64 layers on tcgen05 (BF16)")
    ap.add_argument("--no-eval", action="store_true", help="skip the held-out comparison at the end")
    args = ap.parse_args()
    w = precond_weights.load(args.init) if args.init else None
    if args.eval_only:
        print(json.dumps(dict(evaluation=evaluate(w))), flush=True)
        return
    log = []
    t0 = time.time()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    for k in range(args.scenes):
        losses = []
        try:
            with tempfile.TemporaryDirectory() as d:
                scene.write_case(d, training_scene(k))
                with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, precond=capi.PRECOND_DIAGONAL,
                                     arith=capi.ARITH_FAST) as s:
                    if w is None:
                        w = _initial_params()
                    # enables the learned stencil; the solve keeps diagonal scaling
                    s.set_precond_params(w)
                    s.precond_train_tensor_cores(args.tensor_cores)
                    for step in range(args.steps):
                        s.step(1)
                        a, _ = s.precond_train(args.iters_per_step, args.lr, seed=(k << 20) + step * 16)
                        losses.append(a)
                    w = s.precond_params()
            error = None
        except capi.MPSError as e:  # a scene that fails keeps the weights of its last good step
            error = str(e)
        rec = dict(scene=k, steps=len(losses), loss_first=losses[0] if losses else None,
                   loss_mean_last50=float(np.mean(losses[-50:])) if losses else None,
                   seconds=round(time.time() - t0, 1), error=error)
        log.append(rec)
        print(json.dumps(rec), flush=True)
        np.save(args.out, w.astype(np.float32))
    ev = None if args.no_eval else evaluate(w)
    if ev is not None:
        print(json.dumps(dict(evaluation=ev)), flush=True)
    if args.log:
        with open(args.log, "w") as f:
            json.dump(dict(training=log, evaluation=ev), f, indent=1)


def _initial_params() -> np.ndarray:
    """The library's default initial parameters (factor G = I)."""
    with tempfile.TemporaryDirectory() as d:
        scene.write_case(d, scene.small_tank())
        with capi.Simulation(d, method=capi.METHOD_SEMI_IMPLICIT, precond=capi.PRECOND_LEARNED) as s:
            return s.precond_params()


if __name__ == "__main__":
    main()
