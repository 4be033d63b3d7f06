"""Throughput of the MPS particle step on B200: particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload semi|explicit]
                    [--impl ours|reference] [--arith exact|fast] [--size full|small]

One step = one MPS time step of the whole scene (all particles: fluid, wall
and dummy).  `value` = particles x steps / device time of the timed steps
(CUDA events on the library's stream, L2 flushed before every timed step,
max over ranks), `e2e` = the same metric through the C ABI with host
buffers: every step uploads the state from pinned host memory
(mps_set_state), steps (mps_step_async) and reads positions, velocities and
pressures back (mps_get_state), timed by the host clock.

Multi-GPU: the scenes are independent, so N GPUs run N replicas (one scene
per rank, seeded by rank) with no data-path collective; NCCL is used only for
the barrier and the max of the timings.

--impl reference times the reference's CPU step on the host cores, rank 0
only: the reference's own build (oracle/_ref, MPS_CAL_expl_v1.0) for the
explicit workload; for the semi-implicit one, whose dense N x N reference
matrix cannot be held at 310,912 particles, the oracle's sparse FP64
restatement of MPS_CAL_v4.0's rules.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2

# algorithmic bytes per particle per stage (fixed accounting model: float3 =
# 12 B, scalar/type = 4 B, neighbour reads counted once per stage)
STAGE_BYTES = {
    "visc": 52, "collision": 52, "pnd": 24, "dash": 56, "pressure": 8,
    "cell_keys": 20, "radix_sort": 32, "gather": 64, "update_dt": 12,
}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(rows), "reasons": sorted(reasons)}


def make_scene(workload: str, seed: int, size: str = "full"):
    from mps_solvers_b200 import scene
    if size == "small":
        # a ~110k-particle tank at the same resolution, for detailed profiles
        sc = scene.small_tank(seed=seed, interior=(80, 30, 60), fluid=(30, 20, 45), l0=0.01,
                              dt=1e-4 if workload == "explicit" else 5e-4)
        return sc
    if workload == "explicit":
        return scene.dam_break_explicit(seed=seed)
    if workload == "large":
        return scene.large_obstacle(seed=seed)
    return scene.dam_break_semi(seed=seed)


SURFACE_SHAPE = (256, 64, 128)   # vertices along x (length), y (depth), z (height)
SURFACE_EVERY = 20


def write_batch(d: str, seed: int, nscenes: int = 64):
    """The batched workload's scenes (the first nscenes of the 64) as case
    directories under d; returns (dirs, accel, particles per scene)."""
    from mps_solvers_b200 import scene
    dirs, accel, counts = [], [], []
    for k, (sc, amp, freq) in enumerate(scene.batch_scenes(nscenes, seed)):
        sd = os.path.join(d, f"scene{k:02d}")
        pos, _, _ = scene.write_case(sd, sc)
        dirs.append(sd)
        accel.append((amp, freq))
        counts.append(len(pos))
    return dirs, accel, counts


def workload_name(workload: str) -> str:
    if workload == "large":
        return ("semi-implicit dam break with a box obstacle: 2,004,000 fluid particles, l0=0.005 m, "
                "2.4 x 0.6 x 1.2 m tank, 0.15 x 0.15 x 0.3 m obstacle at x=1.0 m, dt=2.5e-4 s, PPE "
                "diagonally scaled CG to 1e-8, marching-cubes surface on a 256 x 64 x 128 vertex "
                "grid every 20 steps inside the timed region")
    if workload == "batch":
        return ("batched semi-implicit dam breaks: 64 tanks at l0=0.01 m, fluid counts log-uniform "
                "in [5k, 60k] (7,421,757 particles, 1,804,829 fluid), tank acceleration "
                "A sin(2 pi f t) x with A in [0, 2] m/s^2, f in [0.5, 2] Hz, one launch per stage "
                "and one persistent PPE launch for all scenes, each scene's PCG to 1e-8")
    if workload == "explicit":
        return ("explicit EOS dam break: 70,912 particles (8,000 fluid), l0=0.02 m, "
                "r0=2.1 l0, rlap=4.0 l0, c0=20 m/s, dt=1e-4 s")
    return ("semi-implicit dam break: 310,912 particles (80,000 fluid), l0=0.01 m, "
            "PPE diagonally scaled CG to 1e-8 relative residual, dt=5e-4 s")


def cpu_baseline(workload: str, case_dir: str, n_particles: int, warm: int, sample_steps: int):
    """Reference CPU step on the host cores: the first `warm` steps of the
    scene run untimed, then `sample_steps` consecutive steps are timed, so the
    timed window is the one the GPU arm times (its steps warm+1 ..)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    window = f"steps {warm + 1}-{warm + sample_steps} of one run from the initial state"
    if workload == "explicit" and oracle.have_reference_build():
        out = os.path.join(case_dir, "ref_bench.bin")
        info = oracle.run_reference("expl", case_dir, warm + sample_steps, 0, out, threads=threads,
                                    timeout=1800, untimed=warm)
        os.unlink(out)
        v = n_particles * sample_steps / info["steps_s"]
        return {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                "sample": f"{window}, MPS_CAL_expl_v1.0 CPU path (GPU_CUDA off) built from the "
                          f"reference sources, {threads} OpenMP threads, step() only",
                "window": [warm + 1, warm + sample_steps], "cpu": _cpu_model()}
    # semi-implicit: the oracle's sparse restatement of the reference rules
    orc = oracle.Oracle(case_dir, oracle.SEMI_JACOBI, 64)
    orc.set_cg(True, 1e-8, 100000)
    if warm:
        orc.step(warm)
    t0 = time.perf_counter()
    orc.step(sample_steps)
    dt = time.perf_counter() - t0
    return {"value": n_particles * sample_steps / dt, "unit": "particle-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"{window}, sparse FP64 restatement of MPS_CAL_v4.0 MPS_CPU_EXPL (the dense "
                      f"reference cannot hold this size), {threads} threads",
            "window": [warm + 1, warm + sample_steps], "cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def max_over_ranks(values, world: int, device="cpu"):
    """Element-wise maximum of `values` over all ranks (every rank gets it):
    the slowest replica's timings.  The process group is NCCL on the GPU box
    and gloo in the CPU tests."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return None
    from mps_solvers_b200 import scene
    with tempfile.TemporaryDirectory() as d:
        if args.workload == "batch":
            # the smallest scene of the batch stands for the batch (the CPU
            # step cost is proportional to the particles)
            sc = min(scene.batch_scenes(64, 0), key=lambda t: len(scene.build(t[0])[0]))[0]
            pos, nb2, nb1 = scene.write_case(d, sc)
        else:
            pos, nb2, nb1 = scene.write_case(d, make_scene(args.workload, 0))
        n = len(pos)
        # the GPU arm's window: `warmup` untimed steps from the initial state,
        # then `steps` timed consecutive steps (the large scene: at most 3 of
        # them, ~8 s each on the host)
        k = max(1, args.steps)
        if args.workload == "large":
            k = min(k, 3)
        if args.ref_sample:
            k = args.ref_sample
        cb = cpu_baseline(args.workload, d, n, args.warmup, k)
    v = float(cb["value"])
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": v, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * n / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.workload == "explicit" else "f64",
        "data": "synthetic", "config": {"workload": workload_name(args.workload), "particles": n,
                                        "sample_scene": "smallest scene of the batch" if
                                        args.workload == "batch" else None},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return line


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    from mps_solvers_b200 import capi, scene

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    method = capi.METHOD_EXPLICIT if args.workload == "explicit" else capi.METHOD_SEMI_IMPLICIT  # batch: semi
    arith = capi.ARITH_EXACT if args.arith == "exact" else capi.ARITH_FAST
    tmpd = tempfile.mkdtemp(prefix=f"mpsb_{rank}_")
    precond = capi.PRECOND_LEARNED if args.precond == "learned" else capi.PRECOND_DIAGONAL
    batch_counts = None

    def make_sim():
        if args.workload == "batch":
            return capi.Simulation.batch(dirs, accel=accel, method=method, arith=arith, device=local_rank,
                                         use_graph=1, precond=precond)
        return capi.Simulation(tmpd, method=method, arith=arith, device=local_rank, use_graph=1,
                               precond=precond if method == capi.METHOD_SEMI_IMPLICIT else capi.PRECOND_DIAGONAL,
                               visc_implicit=int(method == capi.METHOD_SEMI_IMPLICIT and args.visc == "implicit"),
                               ppe_layout=-1 if args.ppe_layout == "sliced" else 0)

    def load_learned(s):
        from mps_solvers_b200 import precond_weights
        s.set_precond_params(precond_weights.load())

    if args.workload == "batch":
        dirs, accel, batch_counts = write_batch(tmpd, rank, 8 if args.size == "small" else 64)
        n = int(sum(batch_counts))
    else:
        pos0, nb2, nb1 = scene.write_case(tmpd, make_scene(args.workload, rank, args.size))
        n = len(pos0)
    learned = method == capi.METHOD_SEMI_IMPLICIT and precond == capi.PRECOND_LEARNED
    # launch shapes picked by the library's autotuner on a scratch handle of
    # the same scene, so that the timed handle's steps start from the initial
    # state: warm-up steps 1..W, timed steps W+1..W+K
    tune = None
    if not args.no_autotune:
        with make_sim() as scratch:
            if learned:
                load_learned(scratch)
            tune = scratch.autotune(2)
    sim = make_sim()
    if args.workload == "batch":
        nb2 = sum(sim.scene_info(s).nb2 for s in range(len(dirs)))
        nb1 = sum(sim.scene_info(s).nb1 for s in range(len(dirs)))
    if tune is not None:
        if args.ppe_layout == "compact" and "ppe_compact" in tune:
            tune = dict(tune, ppe_compact=1)  # the other launch choices stay the autotuner's
        sim.apply_tuning(tune)
    tc_diff = None
    extra_warm = 0
    if learned:
        load_learned(sim)
        sim.step(1)  # a PPE system for the tensor-core check
        extra_warm = 1
        tc_diff = sim.precond_tensor_cores(True)
    stream = torch.cuda.ExternalStream(sim.stream(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    surface = None
    if args.workload == "large":
        sc_large = make_scene("large", rank, args.size)
        origin, spacing = scene.surface_grid(sc_large, SURFACE_SHAPE)
        sim.surface_setup(SURFACE_SHAPE, origin, spacing, 8 << 20)
        surface = {"grid": list(SURFACE_SHAPE), "every": SURFACE_EVERY}
    # warm-up (also captures the step graphs)
    for _ in range(args.warmup - extra_warm):
        sim.step_async(1)
    sim.step(0)
    first_timed = args.warmup + 1

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))  # write > L2 between timed steps
                ev[k][0].record(stream)
                sim.step_async(1)
                if surface is not None and (k + 1) % SURFACE_EVERY == 0:
                    sim.surface_extract(wait=False)
                ev[k][1].record(stream)
        stream.synchronize()
    stats = sim.step(0)
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    clocks = clk.summary()
    if surface is not None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            sim.surface_extract(wait=False)
            e1.record(stream)
        stream.synchronize()
        surface["ms_per_extraction"] = e0.elapsed_time(e1)
        surface["triangles"] = sim.surface_extract()
        surface["extractions_timed"] = args.steps // SURFACE_EVERY

    # e2e: host buffers through the C ABI
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    npart = sim.counts()["np"]
    hpos, hvel, hp = pin((npart, 3)), pin((npart, 3)), pin((npart,))
    sim.get_state_into(hpos, hvel, hp)
    # the learned preconditioner re-evaluates its network every 40 steps: a
    # window of 40 consecutive steps holds exactly one evaluation
    e2e_steps = max(1, min(args.steps, LEARNED_WINDOW if learned else 20))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.set_state(pos=hpos, vel=hvel, press=hp)
        sim.step_async(1)
        sim.get_state_into(hpos, hvel, hp)
    e2e_s = time.perf_counter() - t0
    h2d = npart * (12 + 12 + 4)
    d2h = npart * (12 + 12 + 4)

    # per-stage device times (stage by stage, no graph) for the roofline
    prof = sim.profile(max(3, min(args.steps, 10)))
    prof_steps = max(3, min(args.steps, 10))
    scal = sim.scalars()
    launches = int(scal["launches_per_step"])
    prof_iters, prof_outer = int(scal["cg_iters"]), int(scal["cg_outer"])
    # PPE work of the last solve: every scene's particles x its own iterations
    if batch_counts is not None:
        infos = [sim.scene_info(s) for s in range(len(batch_counts))]
        ppe_work = sum(c * (60 * i.cg_iters + 40 * i.cg_outer) for c, i in zip(batch_counts, infos))
        scene_iters = [i.cg_iters for i in infos]
    else:
        ppe_work = n * (60 * prof_iters + 40 * prof_outer)
        scene_iters = None
    sim.close()
    compare = None
    if method == capi.METHOD_SEMI_IMPLICIT and rank == 0 and not args.no_ppe_compare:
        if batch_counts is None:
            compare = ppe_compare(tmpd, arith, local_rank, args.warmup, max(3, min(args.steps, 10)),
                                  tune_diag=tune if precond == capi.PRECOND_DIAGONAL else None)
        else:
            compare = ppe_compare(dirs, arith, local_rank, args.warmup, max(3, min(args.steps, 5)), accel=accel)

    ms, e2e_s = max_over_ranks([ms, e2e_s], world, dev)
    if rank != 0:
        return None

    value = world * n * args.steps / (ms / 1e3)
    e2e_v = world * n * e2e_steps / e2e_s
    peak, peak_kind = measured_peaks()
    # dominant kernel: the single-launch stage with the largest device time
    kern = {k: v for k, v in prof.items() if k in ("visc", "collision", "pnd", "dash", "ppe_solve")}
    dom = max(kern, key=kern.get)
    dom_ms = kern[dom] / prof_steps
    if dom == "ppe_solve":
        # fixed accounting model: 60 B per particle per CG iteration, 40 B per
        # FP64 defect-correction pass (the last solve's counts, per scene)
        alg_bytes = ppe_work
    else:
        alg_bytes = STAGE_BYTES[dom] * n
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    # the committed traffic figures are for the full-size workloads, and for
    # the PPE per stencil layout (scalar ppe_escaped is -1 on the 8-byte one)
    sliced = method == capi.METHOD_SEMI_IMPLICIT and scal.get("ppe_escaped", 0) < 0
    tkey = ("pressure_sell" if sliced else "pressure") if dom == "ppe_solve" else dom
    traffic = _traffic_from_profiles(tkey, args.workload) if args.size == "full" else None
    # FP32 pipe (the secondary roofline of the stencil stages): pair
    # evaluations of the fixed model, |{j: r_ij < re}| x FLOP per pair (PND 10
    # over all particles at r0; viscosity 16 at rlap, collision 20 and
    # gradient 18 at r0 over the fluid; the CG product 12 at rlap per fluid
    # row and iteration), over the whole step's device time
    nf = int(n - nb2 - nb1)
    flops = n * 32 * 10 + nf * (250 * 16 + 32 * 20 + 32 * 18)
    if method == capi.METHOD_SEMI_IMPLICIT:
        flops += (ppe_work / 60.0) * 250 * 12 * nf / n if n else 0.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = sms * 128 * 2 * 1965e6 / 1e12
    fp32_ach = flops / (ms / args.steps / 1e3) / 1e12
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if method == capi.METHOD_EXPLICIT else "f32+f64",
        "data": "synthetic",
        "config": {"workload": workload_name(args.workload) if args.size == "full" else
                   f"{args.workload} small profiling tank", "particles": n,
                   "precond": args.precond if method == capi.METHOD_SEMI_IMPLICIT else None,
                   "network_every": 40 if learned else None,
                   "fluid": int(n - nb2 - nb1), "arith": args.arith,
                   "viscosity": ("Crank-Nicolson" if args.visc == "implicit" else "explicit"),
                   "ppe_layout": (None if method != capi.METHOD_SEMI_IMPLICIT else
                                  "sliced 8-byte" if sliced else "compact 6-byte")
                   if method == capi.METHOD_SEMI_IMPLICIT else "explicit",
                   "l2": "flushed (256 MB write) before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                     "ms_per_launch": dom_ms,
                     "note": "stencil kernels scan the 27 reference cells and are issue/latency "
                             "bound; see profiles/ for the measured bound"},
        "roofline_fp32": {"bound": "fp32", "achieved": fp32_ach, "peak": fp32_peak,
                          "peak_kind": f"nominal ({sms} SMs x 128 FP32 lanes x 2 x 1965 MHz)",
                          "unit": "TFLOP/s", "frac": fp32_ach / fp32_peak, "flops_per_step": flops,
                          "note": "pair-evaluation model over the whole step; the stages scan ~5-50x "
                                  "more candidates than they keep"},
        "value_fluid_only": value * nf / n if n else None,
        "stage_ms_per_step": {k: v / prof_steps for k, v in prof.items()},
        "e2e": {"value": e2e_v, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "timed_steps": [first_timed, first_timed + args.steps - 1],
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
        "autotune": tune,
        "learned_tensor_core_rel_diff": tc_diff,
        "surface": surface,
        "ppe_compare": compare,
        "batch": None if scene_iters is None else {
            "scenes": len(scene_iters), "particles_min": int(min(batch_counts)),
            "particles_max": int(max(batch_counts)), "cg_iters_min": int(min(scene_iters)),
            "cg_iters_max": int(max(scene_iters))},
        "final": {"np": stats.np, "step": stats.step, "time": stats.time, "dt": stats.dt,
                  "cg_iters": stats.cg_iters, "cg_outer": stats.cg_outer,
                  "cg_relres": stats.cg_relres},
    }
    return line


def ppe_compare(case_dir, arith: int, device: int, warm: int, steps: int, accel=None, tune_diag=None):
    """PPE solve milliseconds and PCG iterations per step (FP64 true residual
    to 1e-8) with diagonal scaling and with the trained learned factor, each
    on a fresh copy of the scene (or of the batch, when case_dir is a list of
    scene directories: iterations are then the mean over scenes) after
    `warm` steps.  A single scene runs each arm with its own autotuned launch
    shapes and stencil layout (the diagonal arm with the main run's)."""
    from mps_solvers_b200 import capi, precond_weights
    out = {"tolerance": 1e-8, "steps": steps, "warmup": warm,
           "weights": os.path.relpath(precond_weights.PATH, ROOT)}
    batch = isinstance(case_dir, (list, tuple))
    for name, pc in (("diagonal", capi.PRECOND_DIAGONAL), ("learned", capi.PRECOND_LEARNED)):
        if batch:
            sim = capi.Simulation.batch(case_dir, accel=accel, method=capi.METHOD_SEMI_IMPLICIT, arith=arith,
                                        device=device, precond=pc)
        else:
            mk = lambda: capi.Simulation(case_dir, method=capi.METHOD_SEMI_IMPLICIT, arith=arith, device=device,
                                         precond=pc)
            tune = tune_diag if pc == capi.PRECOND_DIAGONAL else None
            if pc == capi.PRECOND_LEARNED:
                with mk() as scratch:
                    scratch.set_precond_params(precond_weights.load())
                    tune = scratch.autotune(2)
            sim = mk()
        with sim as s:
            if not batch and tune is not None:
                s.apply_tuning(tune)
            if pc == capi.PRECOND_LEARNED:
                s.set_precond_params(precond_weights.load())
                s.step(1)
                out["learned_tensor_core_rel_diff"] = s.precond_tensor_cores(True)
            s.step(warm)
            iters, worst = 0, 0.0
            for _ in range(steps):
                st = s.step(1)
                if batch:
                    iters += float(np.mean([s.scene_info(k).cg_iters for k in range(len(case_dir))]))
                else:
                    iters += st.cg_iters
                worst = max(worst, st.cg_relres)
            prof = s.profile(steps)
            out[name] = {"ppe_solve_ms": prof["ppe_solve"] / steps,
                         "ppe_total_ms": (prof["ppe_solve"] + prof.get("pressure", 0.0)) / steps,
                         "cg_iters": iters / steps, "max_relres": worst,
                         "step_ms": sum(prof.values()) / steps}
    out["iters_ratio"] = out["learned"]["cg_iters"] / out["diagonal"]["cg_iters"]
    out["ppe_solve_ratio"] = out["learned"]["ppe_solve_ms"] / out["diagonal"]["ppe_solve_ms"]
    return out


def _traffic_from_profiles(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any
    (a line `traffic_bytes_per_launch: <kernel> <workload> <bytes>`)."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, f)):
            if line.startswith("traffic_bytes_per_launch:"):
                parts = line.split()
                if len(parts) >= 4 and parts[1] == kernel and parts[2] == workload:
                    return float(parts[3])
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="semi", choices=["explicit", "semi", "batch", "large"],
                    help="semi (default): the 310,912-particle semi-implicit dam break the "
                         "metric is quoted on; explicit: the 70,912-particle EOS dam break; "
                         "batch: 64 semi-implicit tanks of 5k-60k fluid particles with tank "
                         "acceleration, stepped as one batch; large: the 3.7M-particle obstacle "
                         "scene (2M fluid) with a marching-cubes surface every 20 steps")
    ap.add_argument("--arith", default=None, choices=["exact", "fast"],
                    help="default: exact for the explicit workload (bit-identical to the "
                         "reference), fast for the semi-implicit one")
    ap.add_argument("--size", default="full", choices=["full", "small"],
                    help="small (profiling): a ~110k-particle tank of the same kernels; with "
                         "--workload batch the first 8 of the 64 scenes; with --workload large the "
                         "small tank with the surface extraction")
    ap.add_argument("--visc", default="explicit", choices=["explicit", "implicit"],
                    help="semi-implicit viscosity: explicit (default) or Crank-Nicolson")
    ap.add_argument("--ref-sample", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precond", default="diagonal", choices=["diagonal", "learned"],
                    help="PPE preconditioner of the semi-implicit timed run")
    ap.add_argument("--no-ppe-compare", action="store_true",
                    help="skip the diagonal-vs-learned PPE comparison (semi-implicit)")
    ap.add_argument("--ppe-layout", default="auto", choices=["auto", "compact", "sliced"],
                    help="PPE stencil layout (auto: the library's default and the autotuner's choice)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (short launch lists for profiling)")
    ap.add_argument("--no-sub-runs", action="store_true",
                    help="skip the short runs of the explicit, batched and large workloads that the "
                         "default semi-implicit run adds under 'workloads'")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.arith is None:
        args.arith = "exact" if args.workload == "explicit" else "fast"


    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    line = run_ours(args, rank, world, local_rank)
    if line is not None and world == 1 and not args.no_cpu_baseline:
        from mps_solvers_b200 import scene
        with tempfile.TemporaryDirectory() as d:
            if args.workload == "batch":
                sc = min(scene.batch_scenes(64, 0), key=lambda t: len(scene.build(t[0])[0]))[0]
            else:
                sc = make_scene(args.workload, 0)
            pos, _, _ = scene.write_case(d, sc)
            # the GPU arm's first timed steps (all of them for the explicit
            # scene, at most 20 for the semi-implicit ones, 2 for the large)
            k = args.steps if args.workload == "explicit" else min(args.steps, 2 if args.workload == "large" else 20)
            line["cpu_baseline"] = cpu_baseline(args.workload, d, len(pos), args.warmup, k)
            if args.workload == "batch":
                line["cpu_baseline"]["sample"] += " (the batch's smallest scene)"
    if line is not None and world == 1 and args.workload == "semi" and args.size == "full" and not args.no_sub_runs:
        line["workloads"] = sub_runs(args, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


# The other configurations, measured briefly in the default run: (steps,
# warm-up, CPU-baseline steps) each; the CPU baseline times the first of the
# GPU arm's timed steps on the same scene.
# (workload, timed steps, warm-up, CPU-baseline steps); the learned runs
# (batch, large) time LEARNED_WINDOW steps so that the network's evaluation
# every 40 steps is inside the window once
LEARNED_WINDOW = 40
SUB_RUNS = (("explicit", 200, 10, 200), ("batch", LEARNED_WINDOW, 3, 10), ("large", LEARNED_WINDOW, 3, 1))
SUB_KEYS = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "timed_steps", "dtype", "config",
            "roofline", "roofline_fp32", "value_fluid_only", "stage_ms_per_step", "e2e", "gpu_launches",
            "clocks", "autotune", "surface", "batch", "final")


def sub_runs(args, local_rank: int):
    """Short runs of the explicit, batched and large workloads (single GPU),
    each with its own timing, roofline, e2e and windowed CPU baseline."""
    import copy
    from mps_solvers_b200 import scene
    out = {}
    for wl, steps, warm, cpu_steps in SUB_RUNS:
        a = copy.copy(args)
        a.workload, a.steps, a.warmup = wl, steps, warm
        a.arith = "exact" if wl == "explicit" else "fast"
        a.no_ppe_compare = True
        # the batched and large configurations name the learned preconditioner
        a.precond = "learned" if wl in ("batch", "large") else "diagonal"
        try:
            sub = run_ours(a, 0, 1, local_rank)
            res = {k: sub.get(k) for k in SUB_KEYS}
            if not args.no_cpu_baseline:
                with tempfile.TemporaryDirectory() as d:
                    if wl == "batch":
                        sc = min(scene.batch_scenes(64, 0), key=lambda t: len(scene.build(t[0])[0]))[0]
                    else:
                        sc = make_scene(wl, 0)
                    pos, _, _ = scene.write_case(d, sc)
                    cb = cpu_baseline(wl, d, len(pos), warm, cpu_steps)
                    if wl == "batch":
                        cb["sample"] += " (the batch's smallest scene)"
                    res["cpu_baseline"] = cb
        except Exception as e:  # one workload failing must not lose the others
            res = {"error": f"{type(e).__name__}: {e}"}
        out[wl] = res
    return out


if __name__ == "__main__":
    main()
