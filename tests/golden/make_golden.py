"""Regenerate the golden fixtures in this directory from the reference itself.

Runs the reference's own CPU step classes, compiled from the reference
sources by oracle/Makefile (oracle/_ref/ref_expl = MPS_CAL_expl_v1.0
MPS_GPU_EXPL with GPU_CUDA off; oracle/_ref/ref_semi = MPS_CAL_v4.0
MPS_CPU_EXPL in 3D; oracle/_ref/ref_impl = MPS_CAL_v4.0 MPS_CPU_IMPL in 3D),
on three small seeded tanks, one thread, and stores the
inputs (input.dat, GEO.dat text) and the reference's state dumps.

    make -C oracle REF=/path/to/reference
    python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from mps_solvers_b200 import scene  # noqa: E402
import oracle  # noqa: E402

def _viscous(sc, niu=1e-2):
    sc.params.niu = niu
    return sc


CASES = {
    # name: (reference binary, scene, steps, dump_every)
    "expl_tank": ("expl", scene.small_tank(seed=1), 60, 30),
    "semi_tank": ("semi", scene.small_tank(seed=2, interior=(10, 4, 14), fluid=(6, 4, 12),
                                           dt=5e-4), 8, 4),
    # MPS_CPU_IMPL (Crank-Nicolson viscosity), viscous enough for it to matter
    "impl_tank": ("impl", _viscous(scene.small_tank(seed=3, interior=(10, 4, 14), fluid=(6, 4, 12),
                                                    dt=5e-4)), 6, 3),
}


def main():
    assert oracle.have_reference_build(), "build the reference first: make -C oracle"
    here = os.path.dirname(os.path.abspath(__file__))
    only = sys.argv[1:]
    for name, (kind, sc, steps, every) in CASES.items():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as d:
            scene.write_case(d, sc)
            oracle.run_reference(kind, d, steps, every, os.path.join(d, "ref.bin"), threads=1)
            R = oracle.read_dump(os.path.join(d, "ref.bin"))
            inp = open(os.path.join(d, "input.dat")).read()
            geo = open(os.path.join(d, "GEO.dat")).read()
        out = dict(input_dat=np.frombuffer(inp.encode(), np.uint8),
                   geo_dat=np.frombuffer(geo.encode(), np.uint8),
                   nzero=R["nzero"], lambda_=R["lambda_"], cell_of=R["cell_of"],
                   cell_start=R["cell_start"], cell_end=R["cell_end"],
                   grid=np.array([R["cdx"], R["cdy"], R["cdz"], R["ncells"]], np.uint32),
                   steps=np.array([s["step"] for s in R["steps"]], np.int32))
        for s in R["steps"]:
            k = s["step"]
            for f in ("id", "type", "pos", "vel", "press", "n"):
                out[f"s{k}_{f}"] = s[f]
            out[f"s{k}_dt"] = np.float64(s["dt"])
            out[f"s{k}_time"] = np.float64(s["time"])
        np.savez_compressed(os.path.join(here, f"{name}.npz"), **out)
        print(name, "np", R["np"], "steps", list(out["steps"]))


if __name__ == "__main__":
    main()
