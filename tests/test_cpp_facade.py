"""The C++ drop-in class (include/mps_gpu_expl.hpp) compiles and links against
libmps_b200.so, and on a GPU runs a reference-style main end to end."""
import os
import subprocess

import pytest

from helpers import HERE

ROOT = os.path.dirname(HERE)
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_main(out):
    lib_dir = os.path.join(ROOT, "mps_solvers_b200")
    cmd = [GXX, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "cpp", "drop_in_main.cpp"), "-o", out, "-L", lib_dir, "-lmps_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True)


def test_facade_compiles_and_links(tmp_path, capi):
    exe = str(tmp_path / "drop_in")
    build_main(exe)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_runs_reference_style_main(tmp_path, capi):
    from mps_solvers_b200 import scene
    sc = scene.small_tank(seed=3)
    sc.params.tt = 10 * 1e-4
    sc.params.tout = 5 * 1e-4
    d = str(tmp_path / "case")
    pos, nb2, nb1 = scene.write_case(d, sc)
    exe = str(tmp_path / "drop_in")
    build_main(exe)
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    outs = sorted(os.listdir(os.path.join(d, "out")))
    assert outs[:2] == ["0000.out", "0001.out"]
    tok = open(os.path.join(d, "out", "0000.out")).read().split()
    assert len(tok) == 9 * len(pos)
