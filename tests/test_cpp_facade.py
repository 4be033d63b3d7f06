"""The C++ drop-in class (include/mps_gpu_expl.hpp) compiles and links against
libmps_b200.so, and on a GPU runs a reference-style main end to end."""
import os
import subprocess

import pytest

from helpers import HERE

ROOT = os.path.dirname(HERE)
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_main(out, src="drop_in_main.cpp"):
    lib_dir = os.path.join(ROOT, "mps_solvers_b200")
    cmd = [GXX, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "cpp", src), "-o", out, "-L", lib_dir, "-lmps_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True)


def test_facade_compiles_and_links(tmp_path, capi):
    exe = str(tmp_path / "drop_in")
    build_main(exe)
    assert os.path.exists(exe)
    exe2 = str(tmp_path / "renderer_style")
    build_main(exe2, "renderer_style_main.cpp")
    assert os.path.exists(exe2)


@pytest.mark.gpu
def test_mps_gpu_class_steps_like_the_explicit_handle(tmp_path, capi, oracle_mod):
    """new MPS_GPU(); Initial(); step() x 10 (the GL build's driving style,
    MPS_CAL_/Renderer.h:54-56,312): the getters' fluid sums equal those of
    the CPU oracle's explicit step bit for bit (same float state), printed
    with 10 significant digits."""
    import numpy as np
    from mps_solvers_b200 import scene
    d = str(tmp_path / "case")
    scene.write_case(d, scene.small_tank(seed=5))
    exe = str(tmp_path / "renderer_style")
    build_main(exe, "renderer_style_main.cpp")
    r = subprocess.run([exe, "10"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    np0, np1, fluid, sz, sw, sp, np2 = r.stdout.split()
    orc = oracle_mod.Oracle(d, oracle_mod.EXPL, 32)
    orc.step(10)
    st = orc.state()
    f = st["type"] == 0
    assert int(np1) == int(np0) == len(st["id"]) == int(np2)
    assert int(fluid) == int(f.sum())
    # the same summation in double over the same sorted float arrays
    ez = sum(float(v) for v in st["pos"][f, 2])
    ew = sum(float(v) for v in st["vel"][f, 2])
    ep = sum(float(v) for v in st["press"][f])
    assert float(sz) == float(f"{ez:.9e}") and float(sw) == float(f"{ew:.9e}") and float(sp) == float(f"{ep:.9e}")


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
