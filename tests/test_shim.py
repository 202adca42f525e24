"""The C++ binding (include/gev_shim.hpp): it compiles and links against the
library with the host compiler; on the GPU, two cycles written in main.cu's
call order through it match gev_step."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gevolution-2.0_b200")


def _build(out):
    cmd = ["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "shim_cycle.cpp"),
           "-L" + LIBDIR, "-lgevb200", "-Wl,-rpath," + LIBDIR, "-o", str(out)]
    return subprocess.run(cmd, capture_output=True, text=True)


def test_shim_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libgevb200.so")):
        pytest.skip("library not built")
    r = _build(tmp_path / "shim_cycle")
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_shim_cycle_matches_gev_step(tmp_path):
    r = _build(tmp_path / "shim_cycle")
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(tmp_path / "shim_cycle")], capture_output=True, text=True, timeout=300)
    print(run.stdout)
    assert run.returncode == 0, run.stdout + run.stderr
