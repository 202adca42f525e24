"""The C++ bindings: include/gev_shim.hpp (the library's calls under the
reference's cycle names) and include/gev_latfield.hpp (the reference's own
per-cycle types and call signatures).  Both compile and link against the
library with the host compiler; on the GPU, cycles written in main.cu's call
order through them match gev_step."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gevolution-2.0_b200")


def _build(out, src="shim_cycle.cpp"):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", src), "-L" + LIBDIR, "-lgevb200", "-Wl,-rpath," + LIBDIR, "-o", str(out)]
    return subprocess.run(cmd, capture_output=True, text=True)


@pytest.mark.parametrize("src", ["shim_cycle.cpp", "latfield_cycle.cpp"])
def test_shim_compiles_and_links(tmp_path, src):
    if not os.path.exists(os.path.join(LIBDIR, "libgevb200.so")):
        pytest.skip("library not built")
    r = _build(tmp_path / "prog", src)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_reference_signature_cycle_matches_gev_step(tmp_path):
    """Three cycles written with the reference's calls (projection_T00_project,
    prepareFTsource, PlanFFT::execute, solveModifiedPoissonFT, projectFTscalar,
    projectFTvector / evolveFTvector, projectFTtensor / evolveFTtensor,
    updateVel, moveParticles) against gev_step: FP64 elliptic, and mixed
    precision with the parabolic method and the tensor state."""
    r = _build(tmp_path / "latfield_cycle", "latfield_cycle.cpp")
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(tmp_path / "latfield_cycle")], capture_output=True, text=True, timeout=300)
    print(run.stdout)
    assert run.returncode == 0, run.stdout + run.stderr


@pytest.mark.gpu
def test_shim_cycle_matches_gev_step(tmp_path):
    r = _build(tmp_path / "shim_cycle")
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(tmp_path / "shim_cycle")], capture_output=True, text=True, timeout=300)
    print(run.stdout)
    assert run.returncode == 0, run.stdout + run.stderr
