"""Index arithmetic of the particle kernels, from the library's own headers
built with nvcc and run on the host (no GPU): the tile-local cell order that
the re-binning sorts by and the deposit's single-chunk path relies on (each
reach cell's records form one run), and the multiply-shift cell decode."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_class_ord_is_bucket_then_cell_order(tmp_path):
    exe = tmp_path / "tile_order_check"
    cmd = ["nvcc", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "gevolution-2.0_b200", "csrc"),
           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "tile_order_check.cu"),
           "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
