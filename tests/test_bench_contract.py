"""The reference arm of bench.py on the host (no GPU): one JSON line with the
GPU arm's metric and unit, `impl` "reference", a `cpu_baseline` of kind
"reference" that names its sample, and an `e2e` block without copies; under a
multi-rank launch only rank 0 prints.  A small box (32^3) keeps it to seconds."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libgevref.so")
METRIC = "Mpart-steps/s at 512^3 (mixed vs FP64 GPU, P(k) err<1e-4); grad/fwd ratio"

pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference build (oracle/_ref) is absent")


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="2", **env_extra)
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
           "--cpu-sample-N", "32"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == METRIC and d["unit"] == "Mpart-steps/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["ms_per_step"] > 0 and d["ms_per_step_grid"] == "32^3"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and "32^3" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "32" in json.dumps(d["config"])


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
