"""Host logic of the multi-GPU path (one independent replica per rank):
max-over-ranks timing and the whole-job rate, run as two gloo ranks on CPU,
and the reference arm's rank handling."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank           # rank 1 is the slow one
        m = bench.max_over_ranks(ms, world, "cpu")
        out[rank] = (m, bench.job_rate(world, 1000, 4, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_rate():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 15.0
    # 2 replicas x 1000 particles x 4 cycles in 15 ms
    assert abs(out[0][1] - 2 * 1000 * 4 / 15e-3 / 1e6) < 1e-12
    assert out[0][1] == out[1][1]


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_rank_handling(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1", "--cpu-sample-N", "16"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if rank == 0:
        assert len(lines) == 1
        d = json.loads(lines[0])
        assert d["impl"] == "reference"
        if "unavailable" in d:   # the reference's functions were not built in this tree
            assert not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libgevref.so"))
            return
        assert d["value"] > 0 and d["config"]["N"] == 16
        assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
    else:
        assert lines == []
