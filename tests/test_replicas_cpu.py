"""Multi-GPU runs are replicas (no data-path collective): the process group
carries only the barriers and the max over ranks of each timing.  This checks
that host logic with two gloo ranks on the CPU, and that under torchrun the
CPU reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    _, world, _, dist = bench.dist_setup(2, backend="gloo")
    bench.dist_barrier(dist)
    out[rank] = bench.dist_max(dist, 1.5 + rank, rank)  # per-rank step time; the job time is the max
    bench.dist_barrier(dist)
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1] == 2.5


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
