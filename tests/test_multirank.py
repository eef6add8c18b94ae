"""The N > 1 host logic of bench.py on CPU: two gloo ranks (127.0.0.1)
reduce their timings to the slowest rank's, the whole-job rate counts every
replica's work over that time, and the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

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
        # rank r timed (1 + r) ms and (10 - r) ms
        res = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == [2.0, 10.0]
    assert out[1] == [2.0, 10.0]


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks([3.0, 4.5], None, "cpu") == [3.0, 4.5]


def test_job_rate_counts_every_replica():
    # 2 replicas each doing 6.7e9 flops in 0.5 ms (slowest rank) -> 26.8 TFLOP/s
    assert abs(bench.job_rate(6.7e9, 2, 0.5) - 2.68e13) < 1e6
    assert bench.job_rate(1.0, 1, 1.0) == 1000.0


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
