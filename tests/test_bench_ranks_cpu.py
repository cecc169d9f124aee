"""The N > 1 path of bench.py without a GPU: two gloo ranks on the CPU run
the same barrier / max-over-ranks calls the GPU ranks make over NCCL, and
the whole-job rate is every rank's units over the slowest rank's time.  The
reference arm runs on rank 0 only; other ranks exit without output."""
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
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        r = bench.Ranks(world, torch.device("cpu"))
        r.barrier()
        # rank k took (k + 1) seconds for its 1000 units
        slowest = r.max(float(rank + 1))
        out[rank] = (slowest, bench.whole_job_rate(1000.0, slowest, world))
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1] == (2.0, 1000.0)


def test_single_rank_needs_no_process_group():
    r = bench.Ranks(1, torch.device("cpu"))
    r.barrier()
    assert r.max(3.5) == 3.5
    assert bench.whole_job_rate(500.0, 2.0, 1) == 250.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
