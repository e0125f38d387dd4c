"""The multi-GPU form of the benchmark is replicas only: every rank runs its
own frequencies with no collective on the data path; the only collectives
are the barrier before timing and the max over ranks of the measured times.
This covers that host logic with two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times):
    sys.path.insert(0, ROOT)
    import bench as b
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        dist.barrier()
        t = b.max_over_ranks(times[rank], world, device="cpu")
        assert t == max(times), (rank, t)
        # every rank derives the same whole-job figure from the slowest rank
        v = b.whole_job_seconds_per_frequency(t, steps=3, world=world)
        assert abs(v - max(times) / (3 * world)) <= 1e-15
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_two_gloo_ranks():
    mp.spawn(_rank, args=(2, _free_port(), [1.25, 2.5]), nprocs=2, join=True)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(0.7, 1) == 0.7
    assert bench.whole_job_seconds_per_frequency(3.0, steps=3, world=1) == 1.0


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_runs_on_rank_zero_only(rank):
    """Under a multi-rank launch the CPU reference arm runs on rank 0; the
    other ranks exit 0 without output and without work."""
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
