"""The benchmark's multi-rank host logic on CPU: two gloo ranks on 127.0.0.1.

Each GPU runs its own replica of the stage (no collective on the data path);
the only cross-rank steps are the barrier around the timed region and the
maximum of the ranks' times, which these tests run with gloo in place of NCCL.
"""
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, world)  # rank 1 is the slow one
        results.put((rank, slowest, bench.whole_job_rate(world, 1000, 4, slowest / 1e3)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    results = ctx.SimpleQueue()
    mp.start_processes(_rank, args=(2, _free_port(), results), nprocs=2, join=True, start_method="spawn")
    got = sorted(results.get() for _ in range(2))
    assert [r for r, _, _ in got] == [0, 1]
    for _, slowest, rate in got:
        assert slowest == 15.0  # every rank sees the slowest rank's time
        assert abs(rate - 2 * 1000 * 4 / 0.015 / 1e9) < 1e-12  # both replicas' cells over that time


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
