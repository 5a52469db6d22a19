"""The multi-GPU (replica) path of bench.py, exercised with two gloo ranks on the CPU.

Pairs are independent, so N GPUs run N replicas with no collective on the data path; the only
collectives are the max-over-ranks reduction of the timed region and barriers.  These tests run
the same helpers under a world of two CPU processes."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench
    from pose_b200.synthetic import spec_for

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # Each rank times a different amount of work; the job takes as long as the slowest.
        mine = 0.5 + rank
        slowest = bench.max_over_ranks(mine, dist, "cpu")
        value = bench.replica_throughput(1_000_000_000, 4, world, slowest)
        # Replicas get distinct seeded pairs (seed + rank) of the same shape.
        spec = spec_for("cfg0", seed_offset=rank)
        dist.barrier()
        queue.put((rank, slowest, value, spec.seed, spec.width, spec.height))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    queue = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(queue.get() for _ in range(2))
    assert [g[1] for g in got] == [1.5, 1.5]                 # max over ranks on both
    assert got[0][2] == got[1][2] == pytest.approx(1e9 * 4 * 2 / 1.5 / 1e9)
    assert got[0][3] != got[1][3]                            # distinct replica seeds
    assert got[0][4:] == got[1][4:]                          # same shape on every rank


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
