"""bench.py's multi-rank logic on the CPU: two gloo ranks (world size 2).

One process per GPU shards the nodes (each rank its own seeded 1M-node shard,
weak scaling) and reduces nothing but the timings, as the maximum over ranks.
Under torchrun the reference arm runs on rank 0 only; other ranks exit 0.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank 0 is slower in the first value, rank 1 in the second
        vals = bench.max_over_ranks([10.0 - rank, 3.0 + rank, 7.0], dist, "cpu")
        _, y0, fp = bench.inputs(64, rank)
        out.put((rank, vals, float(y0.sum()), float(fp.sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timings_by_max_and_shard_inputs():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res[0][1] == res[1][1] == [10.0, 4.0, 7.0]
    assert res[0][2] != res[1][2] and res[0][3] != res[1][3]   # different shards


def test_max_over_ranks_without_process_group_is_identity():
    assert bench.max_over_ranks([1.5, 2.0], None, "cpu") == [1.5, 2.0]


def test_shards_have_the_workload_shape():
    md, y0, fp = bench.inputs(128, 3)
    assert y0.shape == (128, len(md["state_names"])) and fp.shape == (128, len(bench.FIELDS))
    assert np.all(fp > 0)


def test_reference_arm_on_a_non_zero_rank_exits_without_output():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                          env=env, capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0
    assert proc.stdout.strip() == ""


def test_side_legs_run_at_one_process_only():
    class A:
        skip_fp64 = False

    assert bench.side_legs(A, 1)
    assert not bench.side_legs(A, 2) and not bench.side_legs(A, 8)
    A.skip_fp64 = True
    assert not bench.side_legs(A, 1)
