"""World-size-2 checks of bench.py's multi-GPU plumbing on CPU (gloo).

The path shards by independent proofs: every rank proves its own trace
(seeded by its rank) and the only cross-rank traffic is a barrier and the
max-over-ranks reduction of the device-timed duration. Here two gloo ranks
exercise exactly those pieces, plus the reference arm's rank-0-only rule."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_setup(world)  # gloo (no CUDA here)
    assert (ws, r, local) == (world, rank, rank)
    t = bench.dist_max(10.0 + rank, ws)  # each rank reports its own time; all see the max
    bench.barrier(ws)
    tr = bench.make_trace(rank)
    q.put((rank, t, int(tr[0, 0]), int(tr[-1, -1])))
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_max_timing_and_independent_shards():
    world, port = 2, 29500 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]  # max over ranks, on every rank
    assert out[0][2:] != out[1][2:]  # each rank proves a different trace


def test_reference_arm_only_rank0_prints():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--gpus", "2"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
