"""bench.py's multi-GPU path on CPU: world_size 2 over gloo.  Queries shard across ranks with the
BVH replicated and no data-path collective; each rank traces its own rays and the job rate is all
ranks' rays over the slowest rank's time (all-reduce MAX), the only collective."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
        slowest = bench.max_over_ranks(ms, ws)
        rate = bench.weak_scaling_rate(ws, 1_000_000, 4, slowest)
        out[rank] = (slowest, rate, bench.incoherent_seed(rank))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_weak_scaling():
    port = 29500 + (os.getpid() % 2000)
    ws = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_worker, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    assert res[0][1] == pytest.approx(2 * 1_000_000 * 4 / 0.015 / 1e6)
    assert res[0][2] != res[1][2]                  # different rays per rank


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.weak_scaling_rate(1, 1000, 1, 1.0) == pytest.approx(1.0)
