"""The multi-rank timing reduction of bench.py on two gloo ranks (CPU).

The step does not shard, so `bench.py --gpus N` runs N independent replicas. The only
exchange is at the end: the slowest rank's device time (MAX) and the whole job's units
(SUM), which `reduce_over_ranks` computes. These tests run it as two spawned processes
over gloo on 127.0.0.1 and check both numbers and the resulting whole-job throughput.
"""
from __future__ import annotations

import os
import socket

import pytest

from conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, REPO)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: time 10*(r+1) ms, agent-steps 1000*(r+1), voxel updates 7*(r+1)
        t = torch.tensor([10.0 * (rank + 1), 1000.0 * (rank + 1), 7.0 * (rank + 1)],
                         dtype=torch.float64)
        ms_max, tot = bench.reduce_over_ranks(dist, t)
        # a second reduction in the same order, as the e2e leg makes it
        t2 = torch.tensor([0.5 + rank, 3.0], dtype=torch.float64)
        s_max, t2 = bench.reduce_over_ranks(dist, t2)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(" ".join(repr(x) for x in [ms_max, *tot.tolist(), s_max, *t2.tolist()]))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        vals = [float(x) for x in (tmp_path / f"r{r}.txt").read_text().split()]
        ms_max, tot_ms, agents, vox, s_max, tot_s, e2e_units = vals
        assert ms_max == 20.0                      # slowest rank
        assert (tot_ms, agents, vox) == (30.0, 3000.0, 21.0)   # sums over ranks
        assert s_max == 1.5 and tot_s == 2.0 and e2e_units == 6.0
        # whole-job throughput as bench.py reports it: sum of units / slowest time
        assert agents / (ms_max / 1e3) == pytest.approx(150000.0)


def test_reduce_over_ranks_single_rank_is_identity():
    import sys

    import torch

    sys.path.insert(0, REPO)
    import bench

    t = torch.tensor([12.5, 4.0], dtype=torch.float64)
    ms, out = bench.reduce_over_ranks(None, t)
    assert ms == 12.5 and out is t and out.tolist() == [12.5, 4.0]
