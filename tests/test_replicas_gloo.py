"""Multi-GPU is replicas only: each rank runs its own batch with its own
seeds, and the only collective is the max over ranks of the timed region.
This checks that host logic with two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, e2e = bench.max_over_ranks(dist, torch, [10.0 + rank, 30.0 - rank], "cpu")
        seeds = bench.rank_seeds(rank, 4)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        out[rank] = (ms, e2e, gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_distinct_seeds():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that already runs threads
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, e2e, gathered = res[rank]
        assert ms == 11.0 and e2e == 30.0  # the slowest rank's time, per field
        flat = [s for seeds in gathered for s in seeds]
        assert len(flat) == len(set(flat)) == 4 * world


def test_single_rank_needs_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(None, torch, [1.5, 2.5], "cpu") == [1.5, 2.5]
