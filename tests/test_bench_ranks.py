"""The multi-rank timing of bench.py on CPU: two gloo ranks, each with its
own time, both end up with the slowest rank's time (the rule for every
number a multi-GPU bench run reports)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = 10.0 + 5.0 * rank
        out[rank] = (bench.max_over_ranks(mine, dist, "cpu"), bench.max_over_ranks(mine / 2, dist, "cpu"))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world_size_2():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res == {0: (15.0, 7.5), 1: (15.0, 7.5)}


def test_max_over_ranks_without_a_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25
