"""The multi-process path of bench.py on the CPU: two gloo ranks (one process per rank, as
torchrun starts them), max-over-ranks timing, the barrier, and the replicas' disjoint slices
of the sweep."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(REPO))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.dist_max(10.0 * (rank + 1), world)
        bench.barrier(world)
        sweep = 1408
        first = bench.rank_first_frame(rank, sweep)
        q.put((rank, t, first, first + sweep))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_and_disjoint_slices():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [20.0, 20.0]          # both ranks report the slowest rank's time
    (_, _, a0, a1), (_, _, b0, b1) = out
    assert a1 <= b0 and a0 == 0                          # the replicas' frame ranges do not overlap
