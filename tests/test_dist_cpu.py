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


def _sum_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(REPO))
    import datetime

    import numpy as np
    import torch

    sys.path.insert(0, str(REPO / "tests"))
    import oracle
    from conftest import load_kernels_case
    from midas_b200 import sweep
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = load_kernels_case("a")
        nb = g["n_r"] * g["n_eta"]
        frames = [g["image"] * (1.0 + 0.1 * k) for k in range(7)]
        first, count = sweep.frame_slice(rank, world, len(frames))
        s = sweep.SweepSum(n_bins=nb, device="cpu")
        for f in frames[first:first + count]:       # this rank's cakes (the oracle's, on the host)
            ck, _ = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], f, mode="bilinear",
                                     bc_y=g["bc_y"], bc_z=g["bc_z"])
            s.total += torch.from_numpy(ck)
        q.put((rank, first, count, s.reduce().numpy().copy()))
    finally:
        dist.destroy_process_group()


def test_sum_images_all_reduced_over_ranks():
    """SumImages of a sweep sharded over two ranks: contiguous frame slices, one all-reduce,
    and every rank holds the sum over all frames."""
    import numpy as np

    import oracle
    from conftest import load_kernels_case
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_sum_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    out = sorted((q.get(timeout=10) for _ in range(2)), key=lambda o: o[0])
    assert [(o[1], o[2]) for o in out] == [(0, 4), (4, 3)]
    g = load_kernels_case("a")
    nb = g["n_r"] * g["n_eta"]
    want = sum(oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"] * (1.0 + 0.1 * k),
                                mode="bilinear", bc_y=g["bc_y"], bc_z=g["bc_z"])[0] for k in range(7))
    for o in out:
        np.testing.assert_allclose(o[3], want, rtol=1e-13, atol=1e-9)


def test_frame_slices_cover_the_sweep():
    from midas_b200 import sweep
    for n, w in ((1408, 8), (10, 3), (2, 4)):
        sl = [sweep.frame_slice(r, w, n) for r in range(w)]
        assert sum(c for _, c in sl) == n and sl[0][0] == 0
        assert all(a + c == b for (a, c), (b, _) in zip(sl, sl[1:]))
