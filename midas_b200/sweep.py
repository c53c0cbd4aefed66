"""Sharded sweeps: one process per GPU, each caking its own contiguous slice of a sweep's
frames with its own copy of the plan (the map is read-only; no frame data crosses
between GPUs), and the one collective of the path: the SumImages running cake
(IntegratorFitPeaksGPUStream.cu:1043-1046, the dSumMatrix of :2141-2144) summed over the
ranks at the end of the sweep with one all-reduce (NCCL between GPUs; any process group
whose backend takes the tensor's device, e.g. gloo for CPU tensors).

    s = SweepSum(plan)                     # FP64 n_r x n_eta zeros on the plan's device
    for batch in my_slice_batches:
        plan.integrate(batch, sum_into=s.total)
    total = s.reduce()                     # every rank: the sum over all ranks' frames
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch


def frame_slice(rank: int, world: int, n_frames: int) -> Tuple[int, int]:
    """Contiguous share of rank ``rank``: (first frame, count); the first n_frames % world
    ranks take one frame more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(int(n_frames), world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_sum_images(total: torch.Tensor, group=None) -> torch.Tensor:
    """Sum a float64 SumImages cake over the ranks of ``group`` in place (all-reduce, SUM);
    a no-op without an initialised process group of more than one rank."""
    import torch.distributed as dist
    if total.dtype != torch.float64 or not total.is_contiguous():
        raise ValueError("the SumImages cake is a contiguous float64 tensor")
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return total


class SweepSum:
    """The FP64 SumImages cake of one rank's frames, and its sum over the ranks."""

    def __init__(self, plan=None, *, n_bins: Optional[int] = None, device=None):
        if plan is not None:
            n_bins, device = plan.n_r * plan.n_eta, plan.device
        if n_bins is None:
            raise ValueError("a plan or n_bins is needed")
        self.total = torch.zeros(int(n_bins), dtype=torch.float64, device=device)
        self.frames = 0

    def add(self, plan, frames: torch.Tensor, **kw):
        """Cake a batch with ``plan`` and add its cakes to the running sum; returns what
        ``plan.integrate`` returns."""
        out = plan.integrate(frames, sum_into=self.total, **kw)
        self.frames += int(frames.shape[0]) if frames.dim() == 3 else 1
        return out

    def reduce(self, group=None) -> torch.Tensor:
        return reduce_sum_images(self.total, group)
