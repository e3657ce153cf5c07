"""Shot-parallel gradients over torch.distributed (one process per GPU).

Shots are independent, so the only exchange of a gradient evaluation is one
sum over ranks of the misfit and of the lambda, mu and rho images -- the
reference sums its per-GPU gradients on the host (Torch_Fwi.cpp:89-94) after
splitting the shot list by linspace(0, n, ngpu + 1) (Torch_Fwi.cpp:53-54).
Here each rank owns a contiguous shard of the shot list by the same rule and
the sum is an all-reduce (NCCL over NVLink on GPUs; gloo for CPU tests).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import torch
import torch.distributed as dist


def shard_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[lo, hi) of rank's shard of n items: the reference's
    linspace(0, n, world + 1) boundaries truncated to integers."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    bars = torch.linspace(0, n, world + 1, dtype=torch.float32)
    return int(bars[rank].item()), int(bars[rank + 1].item())


def shard(ids: Sequence[int], rank: int, world: int) -> List[int]:
    lo, hi = shard_bounds(len(ids), rank, world)
    return [int(i) for i in ids[lo:hi]]


class ShotParallel:
    """Gradient of the summed misfit of a shot list whose shards live on
    the ranks of `group`.  `prop` is this rank's engine (an
    efwi.engine.Propagator, or any object with the same `gradient`)."""

    def __init__(self, prop, group=None):
        self.prop = prop
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0

    def local_ids(self, ids: Sequence[int]) -> List[int]:
        return shard(ids, self.rank, self.world)

    def gradient(self, local_ids: Sequence[int], obs_local: torch.Tensor, mode: str = "reference"):
        """Runs this rank's shots, then sums J and the three images over
        the ranks.  Every rank must call it (collective)."""
        J, gl, gm, gr = self.prop.gradient(list(local_ids), obs_local, mode=mode)
        if self.world > 1:
            jt = torch.tensor([J], dtype=torch.float64, device=gl.device)
            for t in (gl, gm, gr):
                dist.all_reduce(t, group=self.group)
            dist.all_reduce(jt, group=self.group)
            J = float(jt.item())
        return J, gl, gm, gr
