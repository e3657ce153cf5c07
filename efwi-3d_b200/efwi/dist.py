"""Shot-parallel gradients over torch.distributed (one process per GPU).

Shots are independent, so the only exchange of a gradient evaluation is one
sum over ranks of the misfit and of the lambda, mu and rho images -- the
reference sums its per-GPU gradients on the host (Torch_Fwi.cpp:89-94) after
splitting the shot list by linspace(0, n, ngpu + 1) (Torch_Fwi.cpp:53-54).
Here each rank owns a contiguous shard of the shot list by the same rule and
the sum is ONE all-reduce of a stacked buffer (NCCL over NVLink on GPUs;
gloo for CPU tests): the three images followed by the misfit, carried as
two float32 words (a high part and the remainder) so that the sum keeps
more than float32 precision.
"""
from __future__ import annotations

import inspect
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


def pack_misfit(buf: torch.Tensor, J: float) -> None:
    """Writes J into the last two float32 words of buf (high part, rest)."""
    hi = float(torch.tensor(J, dtype=torch.float32).item())
    buf[-2:] = torch.tensor([hi, J - hi], dtype=torch.float32)


def unpack_misfit(buf: torch.Tensor) -> float:
    two = buf[-2:].double().cpu()
    return float(two[0].item()) + float(two[1].item())


class ShotParallel:
    """Gradient of the summed misfit of a shot list whose shards live on
    the ranks of `group`.  `prop` is this rank's engine (an
    efwi.engine.Propagator, or any object with the same `gradient`)."""

    def __init__(self, prop, group=None):
        self.prop = prop
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self._buf = None
        try:
            self._takes_out = "out" in inspect.signature(prop.gradient).parameters
        except (TypeError, ValueError):
            self._takes_out = False

    def local_ids(self, ids: Sequence[int]) -> List[int]:
        return shard(ids, self.rank, self.world)

    def _stacked(self, n: int, device) -> torch.Tensor:
        if self._buf is None or self._buf.numel() != 3 * n + 2 or self._buf.device != device:
            self._buf = torch.empty(3 * n + 2, dtype=torch.float32, device=device)
        return self._buf

    def gradient(self, local_ids: Sequence[int], obs_local: torch.Tensor, mode: str = "reference"):
        """Runs this rank's shots, then sums J and the three images over
        the ranks with one all-reduce.  Every rank must call it
        (collective).  The returned images are views of one buffer that the
        next call overwrites."""
        if self.world == 1:
            return self.prop.gradient(list(local_ids), obs_local, mode=mode)
        grid = getattr(self.prop, "grid", None)
        if self._takes_out and grid is not None:
            n = grid.ncell
            buf = self._stacked(n, getattr(self.prop, "device", torch.device("cpu")))
            J, gl, gm, gr = self.prop.gradient(list(local_ids), obs_local, mode=mode, out=buf)
        else:
            J, gl, gm, gr = self.prop.gradient(list(local_ids), obs_local, mode=mode)
            n = gl.numel()
            buf = self._stacked(n, gl.device)
            for k, t in enumerate((gl, gm, gr)):
                buf[k * n:(k + 1) * n].copy_(t.reshape(-1))
        shape = gl.shape
        pack_misfit(buf, J)
        dist.all_reduce(buf, group=self.group)
        views = [buf[k * n:(k + 1) * n].view(shape) for k in range(3)]
        return (unpack_misfit(buf), *views)
