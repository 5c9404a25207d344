"""Multi-GPU form of the path: independent replicas, one system per rank.

The hot path of one system does not shard (a single GPU holds the largest
workload with room to spare), so N GPUs run N independent systems with their
own seeds and no data-path collective.  The only communication is timing:
every rank's elapsed device time is reduced with MAX and the whole-job rate
is the beads of all ranks times the sweeps over that maximum.
"""
from __future__ import annotations

from typing import Sequence


def replica_seed(base: int, rank: int) -> int:
    """Seed of the system on `rank` (ranks run distinct, reproducible chains)."""
    return base + rank


def whole_job_rate(beads_per_rank: Sequence[int], sweeps: int, elapsed_s_max: float) -> float:
    """Bead-moves/s of all replicas, timed by the slowest rank."""
    return float(sum(beads_per_rank)) * sweeps / elapsed_s_max


def reduce_max(value: float, dist=None, device: str = "cpu") -> float:
    """MAX over ranks of `value` (identity without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_ints(value: int, dist=None, device: str = "cpu"):
    """All ranks' `value`, in rank order."""
    if dist is None or not dist.is_initialized():
        return [int(value)]
    import torch
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [int(x.item()) for x in out]
