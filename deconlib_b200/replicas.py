"""Multi-GPU: independent replicas, one process per GPU.

The deconvolution path has no exchange step: a volume's FFTs and stencils
need the whole volume, and separate jobs / tiles / volumes are independent.
So N GPUs run N replicas (each its own jobs, OTFs and HBM budget) and the
only collectives are the measurement ones: the maximum of the ranks' device
times and the sum of the work they did.  No collective is on the data path.
"""

from __future__ import annotations

from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of independent jobs / tiles / volumes for ``rank``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} for world size {world}")
    return list(items[rank::world])


def aggregate(ms: float, units: float, group=None) -> Tuple[float, float]:
    """(max device time over ranks, total units over ranks); identity when
    torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), float(units)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    u = torch.tensor([float(units)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(u.item())
