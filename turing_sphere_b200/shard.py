"""Instance sharding over GPUs, one process per GPU.

Instances of a batched model (a parameter sweep, independent fields of a
transform batch) never exchange data during a step, so N GPUs each advance a
contiguous block of the instances with no collective on the data path.  The
only communication is at the edges: the maximum device time over ranks for
reporting, and an optional gather of final states, losses or gradients to
rank 0 once a run has finished.

The helpers take any initialised torch.distributed process group: NCCL with
CUDA tensors on a GPU node, gloo with CPU tensors in tests.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """(start, count) of rank's contiguous block when n instances are split
    over world ranks; the first n % world ranks take one extra instance."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if n < 0:
        raise ValueError("negative instance count")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """The maximum of x over all ranks (device-time reporting)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_instances(local: np.ndarray, n_total: int) -> np.ndarray | None:
    """Concatenate every rank's block of instances (leading axis) in rank
    order on rank 0; other ranks get None.  Blocks may differ in length by
    one (shard_range): they are padded to the longest for the all-gather."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local)
    if not dist.is_initialized() or dist.get_world_size() == 1:
        if local.shape[0] != n_total:
            raise ValueError(f"{local.shape[0]} instances, expected {n_total}")
        return local
    world, rank = dist.get_world_size(), dist.get_rank()
    counts = [shard_range(n_total, r, world)[1] for r in range(world)]
    if local.shape[0] != counts[rank]:
        raise ValueError(f"rank {rank} holds {local.shape[0]} instances, expected {counts[rank]}")
    width = max(counts)
    dev = _device()
    pad = np.zeros((width,) + local.shape[1:], dtype=local.dtype)
    pad[:local.shape[0]] = local
    t = torch.from_numpy(pad).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    if rank != 0:
        return None
    return np.concatenate([p.cpu().numpy()[:c] for p, c in zip(parts, counts)], axis=0)
