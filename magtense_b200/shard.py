"""Instance sharding over ranks, one process per GPU.

Independent instances (the batching, hysteresis-sweep and dataset workloads)
partition across ranks with no exchange in the data path: each rank integrates
its own contiguous slice of the global instance list on its own GPU with its
own copy of the demag tensor.  The only collectives are host-side bookkeeping:
the max over ranks of a timing, and an optional final gather of per-instance
results (for example <m>(t)) to rank 0.  They run on whatever process group is
initialised (NCCL on GPUs, gloo on CPUs); without one they act on the single
local rank.
"""
from __future__ import annotations

import numpy as np
import torch


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def world():
    """(world_size, rank) of the initialised process group, (1, 0) without one."""
    d = _dist()
    return (d.get_world_size(), d.get_rank()) if d else (1, 0)


def shard_range(total: int, world_size: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [start, stop) of ``total`` instances owned by ``rank``:
    the first ``total % world_size`` ranks take one instance more."""
    if total < 0 or world_size < 1 or not (0 <= rank < world_size):
        raise ValueError("bad shard arguments")
    base, extra = divmod(total, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device():
    d = _dist()
    if d and d.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(values):
    """Element-wise max of a list of floats over all ranks (every rank gets it)."""
    d = _dist()
    if not d:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device())
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def gather_to_root(local: np.ndarray, total: int):
    """Concatenate every rank's slice (first axis, sizes from ``shard_range``)
    on rank 0, in rank order; other ranks get None.  All ranks must call it."""
    d = _dist()
    local = np.ascontiguousarray(local, dtype=np.float64)
    if not d:
        return local
    ws, rank = d.get_world_size(), d.get_rank()
    sizes = [shard_range(total, ws, r) for r in range(ws)]
    if local.shape[0] != sizes[rank][1] - sizes[rank][0]:
        raise ValueError("local slice does not match shard_range")
    rest = local.shape[1:]
    width = max(b - a for a, b in sizes)
    buf = torch.zeros((width,) + rest, dtype=torch.float64, device=_device())
    buf[: local.shape[0]] = torch.from_numpy(local).to(buf.device)
    parts = [torch.empty_like(buf) for _ in range(ws)]
    d.all_gather(parts, buf)
    if rank != 0:
        return None
    return np.concatenate([parts[r][: b - a].cpu().numpy() for r, (a, b) in enumerate(sizes)], axis=0)
