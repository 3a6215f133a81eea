"""Instance sharding over ranks, one process per GPU.

Independent instances (the batching, hysteresis-sweep and dataset workloads)
partition across ranks with no exchange in the data path: each rank integrates
its own contiguous slice of the global instance list on its own GPU with its
own copy of the demag tensor.  The only collectives are host-side bookkeeping:
the max over ranks of a timing, and an optional final gather of per-instance
results (for example <m>(t)) to rank 0.  They run on whatever process group is
initialised (NCCL on GPUs, gloo on CPUs); without one they act on the single
local rank.

One instance too large for one GPU is split by receiver rows instead
(``Solver(shard=(rank, world))``): each rank holds the tensor rows of its own
cells, and the integrator exchanges stage arguments and error norms between the
ranks' kernels through peer memory (CUDA IPC of each rank's exchange region).
``link_row_shard`` sets that up over the process group; ``gather_rows`` collects
the ranks' rows of the trajectory.
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


def exchange_bytes(blob: bytes) -> list[bytes]:
    """Every rank's ``blob`` in rank order (all ranks must call it)."""
    d = _dist()
    if not d:
        return [bytes(blob)]
    out = [None] * d.get_world_size()
    d.all_gather_object(out, bytes(blob))
    return out


def link_row_shard(solver) -> None:
    """Map every other rank's exchange region into this rank's row shard: each rank
    publishes the CUDA IPC handle of its region and opens the others'.  The
    solver's shard must be (rank, world) of the initialised process group."""
    ws, rank = world()
    if solver.shard != (rank, ws):
        raise ValueError(f"solver shard {solver.shard} is not (rank, world) = {(rank, ws)}")
    handles = exchange_bytes(solver.shard_ipc_handle())
    solver.shard_open_peers(handles)


def gather_rows(y_local, n: int):
    """Whole-instance trajectory from the row shards' outputs: ``y_local`` (nt, 3n)
    holds valid values in this rank's cells [c0, c0 + nc) of each component (the
    first sample everywhere); every rank gets the (nt, 3n) array with each rank's
    cells taken from that rank.  All ranks must call it."""
    d = _dist()
    y = torch.as_tensor(y_local)
    if not d:
        return y
    ws, rank = d.get_world_size(), d.get_rank()
    nt = y.shape[0]
    rows = [((n * r) // ws, (n * (r + 1)) // ws - (n * r) // ws) for r in range(ws)]
    width = max(nc for _, nc in rows)
    dev = _device()
    c0, nc = rows[rank]
    buf = torch.zeros((nt, 3, width), dtype=torch.float64, device=dev)
    buf[:, :, :nc] = y.reshape(nt, 3, n)[:, :, c0:c0 + nc].to(dev)
    parts = [torch.empty_like(buf) for _ in range(ws)]
    d.all_gather(parts, buf)
    full = torch.empty((nt, 3, n), dtype=torch.float64, device=dev)
    for r, (a, k) in enumerate(rows):
        full[:, :, a:a + k] = parts[r][:, :, :k]
    return full.reshape(nt, 3 * n).to(y.device)
