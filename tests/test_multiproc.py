"""Instance sharding over ranks (magtense_b200/shard.py) with world_size-2
gloo process groups on the CPU: the slices partition the instance list, the
max over ranks and the gather to rank 0 are exact and in rank order, the row
shards of one instance gather their rows and swap their IPC handles in rank
order, and a
rank that leaves before a collective makes the other rank's collective fail
within the process-group timeout instead of hanging."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s=30):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _worker_collectives(rank, world, port, total, out):
    dist = _init(rank, world, port)
    from magtense_b200.shard import gather_to_root, max_over_ranks, shard_range, world as get_world
    assert get_world() == (world, rank)
    a, b = shard_range(total, world, rank)
    # per-instance results: instance k carries k in every entry of its (t, 3) block
    local = np.arange(a, b, dtype=np.float64)[:, None, None] * np.ones((1, 5, 3))
    full = gather_to_root(local, total)
    mx = max_over_ranks([rank + 0.5, -rank])
    if rank == 0:
        out.put(("gather", full))
    out.put(("max", rank, mx))
    dist.barrier()
    dist.destroy_process_group()


def _worker_rows(rank, world, port, n, out):
    """Row shards' host side: every rank fills only its own cells of a (nt, 3n)
    trajectory (NaN elsewhere, the first sample everywhere) and exchanges a
    64-byte blob standing in for its IPC handle."""
    dist = _init(rank, world, port)
    import torch
    from magtense_b200.shard import exchange_bytes, gather_rows
    from magtense_b200.solver import shard_rows
    nt = 4
    ref = torch.arange(nt * 3 * n, dtype=torch.float64).reshape(nt, 3 * n)
    y = torch.full_like(ref, float("nan"))
    y[0] = ref[0]
    c0, nc = shard_rows(n, rank, world)
    for a in range(3):
        y[1:, a * n + c0:a * n + c0 + nc] = ref[1:, a * n + c0:a * n + c0 + nc]
    full = gather_rows(y, n)
    blobs = exchange_bytes(bytes([rank]) * 64)
    out.put((rank, bool(torch.equal(full, ref)), blobs))
    dist.barrier()
    dist.destroy_process_group()


def _worker_leaver(rank, world, port, out):
    dist = _init(rank, world, port, timeout_s=5)
    from magtense_b200.shard import max_over_ranks
    if rank == 1:
        return                               # leaves without joining the collective
    try:
        max_over_ranks([1.0])
        out.put(("no error", None))
    except Exception as e:                   # the timeout surfaces on the host as an exception
        out.put(("error", type(e).__name__))


def test_shard_range_partitions():
    from magtense_b200.shard import shard_range
    for total in (0, 1, 7, 256, 1001):
        for ws in (1, 2, 3, 8):
            cover = []
            for r in range(ws):
                a, b = shard_range(total, ws, r)
                assert 0 <= b - a <= -(-total // ws)
                cover.extend(range(a, b))
            assert cover == list(range(total))
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


@pytest.mark.parametrize("total", [7, 256])
def test_gloo_two_ranks_gather_and_max(total):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_collectives, args=(r, 2, port, total, out)) for r in range(2)]
    for p in procs:
        p.start()
    msgs = [out.get(timeout=120) for _ in range(3)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = [m[1] for m in msgs if m[0] == "gather"][0]
    assert full.shape == (total, 5, 3)
    np.testing.assert_array_equal(full[:, 0, 0], np.arange(total))
    for m in msgs:
        if m[0] == "max":
            assert m[2] == [1.5, 0.0]


def test_gloo_rank_that_leaves_is_detected():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_leaver, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    kind, info = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert kind == "error", info


@pytest.mark.parametrize("world,n", [(2, 640), (3, 814)])
def test_gloo_row_shards_gather_rows_and_handles(world, n):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_rows, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    msgs = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, blobs in msgs:
        assert ok, rank
        assert blobs == [bytes([r]) * 64 for r in range(world)]


def test_row_partition_matches_the_library():
    """shard_rows restates mt_set_row_shard's split: contiguous, covering, sizes
    differing by at most one."""
    from magtense_b200.solver import shard_rows
    for n in (2, 7, 640, 814, 32768):
        for w in range(2, 9):
            if n < w:
                continue
            cells = []
            for r in range(w):
                c0, nc = shard_rows(n, r, w)
                assert nc in (n // w, n // w + 1)
                cells.extend(range(c0, c0 + nc))
            assert cells == list(range(n))
