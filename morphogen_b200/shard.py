"""Sharding one table over several GPUs.

A table is split into contiguous row ranges, one per rank (a row-range table
on each GPU, mg_table_create_range); every rank answers the same keys over its
rows, and the rank shares XOR to the share of the whole table.  NCCL has no
XOR reduction, so the shares (a few hundred bytes) are all-gathered and XORed
locally.  With a CPU process group (gloo) the same code runs without GPUs.
"""
from __future__ import annotations

import numpy as np


def shard_range(total_rows: int, world: int, rank: int, align: int = 1 << 20) -> tuple[int, int]:
    """Contiguous rows [first, first + count) of rank `rank`: boundaries are
    multiples of `align` (except the end) and spread the units evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    units = (total_rows + align - 1) // align
    lo = units * rank // world
    hi = units * (rank + 1) // world
    first = min(lo * align, total_rows)
    last = min(hi * align, total_rows)
    return first, last - first


def xor_shares(parts: list[list[bytes]]) -> list[bytes]:
    """XOR the per-rank shares key by key."""
    out = [np.frombuffer(s, np.uint8).copy() for s in parts[0]]
    for p in parts[1:]:
        for i, s in enumerate(p):
            out[i] ^= np.frombuffer(s, np.uint8)
    return [o.tobytes() for o in out]


def combine_shares(local: list[bytes], group=None, device=None) -> list[bytes]:
    """All-gather every rank's shares (same key order and sizes on every rank)
    and XOR them: the shares of the whole table, on every rank."""
    import torch
    import torch.distributed as dist

    sizes = [len(s) for s in local]
    flat = np.frombuffer(b"".join(local), np.uint8)
    t = torch.from_numpy(flat.copy())
    if device is not None:
        t = t.to(device)
    world = dist.get_world_size(group)
    bufs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(bufs, t, group=group)
    acc = bufs[0].cpu().numpy().copy()
    for b in bufs[1:]:
        acc ^= b.cpu().numpy()
    out, off = [], 0
    for n in sizes:
        out.append(acc[off:off + n].tobytes())
        off += n
    return out
