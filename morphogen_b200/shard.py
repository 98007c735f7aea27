"""Sharding one table over several GPUs.

A table is split into contiguous row ranges, one per rank (a row-range table
on each GPU, mg_table_create_range); every rank answers the same keys over its
rows, and the rank shares XOR to the share of the whole table.  NCCL has no
XOR reduction, so the shares (a few hundred bytes) are all-gathered and XORed
locally.  With a CPU process group (gloo) the same code runs without GPUs.
The reference's counterpart is a timing sketch only
(crates/morphogen-gpu-dpf/src/bin/bench_sharded.rs:14-110: one page range per
GPU thread, max latency over the threads, no combine).
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

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return list(local)
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


def device_view(ptr: int, nbytes: int, device: int):
    """A torch uint8 tensor over `nbytes` of device memory at `ptr` (no copy)."""
    import torch

    class _Buf:
        pass

    b = _Buf()
    b.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                  "version": 3, "strides": None, "stream": None}
    return torch.as_tensor(b, device=f"cuda:{device}")


def combine_tensor(local, gathered, out, world: int, group=None):
    """out = XOR over the ranks of `local` (uint8 tensors; `gathered` holds
    world x local.numel() bytes).  Device tensors go over NCCL, host tensors
    over gloo."""
    import torch
    import torch.distributed as dist

    if world == 1:
        out.copy_(local)
        return out
    dist.all_gather_into_tensor(gathered, local, group=group)
    parts = gathered.view(world, -1)
    torch.bitwise_xor(parts[0], parts[1], out=out)
    for r in range(2, world):
        out.bitwise_xor_(parts[r])
    return out


class ShardCombiner:
    """XOR-combines a workspace's device share buffer across the ranks of a
    process group, on the device: NCCL all-gather of the shares into one
    buffer, then an XOR fold over the ranks.  The result stays on the device
    in `out`; on one rank it is a copy of the local shares."""

    def __init__(self, device: int, group=None):
        import torch.distributed as dist

        self.device = device
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
        self._key = None

    def _bind(self, ws):
        import torch
        ptr, n = ws.shares_device()
        if self._key != (ptr, n):
            self.local = device_view(ptr, n, self.device)
            self.gathered = torch.empty(self.world * n, dtype=torch.uint8, device=f"cuda:{self.device}")
            self.out = torch.empty(n, dtype=torch.uint8, device=f"cuda:{self.device}")
            self._key = (ptr, n)

    def combine(self, ws, stream=None):
        """Enqueue the combine of `ws`'s last pass on `stream` (a torch stream;
        the workspace's pass must have been launched on the same stream)."""
        import torch

        self._bind(ws)
        with torch.cuda.stream(stream) if stream is not None else _null():
            combine_tensor(self.local, self.gathered, self.out, self.world, self.group)
        return self.out


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class ShardedTable:
    """One logical table split into contiguous row ranges over several GPUs
    of this process (the layout of crates/morphogen-gpu-dpf/src/bin/
    bench_sharded.rs, which gives each GPU thread one page range): every scan
    runs the same keys on every range at once, one host thread per range,
    and XORs the range shares into the shares of the whole table.

    scanners: one GpuScanner per range (ranges may share a device)."""

    def __init__(self, scanners, total_rows: int, row_bytes: int, align: int = 1 << 20):
        from morphogen_b200 import gpu_dpf as G

        self.scanners = list(scanners)
        self.total_rows, self.row_bytes = total_rows, row_bytes
        self.spans = [shard_range(total_rows, len(self.scanners), r, align) for r in range(len(self.scanners))]
        self.tables = [G.GpuPageMatrix.range(sc, first, n, row_bytes)
                       for sc, (first, n) in zip(self.scanners, self.spans)]
        from concurrent.futures import ThreadPoolExecutor
        self._pool = ThreadPoolExecutor(max_workers=len(self.tables))

    def fill_splitmix(self, seed: int) -> None:
        for t in self.tables:
            t.fill_splitmix(seed)

    def write_rows(self, first_row: int, rows) -> None:
        """Host rows (n x row_bytes) at logical row first_row, split over the ranges."""
        data = np.ascontiguousarray(rows, dtype=np.uint8).reshape(-1, self.row_bytes)
        end = first_row + data.shape[0]
        for t, (f, n) in zip(self.tables, self.spans):
            lo, hi = max(first_row, f), min(end, f + n)
            if lo < hi:
                t.update_pages(lo - f, data[lo - first_row:hi - first_row])

    def scan(self, keys, timeout_ms: int = 0) -> list[bytes]:
        """One share per key over the whole logical table."""
        kb = [bytes(k) for k in keys]
        parts = list(self._pool.map(lambda st: st[0].scan_keys(st[1], kb, timeout_ms)[0],
                                    zip(self.scanners, self.tables)))
        return xor_shares(parts)

    def close(self) -> None:
        self._pool.shutdown(wait=True)
        for t in self.tables:
            t.close()
