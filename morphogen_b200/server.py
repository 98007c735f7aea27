"""Continuous-batching answer loop (the C++ engine in mg_server.cu) and a
Poisson load generator.

The reference answers GPU queries from tokio handlers, one locked scan per
request (crates/morphogen-server/src/network/api/mod.rs:544-838).  PirServer
keeps the tables and their epoch delta buffers resident and folds every
request that arrives while the GPU is busy into the next pass; passes of its
workspaces overlap on the device.  Latency is measured by the engine from
submission to answer.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from typing import Callable, Sequence

import numpy as np

from . import _native as N
from .gpu_dpf import GpuPageMatrix, GpuScanner


class PirServer:
    def __init__(self, scanner: GpuScanner, slots: int = 2, max_keys_per_pass: int = 0,
                 memory_reserve: int = 1 << 30):
        self._scanner = scanner
        cfg = N.ServerConfig(slots, max_keys_per_pass, memory_reserve)
        h = C.c_void_p()
        N.check(N.lib().mg_server_create(scanner._ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h
        self._share_bytes: dict[int, list[int]] = {}
        self._lock = threading.Lock()

    def submit(self, items: Sequence[tuple[GpuPageMatrix, object]]) -> int:
        """Queue one request: (table, key) pairs; returns its id."""
        ka = N.KeyArray([bytes(k) for _, k in items])
        tarr = (C.c_void_p * ka.n)(*[t.handle.value for t, _ in items])
        rid = C.c_uint64()
        N.check(N.lib().mg_server_submit(self.handle, tarr, ka.ptrs, ka.lens, ka.n, C.byref(rid)))
        with self._lock:
            self._share_bytes[rid.value] = [t.row_bytes for t, _ in items]
        return rid.value

    def wait(self, rid: int, timeout_ms: int = 0) -> tuple[list[bytes], float]:
        with self._lock:
            sizes = self._share_bytes[rid]
        out = (C.c_uint8 * sum(sizes))()
        lat = C.c_double()
        N.check(N.lib().mg_server_wait(self.handle, rid, out, timeout_ms, C.byref(lat)))
        with self._lock:
            del self._share_bytes[rid]
        raw, res, off = bytes(out), [], 0
        for n in sizes:
            res.append(raw[off:off + n])
            off += n
        return res, lat.value

    def answer(self, items) -> list[bytes]:
        return self.wait(self.submit(items))[0]

    def pause(self, timeout_ms: int = 0) -> None:
        """Stop dispatching and drain the passes on the GPU (for epoch merges)."""
        N.check(N.lib().mg_server_pause(self.handle, timeout_ms))

    def resume(self) -> None:
        N.check(N.lib().mg_server_resume(self.handle))

    def merge(self, tables: Sequence[GpuPageMatrix], timeout_ms: int = 0) -> None:
        """Epoch advance: drain, XOR-patch every table with its pending delta, resume."""
        self.pause(timeout_ms)
        try:
            for t in tables:
                t.delta_merge()
        finally:
            self.resume()

    def stats(self) -> dict:
        st = N.ServerStats()
        N.check(N.lib().mg_server_get_stats(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def reset_stats(self) -> None:
        N.check(N.lib().mg_server_reset_stats(self.handle))

    def close(self) -> None:
        if self.handle:
            N.lib().mg_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ShardedPirServer:
    """Continuous batching over a table sharded into row ranges across GPUs
    (morphogen_b200.shard.ShardedTable): one PirServer per range, each
    request submitted to every range's server (so each GPU folds it into its
    own next pass) and the range shares XORed when all have answered.  A
    request's latency is the slowest range's, about 1/N of one GPU's pass."""

    def __init__(self, sharded, slots: int = 2, max_keys_per_pass: int = 0, memory_reserve: int = 1 << 30):
        self.sharded = sharded
        self.servers = [PirServer(sc, slots, max_keys_per_pass, memory_reserve) for sc in sharded.scanners]
        self._next = 0
        self._ids: dict[int, list[int]] = {}
        self._lock = threading.Lock()

    def submit(self, keys: Sequence) -> int:
        """Queue one request: its keys over the sharded table; returns its id."""
        kb = [bytes(k) for k in keys]
        rids: list[int] = []
        try:
            for srv, t in zip(self.servers, self.sharded.tables):
                rids.append(srv.submit([(t, k) for k in kb]))
        except Exception:
            for srv, r in zip(self.servers, rids):  # release what was already queued
                srv.wait(r)
            raise
        with self._lock:
            rid = self._next
            self._next += 1
            self._ids[rid] = rids
        return rid

    def wait(self, rid: int, timeout_ms: int = 0) -> tuple[list[bytes], float]:
        """The request's shares over the whole table and its latency (ms, the
        slowest range)."""
        with self._lock:
            rids = self._ids.pop(rid)
        parts, lat = [], 0.0
        for srv, r in zip(self.servers, rids):
            sh, lt = srv.wait(r, timeout_ms)
            parts.append(sh)
            lat = max(lat, lt)
        from .shard import xor_shares
        return xor_shares(parts), lat

    def answer(self, keys) -> list[bytes]:
        return self.wait(self.submit(keys))[0]

    def close(self) -> None:
        for srv in self.servers:
            srv.close()


def geometric_lookups(rng: np.random.Generator, mean: float = 4.0, lo: int = 1, hi: int = 32) -> int:
    """Lookups per request: geometric on {1, 2, ...} with the given mean, capped to [lo, hi]."""
    return int(min(hi, max(lo, rng.geometric(1.0 / mean))))


def poisson_load(server: PirServer, make_request: Callable[[np.random.Generator], list], rate_hz: float,
                 duration_s: float, seed: int = 0, tick: Callable[[float], None] | None = None) -> dict:
    """Open-loop Poisson arrivals for duration_s; waits for every answer.
    make_request(rng) returns the (table, key) items of one request; tick(t)
    is called from the submitting thread between arrivals (e.g. epoch merges).
    Returns the engine's statistics for the run plus offered/answered rates."""
    rng = np.random.default_rng(seed)
    server.reset_stats()
    ids: list[int] = []
    lookups = 0
    t0 = time.perf_counter()
    t_next = t0
    while True:
        t_next += rng.exponential(1.0 / rate_hz)
        if t_next - t0 > duration_s:
            break
        while True:
            now = time.perf_counter()
            if tick:
                tick(now - t0)
            if now >= t_next:
                break
            time.sleep(min(0.002, t_next - now))
        items = make_request(rng)
        lookups += len(items)
        ids.append(server.submit(items))
    for rid in ids:
        server.wait(rid)
    st = server.stats()
    # Offered load over the whole window (arrivals are open-loop).
    st.update({"offered_req_per_s": len(ids) / duration_s, "requests": len(ids), "keys": lookups,
               "answered_keys_per_s": st["keys_completed"] / max(st["wall_s"], 1e-9)})
    return st
