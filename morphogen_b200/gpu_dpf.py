"""Host-side mirror of the reference's morphogen-gpu-dpf interface, on the sm_100a library.

Names, argument meaning and error behaviour follow
crates/morphogen-gpu-dpf/src/{dpf,kernel,storage}.rs so that callers of the
reference's `GpuScanner` / `GpuPageMatrix` / `ChaChaKey` find the same surface:

* ``ChaChaParams``, ``ChaChaKey`` (wire format of dpf.rs:259-316),
  ``generate_chacha_dpf_keys`` (dpf.rs:322-432);
* ``GpuPageMatrix`` (storage.rs:18-124) generalised to R-byte rows
  (``row_bytes`` defaults to the reference's 4096-byte page);
* ``GpuScanner`` with ``scan`` / ``scan_batch*`` / multistream
  (kernel.rs:685-1210) returning ``PirResult`` with ``KernelTiming``
  (kernel.rs:1214-1240).

Every scan runs in libmorphogen_gpu.so; nothing here evaluates a DPF on the
host except key generation, which is client-side work in the reference too.
"""
from __future__ import annotations

import ctypes as C
import os
import secrets
import threading
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _native as N

PAGE_SIZE_BYTES = 4096            # storage.rs:14
SUBTREE_SIZE = 2048               # kernel.rs:39 (CPU tile; the device path tunes its own)
THREADS_PER_BLOCK = 256           # kernel.rs:42
MAX_DOMAIN_BITS = N.MAX_DOMAIN_BITS  # reference kernel: 25 (kernel.rs:45); this path: 32
MAX_KERNEL_BATCH_SIZE = 16        # kernel.rs:48
DEFAULT_WORKSPACE_POOL_SIZE = 4   # kernel.rs:50
MAX_WORKSPACE_POOL_SIZE = 8       # kernel.rs:52
GPU_WORKSPACE_POOL_SIZE_ENV = "MORPHOGEN_GPU_WORKSPACE_POOL_SIZE"  # kernel.rs:54
KEYS_PER_QUERY = 3                # kernel.rs:56
VERIF_BYTES_PER_KEY = 16          # kernel.rs:58

GpuDpfError = N.GpuDpfError
DriverError = N.DriverError


# ---- host policy helpers (kernel.rs:61-105) --------------------------------

def parse_workspace_pool_size(raw: str | None) -> int:
    """kernel.rs:61-66: positive integers clamp to the max; anything else -> default."""
    try:
        v = int(raw) if raw is not None else 0
    except ValueError:
        v = 0
    return min(v, MAX_WORKSPACE_POOL_SIZE) if v > 0 else DEFAULT_WORKSPACE_POOL_SIZE


def select_workspace_pool_slot(ticket: int, pool_size: int) -> int:
    """kernel.rs:69-72"""
    assert pool_size > 0
    return ticket % pool_size


def clamp_tiled_launch_limit(tile_size: int) -> int:
    """kernel.rs:75-77"""
    return max(1, min(tile_size, MAX_KERNEL_BATCH_SIZE))


def select_tiled_launch_batch_size(remaining: int, tile_size: int) -> int:
    """kernel.rs:80-93: largest of 16/8/4/2/1 not above min(remaining, tile)."""
    capped = min(remaining, clamp_tiled_launch_limit(tile_size))
    for b in (16, 8, 4, 2):
        if capped >= b:
            return b
    return 1


def plan_tiled_launch_batch_sizes(total_queries: int, tile_size: int) -> list[int]:
    """kernel.rs:96-105"""
    plan, remaining = [], total_queries
    while remaining > 0:
        b = select_tiled_launch_batch_size(remaining, tile_size)
        plan.append(b)
        remaining -= b
    return plan


# ---- keys (dpf.rs) ----------------------------------------------------------

class ChaChaParams:
    """dpf.rs:59-86"""

    def __init__(self, domain_bits: int):
        if domain_bits == 0:
            raise GpuDpfError(N.MG_EKEY, f"Invalid domain bits {domain_bits}: must be > 0")
        if domain_bits > 32:
            raise GpuDpfError(N.MG_EKEY, f"Invalid domain bits {domain_bits}: must be <= 32")
        self.domain_bits = domain_bits

    @classmethod
    def new(cls, domain_bits: int) -> "ChaChaParams":
        return cls(domain_bits)

    def max_pages(self) -> int:
        return 1 << self.domain_bits


@dataclass(frozen=True)
class CorrectionWord:
    """dpf.rs:43-48"""
    seed_cw: bytes
    t_cw_left: int
    t_cw_right: int


class ChaChaKey:
    """One party's DPF key, held in the reference's wire format (dpf.rs:259-316)."""

    __slots__ = ("_bytes", "domain_bits", "party")

    def __init__(self, wire: bytes):
        wire = bytes(wire)
        d = C.c_uint32()
        party = C.c_uint8()
        N.check(N.lib().mg_key_check(N.u8ptr(wire), len(wire), C.byref(d), C.byref(party)))
        self._bytes = wire
        self.domain_bits = d.value
        self.party = party.value

    @classmethod
    def from_bytes(cls, wire: bytes) -> "ChaChaKey":
        return cls(wire)

    def to_bytes(self) -> bytes:
        return self._bytes

    def __bytes__(self) -> bytes:
        return self._bytes

    def __eq__(self, other) -> bool:
        return isinstance(other, ChaChaKey) and other._bytes == self._bytes

    def __hash__(self) -> int:
        return hash(self._bytes)

    @property
    def root_seed(self) -> bytes:
        return self._bytes[0:16]

    @property
    def root_t(self) -> int:
        return self._bytes[16]

    @property
    def correction_words(self) -> list[CorrectionWord]:
        out, off = [], 19
        for _ in range(self.domain_bits):
            b = self._bytes[off:off + 18]
            out.append(CorrectionWord(b[:16], b[16], b[17]))
            off += 18
        return out

    @property
    def final_cw(self) -> bytes:
        return self._bytes[-16:]

    def max_pages(self) -> int:
        return 1 << self.domain_bits

    def is_party1(self) -> bool:
        return self.party == 1


def key_size(domain_bits: int) -> int:
    return int(N.lib().mg_key_size(domain_bits))


def generate_chacha_dpf_keys(params: ChaChaParams, target: int,
                             rng: np.random.Generator | None = None) -> tuple[ChaChaKey, ChaChaKey]:
    """dpf.rs:322-432.  Root seeds come from `secrets` (unseeded, like the
    reference's rand::random) or from `rng` when a seeded run is wanted."""
    if target < 0:
        raise GpuDpfError(N.MG_ERANGE, f"Page index {target} exceeds max {params.max_pages()}")
    if rng is None:
        r0, r1 = secrets.token_bytes(16), secrets.token_bytes(16)
    else:
        r0 = rng.integers(0, 256, 16, dtype=np.uint8).tobytes()
        r1 = rng.integers(0, 256, 16, dtype=np.uint8).tobytes()
    n = key_size(params.domain_bits)
    b0 = (C.c_uint8 * n)()
    b1 = (C.c_uint8 * n)()
    N.check(N.lib().mg_keygen(params.domain_bits, target, N.u8ptr(r0), N.u8ptr(r1), b0, b1))
    return ChaChaKey(bytes(b0)), ChaChaKey(bytes(b1))


# ---- results ----------------------------------------------------------------

@dataclass
class KernelTiming:
    """kernel.rs:1214-1228 (per-query averages, nanoseconds)."""
    dpf_eval_ns: int = 0
    xor_accumulate_ns: int = 0
    h2d_ns: int = 0
    kernel_ns: int = 0
    d2h_ns: int = 0
    total_ns: int = 0


@dataclass
class PirResult:
    """kernel.rs:1231-1240: one share per Cuckoo key.  The verif fields mirror
    the reference's Binius outputs, which are all-zero there as well
    (ENABLE_BINIUS is off in cuda/fused_kernel.cu)."""
    page0: bytes
    page1: bytes
    page2: bytes
    verif0: bytes = bytes(VERIF_BYTES_PER_KEY)
    verif1: bytes = bytes(VERIF_BYTES_PER_KEY)
    verif2: bytes = bytes(VERIF_BYTES_PER_KEY)
    timing: KernelTiming = field(default_factory=KernelTiming)

    @property
    def pages(self) -> list[bytes]:
        return [self.page0, self.page1, self.page2]


# ---- device objects -----------------------------------------------------------

class _Context:
    def __init__(self, device: int):
        h = C.c_void_p()
        N.check(N.lib().mg_context_create(device, C.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            N.lib().mg_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuPageMatrix:
    """storage.rs:18-124: a device-resident table of `num_pages` rows of `row_bytes`."""

    def __init__(self, scanner: "GpuScanner", num_rows: int, row_bytes: int = PAGE_SIZE_BYTES,
                 first_row: int = 0):
        self._scanner = scanner  # keeps the context alive
        h = C.c_void_p()
        N.check(N.lib().mg_table_create_range(scanner._ctx.handle, first_row, num_rows, row_bytes, C.byref(h)))
        self.handle = h
        self.row_bytes = row_bytes
        self.first_row = first_row
        self._rows = num_rows

    @classmethod
    def range(cls, scanner: "GpuScanner", first_row: int, num_rows: int, row_bytes: int) -> "GpuPageMatrix":
        """Rows [first_row, first_row + num_rows) of a larger logical table (a shard)."""
        return cls(scanner, num_rows, row_bytes, first_row)

    # storage.rs:27-43
    @classmethod
    def new(cls, scanner: "GpuScanner", cpu_data, row_bytes: int = PAGE_SIZE_BYTES) -> "GpuPageMatrix":
        data = np.frombuffer(bytes(cpu_data), np.uint8) if not isinstance(cpu_data, np.ndarray) else cpu_data
        data = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        if data.size % row_bytes:
            raise ValueError("cpu_data length must be multiple of row_bytes")
        m = cls(scanner, data.size // row_bytes, row_bytes)
        m.update_pages(0, data)
        return m

    # storage.rs:45-86
    @classmethod
    def from_chunked_matrix(cls, scanner: "GpuScanner", matrix, row_bytes: int = PAGE_SIZE_BYTES) -> "GpuPageMatrix":
        """Build from a chunked CPU matrix: `matrix` is a sequence of byte
        chunks, or an object with num_chunks() / chunk(i) like the storage
        crate's ChunkedMatrix.  The total is padded with zeros to whole rows;
        each chunk is uploaded at row offset // row_bytes of its byte offset,
        a chunk that is not a whole number of rows padded with zeros first."""
        if hasattr(matrix, "num_chunks"):
            chunks = [matrix.chunk(i) for i in range(matrix.num_chunks())]
        else:
            chunks = list(matrix)
        views = [np.frombuffer(bytes(c), np.uint8) if not isinstance(c, np.ndarray)
                 else np.ascontiguousarray(c, dtype=np.uint8).reshape(-1) for c in chunks]
        total = sum(v.size for v in views)
        m = cls(scanner, (total + row_bytes - 1) // row_bytes, row_bytes)
        offset = 0
        for v in views:
            size = v.size
            if size % row_bytes:
                v = np.concatenate([v, np.zeros(row_bytes - size % row_bytes, np.uint8)])
            if size:
                m.update_pages(offset // row_bytes, v)
            offset += size
        return m

    @property
    def device(self) -> int:
        """CUDA device ordinal holding the table."""
        return self._scanner.device

    def as_slice(self) -> tuple[int, int]:
        """(device pointer, bytes) of the resident rows."""
        return self.device_ptr(), self.size_bytes()

    # storage.rs:89-101
    @classmethod
    def alloc_empty(cls, scanner: "GpuScanner", num_rows: int, row_bytes: int = PAGE_SIZE_BYTES):
        return cls(scanner, num_rows, row_bytes)

    @classmethod
    def from_seed(cls, scanner: "GpuScanner", num_rows: int, row_bytes: int, seed: int,
                  first_row: int = 0) -> "GpuPageMatrix":
        """Synthetic SplitMix64 rows; a row-range table gets the logical table's rows."""
        m = cls(scanner, num_rows, row_bytes, first_row)
        m.fill_splitmix(seed)
        return m

    # storage.rs:104-124
    def update_pages(self, start_row: int, cpu_rows) -> None:
        data = np.ascontiguousarray(np.frombuffer(bytes(cpu_rows), np.uint8)
                                    if not isinstance(cpu_rows, np.ndarray) else cpu_rows,
                                    dtype=np.uint8).reshape(-1)
        if data.size % self.row_bytes:
            raise ValueError("cpu_pages length must be multiple of row_bytes")
        N.check(N.lib().mg_table_write_rows(self.handle, start_row, data.ctypes.data_as(C.c_void_p),
                                            data.size // self.row_bytes))

    def read_rows(self, start_row: int, nrows: int) -> np.ndarray:
        out = np.empty(nrows * self.row_bytes, np.uint8)
        N.check(N.lib().mg_table_read_rows(self.handle, start_row, out.ctypes.data_as(C.c_void_p), nrows))
        return out

    def fill_splitmix(self, seed: int) -> None:
        N.check(N.lib().mg_table_fill_splitmix(self.handle, seed))

    def xor_rows(self, row_idx, diffs) -> None:
        """Epoch merge: rows[row_idx[i]] ^= diffs[i] in place."""
        idx = np.ascontiguousarray(row_idx, dtype=np.uint64)
        d = np.ascontiguousarray(diffs, dtype=np.uint8).reshape(-1)
        if d.size != idx.size * self.row_bytes:
            raise ValueError("diffs must hold one row per index")
        N.check(N.lib().mg_table_xor_rows(self.handle, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          d.ctypes.data_as(C.c_void_p), idx.size))

    # -- epoch delta (DeltaBuffer / scan_delta_for_gpu / epoch merge) -------
    def delta_reserve(self, capacity: int) -> None:
        N.check(N.lib().mg_table_delta_reserve(self.handle, capacity))

    def delta_push(self, row_idx, diffs) -> None:
        idx = np.ascontiguousarray(row_idx, dtype=np.uint64)
        d = np.ascontiguousarray(diffs, dtype=np.uint8).reshape(-1)
        if d.size != idx.size * self.row_bytes:
            raise ValueError("diffs must hold one row per index")
        N.check(N.lib().mg_table_delta_push(self.handle, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                            d.ctypes.data_as(C.c_void_p), idx.size))

    def delta_count(self) -> int:
        return int(N.lib().mg_table_delta_count(self.handle))

    def delta_clear(self) -> None:
        N.check(N.lib().mg_table_delta_clear(self.handle))

    def delta_merge(self) -> None:
        N.check(N.lib().mg_table_delta_merge(self.handle))

    def epoch(self) -> int:
        return int(N.lib().mg_table_epoch(self.handle))

    def num_pages(self) -> int:
        return self._rows

    num_rows = num_pages

    def size_bytes(self) -> int:
        return self._rows * self.row_bytes

    def device_ptr(self) -> int:
        return int(N.lib().mg_table_device_ptr(self.handle) or 0)

    def close(self):
        if self.handle:
            N.lib().mg_table_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Workspace:
    """One mg_batch: device key buffer, partials, shares, stream, graph cache
    (the reference's BatchWorkspace, kernel.rs:163-171)."""

    def __init__(self, scanner: "GpuScanner"):
        self._scanner = scanner
        h = C.c_void_p()
        N.check(N.lib().mg_batch_create(scanner._ctx.handle, C.byref(h)))
        self.handle = h
        self.lock = threading.Lock()
        self._share_bytes = 0
        self._tables = None
        self._keys = None

    def set_shape(self, subtree_bits: int = 0, keys_per_cta: int = 0) -> None:
        N.check(N.lib().mg_batch_set_shape(self.handle, subtree_bits, keys_per_cta))

    def set_kernel(self, kind: str = "auto") -> None:
        """'auto', 'cta' (any row size) or 'warp' (rows of 16..512 B)."""
        code = {"auto": N.KERNEL_AUTO, "cta": N.KERNEL_CTA, "warp": N.KERNEL_WARP}[kind]
        N.check(N.lib().mg_batch_set_kernel(self.handle, code))

    def set_keys(self, tables: Sequence[GpuPageMatrix], keys: Sequence) -> None:
        if len(tables) != len(keys):
            raise ValueError("one table per key")
        ka = N.KeyArray(keys)
        tarr = (C.c_void_p * ka.n)(*[t.handle.value for t in tables])
        N.check(N.lib().mg_batch_set_keys(self.handle, tarr, ka.ptrs, ka.lens, ka.n))
        self._tables, self._keys = list(tables), ka
        self._share_bytes = sum(t.row_bytes for t in tables)
        self._row_bytes = [t.row_bytes for t in tables]

    def autotune(self, budget_ms: int = 0) -> dict:
        """Time candidate launch shapes for the current keys and keep the
        fastest (also for later passes of the same workload on this scanner)."""
        info = N.PlanInfo()
        ms = C.c_double()
        N.check(N.lib().mg_batch_autotune(self.handle, budget_ms, C.byref(info), C.byref(ms)))
        out = {f: getattr(info, f) for f, _ in info._fields_}
        out["ms"] = ms.value
        return out

    def launch(self, stream: int | None = None, graph: bool = False) -> None:
        f = N.lib().mg_batch_launch_graph if graph else N.lib().mg_batch_launch
        N.check(f(self.handle, C.c_void_p(stream) if stream else None))

    def read(self, stream: int | None = None) -> list[bytes]:
        out = (C.c_uint8 * self._share_bytes)()
        N.check(N.lib().mg_batch_read(self.handle, out, C.c_void_p(stream) if stream else None))
        raw = bytes(out)
        res, off = [], 0
        for rb in self._row_bytes:
            res.append(raw[off:off + rb])
            off += rb
        return res

    def sync(self, timeout_ms: int = 0) -> None:
        N.check(N.lib().mg_batch_sync(self.handle, timeout_ms))

    def plan(self) -> dict:
        info = N.PlanInfo()
        N.check(N.lib().mg_batch_plan(self.handle, C.byref(info)))
        return {f: getattr(info, f) for f, _ in info._fields_}

    def last_kernel_ns(self) -> int:
        v = C.c_uint64()
        N.check(N.lib().mg_batch_last_kernel_ns(self.handle, C.byref(v)))
        return v.value

    def last_scan_ns(self) -> int:
        v = C.c_uint64()
        N.check(N.lib().mg_batch_last_scan_ns(self.handle, C.byref(v)))
        return v.value

    def shares_device(self) -> tuple[int, int]:
        p = C.c_void_p()
        n = C.c_size_t()
        N.check(N.lib().mg_batch_shares_device(self.handle, C.byref(p), C.byref(n)))
        return int(p.value or 0), n.value

    def close(self):
        if self.handle:
            N.lib().mg_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuScanner:
    """kernel.rs:156-1211 on the sm_100a library."""

    def __init__(self, device_ord: int = 0):
        self.device = device_ord
        self._ctx = _Context(device_ord)
        size = parse_workspace_pool_size(os.environ.get(GPU_WORKSPACE_POOL_SIZE_ENV))
        self._pool: list[Workspace | None] = [None] * size
        self._pool_lock = threading.Lock()
        self._ticket = 0

    @classmethod
    def new(cls, device_ord: int = 0) -> "GpuScanner":
        return cls(device_ord)

    # -- helpers -------------------------------------------------------------
    def device_info(self) -> dict:
        sms = C.c_int()
        free = C.c_uint64()
        total = C.c_uint64()
        N.check(N.lib().mg_device_info(self._ctx.handle, C.byref(sms), C.byref(free), C.byref(total)))
        return {"sm_count": sms.value, "free_bytes": free.value, "total_bytes": total.value}

    def prg_peak(self, iters: int = 256) -> float:
        """Node expansions/s of the device ChaCha8 PRG alone (ALU ceiling)."""
        v = C.c_double()
        N.check(N.lib().mg_prg_peak(self._ctx.handle, iters, C.byref(v)))
        return v.value

    def workspace(self) -> Workspace:
        return Workspace(self)

    def _slot(self) -> Workspace:
        with self._pool_lock:
            ticket = self._ticket
            self._ticket += 1
            i = select_workspace_pool_slot(ticket, len(self._pool))
            if self._pool[i] is None:
                self._pool[i] = Workspace(self)
            return self._pool[i]

    def _run_pass(self, ws: Workspace, tables, keys, graph: bool) -> tuple[list[bytes], int]:
        ws.set_keys(tables, keys)
        ws.launch(graph=graph)
        shares = ws.read()
        return shares, ws.last_kernel_ns()

    @staticmethod
    def _flatten(queries) -> list:
        keys = []
        for q in queries:
            if len(q) != KEYS_PER_QUERY:
                raise ValueError(f"each query carries {KEYS_PER_QUERY} keys")
            keys.extend(bytes(k) for k in q)
        return keys

    # -- the reference's entry points -------------------------------------------
    def scan(self, db: GpuPageMatrix, keys: Sequence) -> PirResult:
        """kernel.rs:927-935"""
        return self.scan_batch(db, [list(keys)])[0]

    def scan_batch(self, db: GpuPageMatrix, queries, *, use_cuda_graph: bool = False,
                   max_tile_size: int | None = None) -> list[PirResult]:
        """kernel.rs:685-924: all queries' keys in passes of at most
        `max_tile_size` queries (default: the whole batch in one pass)."""
        queries = list(queries)
        if not queries:
            return []
        import time
        t_start = time.perf_counter_ns()
        plan = ([len(queries)] if max_tile_size is None
                else plan_tiled_launch_batch_sizes(len(queries), max_tile_size))
        ws = self._slot()
        results: list[PirResult] = []
        kernel_ns = 0
        with ws.lock:
            done = 0
            for q in plan:
                keys = self._flatten(queries[done:done + q])
                shares, kns = self._run_pass(ws, [db] * len(keys), keys, use_cuda_graph)
                kernel_ns += kns
                for i in range(q):
                    results.append(PirResult(*shares[3 * i:3 * i + 3]))
                done += q
        total = time.perf_counter_ns() - t_start
        n = len(queries)
        for r in results:
            r.timing = KernelTiming(dpf_eval_ns=kernel_ns // n, kernel_ns=kernel_ns // n,
                                    total_ns=total // n, h2d_ns=0, d2h_ns=0)
        return results

    def scan_batch_optimized(self, db, queries):
        return self.scan_batch(db, queries)

    def scan_batch_optimized_with_graph(self, db, queries, use_cuda_graph: bool):
        return self.scan_batch(db, queries, use_cuda_graph=use_cuda_graph)

    def scan_batch_optimized_tiled(self, db, queries, tile_size: int):
        return self.scan_batch(db, queries, max_tile_size=tile_size)

    def scan_batch_optimized_tiled_with_graph(self, db, queries, tile_size: int, use_cuda_graph: bool):
        return self.scan_batch(db, queries, use_cuda_graph=use_cuda_graph, max_tile_size=tile_size)

    def scan_batch_single_query_multistream_optimized(self, db, queries, stream_count: int):
        return self.scan_batch_single_query_multistream_optimized_with_graph(db, queries, stream_count, False)

    def scan_batch_single_query_multistream_optimized_with_graph(self, db, queries, stream_count: int,
                                                                 use_cuda_graph: bool):
        """kernel.rs:955-1097: one pass per query, round-robin over
        `stream_count` workspaces whose streams overlap on the device."""
        queries = list(queries)
        if not queries:
            return []
        stream_count = max(1, min(stream_count, len(queries)))
        if stream_count <= 1:
            return self.scan_batch(db, queries, use_cuda_graph=use_cuda_graph)
        wss = [Workspace(self) for _ in range(stream_count)]
        out: list[PirResult | None] = [None] * len(queries)
        for start in range(0, len(queries), stream_count):
            active = []
            for j, qi in enumerate(range(start, min(start + stream_count, len(queries)))):
                ws = wss[j]
                keys = self._flatten([queries[qi]])
                ws.set_keys([db] * 3, keys)
                ws.launch(graph=use_cuda_graph)
                active.append((qi, ws))
            for qi, ws in active:
                shares = ws.read()
                kns = ws.last_kernel_ns()
                out[qi] = PirResult(*shares, timing=KernelTiming(dpf_eval_ns=kns, kernel_ns=kns))
        for ws in wss:
            ws.close()
        return out  # type: ignore[return-value]

    def scan_multi(self, items: Iterable[tuple[GpuPageMatrix, object]], *, timeout_ms: int = 0,
                   use_cuda_graph: bool = False) -> list[bytes]:
        """Mixed-size batching: any number of (table, key) pairs over several
        resident tables answered in one pass; one share per pair."""
        items = list(items)
        if not items:
            return []
        ws = self._slot()
        with ws.lock:
            ws.set_keys([t for t, _ in items], [bytes(k) for _, k in items])
            ws.launch(graph=use_cuda_graph)
            if timeout_ms:
                ws.sync(timeout_ms)
            return ws.read()

    def scan_keys(self, db, keys: Sequence, timeout_ms: int = 0) -> tuple[list[bytes], dict]:
        """The one-call C entry point mg_scan: host keys in, host shares out.
        `db` is one table for every key, or a sequence with one table per key."""
        ka = N.KeyArray(keys)
        tabs = list(db) if isinstance(db, (list, tuple)) else [db] * ka.n
        if len(tabs) != ka.n:
            raise ValueError("one table per key")
        tarr = (C.c_void_p * ka.n)(*[t.handle.value for t in tabs])
        sizes = [t.row_bytes for t in tabs]
        out = (C.c_uint8 * sum(sizes))()
        tm = N.Timing()
        N.check(N.lib().mg_scan(self._ctx.handle, tarr, ka.ptrs, ka.lens, ka.n, out, timeout_ms, C.byref(tm)))
        raw = bytes(out)
        res, off = [], 0
        for rb in sizes:
            res.append(raw[off:off + rb])
            off += rb
        return res, {
            "h2d_ns": tm.h2d_ns, "kernel_ns": tm.kernel_ns, "d2h_ns": tm.d2h_ns, "total_ns": tm.total_ns}

    def eval_points(self, key, indices) -> np.ndarray:
        """ChaChaKey::eval (dpf.rs:103-142) at each index, on the device."""
        kb = bytes(key)
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        out = np.empty(idx.size * 16, np.uint8)
        N.check(N.lib().mg_eval_points(self._ctx.handle, N.u8ptr(kb), len(kb),
                                       idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size,
                                       out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.reshape(-1, 16)

    def close(self):
        """Release the workspace pool.  The context itself is released when the
        last table or workspace referring to this scanner is gone."""
        for w in self._pool:
            if w is not None:
                w.close()
        self._pool = []
