"""mg_scan_noalloc: the scan entry point for callers that cannot call
cudaMalloc (their device memory belongs to a host application or pool, or an
allocation would stall a latency-bound serving loop).  It must give exactly
the oracle's shares -- and so mg_scan's -- for the same table and keys, call
after call, while the keys and partial rows live in the library's fixed
device array.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle_keypair

from morphogen_b200 import _native as N
from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu


def scan_noalloc(table: G.GpuPageMatrix, keys, out: G.GpuPageMatrix, rows: int | None = None,
                 stream=None) -> list[bytes]:
    """Call the entry point through the C ABI.  The output buffer is device
    memory the caller owns (here a table of at least len(keys) rows)."""
    ka = N.KeyArray([bytes(k) for k in keys])
    n = table.num_rows() if rows is None else rows
    st = C.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = N.lib().mg_scan_noalloc(0, C.c_void_p(table.device_ptr()), n, table.row_bytes,
                                 ka.ptrs, ka.lens, ka.n, C.c_void_p(out.device_ptr()), st)
    N.check(rc)
    if stream is not None:
        stream.synchronize()
    # The legacy default stream orders this synchronous copy after the scan.
    raw = out.read_rows(0, ka.n).tobytes()
    rb = table.row_bytes
    return [raw[i * rb:(i + 1) * rb] for i in range(ka.n)]


def host_table(scanner, oracle_mod, nrows, row_bytes, seed):
    host = oracle_mod.fill_splitmix(0, nrows * row_bytes, seed)
    return G.GpuPageMatrix.new(scanner, host, row_bytes), host.reshape(nrows, row_bytes)


def test_noalloc_matches_oracle_two_calls_in_a_row(scanner, oracle_mod):
    t32, rows32 = host_table(scanner, oracle_mod, 1 << 18, 32, seed=31)
    t256, rows256 = host_table(scanner, oracle_mod, 50_000, 256, seed=32)
    out = G.GpuPageMatrix(scanner, 8, 256)
    out32 = G.GpuPageMatrix(scanner, 8, 32)

    # Call 1: one query (3 keys, 18-bit) over 2^18 rows of 32 B.
    keys1 = [oracle_keypair(oracle_mod, 18, t, seed=33, i=j)[0] for j, t in enumerate((5, 99_999, 262_143))]
    want1 = oracle_mod.scan_fused(keys1, rows32, 32)
    got1 = scan_noalloc(t32, keys1, out32)
    assert got1 == want1
    assert got1 == scanner.scan_keys(t32, keys1)[0]

    # Call 2, right after: another table, row size and key count; the shared
    # array still holds call 1's keys and partial rows.
    keys2 = [oracle_keypair(oracle_mod, 20, (j * 7717) % 50_000, seed=34, i=j)[0] for j in range(5)]
    got2 = scan_noalloc(t256, keys2, out)
    assert got2 == oracle_mod.scan_fused(keys2, rows256, 256)
    assert got2 == scanner.scan_keys(t256, keys2)[0]

    # And call 1 again: nothing from call 2 leaks into it.
    assert scan_noalloc(t32, keys1, out32) == want1


@pytest.mark.parametrize("d,nrows", [(1, 2), (1, 1), (5, 32), (5, 19)])
def test_noalloc_small_domains(scanner, oracle_mod, d, nrows):
    # d < 8: the tile is the whole domain and fewer than 8 breadth-first levels.
    t, rows = host_table(scanner, oracle_mod, nrows, 64, seed=40 + d)
    out = G.GpuPageMatrix(scanner, 4, 64)
    keys = [oracle_keypair(oracle_mod, d, (3 * j) % nrows, seed=41, i=j)[0] for j in range(4)]
    assert scan_noalloc(t, keys, out) == oracle_mod.scan_fused(keys, rows, 64)


def test_noalloc_empty_table_gives_zero_shares(scanner, oracle_mod):
    t, _ = host_table(scanner, oracle_mod, 16, 48, seed=43)
    out = G.GpuPageMatrix(scanner, 3, 48)
    out.update_pages(0, np.full(3 * 48, 0xA5, np.uint8))  # stale bytes the call must overwrite
    keys = [oracle_keypair(oracle_mod, 9, j, seed=44, i=j)[0] for j in range(3)]
    assert scan_noalloc(t, keys, out, rows=0) == [bytes(48)] * 3


def test_noalloc_on_a_created_stream(scanner, oracle_mod):
    import torch
    t, rows = host_table(scanner, oracle_mod, 40_000, 128, seed=45)
    out = G.GpuPageMatrix(scanner, 3, 128)
    keys = [oracle_keypair(oracle_mod, 16, (11 * j + 5) % 40_000, seed=46, i=j)[0] for j in range(3)]
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    assert scan_noalloc(t, keys, out, stream=stream) == oracle_mod.scan_fused(keys, rows, 128)


def test_noalloc_and_mg_scan_share_the_kernels_smem_limit(scanner, oracle_mod):
    # Both entry points launch the one-key CTA kernel.  A 14-level tile needs
    # 34,928 B of shared memory, a 10-level tile 17,520 B; whichever runs
    # second must not lower the limit under the other's larger shape.
    big, rows_big = host_table(scanner, oracle_mod, 20_000, 1024, seed=47)
    keys_big = [oracle_keypair(oracle_mod, 16, 12_345, seed=48)[0]]
    want_big = oracle_mod.scan_fused(keys_big, rows_big, 1024)
    small, rows_small = host_table(scanner, oracle_mod, 1000, 1024, seed=49)
    keys_small = [oracle_keypair(oracle_mod, 10, 999, seed=50)[0]]
    want_small = oracle_mod.scan_fused(keys_small, rows_small, 1024)
    out = G.GpuPageMatrix(scanner, 1, 1024)

    # Order 1: the workspace path with the large pinned shape, then the
    # allocation-free path with a 10-bit key, then the workspace again.
    ws = scanner.workspace()
    ws.set_kernel("cta")
    ws.set_shape(14, 1)
    ws.set_keys([big], keys_big)
    ws.launch()
    assert ws.read() == want_big
    assert scan_noalloc(small, keys_small, out) == want_small
    ws.launch()
    assert ws.read() == want_big

    # Order 2: the allocation-free path (its planner tries the 14-level tile
    # for a 16-bit key first), then a fresh context's workspace with the
    # small pinned shape, then the first workspace's large shape and the
    # allocation-free path again.
    assert scan_noalloc(big, keys_big, out) == want_big
    other = G.GpuScanner(0)
    small2, _ = host_table(other, oracle_mod, 1000, 1024, seed=49)
    ws2 = other.workspace()
    ws2.set_kernel("cta")
    ws2.set_shape(10, 1)
    ws2.set_keys([small2], keys_small)
    ws2.launch()
    assert ws2.read() == want_small
    ws.launch()
    assert ws.read() == want_big
    assert scan_noalloc(big, keys_big, out) == want_big
    assert scan_noalloc(small, keys_small, out) == want_small
    for o in (ws2, small2, ws):
        o.close()
    other.close()


def test_noalloc_rejects_requests_beyond_its_array(scanner, oracle_mod):
    t = G.GpuPageMatrix.from_seed(scanner, 1 << 12, 4096, seed=35)
    out = G.GpuPageMatrix(scanner, 64, 4096)
    k = oracle_keypair(oracle_mod, 12, 7, seed=36)[0]
    with pytest.raises(N.MgError) as e:
        scan_noalloc(t, [k] * 32, out)  # 32 keys x 4 KB rows: partial rows exceed the array
    assert e.value.code == N.MG_ERANGE and "MG_NOALLOC_SCRATCH_BYTES" in e.value.message
    with pytest.raises(N.MgError) as e:
        scan_noalloc(t, [k] * 65, out)
    assert e.value.code == N.MG_ERANGE and "MG_NOALLOC_MAX_KEYS" in e.value.message
    # A request inside the limits still works after the rejections.
    want, _ = scanner.scan_keys(t, [k, k])
    assert scan_noalloc(t, [k, k], out) == want
