"""mg_scan_noalloc: the scan entry point for callers that cannot call
cudaMalloc (their device memory belongs to a host application or pool, or an
allocation would stall a latency-bound serving loop).  It must give exactly
the shares mg_scan gives for the same table and keys, call after call, while
the keys and partial rows live in the library's fixed device array.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle_keypair

from morphogen_b200 import _native as N
from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu


def scan_noalloc(table: G.GpuPageMatrix, keys, out: G.GpuPageMatrix) -> list[bytes]:
    """Call the entry point through the C ABI.  The output buffer is device
    memory the caller owns (here a table of len(keys) rows)."""
    ka = N.KeyArray([bytes(k) for k in keys])
    rc = N.lib().mg_scan_noalloc(0, C.c_void_p(table.device_ptr()), table.num_rows(), table.row_bytes,
                                 ka.ptrs, ka.lens, ka.n, C.c_void_p(out.device_ptr()), None)
    N.check(rc)
    # The legacy default stream orders this synchronous copy after the scan.
    raw = out.read_rows(0, ka.n).tobytes()
    rb = table.row_bytes
    return [raw[i * rb:(i + 1) * rb] for i in range(ka.n)]


def test_noalloc_matches_mg_scan_two_calls_in_a_row(scanner, oracle_mod):
    t32 = G.GpuPageMatrix.from_seed(scanner, 1 << 18, 32, seed=31)
    t256 = G.GpuPageMatrix.from_seed(scanner, 50_000, 256, seed=32)
    out = G.GpuPageMatrix(scanner, 8, 256)

    # Call 1: one query (3 keys, 18-bit) over 2^18 rows of 32 B.
    keys1 = [oracle_keypair(oracle_mod, 18, t, seed=33, i=j)[0] for j, t in enumerate((5, 99_999, 262_143))]
    want1, _ = scanner.scan_keys(t32, keys1)
    out32 = G.GpuPageMatrix(scanner, 8, 32)
    got1 = scan_noalloc(t32, keys1, out32)
    assert got1 == want1

    # Call 2, right after: another table, row size and key count; the shared
    # array still holds call 1's keys and partial rows.
    keys2 = [oracle_keypair(oracle_mod, 20, (j * 7717) % 50_000, seed=34, i=j)[0] for j in range(5)]
    want2, _ = scanner.scan_keys(t256, keys2)
    got2 = scan_noalloc(t256, keys2, out)
    assert got2 == want2

    # And call 1 again: nothing from call 2 leaks into it.
    assert scan_noalloc(t32, keys1, out32) == want1


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
