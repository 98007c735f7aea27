"""The one-call scan (mg_scan; the reference's GpuScanner::scan,
kernel.rs:685-760) called again with the same tables and key depths replays
one CUDA graph that holds the key upload, the pass and the share download.
Every call here brings new keys, changed rows or another workload, and every
share is compared with the oracle, so a replay that kept the previous call's
keys, shares or plan would be caught."""
import numpy as np
import pytest

from conftest import oracle_keypair

from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu


def host_table(scanner, oracle_mod, nrows, row_bytes, seed):
    host = oracle_mod.fill_splitmix(0, nrows * row_bytes, seed)
    return G.GpuPageMatrix.new(scanner, host, row_bytes), host.reshape(nrows, row_bytes).copy()


def test_repeated_calls_follow_each_calls_keys(scanner, oracle_mod):
    n = 1 << 14
    db, rows = host_table(scanner, oracle_mod, n, 256, seed=61)
    for r in range(6):
        keys = [oracle_keypair(oracle_mod, 14, (r * 977 + j * 31) % n, seed=62 + r, i=j)[0] for j in range(3)]
        got, tm = scanner.scan_keys(db, keys)
        assert got == oracle_mod.scan_fused(keys, rows, 256)
        assert tm["kernel_ns"] > 0 and tm["total_ns"] >= tm["kernel_ns"]
    db.close()


def test_replay_sees_row_updates_and_survives_other_workloads(scanner, oracle_mod):
    db, rows = host_table(scanner, oracle_mod, 4096, 32, seed=70)
    other, rows_o = host_table(scanner, oracle_mod, 3000, 64, seed=71)
    ka = [oracle_keypair(oracle_mod, 12, 7 + 5 * j, seed=72, i=j)[0] for j in range(3)]
    want = oracle_mod.scan_fused(ka, rows, 32)
    assert scanner.scan_keys(db, ka)[0] == want  # planned
    assert scanner.scan_keys(db, ka)[0] == want  # replayed

    # Rows change between replays: the graph reads the table, not a copy.
    idx = np.array([7, 12, 4095, 7], np.uint64)
    diffs = oracle_mod.fill_splitmix(0, idx.size * 32, 73).reshape(-1, 32)
    db.xor_rows(idx, diffs)
    for i, r in enumerate(idx):
        rows[r] ^= diffs[i]
    assert scanner.scan_keys(db, ka)[0] == oracle_mod.scan_fused(ka, rows, 32)

    # Another table and row size, then four keys instead of three: new plans.
    kb = [oracle_keypair(oracle_mod, 12, 2999 - j, seed=74, i=j)[0] for j in range(3)]
    for _ in range(2):
        assert scanner.scan_keys(other, kb)[0] == oracle_mod.scan_fused(kb, rows_o, 64)
    kc = ka + [oracle_keypair(oracle_mod, 12, 4000, seed=75)[0]]
    for _ in range(2):
        assert scanner.scan_keys(db, kc)[0] == oracle_mod.scan_fused(kc, rows, 32)

    # Back to the first workload: planned again, then replayed.
    for _ in range(2):
        assert scanner.scan_keys(db, ka)[0] == oracle_mod.scan_fused(ka, rows, 32)
    db.close()
    other.close()
