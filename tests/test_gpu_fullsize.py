"""The mainnet-scale configuration at full size: 2^31 rows x 32 B (64 GiB,
SplitMix64 bytes from seed 0), 3 key pairs over the 31-bit domain.  The
oracle cannot scan 64 GiB in a test, so parity at this size goes through
size-independent properties (tolerance: bit-exact):
  * the two servers' shares XOR to the target rows (regenerated on the host);
  * a pending delta changes each share by exactly the oracle's delta term
    (linearity of the scan, scan.rs:434-485);
  * the keys' shares over a 2^20-row window deep in the domain equal the
    oracle's scan of the same window at the same logical rows;
  * with a 2^28 x 64 B accounts table resident beside it, one pass over both
    tables reconstructs every target row of both;
  * a batched pass of 16 queries (48 keys) reconstructs every target row."""
import numpy as np
import pytest

from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu

ROWS, RB, D = 1 << 31, 32, 31


@pytest.fixture(scope="module")
def big(scanner):
    free = scanner.device_info()["free_bytes"]
    if free < ROWS * RB + (8 << 30):
        pytest.skip(f"needs {ROWS * RB >> 30} GiB of free device memory")
    t = G.GpuPageMatrix.from_seed(scanner, ROWS, RB, seed=0)
    yield t
    t.close()


def test_full_size_shares_reconstruct_targets(scanner, oracle_mod, big):
    targets = [int(x) for x in np.random.default_rng(0).integers(0, ROWS, 3)]
    targets[0] = ROWS - 1  # the last row of the domain
    pairs = [oracle_keypair(oracle_mod, D, t, seed=31, i=j) for j, t in enumerate(targets)]
    a, _ = scanner.scan_keys(big, [p[0] for p in pairs])
    b, _ = scanner.scan_keys(big, [p[1] for p in pairs])
    for j, t in enumerate(targets):
        assert xor_bytes(a[j], b[j]) == oracle_mod.fill_splitmix(t * RB, RB, 0).tobytes()


def test_full_size_delta_is_linear(scanner, oracle_mod, big):
    pairs = [oracle_keypair(oracle_mod, D, 12345 + j, seed=32, i=j) for j in range(3)]
    k0 = [p[0] for p in pairs]
    before, _ = scanner.scan_keys(big, k0)
    idx = np.array([0, 12346, ROWS - 1], np.uint64)
    diffs = oracle_mod.fill_splitmix(77, 3 * RB, 33).reshape(3, RB)
    big.delta_reserve(8)
    big.delta_push(idx, diffs)
    try:
        after, _ = scanner.scan_keys(big, k0)
        delta = oracle_mod.delta_apply(k0, idx, diffs, RB)
        assert [xor_bytes(x, y) for x, y in zip(before, after)] == delta
    finally:
        big.delta_clear()


def test_deep_window_matches_oracle(scanner, oracle_mod):
    first, n = (1 << 30) + (1 << 22), 1 << 20
    win = G.GpuPageMatrix.from_seed(scanner, n, RB, seed=0, first_row=first)
    keys = [oracle_keypair(oracle_mod, D, first + 1000 * j, seed=34, i=j)[0] for j in range(3)]
    got, _ = scanner.scan_keys(win, keys)
    host = oracle_mod.fill_splitmix(first * RB, n * RB, 0)
    assert got == oracle_mod.scan_fused(keys, host, RB, row_base=first)
    win.close()


def test_full_size_mixed_tables_one_pass_reconstruct(scanner, oracle_mod, big):
    """Two resident tables in one pass at full size: an accounts table of
    2^28 rows x 64 B (16 GiB, 28-bit keys) beside the 2^31 x 32 B storage
    table (31-bit keys).  Both servers' passes hold 2 accounts queries and 1
    storage query; every share pair XORs to its target row."""
    arows, arb, ad = 1 << 28, 64, 28
    free = scanner.device_info()["free_bytes"]
    if free < arows * arb + (4 << 30):
        pytest.skip(f"needs {arows * arb >> 30} GiB more free device memory")
    acc = G.GpuPageMatrix.from_seed(scanner, arows, arb, seed=1)
    try:
        at = [int(x) for x in np.random.default_rng(5).integers(0, arows, 6)]
        at[0] = arows - 1
        st = [int(x) for x in np.random.default_rng(6).integers(0, ROWS, 3)]
        pairs = [oracle_keypair(oracle_mod, ad, t, seed=35, i=j) for j, t in enumerate(at)]
        pairs += [oracle_keypair(oracle_mod, D, t, seed=36, i=j) for j, t in enumerate(st)]
        tables = [acc] * 6 + [big] * 3
        shares = []
        for side in (0, 1):
            ws = scanner.workspace()
            ws.set_keys(tables, [p[side] for p in pairs])
            ws.launch()
            shares.append(ws.read())
            assert ws.plan()["segments"] == 2
            ws.close()
        for j, t in enumerate(at):
            want = oracle_mod.fill_splitmix(t * arb, arb, 1).tobytes()
            assert xor_bytes(shares[0][j], shares[1][j]) == want
        for j, t in enumerate(st):
            want = oracle_mod.fill_splitmix(t * RB, RB, 0).tobytes()
            assert xor_bytes(shares[0][6 + j], shares[1][6 + j]) == want
    finally:
        acc.close()


def test_full_size_batched_pass_reconstructs(scanner, oracle_mod, big):
    """16 queries (48 keys, one key group each) in one pass over the
    2^31 x 32 B table, replayed from a CUDA graph: every share pair XORs to
    its target row."""
    targets = [int(x) for x in np.random.default_rng(7).integers(0, ROWS, 48)]
    pairs = [oracle_keypair(oracle_mod, D, t, seed=37, i=j) for j, t in enumerate(targets)]
    shares = []
    for side in (0, 1):
        ws = scanner.workspace()
        ws.set_keys([big] * 48, [p[side] for p in pairs])
        ws.launch(graph=True)
        shares.append(ws.read())
        ws.close()
    for j, t in enumerate(targets):
        assert xor_bytes(shares[0][j], shares[1][j]) == oracle_mod.fill_splitmix(t * RB, RB, 0).tobytes()
