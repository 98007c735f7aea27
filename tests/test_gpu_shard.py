"""Row-range tables (one table sharded over GPUs): a table holding rows
[first_row, first_row + n) of a larger logical table answers keys at the
logical row indices; the range shares XOR to the whole table's share
(bit-exact), on both kernel families, with pending deltas and after merges.
Two ranges on one GPU stand in for two GPUs: the shards do not exchange
anything until the host XOR."""
import numpy as np
import pytest

from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import gpu_dpf as G
from morphogen_b200.shard import shard_range, xor_shares

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["auto", "cta", "warp"])
@pytest.mark.parametrize("rb,nrows,d,world,align", [
    (32, 1 << 18, 18, 2, 1 << 16),       # power-of-two halves
    (32, 300_001, 20, 3, 4096),          # ragged end, domain larger than the table
    (64, 100_000, 17, 2, 1),             # split at an odd row
    (32, 100_003, 17, 3, 1),             # 32-B rows (own-rows path), odd splits
    (16, 50_001, 31, 2, 1),              # 16-B rows, 31-bit keys
    (4096, 600, 10, 4, 7),               # page rows, odd boundaries
])
def test_ranges_xor_to_whole_table(scanner, oracle_mod, kernel, rb, nrows, d, world, align):
    if kernel == "warp" and rb > 512:
        pytest.skip("the warp kernel takes rows of 16..512 B")
    whole_host = oracle_mod.fill_splitmix(0, nrows * rb, 40 + rb).reshape(nrows, rb)
    targets = [0, nrows // 2, nrows - 1]
    keys = [oracle_keypair(oracle_mod, d, t, seed=41, i=j)[0] for j, t in enumerate(targets)]
    want = oracle_mod.scan_fused(keys, whole_host, rb)
    parts = []
    for r in range(world):
        first, n = shard_range(nrows, world, r, align)
        t = G.GpuPageMatrix.from_seed(scanner, n, rb, 40 + rb, first_row=first)
        assert t.first_row == first
        assert (t.read_rows(0, n).reshape(n, rb) == whole_host[first:first + n]).all()
        ws = scanner.workspace()
        ws.set_kernel(kernel)
        ws.set_keys([t] * len(keys), keys)
        ws.launch()
        got = ws.read()
        ws.close()
        assert got == oracle_mod.scan_fused(keys, whole_host[first:first + n], rb, row_base=first)
        parts.append(got)
        t.close()
    assert xor_shares(parts) == want


def test_range_delta_and_merge(scanner, oracle_mod):
    rb, nrows, d = 32, 1 << 16, 16
    whole = oracle_mod.fill_splitmix(0, nrows * rb, 77).reshape(nrows, rb).copy()
    first, n = 20_000, 30_000
    t = G.GpuPageMatrix.range(scanner, first, n, rb)
    t.update_pages(0, whole[first:first + n])
    t.delta_reserve(64)
    local_idx = np.array([0, 5, n - 1, 5], np.uint64)  # indices within the range
    diffs = oracle_mod.fill_splitmix(3, local_idx.size * rb, 78).reshape(-1, rb)
    t.delta_push(local_idx, diffs)
    patched = whole.copy()
    for i, r in enumerate(local_idx):
        patched[first + int(r)] ^= diffs[i]
    pairs = [oracle_keypair(oracle_mod, d, first + x, seed=79, i=j) for j, x in enumerate((0, 5, n - 1))]
    k0 = [p[0] for p in pairs]
    got, _ = scanner.scan_keys(t, k0)
    assert got == oracle_mod.scan_fused(k0, patched[first:first + n], rb, row_base=first)
    t.delta_merge()
    after, _ = scanner.scan_keys(t, k0)
    assert after == got and t.delta_count() == 0
    # With the other server's shares, the updated logical rows come back.
    got1, _ = scanner.scan_keys(t, [p[1] for p in pairs])
    for j, x in enumerate((0, 5, n - 1)):
        assert xor_bytes(after[j], got1[j]) == patched[first + x].tobytes()
    t.close()


def test_range_limits(scanner, oracle_mod):
    with pytest.raises(G.GpuDpfError):
        G.GpuPageMatrix.range(scanner, (1 << 32) - 10, 11, 32)  # past the largest domain
    t = G.GpuPageMatrix.range(scanner, 1000, 100, 32)
    k_small = oracle_keypair(oracle_mod, 10, 3, seed=1)[0]  # domain 1024 < 1100
    with pytest.raises(G.GpuDpfError):
        scanner.scan_keys(t, [k_small])
    k_ok = oracle_keypair(oracle_mod, 11, 1050, seed=2)[0]
    got, _ = scanner.scan_keys(t, [k_ok])
    assert len(got[0]) == 32
    t.close()


def test_device_combiner_single_rank(scanner, oracle_mod):
    from morphogen_b200.shard import ShardCombiner
    rb, nrows, d = 64, 50_000, 16
    t = G.GpuPageMatrix.from_seed(scanner, nrows, rb, 5)
    keys = [oracle_keypair(oracle_mod, d, 7 * j, seed=3, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_keys([t] * 3, keys)
    ws.launch()
    comb = ShardCombiner(scanner.device_ord if hasattr(scanner, "device_ord") else 0)
    out = comb.combine(ws)
    assert out.cpu().numpy().tobytes() == b"".join(ws.read())
    ws.close()
    t.close()


def test_in_process_sharded_table(scanner, oracle_mod):
    """Three ranges scanned concurrently from host threads (here all on one
    GPU; one per GPU in production) XOR to the whole table's shares, and the
    two servers' combined shares give the target rows."""
    from morphogen_b200.shard import ShardedTable
    rows, rb, d = 300_001, 32, 19
    whole = oracle_mod.fill_splitmix(0, rows * rb, 51).reshape(rows, rb)
    st = ShardedTable([scanner] * 3, rows, rb, align=4096)
    st.write_rows(0, whole)
    for t, (f, n) in zip(st.tables, st.spans):
        assert (t.read_rows(0, n).reshape(n, rb) == whole[f:f + n]).all()
    targets = [5, 150_000, rows - 1]
    pairs = [oracle_keypair(oracle_mod, d, t, seed=52, i=j) for j, t in enumerate(targets)]
    a = st.scan([p[0] for p in pairs])
    b = st.scan([p[1] for p in pairs])
    assert a == oracle_mod.scan_fused([p[0] for p in pairs], whole, rb)
    for j, t in enumerate(targets):
        assert xor_bytes(a[j], b[j]) == whole[t].tobytes()
    st.close()


def test_sharded_serving_loop(scanner, oracle_mod):
    """Requests folded into passes on every range's serving loop (two ranges
    on one GPU here) answer exactly what one whole-table scan answers."""
    from morphogen_b200.server import ShardedPirServer
    from morphogen_b200.shard import ShardedTable
    rows, rb, d = 200_003, 32, 18
    whole = oracle_mod.fill_splitmix(0, rows * rb, 61).reshape(rows, rb)
    st = ShardedTable([scanner] * 2, rows, rb, align=1024)
    st.write_rows(0, whole)
    srv = ShardedPirServer(st, slots=2)
    reqs = [[oracle_keypair(oracle_mod, d, (7919 * (3 * r + j)) % rows, seed=62, i=3 * r + j)[0] for j in range(3)]
            for r in range(6)]
    for s_ in srv.servers:
        s_.pause()
    ids = [srv.submit(keys) for keys in reqs]
    for s_ in srv.servers:
        s_.resume()
    for rid, keys in zip(ids, reqs):
        shares, lat = srv.wait(rid)
        assert shares == oracle_mod.scan_fused(keys, whole, rb) and lat > 0
    srv.close()
    st.close()
