"""GPU parity: shares from the sm_100a library, through the C ABI, equal the
oracle's shares byte for byte, and the XOR of the two servers' shares equals
the target row.  Restates the reference's GPU tests
(crates/morphogen-gpu-dpf/src/kernel.rs:1563-1677) and widens them to row
mode, deep domains, every launch shape and mixed tables."""
import numpy as np
import pytest

from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import gpu_dpf as G
from morphogen_b200 import _native as N

pytestmark = pytest.mark.gpu


def make_table(scanner, oracle_mod, nrows, row_bytes, seed=0, pattern="splitmix"):
    if pattern == "pages":
        host = oracle_mod.fill_test_rows(nrows, row_bytes)
    else:
        host = oracle_mod.fill_splitmix(0, nrows * row_bytes, seed)
    t = G.GpuPageMatrix.new(scanner, host, row_bytes)
    return t, host.reshape(nrows, row_bytes)


def test_gpu_fused_3dpf_recovers_all_targets(scanner, oracle_mod):
    # kernel.rs:1563-1610: 256 pages of 4 KB, 8-bit keys.
    db, pages = make_table(scanner, oracle_mod, 256, 4096, pattern="pages")
    targets = [10, 100, 200]
    pairs = [oracle_keypair(oracle_mod, 8, t, seed=1, i=j) for j, t in enumerate(targets)]
    r0 = scanner.scan(db, [G.ChaChaKey(p[0]) for p in pairs])
    r1 = scanner.scan(db, [G.ChaChaKey(p[1]) for p in pairs])
    want0 = oracle_mod.scan_fused([p[0] for p in pairs], pages, 4096)
    for j, t in enumerate(targets):
        assert r0.pages[j] == want0[j]
        assert xor_bytes(r0.pages[j], r1.pages[j]) == pages[t].tobytes()
    assert r0.verif0 == bytes(16)


def test_gpu_tiled_batch_matches_default_optimized_outputs(scanner, oracle_mod):
    # kernel.rs:1612-1677
    db, pages = make_table(scanner, oracle_mod, 256, 4096, pattern="pages")
    queries = []
    for i in range(32):
        ts = (i % 256, (i * 7 + 13) % 256, (i * 11 + 29) % 256)
        queries.append([G.ChaChaKey(oracle_keypair(oracle_mod, 8, t, seed=2, i=3 * i + j)[0])
                        for j, t in enumerate(ts)])
    for q in (1, 2, 4, 8, 16, 32):
        base = scanner.scan_batch_optimized(db, queries[:q])
        tiled = scanner.scan_batch_optimized_tiled(db, queries[:q], 4)
        assert len(base) == len(tiled) == q
        for a, b in zip(base, tiled):
            assert a.pages == b.pages and a.verif0 == b.verif0
    want = oracle_mod.scan_fused([k.to_bytes() for q in queries for k in q], pages, 4096)
    got = [p for r in base for p in r.pages]
    assert got == want


SWEEP = [
    # (row_bytes, domain_bits, rows)
    (16, 1, 2), (16, 1, 1), (32, 2, 3), (32, 5, 32), (32, 9, 300), (32, 12, 4096),
    (48, 10, 1000), (64, 13, 8000), (80, 11, 2048), (256, 14, 16384), (32, 16, 65536),
    (32, 18, 200001), (512, 9, 512), (4096, 10, 700), (1024, 12, 4000), (2048, 8, 256),
    (32, 24, 1 << 20),
    # the largest domain over small tables (frontier chain past level 31), and
    # 16-B rows with 31-bit keys
    (32, 32, 70_001), (16, 32, 3), (16, 31, 100_000), (64, 28, 3000),
]


@pytest.mark.parametrize("row_bytes,d,nrows", SWEEP)
def test_shares_match_oracle(scanner, oracle_mod, row_bytes, d, nrows):
    db, rows = make_table(scanner, oracle_mod, nrows, row_bytes, seed=row_bytes * 131 + d)
    rng = np.random.default_rng(d * 1000 + row_bytes)
    targets = [int(x) for x in rng.integers(0, nrows, 3)]
    pairs = [oracle_keypair(oracle_mod, d, t, seed=d, i=j) for j, t in enumerate(targets)]
    k0 = [p[0] for p in pairs]
    got0, _ = scanner.scan_keys(db, k0)
    got1, _ = scanner.scan_keys(db, [p[1] for p in pairs])
    assert got0 == oracle_mod.scan_fused(k0, rows, row_bytes)
    for j, t in enumerate(targets):
        assert xor_bytes(got0[j], got1[j]) == rows[t].tobytes()


@pytest.mark.parametrize("subtree_bits", [1, 3, 8, 9, 10, 12, 14, 16])
@pytest.mark.parametrize("keys_per_cta", [1, 2, 3, 4, 8])
def test_every_cta_kernel_shape_is_bit_exact(scanner, oracle_mod, subtree_bits, keys_per_cta):
    row_bytes, d, nrows = 32, 17, 100_003
    db, rows = make_table(scanner, oracle_mod, nrows, row_bytes, seed=5)
    keys = [oracle_keypair(oracle_mod, d, (7919 * j) % nrows, seed=6, i=j)[0] for j in range(7)]
    ws = scanner.workspace()
    ws.set_kernel("cta")
    ws.set_shape(subtree_bits, keys_per_cta)
    g = min(keys_per_cta, 7)
    g = g if g in (1, 2, 3, 4, 8) else 4
    S = min(subtree_bits, d)
    M = S - min(8, S - 1)
    if g * (624 + 2 * 256 * 16 + max(M, 2) * 256 * 17) > 232448:  # 227 KB per CTA
        with pytest.raises(N.MgError) as e:
            ws.set_keys([db] * len(keys), keys)
        assert e.value.code == N.MG_EINVAL
        ws.close()
        return
    ws.set_keys([db] * len(keys), keys)
    ws.launch()
    got = ws.read()
    assert got == oracle_mod.scan_fused(keys, rows, row_bytes)
    plan = ws.plan()
    assert plan["kernel"] == N.KERNEL_CTA and plan["keys_per_cta"] == g
    ws.close()


@pytest.mark.parametrize("warp_tile_bits", [6, 7, 9, 12, 15])
@pytest.mark.parametrize("keys_per_item", [1, 2, 3, 4])
@pytest.mark.parametrize("row_bytes", [16, 32, 64, 128, 256, 512])
def test_every_warp_kernel_shape_is_bit_exact(scanner, oracle_mod, warp_tile_bits, keys_per_item, row_bytes):
    d, nrows = 17, 70_001
    db, rows = make_table(scanner, oracle_mod, nrows, row_bytes, seed=7)
    keys = [oracle_keypair(oracle_mod, d, (104729 * j) % nrows, seed=8, i=j)[0] for j in range(7)]
    ws = scanner.workspace()
    ws.set_kernel("warp")
    ws.set_shape(warp_tile_bits, keys_per_item)
    ws.set_keys([db] * len(keys), keys)
    ws.launch()
    got = ws.read()
    assert got == oracle_mod.scan_fused(keys, rows, row_bytes)
    plan = ws.plan()
    assert plan["kernel"] == N.KERNEL_WARP and plan["subtree_bits"] == warp_tile_bits
    assert plan["keys_per_cta"] == keys_per_item
    ws.close()


@pytest.mark.parametrize("rb", [32, 64])
@pytest.mark.parametrize("d,M", [(16, 5), (20, 10), (21, 10), (22, 1), (30, 10), (31, 10), (32, 2), (32, 1)])
def test_frontier_chain_depths_are_bit_exact(scanner, oracle_mod, d, M, rb):
    # F = d - M frontier levels: one step from the roots up to 10 levels,
    # else steps of 10 levels whose first reaches its roots by a path walk
    # of F - 10 * steps levels (1..10).  The table is a row range that does
    # not start on a tile boundary, so every step keeps only the nodes that
    # meet the rows.  32-B rows use reduce_kernel, 64-B rows reduce in-kernel
    # with the shares zeroed by the first frontier step.
    n = 40_000
    first = ((1 << d) - n) // 3 + 3
    db = G.GpuPageMatrix.from_seed(scanner, n, rb, seed=81, first_row=first)
    host = oracle_mod.fill_splitmix(first * rb, n * rb, 81).reshape(n, rb)
    keys = [oracle_keypair(oracle_mod, d, first + (12_347 * j) % n, seed=82, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_kernel("warp")
    ws.set_shape(M + 5, 1)
    ws.set_keys([db] * 3, keys)
    ws.launch()
    assert ws.read() == oracle_mod.scan_fused(keys, host, rb, row_base=first)
    F = d - M
    steps = 1 if F <= 10 else (F - 1) // 10
    plan = ws.plan()
    assert plan["subtree_bits"] == M + 5
    assert plan["kernels"] == steps + (1 if rb > 32 else 2)
    ws.launch(graph=True)
    assert ws.read() == oracle_mod.scan_fused(keys, host, rb, row_base=first)
    ws.close()
    db.close()


def test_domain_zero_key(scanner, oracle_mod):
    # from_bytes accepts d = 0 (a one-leaf domain, dpf.rs:277-316).
    k0, _ = oracle_keypair(oracle_mod, 4, 3)
    k = bytearray(k0[:19] + k0[-16:])
    k[18] = 0
    k[16] = 1  # root_t == 1 applies final_cw
    db, rows = make_table(scanner, oracle_mod, 1, 64, seed=3)
    got, _ = scanner.scan_keys(db, [bytes(k)])
    assert got == oracle_mod.scan_fused([bytes(k)], rows, 64)


def test_nonbinary_t_bytes(scanner, oracle_mod):
    k0, _ = oracle_keypair(oracle_mod, 14, 77, seed=8)
    b = bytearray(k0)
    b[16] = 1
    for lvl in range(0, 14, 3):
        b[19 + 18 * lvl + 16] = 3
        b[19 + 18 * lvl + 17] = 0x81
    db, rows = make_table(scanner, oracle_mod, 1 << 14, 32, seed=4)
    got, _ = scanner.scan_keys(db, [bytes(b), k0])
    assert got == oracle_mod.scan_fused([bytes(b), k0], rows, 32)


def test_mixed_tables_one_pass(scanner, oracle_mod):
    # Two resident tables of different row sizes and domains in one launch.
    acc, acc_rows = make_table(scanner, oracle_mod, 30_000, 64, seed=10)
    sto, sto_rows = make_table(scanner, oracle_mod, 70_000, 32, seed=11)
    items, want_keys = [], {"a": [], "s": []}
    for j in range(5):
        ka = oracle_keypair(oracle_mod, 15, (j * 977) % 30_000, seed=12, i=j)[0]
        ks = oracle_keypair(oracle_mod, 17, (j * 1231) % 70_000, seed=13, i=j)[0]
        items += [(acc, ka), (sto, ks)]
        want_keys["a"].append(ka)
        want_keys["s"].append(ks)
    got = scanner.scan_multi(items)
    wa = oracle_mod.scan_fused(want_keys["a"], acc_rows, 64)
    wsx = oracle_mod.scan_fused(want_keys["s"], sto_rows, 32)
    assert got[0::2] == wa and got[1::2] == wsx


def test_keys_of_different_domains_on_one_table(scanner, oracle_mod):
    db, rows = make_table(scanner, oracle_mod, 5000, 32, seed=14)
    keys = [oracle_keypair(oracle_mod, d, 4999, seed=15, i=d)[0] for d in (13, 14, 20, 13, 31, 32)]
    got, _ = scanner.scan_keys(db, keys)
    assert got == oracle_mod.scan_fused(keys, rows, 32)


def test_rejects_more_rows_than_domain(scanner, oracle_mod):
    db, _ = make_table(scanner, oracle_mod, 300, 32)
    k = oracle_keypair(oracle_mod, 8, 3)[0]
    with pytest.raises(G.GpuDpfError) as e:
        scanner.scan_keys(db, [k])
    assert e.value.code == N.MG_ERANGE


def test_eval_points_match_oracle(scanner, oracle_mod):
    for d in (1, 8, 25, 31, 32):
        k = oracle_keypair(oracle_mod, d, (1 << d) - 1, seed=16, i=d)[0]
        idx = np.random.default_rng(d).integers(0, 1 << d, 200, dtype=np.uint64)
        idx[:2] = [0, (1 << d) - 1]
        got = scanner.eval_points(G.ChaChaKey(k), idx)
        for i, x in enumerate(idx):
            assert got[i].tobytes() == oracle_mod.eval_point(k, int(x))


def test_fill_splitmix_matches_oracle_generator(scanner, oracle_mod):
    db = G.GpuPageMatrix.from_seed(scanner, 10_000, 48, seed=99)
    for start, n in ((0, 5), (4321, 17), (9990, 10)):
        assert (db.read_rows(start, n) == oracle_mod.fill_splitmix(start * 48, n * 48, 99)).all()


def test_xor_rows_then_rescan(scanner, oracle_mod):
    db, rows = make_table(scanner, oracle_mod, 4096, 32, seed=17)
    rows = rows.copy()
    idx = np.array([0, 5, 4095, 5, 100], np.uint64)
    diffs = oracle_mod.fill_splitmix(0, idx.size * 32, 18).reshape(-1, 32)
    keys = [oracle_keypair(oracle_mod, 12, int(t), seed=19, i=j)[0] for j, t in enumerate((5, 100, 7))]
    before, _ = scanner.scan_keys(db, keys)
    db.xor_rows(idx, diffs)
    for i, r in enumerate(idx):
        rows[r] ^= diffs[i]
    after, _ = scanner.scan_keys(db, keys)
    assert after == oracle_mod.scan_fused(keys, rows, 32)
    delta = oracle_mod.delta_apply(keys, idx, diffs, 32)
    assert [xor_bytes(a, b) for a, b in zip(before, delta)] == after


def test_graph_and_multistream_match_direct(scanner, oracle_mod):
    db, rows = make_table(scanner, oracle_mod, 1 << 16, 64, seed=20)
    queries = [[G.ChaChaKey(oracle_keypair(oracle_mod, 16, (q * 3 + j) * 101, seed=21, i=3 * q + j)[0])
                for j in range(3)] for q in range(6)]
    direct = scanner.scan_batch(db, queries)
    graph1 = scanner.scan_batch(db, queries, use_cuda_graph=True)
    graph2 = scanner.scan_batch(db, queries, use_cuda_graph=True)  # replay
    multi = scanner.scan_batch_single_query_multistream_optimized(db, queries, 3)
    for a, b, c, d in zip(direct, graph1, graph2, multi):
        assert a.pages == b.pages == c.pages == d.pages
    want = oracle_mod.scan_fused([k.to_bytes() for q in queries for k in q], rows, 64)
    assert [p for r in direct for p in r.pages] == want


def test_deadline_returns_timeout_then_recovers(scanner, oracle_mod):
    # A host deadline shorter than the pass: MG_ETIMEDOUT, then MG_EBUSY while
    # the pass drains, then normal service.  No GPU fault is involved.
    big = G.GpuPageMatrix.from_seed(scanner, 1 << 26, 32, seed=22)
    keys = [oracle_keypair(oracle_mod, 26, 5 + j, seed=23, i=j)[0] for j in range(3)]
    with pytest.raises(N.Timeout):
        scanner.scan_keys(big, keys, timeout_ms=1)
    import time
    for _ in range(2000):
        try:
            shares, _ = scanner.scan_keys(big, keys)
            break
        except N.MgError as e:
            assert e.code == N.MG_EBUSY
            time.sleep(0.005)
    else:
        pytest.fail("pass never drained")
    rows5 = big.read_rows(5, 3)
    k1 = [oracle_keypair(oracle_mod, 26, 5 + j, seed=23, i=j)[1] for j in range(3)]
    other, _ = scanner.scan_keys(big, k1)
    for j in range(3):
        assert xor_bytes(shares[j], other[j]) == rows5[j * 32:(j + 1) * 32].tobytes()
    big.close()


def test_plain_single_query_cpu_runnable_config(scanner, oracle_mod):
    """The CPU-runnable plain single query: 2^20 rows x 256 B from seed 0,
    3 key pairs over a 20-bit domain, targets uniform; bit-exact vs oracle."""
    nrows, rb, d = 1 << 20, 256, 20
    db = G.GpuPageMatrix.from_seed(scanner, nrows, rb, seed=0)
    host = oracle_mod.fill_splitmix(0, nrows * rb, 0).reshape(nrows, rb)
    targets = [int(t) for t in np.random.default_rng(0).integers(0, nrows, 3)]
    pairs = [oracle_keypair(oracle_mod, d, t, seed=0, i=j) for j, t in enumerate(targets)]
    a = scanner.scan(db, [G.ChaChaKey(p[0]) for p in pairs])
    b = scanner.scan(db, [G.ChaChaKey(p[1]) for p in pairs])
    assert a.pages == oracle_mod.scan_fused([p[0] for p in pairs], host, rb)
    assert b.pages == oracle_mod.scan_fused([p[1] for p in pairs], host, rb)
    for j, t in enumerate(targets):
        assert xor_bytes(a.pages[j], b.pages[j]) == host[t].tobytes()


def test_autotuner_keeps_shares_and_caches_the_shape(scanner, oracle_mod):
    db, rows = make_table(scanner, oracle_mod, 1 << 16, 64, seed=40)
    keys = [oracle_keypair(oracle_mod, 16, 1000 * j + 7, seed=41, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_keys([db] * 3, keys)
    best = ws.autotune(budget_ms=0)
    assert best["ms"] > 0 and best["kernel"] in (N.KERNEL_CTA, N.KERNEL_WARP)
    ws.launch()
    want = oracle_mod.scan_fused(keys, rows, 64)
    assert ws.read() == want
    # A fresh workspace with the same workload picks the tuned shape up.
    ws2 = scanner.workspace()
    other = [oracle_keypair(oracle_mod, 16, 999 * j + 1, seed=42, i=j)[0] for j in range(3)]
    ws2.set_keys([db] * 3, other)
    plan = ws2.plan()
    for f in ("kernel", "subtree_bits", "keys_per_cta"):
        assert plan[f] == best[f]
    ws2.launch()
    assert ws2.read() == oracle_mod.scan_fused(other, rows, 64)
    # ... and so does the one-call entry point.
    got, _ = scanner.scan_keys(db, other)
    assert got == oracle_mod.scan_fused(other, rows, 64)
    ws.close()
    ws2.close()


def test_from_chunked_matrix_pads_like_the_reference(scanner, oracle_mod):
    # storage.rs:45-86: chunks uploaded at their byte offsets, the total and a
    # ragged last chunk padded with zeros to whole pages.
    rb = 4096
    data = oracle_mod.fill_splitmix(0, 5 * rb + 1000, 17)
    chunks = [data[:2 * rb], data[2 * rb:5 * rb], data[5 * rb:]]
    m = G.GpuPageMatrix.from_chunked_matrix(scanner, chunks, rb)
    assert m.num_pages() == 6 and m.size_bytes() == 6 * rb
    want = np.concatenate([data, np.zeros(6 * rb - data.size, np.uint8)])
    assert (m.read_rows(0, 6) == want).all()
    ptr, n = m.as_slice()
    assert ptr == m.device_ptr() and n == 6 * rb and m.device == scanner.device
    k0, k1 = oracle_keypair(oracle_mod, 3, 5, seed=18)
    a = scanner.scan_keys(m, [k0])[0][0]
    b = scanner.scan_keys(m, [k1])[0][0]
    assert bytes(x ^ y for x, y in zip(a, b)) == want[5 * rb:].tobytes()
    m.close()


def test_plan_reuse_restages_keys_and_replans_on_change(scanner, oracle_mod):
    """A workspace keeps its plan across set_keys calls with the same tables,
    depths and shape (only the keys are restaged) and replans on any change;
    every pass stays bit-exact, also through the one-call path, which replays
    repeated workloads from a CUDA graph."""
    rb, n = 32, 5000
    t1, rows1 = make_table(scanner, oracle_mod, n, rb, seed=91)
    ws = scanner.workspace()
    for rep in range(3):
        keys = [oracle_keypair(oracle_mod, 13, (977 * rep + 31 * j) % n, seed=92, i=10 * rep + j)[0] for j in range(3)]
        ws.set_keys([t1] * 3, keys)
        ws.launch()
        assert ws.read() == oracle_mod.scan_fused(keys, rows1, rb)
        got, _ = scanner.scan_keys(t1, keys)
        assert got == oracle_mod.scan_fused(keys, rows1, rb)
    # another depth on the same table
    keys = [oracle_keypair(oracle_mod, 15, 7 + j, seed=93, i=j)[0] for j in range(3)]
    ws.set_keys([t1] * 3, keys)
    ws.launch()
    assert ws.read() == oracle_mod.scan_fused(keys, rows1, rb)
    # a table of another shape, possibly at a recycled address
    t1.close()
    t2, rows2 = make_table(scanner, oracle_mod, 7001, 64, seed=94)
    keys = [oracle_keypair(oracle_mod, 13, 100 * j + 1, seed=95, i=j)[0] for j in range(3)]
    for _ in range(2):
        ws.set_keys([t2] * 3, keys)
        ws.launch()
        assert ws.read() == oracle_mod.scan_fused(keys, rows2, 64)
        got, _ = scanner.scan_keys(t2, keys)
        assert got == oracle_mod.scan_fused(keys, rows2, 64)
    # a delta buffer appears: the pass must fold it
    t2.delta_reserve(16)
    idx = np.array([1, 101], np.uint64)
    diffs = oracle_mod.fill_splitmix(3, 2 * 64, 96).reshape(2, 64)
    t2.delta_push(idx, diffs)
    ws.set_keys([t2] * 3, keys)
    ws.launch()
    patched = rows2.copy()
    for i, r in enumerate(idx):
        patched[r] ^= diffs[i]
    assert ws.read() == oracle_mod.scan_fused(keys, patched, 64)
    ws.close()
    t2.close()


@pytest.mark.parametrize("kernel,rb", [("auto", 32), ("cta", 4096), ("warp", 64)])
def test_empty_table_and_empty_batch(scanner, oracle_mod, kernel, rb):
    """storage.rs:89-101 allows an empty matrix: every share is zero; an
    empty batch returns no results (kernel.rs:711-924)."""
    empty = G.GpuPageMatrix.alloc_empty(scanner, 0, rb)
    keys = [oracle_keypair(oracle_mod, 10, 3 * j, seed=61, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_kernel(kernel)
    ws.set_keys([empty] * 3, keys)
    ws.launch()
    assert ws.read() == [bytes(rb)] * 3
    ws.close()
    got, _ = scanner.scan_keys(empty, keys)
    assert got == [bytes(rb)] * 3
    assert scanner.scan_batch(empty, []) == []
    with pytest.raises(G.GpuDpfError):
        empty.delta_reserve(4)
        empty.delta_push(np.array([0], np.uint64), np.zeros((1, rb), np.uint8))
    empty.close()


def test_many_key_groups_one_pass(scanner, oracle_mod):
    """192 keys (64 queries) over one table in one pass: 192 key groups do not
    divide the persistent warps, so the planner may stride every warp over
    the tile-major items; bit-exact either way."""
    rb, nrows, d = 32, 1 << 16, 16
    db, rows = make_table(scanner, oracle_mod, nrows, rb, seed=71)
    keys = [oracle_keypair(oracle_mod, d, (40503 * j) % nrows, seed=72, i=j)[0] for j in range(192)]
    got, _ = scanner.scan_keys(db, keys)
    assert got == oracle_mod.scan_fused(keys, rows, rb)


def test_prg_peak_and_timers(scanner, oracle_mod):
    """mg_prg_peak (the ChaCha8 ceiling the bench reports against) gives a
    plausible rate, and a pass's scan time lies within its total time."""
    rate = scanner.prg_peak(64)
    assert 1e9 < rate < 1e12
    db, rows = make_table(scanner, oracle_mod, 50_000, 32, seed=81)
    keys = [oracle_keypair(oracle_mod, 16, 7 * j, seed=82, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_keys([db] * 3, keys)
    ws.launch()
    ws.sync()
    assert 0 < ws.last_scan_ns() <= ws.last_kernel_ns()
    assert ws.read() == oracle_mod.scan_fused(keys, rows, 32)
    ws.close()


def test_gpu_matches_recorded_reference_kernel_outputs(scanner, oracle_mod):
    """Shares recorded from the reference's own CUDA kernel (committed
    fixtures, make_test_pages pages, depths 8-25): this library's GPU path
    reproduces every one without the reference present."""
    import hashlib
    import json
    from pathlib import Path
    data = json.loads((Path(__file__).with_name("golden") / "ref_kernel_pages.json").read_text())
    for case in data["cases"]:
        pages = oracle_mod.fill_test_rows(case["pages"], 4096)
        db = G.GpuPageMatrix.new(scanner, pages, 4096)
        keys = [bytes.fromhex(k) for k in case["keys"]]
        got, _ = scanner.scan_keys(db, keys)
        for j, share in enumerate(got):
            assert hashlib.sha256(share).hexdigest() == case["sha256"][j]
            assert share[:64].hex() == case["head"][j] and share[-64:].hex() == case["tail"][j]
        db.close()
