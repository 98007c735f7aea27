"""Device-resident epoch delta (crates/morphogen-core/src/delta.rs,
crates/morphogen-server/src/scan.rs:434-485, epoch.rs:465-549): pending
entries are folded into every pass, a merge XOR-patches the table and
clears them; bit-exact against the oracle's scan of the patched table and
its restatement of scan_delta_for_gpu."""
import numpy as np
import pytest

from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import _native as N
from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu


def setup_table(scanner, oracle_mod, nrows, rb, seed):
    host = oracle_mod.fill_splitmix(0, nrows * rb, seed).reshape(nrows, rb).copy()
    return G.GpuPageMatrix.new(scanner, host, rb), host


@pytest.mark.parametrize("rb,nrows,d", [(32, 1 << 16, 16), (64, 40_000, 17), (256, 5000, 13), (4096, 300, 9)])
def test_delta_folded_into_every_pass(scanner, oracle_mod, rb, nrows, d):
    db, host = setup_table(scanner, oracle_mod, nrows, rb, seed=rb + d)
    db.delta_reserve(1024)
    rng = np.random.default_rng(d)
    idx = rng.integers(0, nrows, 700).astype(np.uint64)
    idx[:4] = [0, nrows - 1, 17, 17]  # edges and a duplicate row
    diffs = oracle_mod.fill_splitmix(123, idx.size * rb, 5).reshape(-1, rb)
    db.delta_push(idx[:400], diffs[:400])
    db.delta_push(idx[400:], diffs[400:])
    assert db.delta_count() == 700
    targets = [int(t) for t in (idx[0], idx[2], idx[500])]
    pairs = [oracle_keypair(oracle_mod, d, t, seed=70, i=j) for j, t in enumerate(targets)]
    k0 = [p[0] for p in pairs]
    got, _ = scanner.scan_keys(db, k0)
    base = oracle_mod.scan_fused(k0, host, rb)
    delta = oracle_mod.delta_apply(k0, idx, diffs, rb)
    assert got == [xor_bytes(a, b) for a, b in zip(base, delta)]
    patched = host.copy()
    for i, r in enumerate(idx):
        patched[r] ^= diffs[i]
    assert got == oracle_mod.scan_fused(k0, patched, rb)
    # The two servers' answers recover the updated rows.
    got1, _ = scanner.scan_keys(db, [p[1] for p in pairs])
    for j, t in enumerate(targets):
        assert xor_bytes(got[j], got1[j]) == patched[t].tobytes()
    # Merge: the table becomes the patched table, the buffer empties, the epoch advances.
    e0 = db.epoch()
    db.delta_merge()
    assert db.delta_count() == 0 and db.epoch() == e0 + 1
    assert (db.read_rows(0, nrows).reshape(nrows, rb) == patched).all()
    after, _ = scanner.scan_keys(db, k0)
    assert after == got


def test_graph_replay_sees_later_pushes(scanner, oracle_mod):
    rb, nrows, d = 32, 1 << 15, 15
    db, host = setup_table(scanner, oracle_mod, nrows, rb, seed=90)
    db.delta_reserve(256)
    keys = [oracle_keypair(oracle_mod, d, 100 * j + 1, seed=91, i=j)[0] for j in range(3)]
    ws = scanner.workspace()
    ws.set_keys([db] * 3, keys)
    ws.launch(graph=True)
    assert ws.read() == oracle_mod.scan_fused(keys, host, rb)
    idx = np.array([1, 101, 201, 5], np.uint64)
    diffs = oracle_mod.fill_splitmix(7, idx.size * rb, 8).reshape(-1, rb)
    db.delta_push(idx, diffs)
    ws.launch(graph=True)  # replay of the captured pass
    patched = host.copy()
    for i, r in enumerate(idx):
        patched[r] ^= diffs[i]
    assert ws.read() == oracle_mod.scan_fused(keys, patched, rb)
    ws.close()


def test_delta_limits(scanner, oracle_mod):
    db, _ = setup_table(scanner, oracle_mod, 1000, 32, seed=3)
    db.delta_reserve(4)
    diffs = np.zeros((5, 32), np.uint8)
    with pytest.raises(G.GpuDpfError) as e:
        db.delta_push(np.arange(5, dtype=np.uint64), diffs)
    assert e.value.code == N.MG_ERANGE and "full" in e.value.message
    with pytest.raises(G.GpuDpfError) as e:
        db.delta_push(np.array([1000], np.uint64), diffs[:1])
    assert e.value.code == N.MG_ERANGE
    db.delta_push(np.array([1, 2], np.uint64), diffs[:2])
    db.delta_reserve(64)  # growing keeps pending entries
    assert db.delta_count() == 2
    db.delta_clear()
    assert db.delta_count() == 0
