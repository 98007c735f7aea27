"""The dynamic shared-memory limit of a scan kernel belongs to the kernel on
its device for the whole process, not to a context.  Two GpuScanners on one
device (the reference's GpuScanner::new, kernel.rs:258-465, sets the limit
once per kernel at start-up, :293-303) must therefore never undo each
other's launch shapes: context A plans a large CTA (or warp) shape, context B
a smaller one, and A's next pass still launches.  Every share is compared
with the oracle."""
import pytest

from conftest import oracle_keypair

from morphogen_b200 import gpu_dpf as G

pytestmark = pytest.mark.gpu


def host_table(scanner, oracle_mod, nrows, row_bytes, seed):
    host = oracle_mod.fill_splitmix(0, nrows * row_bytes, seed)
    return G.GpuPageMatrix.new(scanner, host, row_bytes), host.reshape(nrows, row_bytes)


def pinned(scanner, kind, subtree_bits, keys_per_item):
    ws = scanner.workspace()
    ws.set_kernel(kind)
    ws.set_shape(subtree_bits, keys_per_item)
    return ws


@pytest.mark.parametrize("kind,big,small,row_bytes", [
    # CTA kernel, 4 keys per CTA: tile depth 14 needs 4 x 34,928 B of shared
    # memory, tile depth 8 needs 4 x 17,520 B.
    ("cta", 14, 8, 64),
    # warp kernel, 4 keys per warp: warp tile 2^15 (depth-first M = 10) needs
    # 206,848 B, warp tile 2^6 (M = 1) 50,176 B.
    ("warp", 15, 6, 32),
])
def test_second_context_cannot_lower_the_first_contexts_limit(scanner, oracle_mod, kind, big, small, row_bytes):
    d, nrows = 17, 70_001
    db_a, rows_a = host_table(scanner, oracle_mod, nrows, row_bytes, seed=91)
    keys = [oracle_keypair(oracle_mod, d, (7717 * j) % nrows, seed=92, i=j)[0] for j in range(4)]
    want_a = oracle_mod.scan_fused(keys, rows_a, row_bytes)

    ws_a = pinned(scanner, kind, big, 4)
    ws_a.set_keys([db_a] * 4, keys)
    ws_a.launch()
    assert ws_a.read() == want_a

    other = G.GpuScanner(0)  # a second context on the same device
    db_b, rows_b = host_table(other, oracle_mod, nrows, row_bytes, seed=93)
    ws_b = pinned(other, kind, small, 4)
    ws_b.set_keys([db_b] * 4, keys)
    ws_b.launch()
    assert ws_b.read() == oracle_mod.scan_fused(keys, rows_b, row_bytes)

    # Context A's plan (made before B's) launches again with its larger shape.
    ws_a.launch()
    assert ws_a.read() == want_a
    ws_a.set_keys([db_a] * 4, keys)
    ws_a.launch(graph=True)
    assert ws_a.read() == want_a
    for o in (ws_b, db_b, ws_a, db_a):
        o.close()
    other.close()
