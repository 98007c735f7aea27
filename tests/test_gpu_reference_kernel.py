"""Page-mode parity against the reference's own CUDA kernels.

The reference's cuda/fused_kernel.cu (the single-query kernel its server
calls) and cuda/fused_kernel_optimized.cu (its batched kernel) are compiled
unmodified for sm_100a into oracle/_ref by oracle/ref_build.py.  On the same
table, in the reference's page layout (4096-byte pages, at most 25 levels),
the reference kernels, the oracle and this library must give identical
shares."""
import numpy as np
import pytest

import oracle
from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import gpu_dpf as G

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference tree)")]


def pages_table(scanner, npages, pattern):
    host = (oracle.fill_test_rows(npages, 4096) if pattern == "pages"
            else oracle.fill_splitmix(0, npages * 4096, 77))
    return G.GpuPageMatrix.new(scanner, host, 4096), host.reshape(npages, 4096)


@pytest.mark.parametrize("d,npages,pattern", [(8, 256, "pages"), (10, 500, "pages"), (12, 4096, "splitmix"),
                                              (16, 3001, "splitmix"), (25, 2100, "splitmix")])
def test_baseline_reference_kernel_matches(scanner, oracle_mod, d, npages, pattern):
    db, pages = pages_table(scanner, npages, pattern)
    targets = [(npages * j) // 3 + 1 for j in range(3)]
    pairs = [oracle_keypair(oracle_mod, d, t, seed=50 + d, i=j) for j, t in enumerate(targets)]
    k0 = [p[0] for p in pairs]
    ref, _ = oracle.ref_scan(0, k0, db.device_ptr(), npages)
    mine, _ = scanner.scan_keys(db, k0)
    assert mine == ref
    assert ref == oracle_mod.scan_fused(k0, pages, 4096)
    ref1, _ = oracle.ref_scan(0, [p[1] for p in pairs], db.device_ptr(), npages)
    for j, t in enumerate(targets):
        assert xor_bytes(ref[j], ref1[j]) == pages[t].tobytes()


@pytest.mark.parametrize("batch", [1, 2, 4])
def test_optimized_reference_kernel_matches(scanner, oracle_mod, batch):
    npages, d = 5000, 13
    db, pages = pages_table(scanner, npages, "splitmix")
    keys = [oracle_keypair(oracle_mod, d, (997 * j + 3) % npages, seed=60, i=j)[0] for j in range(3 * batch)]
    ref, _ = oracle.ref_scan(1, keys, db.device_ptr(), npages)
    mine, _ = scanner.scan_keys(db, keys)
    assert mine == ref == oracle_mod.scan_fused(keys, pages, 4096)
