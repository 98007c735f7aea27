"""Record the reference's own CUDA kernel outputs as golden fixtures.

Runs on a GPU box: builds nothing, loads oracle/_ref/libmg_refkernels.so
(the reference's cuda/fused_kernel.cu compiled unmodified for sm_100a),
uploads make_test_pages-pattern pages (kernel.rs:1390-1403), evaluates seeded
keys with the reference's single-query kernel and writes
tests/golden/ref_kernel_pages.json (keys, pages spec, SHA-256 and the first
and last 64 bytes of every share, plus the full shares of the smallest case).
The CPU test test_oracle.py::test_oracle_matches_reference_kernel_fixtures
then checks the oracle against these outputs without a GPU.

Run: python tests/golden/make_ref_fixtures.py [out_dir]
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from conftest import oracle_keypair  # noqa: E402
from morphogen_b200 import gpu_dpf as G  # noqa: E402

CASES = [(8, 256), (11, 1500), (14, 9000), (25, 2500)]


def main(out_dir: Path):
    scanner = G.GpuScanner(0)
    cases = []
    for d, npages in CASES:
        host = oracle.fill_test_rows(npages, 4096)
        db = G.GpuPageMatrix.new(scanner, host, 4096)
        keys = []
        for j in range(3):
            t = (npages * (2 * j + 1)) // 6
            keys.append(oracle_keypair(oracle, d, t, seed=1000 + d, i=j)[0])
        shares, _ = oracle.ref_scan(0, keys, db.device_ptr(), npages)
        case = {"domain_bits": d, "pages": npages, "pattern": "make_test_pages",
                "keys": [k.hex() for k in keys],
                "sha256": [hashlib.sha256(s).hexdigest() for s in shares],
                "head": [s[:64].hex() for s in shares], "tail": [s[-64:].hex() for s in shares]}
        if npages == 256:
            case["shares"] = [s.hex() for s in shares]
        cases.append(case)
        db.close()
    out = {"source": "reference cuda/fused_kernel.cu fused_batch_pir_kernel_1, built for sm_100a, run on B200",
           "cases": cases}
    out_dir.mkdir(parents=True, exist_ok=True)
    (out_dir / "ref_kernel_pages.json").write_text(json.dumps(out, indent=1) + "\n")
    print(out_dir / "ref_kernel_pages.json")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).parent)
