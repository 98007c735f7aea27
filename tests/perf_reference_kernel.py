"""Page-mode comparison with the reference's own CUDA kernels (not a pytest
module; run explicitly on a GPU box).

Workload: the reference's mainnet page matrix shape, 16,817,159 pages of
4096 bytes (68.9 GB, SplitMix64 bytes from seed 0 stand in for the absent
mainnet file), one query = 3 keys over a 25-bit domain (the reference
kernel's maximum).  Times, on the same table and keys:
  * this library's device pass (autotuned shape, CUDA events);
  * the reference's single-query kernel fused_batch_pir_kernel_1 and its
    batched kernel fused_batch_pir_kernel_optimized_1 (both compiled
    unmodified for sm_100a into oracle/_ref), launched with its own recipe;
and checks that all three give identical shares at full size.

Run: python tests/perf_reference_kernel.py [--pages N] [--reps R]
"""
import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from morphogen_b200 import gpu_dpf as G  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pages", type=int, default=16_817_159)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--domain-bits", type=int, default=25)
    args = ap.parse_args()
    scanner = G.GpuScanner(0)
    db = G.GpuPageMatrix.from_seed(scanner, args.pages, 4096, seed=0)
    rng = np.random.default_rng(0)
    p = G.ChaChaParams(args.domain_bits)
    keys = [G.generate_chacha_dpf_keys(p, int(t), rng)[0] for t in rng.integers(0, args.pages, 3)]
    ws = scanner.workspace()
    ws.set_keys([db] * 3, keys)
    ws.launch()
    mine = ws.read()
    tuned = ws.autotune(20000)
    ws.launch()
    assert ws.read() == mine
    times = []
    for _ in range(args.reps):
        ws.launch()
        ws.sync()
        times.append(ws.last_kernel_ns() / 1e6)
    ours = min(times)
    res = {"workload": f"{args.pages} pages x 4096 B ({args.pages * 4096 / 1e9:.1f} GB), 3 x {args.domain_bits}-bit keys",
           "ours_ms": round(ours, 3), "ours_GBps": round(args.pages * 4096 / ours / 1e6, 1),
           "ours_plan": ws.plan()}
    for kind, name in ((0, "reference fused_batch_pir_kernel_1"), (1, "reference fused_batch_pir_kernel_optimized_1")):
        shares, ms = oracle.ref_scan(kind, [k.to_bytes() for k in keys], db.device_ptr(), args.pages, reps=args.reps)
        res[name] = {"ms": round(ms, 3), "GBps": round(args.pages * 4096 / ms / 1e6, 1),
                     "shares_equal": shares == mine}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
