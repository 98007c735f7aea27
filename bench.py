#!/usr/bin/env python
"""Benchmark of the per-server PIR answer path on B200.

Default workload (one step = one scan pass answering one query):
  plain single query at mainnet scale -- a table of 2^31 rows x 32 B (64 GiB)
  of SplitMix64 bytes from seed 0, 3 ChaCha8 DPF keys (one server's shares)
  over a 31-bit domain for 3 uniformly drawn target rows.

`value` is scanned GB/s (table bytes per pass / device time per pass, keys
resident); `e2e` is the same metric through the one-call C entry point
mg_scan with host keys in and host shares out.  `roofline` reports the
dominant kernel against its binding resource: the integer ALU pipe running
ChaCha8 (node expansions per second against the PRG-only ceiling measured
in the same run), with the HBM fraction beside it (`roofline.hbm`).

On one GPU the default run adds, in the same JSON line:
  c1       the full 2^20 rows x 256 B configuration (3 x 20-bit keys),
           autotuned, passes replayed from a CUDA graph;
  batched  Q = 1 and 8 queries (3 keys each) per pass over the 2^31 x 32 B
           table, launch shape autotuned on a 2^26-row window of the same
           table and kept only if faster on the full table, graph replay;
  pages    the reference's own layout (16,817,159 pages x 4096 B, 25-bit
           keys): this library's pass against the reference's
           fused_batch_pir_kernel_1 compiled for sm_100a, on the same table
           and keys, shares compared.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload plain31|plain20|batched31 --queries Q|sharded31|pages|mixed|serve31]
                  [--no-extras] [--no-cpu]

Multi-GPU (torchrun, one process per GPU): by default every rank serves an
independent replica of the table (no collective; weak scaling), timing is the
max over ranks and `value` the aggregate over all replicas.  `sharded31`
splits the one table into contiguous row ranges over the ranks instead; each
pass ends with an NCCL all-gather + XOR of the ranks' shares (strong scaling:
the per-query latency falls with N).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "plain31": dict(name="plain single query, 2^31 rows x 32 B (64 GiB), 31-bit keys",
                    rows=1 << 31, row_bytes=32, d=31),
    "plain31s": dict(name="profiling case: 2^25 rows x 32 B (1 GiB) scanned with 31-bit keys",
                     rows=1 << 25, row_bytes=32, d=31),
    "plain20": dict(name="plain single query, 2^20 rows x 256 B (256 MiB), 20-bit keys",
                    rows=1 << 20, row_bytes=256, d=20),
    "batched31": dict(name="batched queries per pass, 2^31 rows x 32 B (64 GiB), 31-bit keys",
                      rows=1 << 31, row_bytes=32, d=31),
    "sharded31": dict(name="plain single query, 2^31 rows x 32 B (64 GiB) split into contiguous row ranges "
                           "over the ranks, shares XOR-combined by NCCL all-gather", rows=1 << 31, row_bytes=32, d=31),
    "pages": dict(name="page mode (the reference's layout): 16,817,159 pages x 4096 B (68.9 GB), 25-bit keys",
                  rows=16_817_159, row_bytes=4096, d=25),
    "pages_s": dict(name="profiling case: 2^16 pages x 4096 B (256 MiB) scanned with 25-bit keys",
                    rows=1 << 16, row_bytes=4096, d=25),
    "mixed": dict(name="accounts 2^28 x 64 B + storage 2^31 x 32 B in one pass", rows=0, row_bytes=0, d=0),
    "serve31": dict(name="serving loop over 2^31 rows x 32 B (64 GiB): Poisson arrivals, 1-32 lookups per "
                         "request (geometric, mean 4), 3 x 31-bit keys per lookup, 2^16-row epoch delta "
                         "replaced and merged every 12 s", rows=1 << 31, row_bytes=32, d=31),
}
KEYS_PER_QUERY = 3
SEED = 0
CPU_SAMPLE_BYTES = 4 << 30     # aligned window timed on the host cores (cpu_baseline): 2^27 rows of 32 B
REF_SAMPLE_BYTES = 1 << 30     # per-step sample of the reference arm: 2^25 rows of 32 B
PROXY_ROWS = 1 << 26           # window of the 2^31-row table the batched shapes are autotuned on
PAGES = 16_817_159             # the reference's mainnet page matrix (docs/benchmarks/...-h100-matrix.csv)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


def seeded_keys(d: int, rows: int, nqueries: int, seed: int = SEED):
    """Targets uniform in [0, rows), root seeds from a seeded generator;
    returns (party-0 keys, party-1 keys, targets)."""
    from morphogen_b200 import gpu_dpf as G
    rng = np.random.default_rng(seed)
    targets = [int(t) for t in rng.integers(0, rows, nqueries * KEYS_PER_QUERY)]
    k0, k1 = [], []
    p = G.ChaChaParams(d)
    for t in targets:
        a, b = G.generate_chacha_dpf_keys(p, t, rng)
        k0.append(a)
        k1.append(b)
    return k0, k1, targets


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        note = None
        if not self.lines:
            # Timed region shorter than the sampling interval: one reading
            # right after it (the clocks have not settled back to idle yet).
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
                self.lines = [ln.strip() for ln in out.stdout.splitlines() if ln.strip()]
                note = "timed region shorter than the 100 ms sampling interval; one reading right after it"
            except (OSError, subprocess.TimeoutExpired):
                pass
        sm, smax, power, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        res = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
               "reasons": sorted(reasons), "samples": len(sm),
               "power_w_max": max(power) if power else None}
        if note:
            res["note"] = note
        return res


def cpu_info() -> dict:
    """Host CPU model, logical CPUs and physical cores (the baseline's `cores`
    is the OpenMP thread count actually used)."""
    model = "unknown"
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    physical = None
    try:
        import psutil
        physical = psutil.cpu_count(logical=False)
    except Exception:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count(), "physical_cores": physical}


def cpu_scan_sample(keys, rows_total: int, row_bytes: int, sample_rows: int, reps: int = 1,
                    avx512: bool = True, base: int | None = None) -> dict:
    """Time the oracle (the restated reference CPU scan: eval_fused_3dpf_cpu
    with scalar ChaCha8, OpenMP over all host threads) on an aligned window
    of the table.  avx512: the AND/XOR loop in 512-bit registers, eight rows
    per step (the reference server's AVX-512 scan shape, scan.rs:719-895) when
    the host has AVX-512F.  Returns per-rep seconds and GB/s with the host
    description."""
    import oracle
    oracle.build()
    use_avx = avx512 and oracle.avx512_available()
    if base is None:
        base = (rows_total // 2) // sample_rows * sample_rows
    host = oracle.fill_splitmix(base * row_bytes, sample_rows * row_bytes, SEED)
    kb = [bytes(k) for k in keys]
    nthreads = os.cpu_count() or 1
    secs = []
    for _ in range(reps):
        t0 = time.perf_counter()
        oracle.scan_fused(kb, host, row_bytes, row_base=base, nthreads=nthreads, avx512=use_avx)
        secs.append(time.perf_counter() - t0)
    window = sample_rows * row_bytes
    rates = [window / t / 1e9 for t in secs]
    variant = ("AND/XOR in AVX-512 registers, 8 rows per step (scan.rs:719-895 shape); scalar ChaCha8"
               if use_avx else "scalar AND/XOR (kernel.rs:1243-1256); scalar ChaCha8")
    desc = (f"{len(kb)} keys over the aligned window of {sample_rows} rows starting at row {base} "
            f"({window / 2**30:.2f} GiB); GB/s of that window")
    return {"rates": rates, "secs": secs, "threads": nthreads, "window_bytes": window, "variant": variant,
            "avx512": use_avx, "desc": desc, **cpu_info()}


def cpu_baseline_obj(c: dict, scalar: dict | None = None) -> dict:
    v = sum(c["rates"]) / len(c["rates"])
    o = {"value": round(v, 4), "unit": "GB/s", "cores": c["threads"], "kind": "port", "sample": c["desc"],
         "variant": c["variant"], "per_rep_s": [round(x, 4) for x in c["secs"]], "window_bytes": c["window_bytes"],
         "cpu_model": c["cpu_model"], "logical_cpus": c["logical_cpus"], "physical_cores": c["physical_cores"]}
    if scalar:
        o["scalar_variant"] = {"value": round(sum(scalar["rates"]) / len(scalar["rates"]), 4),
                               "per_rep_s": [round(x, 4) for x in scalar["secs"]], "variant": scalar["variant"]}
    return o


def run_reference(args, rank: int, world: int):
    """The reference's CPU implementation of the path (oracle port) on the host cores."""
    if rank != 0:
        return
    if args.workload in ("mixed", "serve31"):
        args.workload = "plain31"
    wl = WORKLOADS[args.workload]
    nq = int(str(args.queries).split(",")[0]) if args.workload == "batched31" else 1
    k0, _, _ = seeded_keys(wl["d"], wl["rows"], nq)
    sample = min(REF_SAMPLE_BYTES // wl["row_bytes"], wl["rows"])
    cpu_scan_sample(k0, wl["rows"], wl["row_bytes"], sample, reps=args.warmup)
    c = cpu_scan_sample(k0, wl["rows"], wl["row_bytes"], sample, reps=args.steps)
    v = sum(c["rates"]) / len(c["rates"])
    gb_pass = wl["rows"] * wl["row_bytes"] / 1e9
    cb = cpu_baseline_obj(c)
    cb["sample"] += "; ms_per_step extrapolates the window's time to the full table"
    line = {
        "impl": "reference", "metric": "scanned GB/s", "value": round(v, 4), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(gb_pass / v * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl["name"], "queries_per_pass": nq, "keys": nq * KEYS_PER_QUERY,
                   "l2": "inputs larger than L2"},
        "cpu_baseline": cb,
        "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_serve(args, local_rank: int):
    """Continuous-batching serving loop at several Poisson arrival rates."""
    import torch

    from morphogen_b200 import gpu_dpf as G
    from morphogen_b200.server import PirServer, geometric_lookups, poisson_load

    torch.cuda.set_device(local_rank)
    wl = WORKLOADS["serve31"]
    rows, rb, d = wl["rows"], wl["row_bytes"], wl["d"]
    scanner = G.GpuScanner(local_rank)
    table = G.GpuPageMatrix.from_seed(scanner, rows, rb, seed=SEED)
    drng = np.random.default_rng(SEED + 1)
    delta_rows = 1 << 16
    table.delta_reserve(delta_rows)

    def new_delta():
        idx = drng.integers(0, rows, delta_rows).astype(np.uint64)
        diffs = drng.integers(0, 256, delta_rows * rb, dtype=np.uint8)
        table.delta_push(idx, diffs)

    new_delta()
    pool, _, _ = seeded_keys(d, rows, 64)  # 64 lookups x 3 keys
    lookups = [pool[3 * i:3 * i + 3] for i in range(64)]

    def make_request(rng):
        n = geometric_lookups(rng, mean=4.0, lo=1, hi=32)
        items = []
        for _ in range(n):
            items += [(table, k) for k in lookups[int(rng.integers(0, len(lookups)))]]
        return items

    srv = PirServer(scanner, slots=2)
    # Single-lookup latency with an idle server (the plain path through the loop).
    for _ in range(2):
        srv.answer(make_request(np.random.default_rng(0))[:3])
    srv.reset_stats()
    for _ in range(5):
        srv.answer([(table, k) for k in lookups[0]])
    idle = srv.stats()
    merges = {"count": 0, "next": 12.0}

    def tick(t):
        if t >= merges["next"]:
            srv.pause()
            table.delta_merge()
            new_delta()
            srv.resume()
            merges["count"] += 1
            merges["next"] += 12.0

    points = []
    rates = [float(x) for x in args.rates.split(",")]
    for rate in rates:
        merges["next"] = 12.0
        dur = args.duration if rate <= 5 else args.overload_duration
        st = poisson_load(srv, make_request, rate, dur, seed=int(rate * 1000), tick=tick)
        points.append({"offered_req_per_s": round(st["offered_req_per_s"], 3), "requests": st["requests"],
                       "lookups": st["keys"] // 3, "answered_lookups_per_s": round(st["answered_keys_per_s"] / 3, 3),
                       "p50_ms": round(st["p50_ms"], 1), "p95_ms": round(st["p95_ms"], 1),
                       "p99_ms": round(st["p99_ms"], 1), "passes": st["passes"], "failed": st["failed"]})
    srv.close()
    best = max(p["answered_lookups_per_s"] for p in points)
    line = {
        "metric": "answered lookups/s (3 keys each) and p50/p95/p99 latency under Poisson load",
        "value": best, "unit": "lookups/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u32",
        "data": "synthetic", "config": {"workload": wl["name"], "slots": 2, "delta_rows": delta_rows,
                                        "merge_interval_s": 12, "epoch_merges": merges["count"]},
        "idle_single_lookup_ms": {"p50": round(idle["p50_ms"], 2), "p99": round(idle["p99_ms"], 2)},
        "load_points": points,
    }
    print(json.dumps(line), flush=True)


def run_serving_point(scanner, table, rb: int, d: int, rows: int, local_rank: int) -> dict:
    """The continuous-batching loop (mg_server) on the 2^31-row table of the
    default line: single-lookup latency on an idle server, then 30 s of
    open-loop Poisson arrivals of single lookups (3 keys each) at 60% of the
    one-GPU capacity.  One lookup's shares are checked
    against the second server's keys (their XOR is the target row)."""
    from morphogen_b200.server import PirServer, poisson_load

    nlook = 16
    k0, k1, targets = seeded_keys(d, rows, nlook, seed=SEED + 7)
    lookups = [k0[3 * i:3 * i + 3] for i in range(nlook)]
    srv = PirServer(scanner, slots=2)
    try:
        for _ in range(2):
            srv.answer([(table, k) for k in lookups[1]])
        got = srv.answer([(table, k) for k in lookups[0]])
        other, _ = scanner.scan_keys(table, k1[0:3])
        want = target_rows(table, targets[0:3], rb, None, local_rank)
        verified = all(bytes(a ^ b for a, b in zip(x, y)) == w for x, y, w in zip(got, other, want))
        srv.reset_stats()
        for j in range(9):
            srv.answer([(table, k) for k in lookups[j]])
        idle = srv.stats()
        pass_s = max(idle["p50_ms"], 1.0) * 1e-3  # one lookup = one pass when idle
        rate = 0.6 / pass_s  # lookups/s at 60% of capacity

        def make_request(rng):
            return [(table, k) for k in lookups[int(rng.integers(0, nlook))]]

        st = poisson_load(srv, make_request, rate, 30.0, seed=SEED + 8)
    finally:
        srv.close()
    if not verified:
        raise SystemExit("bench: serving-loop shares do not reconstruct the target rows")
    return {
        "workload": "serving loop (mg_server, 2 workspaces) over 2^31 rows x 32 B (64 GiB), 31-bit keys, "
                    "3 keys per lookup",
        "idle_single_lookup_ms": {"p50": round(idle["p50_ms"], 2), "p99": round(idle["p99_ms"], 2)},
        "poisson": {"offered_lookups_per_s": round(st["offered_req_per_s"], 3),
                    "offered_load": round(st["offered_req_per_s"] * pass_s, 3), "target_load": 0.6,
                    "lookups": st["requests"], "answered_lookups_per_s": round(st["answered_keys_per_s"] / 3, 3),
                    "p50_ms": round(st["p50_ms"], 1), "p95_ms": round(st["p95_ms"], 1),
                    "p99_ms": round(st["p99_ms"], 1), "passes": st["passes"], "failed": st["failed"],
                    "duration_s": 30.0, "lookups_per_request": 1},
        "verified": verified,
    }


def expansions(first: int, n: int, d: int) -> int:
    """Tree nodes expanded by one key over rows [first, first + n): the
    internal nodes (levels of width 2^1 .. 2^d) whose leaves meet the range."""
    return sum(((first + n - 1) >> s) - (first >> s) + 1 for s in range(1, d + 1)) if n else 0


def target_rows(table, targets, rb: int, dist, local_rank: int) -> list[bytes]:
    """The logical table's rows at `targets`: read by the rank whose range
    holds each one, summed over the ranks (zeros elsewhere)."""
    import torch
    buf = np.zeros((len(targets), rb), np.int32)
    for j, t in enumerate(targets):
        if table.first_row <= t < table.first_row + table.num_pages():
            buf[j] = table.read_rows(t - table.first_row, 1)
    if dist:
        tt = torch.from_numpy(buf).to(f"cuda:{local_rank}")
        dist.all_reduce(tt)
        buf = tt.cpu().numpy()
    return [buf[j].astype(np.uint8).tobytes() for j in range(len(targets))]


def measure(args, scanner, tables, k0, k1, targets_rows, world, local_rank, dist, combiner=None,
            graph=None, autotune=None, steps=None, warmup=None, pin=None):
    """One workload point: correctness gate, optional autotune, K timed device
    passes (CUDA events on the launching stream), e2e passes through mg_scan.
    tables[i] is the table of key i.  With a ShardCombiner every pass is
    followed by the XOR-combine of the ranks' shares (tables are row ranges of
    one logical table).  graph / autotune / steps / warmup override the
    command line for this point; pin = (kernel, subtree_bits, keys_per_item)
    fixes the launch shape.  Returns the fields of the JSON line."""
    import torch

    from morphogen_b200.shard import combine_shares

    graph = args.graph if graph is None else graph
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    nkeys = len(k0)
    host_combine = (lambda sh: combine_shares(sh, device=f"cuda:{local_rank}")) if combiner else (lambda sh: sh)
    ws = scanner.workspace()
    if pin:
        ws.set_kernel(pin[0])
        ws.set_shape(pin[1], pin[2])
    else:
        ws.set_kernel(args.kernel)
        if args.shape:
            S, Gk = (int(x) for x in args.shape.split(","))
            ws.set_shape(S, Gk)
    # Correctness gate (outside timing): both servers' shares XOR to the targets.
    ws.set_keys(tables, k1)
    ws.launch()
    s1 = host_combine(ws.read())
    ws.set_keys(tables, k0)
    ws.launch()
    s0_local = ws.read()
    s0 = host_combine(s0_local)
    if combiner:
        combiner.combine(ws)
        if combiner.out.cpu().numpy().tobytes() != b"".join(s0):
            raise SystemExit("bench: device combine differs from the host combine")
    verified = all(bytes(a ^ b for a, b in zip(x, y)) == row for x, y, row in zip(s0, s1, targets_rows))
    if not verified:
        raise SystemExit("bench: shares do not reconstruct the target rows")
    tuned = None
    budget = args.autotune if autotune is None else autotune
    if budget < 0:
        ws.launch()
        ws.sync()
        budget = 5000 if ws.last_kernel_ns() < 20e6 and args.kernel == "auto" and not pin else 0
    if budget > 0:
        tuned = ws.autotune(budget)
        ws.launch()
        if ws.read() != s0_local:
            raise SystemExit("bench: autotuned shape changed the shares")
    plan = ws.plan()
    if tuned:
        plan["autotuned_ms"] = round(tuned["ms"], 4)

    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    for _ in range(warmup):
        ws.launch(stream=sh, graph=graph)
        if combiner:
            combiner.combine(ws, stream)
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    scan_ns = []
    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(steps):
        ev[i][0].record(stream)
        ws.launch(stream=sh, graph=graph)
        if combiner:
            combiner.combine(ws, stream)
        ev[i][1].record(stream)
        if not graph:
            # Device time of the scan kernels alone (before the reduction);
            # reading it waits for this pass.  A replayed graph is timed as a
            # whole by the step events instead, with no host wait between
            # passes.
            scan_ns.append(ws.last_scan_ns())
    t_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    total_ms = t_start.elapsed_time(t_end)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    if graph:
        scan_ns = [x * 1e6 for x in step_ms]
    if dist:
        tt = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms_per_step = total_ms / steps

    # e2e: host keys in, host shares out, through the one-call C entry point
    # mg_scan (GpuScanner::scan; repeated passes replay from a CUDA graph).
    e2e_ms = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        shares = host_combine(scanner.scan_keys(tables, k0)[0])
        dt = (time.perf_counter() - t0) * 1e3
        if i >= warmup:
            e2e_ms.append(dt)
    if shares != s0:
        raise SystemExit("bench: e2e shares differ")
    e2e_per = sum(e2e_ms) / len(e2e_ms)
    if dist:
        tt = torch.tensor([e2e_per], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_per = float(tt.item())
    ws.close()
    return dict(plan=plan, verified=verified, ms_per_step=ms_per_step, step_ms=step_ms, e2e_ms=e2e_ms,
                e2e_per=e2e_per, scan_avg_s=sum(scan_ns) / len(scan_ns) * 1e-9, clocks=clk, shares0=s0_local,
                steps=steps, warmup=warmup, graph=bool(graph))


def pct3(xs) -> dict:
    a = np.array(xs)
    return {"p50": round(float(np.percentile(a, 50)), 3), "p95": round(float(np.percentile(a, 95)), 3),
            "p99": round(float(np.percentile(a, 99)), 3)}


def rooflines(bytes_scanned: int, nodes: int, seconds: float, prg_peak: float, hbm_peak: float, peaks: dict,
              traffic) -> dict:
    """The dominant kernel against both of its bounds.  `bound` names the
    binding one (the larger fraction); the other sits beside it."""
    a_nodes = nodes / seconds
    a_hbm = bytes_scanned / seconds / 1e9
    alu = {"achieved": round(a_nodes / 1e9, 3), "peak": round(prg_peak / 1e9, 3), "unit": "G node expansions/s",
           "frac": round(a_nodes / prg_peak, 4),
           "peak_source": "mg_prg_peak: device ChaCha8 PRG alone, measured in this run (of measured)"}
    hbm = {"achieved": round(a_hbm, 2), "peak": hbm_peak, "unit": "GB/s", "frac": round(a_hbm / hbm_peak, 4),
           "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "fallback" not in peaks
           else "fallback 6650 GB/s (of fallback)"}
    if alu["frac"] >= hbm["frac"]:
        return {"bound": "alu", "what": "int32 ALU pipe (ChaCha8 node expansions)", **alu, "traffic": traffic,
                "hbm": hbm}
    return {"bound": "hbm", **hbm, "traffic": traffic, "alu": alu}


def traffic_for(traffic_rec: dict, kernel_kind: int, bytes_scanned: int, row_bytes: int = 32):
    """DRAM read + write bytes per launch: the ratio ncu measured on a smaller
    capture of the same kernel (the warp kernel's own-rows and wide-row
    instantiations apart), scaled by the rows scanned."""
    name = "scan_kernel" if kernel_kind != 2 else ("scan_warp_kernel" if row_bytes <= 32 else "scan_warp_kernel_wide")
    rec = traffic_rec.get(name, {})
    if not rec.get("table_bytes"):
        return None
    # Reads grow with the rows scanned; the writes are the per-CTA partial
    # rows and shares, which do not, so they are added as captured.
    return round(rec["dram_read_bytes"] / rec["table_bytes"] * bytes_scanned + rec["dram_write_bytes"])


def run_c1(args, scanner, prg_peak, hbm_peak, peaks, traffic_rec, local_rank) -> dict:
    """The plain single query at 2^20 rows x 256 B (3 x 20-bit keys):
    autotuned shape, passes replayed from a CUDA graph."""
    from morphogen_b200 import gpu_dpf as G
    wl = WORKLOADS["plain20"]
    rows, rb, d = wl["rows"], wl["row_bytes"], wl["d"]
    table = G.GpuPageMatrix.from_seed(scanner, rows, rb, seed=SEED)
    k0, k1, targets = seeded_keys(d, rows, 1)
    m = measure(args, scanner, [table] * 3, k0, k1, target_rows(table, targets, rb, None, local_rank), 1,
                local_rank, None, graph=True, autotune=5000, steps=200, warmup=20)
    nodes = 3 * expansions(0, rows, d)
    bytes_pass = rows * rb
    out = {
        "workload": wl["name"], "keys": 3, "steps": m["steps"], "warmup": m["warmup"], "cuda_graph": True,
        "plan": m["plan"], "ms_per_step": round(m["ms_per_step"], 4),
        "GBps": round(bytes_pass / (m["ms_per_step"] * 1e-3) / 1e9, 2),
        "queries_per_s": round(1e3 / m["ms_per_step"], 1),
        "latency_ms": pct3(m["step_ms"]),
        "e2e": {"value": round(bytes_pass / (m["e2e_per"] * 1e-3) / 1e9, 2), "unit": "GB/s",
                "ms": round(m["e2e_per"], 4), **{f"{k}_ms": v for k, v in pct3(m["e2e_ms"]).items()}},
        "roofline": rooflines(bytes_pass, nodes, m["scan_avg_s"], prg_peak, hbm_peak, peaks,
                              traffic_for(traffic_rec, m["plan"].get("kernel"), bytes_pass, rb)),
        "roofline_note": "a replayed pass is timed as a whole (frontier and scan kernels; the scan reduces in-kernel)",
        "verified": m["verified"], "clocks": m["clocks"], "l2": "table (268 MB) larger than L2 (126 MB)",
    }
    if not args.no_cpu:
        import oracle
        c = cpu_scan_sample(k0, rows, rb, rows, reps=3, base=0)
        sc = cpu_scan_sample(k0, rows, rb, rows, reps=3, base=0, avx512=False)
        out["cpu_baseline"] = cpu_baseline_obj(c, sc)
        host = oracle.fill_splitmix(0, bytes_pass, SEED)
        out["cpu_shares_equal"] = oracle.scan_fused([bytes(k) for k in k0], host, rb, avx512=c["avx512"]) == \
            m["shares0"]
    table.close()
    return out


def run_batched(args, scanner, table, prg_peak, hbm_peak, peaks, local_rank, qlist=(1, 8)) -> dict:
    """Q queries (3 keys each) per pass over the 2^31 x 32 B table.  The
    autotuner runs on a 2^26-row window of the same table with the same keys
    (a full-size candidate pass takes Q x 0.18 s); its shape is kept only if
    it is faster than the planner's on the full table.  Timed passes replay a
    CUDA graph."""
    from morphogen_b200 import gpu_dpf as G
    wl = WORKLOADS["plain31"]
    rows, rb, d = wl["rows"], wl["row_bytes"], wl["d"]
    proxy = G.GpuPageMatrix.from_seed(scanner, PROXY_ROWS, rb, seed=SEED)
    kinds = {1: "cta", 2: "warp"}
    out = {"workload": wl["name"], "tuning": f"autotuned on rows [0, 2^26) of the same table (5 s budget)",
           "points": []}
    for q in qlist:
        k0, k1, targets = seeded_keys(d, rows, q, seed=SEED + 100 + q)
        nk = len(k0)
        wp = scanner.workspace()
        wp.set_keys([proxy] * nk, k0)
        tuned = wp.autotune(5000)
        wp.close()
        cand = (kinds[tuned["kernel"]], tuned["subtree_bits"], tuned["keys_per_cta"])
        # planner's shape vs the proxy's, one full-size pass each
        timings = {}
        for name, pin in (("planner", None), ("autotuned", cand)):
            ws = scanner.workspace()
            if pin:
                ws.set_kernel(pin[0])
                ws.set_shape(pin[1], pin[2])
            ws.set_keys([table] * nk, k0)
            ws.launch()
            ws.sync()
            timings[name] = ws.last_kernel_ns() / 1e6
            ws.close()
        pin = cand if timings["autotuned"] < timings["planner"] else None
        steps, warmup = (5, 2) if q == 1 else (3, 1)
        m = measure(args, scanner, [table] * nk, k0, k1, target_rows(table, targets, rb, None, local_rank), 1,
                    local_rank, None, graph=True, autotune=0, steps=steps, warmup=warmup, pin=pin)
        nodes = nk * expansions(0, rows, d)
        bytes_pass = rows * rb
        out["points"].append({
            "queries_per_pass": q, "keys": nk, "steps": steps, "warmup": warmup, "cuda_graph": True,
            "plan": m["plan"], "shape": "autotuned" if pin else "planner",
            "full_size_candidate_ms": {k: round(v, 2) for k, v in timings.items()},
            "ms_per_pass": round(m["ms_per_step"], 2),
            "queries_per_s": round(q / (m["ms_per_step"] * 1e-3), 3),
            "per_key_GBps": round(nk * bytes_pass / (m["ms_per_step"] * 1e-3) / 1e9, 1),
            "latency_ms": pct3(m["step_ms"]),
            "e2e_queries_per_s": round(q / (m["e2e_per"] * 1e-3), 3),
            "alu_frac": round(nodes / m["scan_avg_s"] / prg_peak, 4),
            "hbm_frac": round(bytes_pass / m["scan_avg_s"] / 1e9 / hbm_peak, 4),
            "verified": m["verified"], "clocks": m["clocks"]})
    proxy.close()
    base = out["points"][0]["queries_per_s"]
    for pt in out["points"]:
        pt["speedup_vs_q1"] = round(pt["queries_per_s"] / base, 3)
    return out


def run_pages(args, scanner, hbm_peak, peaks, traffic_rec, local_rank, pages: int = PAGES) -> dict:
    """Page mode, the reference's own layout: this library's pass against the
    reference's fused_batch_pir_kernel_1 (the server's single-query kernel,
    compiled unmodified for sm_100a into oracle/_ref and launched with the
    reference's recipe) on the same table and keys, shares compared."""
    from morphogen_b200 import gpu_dpf as G
    rb, d = 4096, 25
    table = G.GpuPageMatrix.from_seed(scanner, pages, rb, seed=SEED)
    k0, k1, targets = seeded_keys(d, pages, 1)
    m = measure(args, scanner, [table] * 3, k0, k1, target_rows(table, targets, rb, None, local_rank), 1,
                local_rank, None, graph=True, autotune=5000, steps=20, warmup=5)
    bytes_pass = pages * rb
    ours_best = min(m["step_ms"])
    out = {
        "workload": f"page mode: {pages:,} pages x 4096 B ({bytes_pass / 1e9:.1f} GB), 3 x 25-bit keys",
        "steps": m["steps"], "warmup": m["warmup"], "cuda_graph": True, "plan": m["plan"],
        "ms_per_step": round(m["ms_per_step"], 3), "best_ms": round(ours_best, 3),
        "GBps": round(bytes_pass / (m["ms_per_step"] * 1e-3) / 1e9, 1),
        "latency_ms": pct3(m["step_ms"]),
        "e2e": {"value": round(bytes_pass / (m["e2e_per"] * 1e-3) / 1e9, 1), "unit": "GB/s"},
        "roofline": rooflines(bytes_pass, 3 * expansions(0, pages, d), m["scan_avg_s"], 1e30, hbm_peak, peaks,
                              traffic_for(traffic_rec, m["plan"].get("kernel"), bytes_pass)),
        "verified": m["verified"], "clocks": m["clocks"],
    }
    out["roofline"].pop("alu", None)
    try:
        import oracle
        if not oracle.ref_available():
            raise RuntimeError("oracle/_ref/libmg_refkernels.so was not built")
        shares, ref_best = oracle.ref_scan(0, [bytes(k) for k in k0], table.device_ptr(), pages, reps=5)
        out["reference_kernel"] = {
            "kernel": "fused_batch_pir_kernel_1 (cuda/fused_kernel.cu), compiled for sm_100a, reference launch "
                      "recipe (kernel.rs:293-303,774-787)",
            "best_ms": round(ref_best, 3), "GBps": round(bytes_pass / (ref_best * 1e-3) / 1e9, 1),
            "reps": 5, "shares_equal": shares == m["shares0"],
            "speedup_mean_vs_ref_best": round(ref_best / m["ms_per_step"], 3),
            "speedup_best_vs_best": round(ref_best / ours_best, 3)}
    except Exception as e:  # the baseline leg only; this library's numbers stand
        out["reference_kernel"] = {"unavailable": str(e)}
    table.close()
    return out


def run_pages_line(args, local_rank: int):
    """--workload pages on one GPU: the page-mode point of the default line
    (this library's pass against the reference's kernel on the same table and
    keys) as its own line; --pages sets the page count (profiling cases)."""
    import torch

    from morphogen_b200 import gpu_dpf as G
    torch.cuda.set_device(local_rank)
    scanner = G.GpuScanner(local_rank)
    peaks = measured_peaks()
    try:
        traffic_rec = json.loads((ROOT / "profiles" / "traffic.json").read_text())
    except (OSError, ValueError):
        traffic_rec = {}
    pg = run_pages(args, scanner, float(peaks["hbm_gbs"]), peaks, traffic_rec, local_rank, pages=args.pages)
    line = {"metric": "scanned GB/s", "value": pg["GBps"], "unit": "GB/s", "n_gpus": 1,
            "steps": pg["steps"], "warmup": pg["warmup"], "ms_per_step": pg["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": pg["workload"], "plan": pg["plan"], "cuda_graph": True,
                       "l2": "inputs larger than L2" if args.pages * 4096 > 126e6 else "table fits L2"},
            **{k: v for k, v in pg.items() if k not in ("workload", "plan", "steps", "warmup", "ms_per_step")}}
    print(json.dumps(line), flush=True)


def run_gpu(args, rank: int, world: int, local_rank: int):
    import torch

    from morphogen_b200 import gpu_dpf as G
    from morphogen_b200.shard import ShardCombiner, shard_range

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local_rank)

    wl = WORKLOADS[args.workload]
    rows, rb, d = wl["rows"], wl["row_bytes"], wl["d"]
    sharded = args.workload == "sharded31"
    first, n_local = shard_range(rows, world, rank, 1 << 20) if sharded else (0, rows)
    scanner = G.GpuScanner(local_rank)
    table = G.GpuPageMatrix.from_seed(scanner, n_local, rb, seed=SEED, first_row=first)
    combiner = ShardCombiner(local_rank) if sharded else None
    qlist = [int(q) for q in str(args.queries).split(",")] if args.workload == "batched31" else [1]
    peaks = measured_peaks()
    hbm_peak = float(peaks["hbm_gbs"])
    prg_peak = scanner.prg_peak()
    try:
        traffic_rec = json.loads((ROOT / "profiles" / "traffic.json").read_text())
    except (OSError, ValueError):
        traffic_rec = {}
    bytes_pass = rows * rb
    extras = world == 1 and args.workload == "plain31" and not args.no_extras
    line = None
    for nq in qlist:
        k0, k1, targets = seeded_keys(d, rows, nq)
        nkeys = len(k0)
        m = measure(args, scanner, [table] * nkeys, k0, k1, target_rows(table, targets, rb, dist, local_rank),
                    world, local_rank, dist, combiner)
        plan = m["plan"]
        # Replicas: every rank scans the whole table for its own queries (the
        # aggregate counts each rank's pass).  Sharded: the ranks together
        # scan the table once per pass.
        copies = 1 if sharded else world
        value = copies * bytes_pass / (m["ms_per_step"] * 1e-3) / 1e9
        e2e_value = copies * bytes_pass / (m["e2e_per"] * 1e-3) / 1e9
        # Rooflines of the dominant kernel (this rank's launch): node
        # expansions and bytes of the launch over its CUDA-event time.
        local_bytes = n_local * rb
        nodes = nkeys * expansions(first, n_local, d)
        roof = rooflines(local_bytes, nodes, m["scan_avg_s"], prg_peak, hbm_peak, peaks,
                         traffic_for(traffic_rec, plan.get("kernel"), local_bytes, rb) if nkeys == 3 else None)
        roof["timed"] = "frontier chain + scan kernel of each pass (CUDA events before the reduction)"
        if rank != 0:
            continue
        line = {
            "metric": "scanned GB/s", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(m["ms_per_step"], 3),
            "higher_is_better": True, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": wl["name"], "queries_per_pass": nq, "keys": nkeys,
                       "parallelism": (f"row ranges x{world}" if sharded else f"replicas x{world}")
                       if world > 1 else "single GPU",
                       "rows_per_rank": n_local,
                       "cuda_graph": bool(args.graph), "plan": plan,
                       "l2": "inputs larger than L2" if bytes_pass > 126e6 else "table fits L2"},
            "latency_ms": {**pct3(m["step_ms"]), **{f"e2e_{k}": v for k, v in pct3(m["e2e_ms"]).items()}},
            "queries_per_s": round(copies * nq / (m["ms_per_step"] * 1e-3), 3),
            "per_key_GBps": round(value * nkeys, 2),
            "e2e": {"value": round(e2e_value, 2), "unit": "GB/s",
                    "h2d_bytes_per_step": sum(len(bytes(k)) for k in k0), "d2h_bytes_per_step": nkeys * rb},
            "roofline": roof,
            "gpu_launches": plan["kernels"] * args.steps,
            "clocks": m["clocks"],
            "verified": m["verified"],
        }
        if world == 1 and not args.no_cpu:
            sample = min(CPU_SAMPLE_BYTES // rb, rows)
            c = cpu_scan_sample(k0[:3], rows, rb, sample)
            sc = cpu_scan_sample(k0[:3], rows, rb, sample, avx512=False) if c["avx512"] else None
            line["cpu_baseline"] = cpu_baseline_obj(c, sc)
        if len(qlist) > 1:
            print(json.dumps(line), flush=True)
    if extras and rank == 0:
        line["batched"] = run_batched(args, scanner, table, prg_peak, hbm_peak, peaks, local_rank)
        line["serving"] = run_serving_point(scanner, table, rb, d, rows, local_rank)
        table.close()
        line["c1"] = run_c1(args, scanner, prg_peak, hbm_peak, peaks, traffic_rec, local_rank)
        line["pages"] = run_pages(args, scanner, hbm_peak, peaks, traffic_rec, local_rank)
    if rank == 0 and line is not None and len(qlist) == 1:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_emulated_shards(args, local_rank: int):
    """sharded31 on one GPU, rank by rank: the row range of every rank of an
    R-rank job is created, timed and freed in turn (no collective).  Prints
    one line per R with the slowest range's pass time -- the per-rank compute
    of the R-GPU job; the all-gather of 3 x 32 B is not included."""
    import torch

    from morphogen_b200 import gpu_dpf as G
    from morphogen_b200.shard import shard_range

    torch.cuda.set_device(local_rank)
    wl = WORKLOADS["sharded31"]
    rows, rb, d = wl["rows"], wl["row_bytes"], wl["d"]
    scanner = G.GpuScanner(local_rank)
    k0, k1, targets = seeded_keys(d, rows, 1)
    for R in [int(x) for x in str(args.emulate_ranks).split(",")]:
        per_rank = []
        for r in range(R):
            first, n = shard_range(rows, R, r, 1 << 20)
            t = G.GpuPageMatrix.from_seed(scanner, n, rb, seed=SEED, first_row=first)
            m = measure(args, scanner, [t] * len(k0), k0, k1, target_rows(t, targets, rb, None, local_rank),
                        1, local_rank, None)
            per_rank.append({"first_row": first, "rows": n, "ms_per_step": round(m["ms_per_step"], 3),
                             "e2e_ms": round(m["e2e_per"], 3), "clocks_sm_mhz": m["clocks"]["sm_mhz"]})
            t.close()
        worst = max(x["ms_per_step"] for x in per_rank)
        print(json.dumps({
            "metric": "scanned GB/s (per-rank compute of an R-GPU row-range job, ranks emulated one after another "
                      "on one GPU)", "emulated_ranks": R, "value": round(rows * rb / (worst * 1e-3) / 1e9, 2),
            "unit": "GB/s", "ms_per_step_slowest_rank": worst, "ranks": per_rank,
            "config": {"workload": wl["name"], "keys": len(k0)}}), flush=True)


def run_mixed(args, local_rank: int):
    """Two resident tables in one pass: accounts 2^28 x 64 B (28-bit keys) and
    storage 2^31 x 32 B (31-bit keys); queries per table drawn from U{1..32}."""
    import torch

    from morphogen_b200 import gpu_dpf as G

    torch.cuda.set_device(local_rank)
    scanner = G.GpuScanner(local_rank)
    acc = G.GpuPageMatrix.from_seed(scanner, 1 << 28, 64, seed=SEED)
    sto = G.GpuPageMatrix.from_seed(scanner, 1 << 31, 32, seed=SEED + 1)
    rng = np.random.default_rng(SEED)
    qa, qs = int(rng.integers(1, 33)), int(rng.integers(1, 33))
    a0, a1, at = seeded_keys(28, 1 << 28, qa, seed=SEED + 2)
    s0_, s1_, st_ = seeded_keys(31, 1 << 31, qs, seed=SEED + 3)
    tables = [acc] * len(a0) + [sto] * len(s0_)
    rows = [acc.read_rows(t, 1).tobytes() for t in at] + [sto.read_rows(t, 1).tobytes() for t in st_]
    m = measure(args, scanner, tables, a0 + s0_, a1 + s1_, rows, 1, local_rank, None)
    bytes_pass = (1 << 28) * 64 + (1 << 31) * 32
    nodes = len(a0) * ((1 << 28) - 1) + len(s0_) * ((1 << 31) - 1)
    prg_peak = scanner.prg_peak()
    pct = lambda xs, q: float(np.percentile(np.array(xs), q))  # noqa: E731
    line = {
        "metric": "queries/s, mixed tables in one pass", "value": round((qa + qs) / (m["ms_per_step"] * 1e-3), 3),
        "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(m["ms_per_step"], 3), "higher_is_better": True, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "accounts 2^28 x 64 B (28-bit keys) + storage 2^31 x 32 B (31-bit keys), "
                               "queries per table per pass from U{1..32}",
                   "accounts_queries": qa, "storage_queries": qs, "keys": 3 * (qa + qs), "plan": m["plan"]},
        "scanned_GBps": round(bytes_pass / (m["ms_per_step"] * 1e-3) / 1e9, 2),
        "latency_ms": {"p50": round(pct(m["step_ms"], 50), 3), "e2e_p50": round(pct(m["e2e_ms"], 50), 3)},
        "alu": {"achieved": round(nodes / m["scan_avg_s"] / 1e9, 3), "peak": round(prg_peak / 1e9, 3),
                "unit": "G node expansions/s", "frac": round(nodes / m["scan_avg_s"] / prg_peak, 4)},
        "verified": m["verified"], "clocks": m["clocks"],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mg", choices=["mg", "reference"])
    ap.add_argument("--workload", default="plain31", choices=sorted(WORKLOADS))
    ap.add_argument("--queries", default="1", help="batched31: queries per pass, or a comma list to sweep")
    ap.add_argument("--graph", action="store_true", help="replay the timed passes from a CUDA graph")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--pages", type=int, default=PAGES,
                    help="pages workload: number of 4096-B pages (default: the reference's 16,817,159)")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain31 on one GPU: skip the c1 / batched / pages points of the default line")
    ap.add_argument("--autotune", type=int, default=-1,
                    help="autotuner budget in ms before timing (-1: 5000 when a pass is under 20 ms, else off)")
    ap.add_argument("--rates", default="0.25,0.5,1,2,100",
                    help="serve31: Poisson arrival rates (requests/s) to run")
    ap.add_argument("--duration", type=float, default=20.0, help="serve31: seconds of arrivals per rate")
    ap.add_argument("--overload-duration", type=float, default=1.0,
                    help="serve31: seconds of arrivals for rates above capacity")
    ap.add_argument("--shape", default="",
                    help="pin the launch shape 'S,G' (tile depth, keys per item) instead of the planner's choice")
    ap.add_argument("--emulate-ranks", default="",
                    help="sharded31 on one GPU: time every rank's row range of R-rank jobs (comma list of R)")
    ap.add_argument("--kernel", default="auto", choices=["auto", "cta", "warp"],
                    help="scan kernel for the device-resident passes (default: the planner's choice)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "mg":
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "serve31":
        if rank == 0:
            run_serve(args, local_rank)
    elif args.workload == "sharded31" and args.emulate_ranks and world == 1:
        run_emulated_shards(args, local_rank)
    elif args.workload == "pages" and world == 1:
        run_pages_line(args, local_rank)
    elif args.workload == "mixed":
        if rank == 0:
            run_mixed(args, local_rank)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
