"""The multi-GPU path on CPU: two gloo ranks each answer the same keys over
their row range of one table (the oracle stands in for the GPU), all-gather
and XOR their shares, and obtain the share of the whole table."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from morphogen_b200.shard import shard_range, xor_shares


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch.distributed as dist

    import oracle
    from conftest import oracle_keypair
    from morphogen_b200.shard import combine_shares, shard_range

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    rows, rb, d = 10_000, 32, 14
    first, count = shard_range(rows, world, rank, align=512)
    host = oracle.fill_splitmix(first * rb, count * rb, 9)
    keys = [oracle_keypair(oracle, d, t, seed=12, i=t)[0] for t in (3, 5000, 9999)]
    local = oracle.scan_fused(keys, host, rb, row_base=first)
    full = combine_shares(local)
    # The tensor form the device combiner uses (here on host tensors).
    import torch
    from morphogen_b200.shard import combine_tensor
    lt = torch.from_numpy(np.frombuffer(b"".join(local), np.uint8).copy())
    out = torch.empty_like(lt)
    combine_tensor(lt, torch.empty(world * lt.numel(), dtype=torch.uint8), out, world)
    if rank == 0:
        whole = oracle.scan_fused(keys, oracle.fill_splitmix(0, rows * rb, 9), rb)
        q.put(full == whole and out.numpy().tobytes() == b"".join(whole))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range_partitions_the_rows():
    for total, world, align in [(10_000, 2, 512), (1 << 31, 8, 1 << 20), (7, 3, 1), (100, 4, 64)]:
        spans = [shard_range(total, world, r, align) for r in range(world)]
        assert spans[0][0] == 0 and sum(c for _, c in spans) == total
        for (f0, c0), (f1, _) in zip(spans, spans[1:]):
            assert f0 + c0 == f1 and f1 % align == 0


def test_xor_shares():
    a = [bytes([1, 2]), bytes([3])]
    b = [bytes([1, 0]), bytes([5])]
    assert xor_shares([a, b]) == [bytes([0, 2]), bytes([6])]


def test_two_gloo_ranks_combine_to_the_whole_table_share():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True
