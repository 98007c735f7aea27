"""The continuous-batching answer loop: every request's shares are the same
when it is answered alone and when it is folded into passes with other
requests (tolerance: bit-exact), epoch merges drain and patch while
requests keep arriving, deadlines and bad input fail cleanly."""
import numpy as np
import pytest

from conftest import oracle_keypair, xor_bytes

from morphogen_b200 import _native as N
from morphogen_b200 import gpu_dpf as G
from morphogen_b200.server import PirServer, geometric_lookups, poisson_load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables(scanner):
    import oracle
    a_host = oracle.fill_splitmix(0, (1 << 18) * 32, 201).reshape(-1, 32)
    b_host = oracle.fill_splitmix(0, 20_000 * 64, 202).reshape(-1, 64)
    a = G.GpuPageMatrix.new(scanner, a_host, 32)
    b = G.GpuPageMatrix.new(scanner, b_host, 64)
    return (a, a_host, 18), (b, b_host, 15)


def make_requests(oracle_mod, tables, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for r in range(n):
        items = []
        for q in range(geometric_lookups(rng, mean=2.0, hi=5)):
            t, host, d = tables[int(rng.integers(0, 2))]
            for j in range(3):
                target = int(rng.integers(0, host.shape[0]))
                k0, _ = oracle_keypair(oracle_mod, d, target, seed=seed * 1000 + r, i=10 * q + j)
                items.append((t, k0))
        reqs.append(items)
    return reqs


def test_each_result_is_the_same_alone_and_in_the_mix(scanner, oracle_mod, tables):
    reqs = make_requests(oracle_mod, tables, 16, seed=1)
    srv = PirServer(scanner, slots=2)
    alone = [srv.answer(items) for items in reqs]
    assert srv.stats()["passes"] == len(reqs)
    # Mix 1: everything arrives while dispatch is held, then is folded into
    # as few passes as the workspaces allow.
    srv.reset_stats()
    srv.pause()
    ids = [srv.submit(items) for items in reqs]
    srv.resume()
    mixed = [srv.wait(i)[0] for i in ids]
    st = srv.stats()
    assert mixed == alone
    assert st["completed"] == len(reqs) and st["passes"] <= 2
    srv.close()
    # Mix 2: a cap of 12 keys per pass splits the same requests into several
    # passes that overlap on the two workspaces' streams.
    srv = PirServer(scanner, slots=2, max_keys_per_pass=12)
    srv.pause()
    ids = [srv.submit(items) for items in reqs]
    srv.resume()
    mixed2 = [srv.wait(i)[0] for i in ids]
    st2 = srv.stats()
    assert mixed2 == alone
    assert 2 < st2["passes"] < len(reqs)
    # and both equal the oracle
    for items, shares in zip(reqs[:4], alone):
        for (t, k), s in zip(items, shares):
            host = tables[0][1] if t is tables[0][0] else tables[1][1]
            assert s == oracle_mod.scan_fused([k], host, t.row_bytes)[0]
    srv.close()


def test_merge_while_serving(scanner, oracle_mod):
    rb, nrows, d = 32, 1 << 16, 16
    host = oracle_mod.fill_splitmix(0, nrows * rb, 300).reshape(nrows, rb).copy()
    t = G.GpuPageMatrix.new(scanner, host, rb)
    t.delta_reserve(1 << 12)
    srv = PirServer(scanner, slots=3)
    pairs = [oracle_keypair(oracle_mod, d, 4000 + j, seed=301, i=j) for j in range(3)]
    before = srv.answer([(t, p[0]) for p in pairs])
    idx = np.arange(4000, 4003, dtype=np.uint64)
    diffs = oracle_mod.fill_splitmix(5, 3 * rb, 302).reshape(3, rb)
    t.delta_push(idx, diffs)
    pending = [srv.submit([(t, p[0]) for p in pairs]) for _ in range(4)]
    srv.merge([t])  # drains the passes on the GPU, patches, resumes
    after = srv.answer([(t, p[0]) for p in pairs])
    delta = oracle_mod.delta_apply([p[0] for p in pairs], idx, diffs, rb)
    want = [xor_bytes(a, b) for a, b in zip(before, delta)]
    for rid in pending:  # answered before or after the merge: same (delta or merged)
        assert srv.wait(rid)[0] == want
    assert after == want and t.delta_count() == 0 and t.epoch() == 1
    other = srv.answer([(t, p[1]) for p in pairs])
    for j in range(3):
        assert xor_bytes(after[j], other[j]) == (host[4000 + j] ^ diffs[j]).tobytes()
    srv.close()


def test_poisson_load_generator_answers_everything(scanner, oracle_mod, tables):
    reqs = make_requests(oracle_mod, tables, 8, seed=2)
    srv = PirServer(scanner, slots=2)
    st = poisson_load(srv, lambda rng: reqs[int(rng.integers(0, len(reqs)))], rate_hz=400, duration_s=0.3)
    assert st["failed"] == 0 and st["completed"] == st["requests"] > 0
    assert st["p50_ms"] <= st["p95_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()


def test_deadline_and_bad_input(scanner, oracle_mod):
    big = G.GpuPageMatrix.from_seed(scanner, 1 << 26, 32, seed=5)
    srv = PirServer(scanner, slots=1)
    keys = [oracle_keypair(oracle_mod, 26, 9 + j, seed=6, i=j)[0] for j in range(3)]
    rid = srv.submit([(big, k) for k in keys])
    with pytest.raises(N.Timeout):
        srv.wait(rid, timeout_ms=1)
    shares, lat = srv.wait(rid)  # still answered afterwards
    assert len(shares) == 3 and lat > 0
    with pytest.raises(G.GpuDpfError):
        srv.submit([(big, keys[0][:-1])])
    small_key = oracle_keypair(oracle_mod, 20, 3, seed=7)[0]
    with pytest.raises(G.GpuDpfError):  # more rows than the key's domain
        srv.submit([(big, small_key)])
    srv.close()
    big.close()


def test_destroy_wakes_a_blocked_waiter_with_ebusy(scanner, oracle_mod, tables):
    import threading
    srv = PirServer(scanner, slots=1)
    srv.pause()  # the request stays pending: it is never dispatched
    items = make_requests(oracle_mod, tables, 1, seed=3)[0]
    rid = srv.submit(items)
    got = {}

    def waiter():
        try:
            srv.wait(rid)
            got["rc"] = N.MG_OK
        except N.MgError as e:
            got["rc"] = e.code

    th = threading.Thread(target=waiter)
    th.start()
    th.join(0.2)
    assert th.is_alive()  # blocked in mg_server_wait
    srv.close()  # destroy: the waiter wakes with MG_EBUSY before anything is freed
    th.join(10)
    assert not th.is_alive() and got["rc"] == N.MG_EBUSY


def test_submit_is_not_held_up_by_planning(scanner, oracle_mod):
    # A 96-key pass of 31-bit keys is parsed, planned, staged and launched by
    # the dispatcher with the server's mutex released, so submissions made
    # meanwhile return at once.
    import ctypes as C
    import time
    big = G.GpuPageMatrix.from_seed(scanner, 1 << 24, 32, seed=8)
    srv = PirServer(scanner, slots=2)
    keys = [oracle_keypair(oracle_mod, 31, (2654435761 * j) % (1 << 24), seed=9, i=j)[0] for j in range(96)]
    first = srv.submit([(big, k) for k in keys])
    small = [(big, k) for k in keys[:3]]
    ka = N.KeyArray([bytes(k) for _, k in small])
    tarr = (C.c_void_p * ka.n)(*[t.handle.value for t, _ in small])
    rid = C.c_uint64()
    ids, took = [], []
    t_end = time.perf_counter() + 0.1
    while time.perf_counter() < t_end:
        t0 = time.perf_counter()
        rc = N.lib().mg_server_submit(srv.handle, tarr, ka.ptrs, ka.lens, ka.n, C.byref(rid))
        took.append(time.perf_counter() - t0)
        N.check(rc)
        srv._share_bytes[rid.value] = [32] * 3
        ids.append(rid.value)
        time.sleep(0.001)
    assert max(took) < 1e-3, f"slowest submit {max(took) * 1e3:.3f} ms"
    shares = srv.wait(first)[0]
    assert len(shares) == 96
    alone = scanner.scan_keys(big, keys[:3])[0]
    for i in ids:
        assert srv.wait(i)[0] == alone
    srv.close()
    big.close()


def test_default_pass_size_follows_the_measured_rate(scanner, oracle_mod):
    # max_keys_per_pass = 0: once a pass has been timed, a backlog whose
    # estimated device time is above 50 ms is split into several passes.
    t = G.GpuPageMatrix.from_seed(scanner, 1 << 24, 32, seed=10)
    srv = PirServer(scanner, slots=1)
    keys = [oracle_keypair(oracle_mod, 24, (40503 * j) % (1 << 24), seed=11, i=j)[0] for j in range(120)]
    alone = srv.answer([(t, k) for k in keys[:3]])  # times one pass
    srv.reset_stats()
    srv.pause()
    ids = [srv.submit([(t, k) for k in keys[3 * i:3 * i + 3]]) for i in range(40)]
    srv.resume()
    res = [srv.wait(i)[0] for i in ids]
    st = srv.stats()
    assert st["completed"] == 40 and st["passes"] >= 2
    assert res[0] == alone
    srv.close()
    t.close()
