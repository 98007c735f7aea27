"""Host-side logic of the serving helpers, without a GPU: the lookup-count
distribution and the open-loop Poisson generator (driven against a stand-in
server that answers immediately)."""
import numpy as np

from morphogen_b200.server import geometric_lookups, poisson_load


def test_geometric_lookups_bounds_and_mean():
    rng = np.random.default_rng(0)
    xs = [geometric_lookups(rng, mean=4.0, lo=1, hi=32) for _ in range(20000)]
    assert min(xs) >= 1 and max(xs) <= 32
    assert 3.6 < float(np.mean(xs)) < 4.3


class _FakeServer:
    def __init__(self):
        self.submitted, self.waited, self.resets = [], [], 0

    def reset_stats(self):
        self.resets += 1

    def submit(self, items):
        self.submitted.append(items)
        return len(self.submitted) - 1

    def wait(self, rid, timeout_ms=0):
        self.waited.append(rid)
        return [b""] * len(self.submitted[rid]), 1.0

    def stats(self):
        return {"keys_completed": sum(len(x) for x in self.submitted), "wall_s": 0.5}


def test_poisson_load_submits_at_the_offered_rate_and_waits_for_all():
    srv = _FakeServer()
    ticks = []
    st = poisson_load(srv, lambda rng: [("t", b"k")] * int(rng.integers(1, 4)), rate_hz=400, duration_s=0.25,
                      seed=3, tick=ticks.append)
    n = len(srv.submitted)
    assert 50 < n < 160  # ~100 arrivals expected
    assert sorted(srv.waited) == list(range(n)) and srv.resets == 1
    assert st["requests"] == n and st["keys"] == sum(len(x) for x in srv.submitted)
    assert ticks and all(0 <= t <= 0.5 for t in ticks)
