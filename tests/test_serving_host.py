"""CPU tests of the serving loop's host logic (admission, batching, query
fan-out, latency bookkeeping) with a fake engine and a simulated clock."""
import numpy as np

from galpha_b200 import serving as S


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, d):
        self.t += d


class FakeEngine:
    """Stands in for Engine: each batch costs 1 ms + 1 us per point."""

    def __init__(self, clock):
        self.clock = clock
        self.batches = []
        self.queries = []

    def run_batch(self, sets, bounds=None):
        assert bounds is not None and len(bounds) == len(sets)
        self.batches.append([len(p) for p in sets])
        self.clock.t += 1e-3 + 1e-6 * sum(len(p) for p in sets)

    def batch_query(self, values, by_quantile=False):
        assert by_quantile
        self.queries.append(list(values))
        return [("q", v) for v in values]


def _requests(n, rate, seed, size=1000):
    t = S.poisson_arrivals(rate, n / rate * 2, seed)[:n]
    return [S.Request(i, t[i], np.zeros((size, 2))) for i in range(len(t))]


def test_every_request_served_with_its_queries():
    clk = FakeClock()
    eng = FakeEngine(clk)
    reqs = _requests(200, 1000.0, 1)
    srv = S.Server(eng, hbm_budget=1e12, max_batch_points=10**9)
    srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert all(r.done is not None and r.done >= r.arrival for r in reqs)
    assert all([x[1] for x in r.results] == [0.1, 0.5, 0.9] for r in reqs)
    assert sum(len(b) for b in eng.batches) == len(reqs)
    # three query launches per batch, one value per request of the batch
    assert len(eng.queries) == 3 * len(eng.batches)
    s = S.summary(reqs, srv.batches)
    assert s["requests"] == 200 and s["p50_ms"] <= s["p99_ms"]


def test_admission_respects_budget():
    clk = FakeClock()
    eng = FakeEngine(clk)
    reqs = [S.Request(i, 0.0, np.zeros((3000, 2))) for i in range(10)]
    srv = S.Server(eng, hbm_budget=7000 * S.BYTES_PER_POINT, max_batch_points=10**9)
    srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert all(sum(b) <= 7000 for b in eng.batches)
    assert [len(b) for b in eng.batches] == [2, 2, 2, 2, 2]


def test_oversized_request_runs_alone():
    clk = FakeClock()
    eng = FakeEngine(clk)
    reqs = [S.Request(0, 0.0, np.zeros((50, 2))), S.Request(1, 0.0, np.zeros((500, 2)))]
    srv = S.Server(eng, hbm_budget=1e12, max_batch_points=100)
    srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert eng.batches == [[50], [500]]


def test_fifo_and_latency_accounting():
    clk = FakeClock()
    eng = FakeEngine(clk)
    reqs = [S.Request(i, 0.01 * i, np.zeros((100, 2))) for i in range(5)]
    S.Server(eng).run(reqs, clock=clk, sleep=clk.sleep)
    order = [n for b in eng.batches for n in b]
    assert len(order) == 5
    for r in reqs:
        assert abs(r.latency - (r.done - r.arrival)) < 1e-12 and r.latency > 0


class SleepEngine:
    """A slot that takes real time (5 ms + 0.1 us per point) per batch; records
    how many slots were busy at once."""

    busy = 0
    peak = 0
    lock = None

    def __init__(self, fail=False):
        self.batches = []
        self.fail = fail

    def run_batch(self, sets, bounds=None):
        import time

        assert bounds is not None and len(bounds) == len(sets)
        with SleepEngine.lock:
            SleepEngine.busy += 1
            SleepEngine.peak = max(SleepEngine.peak, SleepEngine.busy)
        try:
            if self.fail:
                raise RuntimeError("slot failed")
            time.sleep(5e-3 + 1e-7 * sum(len(p) for p in sets))
            self.batches.append([len(p) for p in sets])
            self._last = [len(p) for p in sets]
        finally:
            with SleepEngine.lock:
                SleepEngine.busy -= 1

    def batch_query(self, values, by_quantile=False):
        return [(n, v) for n, v in zip(self._last, values)]


def _reset_sleep_engines():
    import threading

    SleepEngine.busy = SleepEngine.peak = 0
    SleepEngine.lock = threading.Lock()


def test_slots_overlap_and_serve_every_request_once():
    _reset_sleep_engines()
    slots = [SleepEngine(), SleepEngine(), SleepEngine()]
    rng = np.random.default_rng(3)
    reqs = [S.Request(i, 0.0 if i < 12 else 0.002 * i, np.zeros((int(rng.integers(100, 3000)), 2)))
            for i in range(40)]
    srv = S.Server(slots, max_batch_points=4000)
    srv.run(reqs)
    # every request answered exactly once, by the batch that held it
    assert all(r.done is not None and r.done >= r.start >= r.arrival - 1e-9 for r in reqs)
    assert all([x for x in r.results] == [(len(r.points), q) for q in (0.1, 0.5, 0.9)] for r in reqs)
    served = sorted(n for e in slots for b in e.batches for n in b)
    assert served == sorted(len(r.points) for r in reqs)
    assert all(sum(b) <= 4000 or len(b) == 1 for e in slots for b in e.batches)
    # the burst at t = 0 kept several slots busy at once, and batch intervals overlap
    assert SleepEngine.peak >= 2
    iv = sorted((b[0], b[1], b[4]) for b in srv.batches)
    assert any(a[2] != b[2] and b[0] < a[1] for a, b in zip(iv, iv[1:]))
    assert len({b[4] for b in srv.batches}) >= 2


def test_slot_budget_share():
    _reset_sleep_engines()
    slots = [SleepEngine(), SleepEngine()]
    reqs = [S.Request(i, 0.0, np.zeros((3000, 2))) for i in range(8)]
    srv = S.Server(slots, hbm_budget=2 * 7000 * S.BYTES_PER_POINT, max_batch_points=10**9)
    assert srv.max_points == 7000
    srv.run(reqs)
    assert all(sum(b) <= 7000 for e in slots for b in e.batches)
    assert sum(len(b) for e in slots for b in e.batches) == 8


def test_failing_slot_raises_after_the_others_finish():
    import pytest

    _reset_sleep_engines()
    slots = [SleepEngine(), SleepEngine(fail=True)]
    reqs = [S.Request(i, 0.0, np.zeros((2000, 2))) for i in range(6)]
    srv = S.Server(slots, max_batch_points=2000)
    with pytest.raises(RuntimeError, match="slot failed"):
        srv.run(reqs)
    assert SleepEngine.busy == 0


def test_warm_runs_every_slot():
    _reset_sleep_engines()
    slots = [SleepEngine(), SleepEngine()]
    sets = [np.zeros((100, 2)), np.zeros((50, 2))]
    slots[0]._last = slots[1]._last = [0, 0]
    S.Server(slots).warm(sets, bounds=np.zeros((2, 4)))
    assert all(e.batches == [[100, 50]] for e in slots)
