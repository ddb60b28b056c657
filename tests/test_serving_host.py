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
