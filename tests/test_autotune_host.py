"""CPU tests of the batch-density autotuner with a fake engine whose device
time depends on the density."""
import json

import numpy as np
import pytest

from galpha_b200 import autotune as A


class FakeStatus:
    def __init__(self, ms):
        self.ms = [0.0] * 12
        self.ms[A.STAGE_TOTAL] = ms


class FakeEngine:
    def __init__(self, cost):
        self.cost = cost
        self.density = 10.0
        self.calls = []

    def set_batch_density(self, d):
        assert 1.0 <= d <= 64.0
        self.density = d

    def run_batch(self, sets, bounds=None, with_alpha=True):
        self.calls.append(self.density)
        return FakeStatus(self.cost(self.density))


def test_picks_fastest_and_leaves_it_set():
    eng = FakeEngine(lambda d: (d - 5.0) ** 2 + 100.0)
    best, table = A.tune_batch_density(eng, [np.zeros((10, 2))], reps=3)
    assert best == 5.0 and eng.density == 5.0
    assert [t[0] for t in table] == list(A.DEFAULT_CANDIDATES)
    # one warm-up and `reps` timed runs per candidate
    assert len(eng.calls) == 4 * len(A.DEFAULT_CANDIDATES)


def test_ties_go_to_the_lower_density_and_roundtrip(tmp_path):
    eng = FakeEngine(lambda d: 1.0)
    best, table = A.tune_batch_density(eng, [], candidates=(8.0, 4.0, 6.0), reps=1)
    assert best == 4.0
    p = tmp_path / "tune.json"
    A.save(str(p), best, table, "fake")
    assert A.load(str(p)) == 4.0 and json.load(open(p))["workload"] == "fake"
    with pytest.raises(ValueError):
        A.tune_batch_density(eng, [], candidates=())
