"""CPU tests of the autotuner (batch density, loop schedule) with a fake
engine whose device time depends on the settings."""
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


class FakeScheduleEngine:
    DEFAULT = dict(shift_group=4, missing_group=2, flip_sync=4, flip_tail_enter=4096, flip_tail_leave=32768)

    def __init__(self, cost):
        self.cost = cost
        self.s = dict(self.DEFAULT)
        self.runs = 0

    def schedule(self):
        return dict(self.s)

    def set_schedule(self, sg, mg, fs, te, tl):
        assert tl >= te
        self.s = dict(shift_group=sg, missing_group=mg, flip_sync=fs, flip_tail_enter=te, flip_tail_leave=tl)

    def run(self):
        self.runs += 1
        return FakeStatus(self.cost(self.s))


def test_schedule_descends_to_the_fastest_and_leaves_it_set():
    want = dict(shift_group=8, missing_group=1, flip_sync=16, flip_tail_enter=16384, flip_tail_leave=131072)
    eng = FakeScheduleEngine(lambda s: 100.0 + 10.0 * sum(abs(s[k] - want[k]) / max(1, want[k]) for k in want))
    best, table = A.tune_schedule(eng, eng.run, reps=3)
    assert best == want and eng.s == want
    # every measured schedule is valid (tail leave >= enter) and measured once
    assert all(t[0]["flip_tail_leave"] >= t[0]["flip_tail_enter"] for t in table)
    keys = [tuple(sorted(t[0].items())) for t in table]
    assert len(keys) == len(set(keys))
    assert eng.runs == 4 * len(table)  # one untimed and three timed runs each


def test_schedule_keeps_the_default_within_noise():
    eng = FakeScheduleEngine(lambda s: 100.0 - 0.5 * (s["flip_sync"] == 8))  # 0.5 % better: below min_gain
    best, _ = A.tune_schedule(eng, eng.run, reps=1)
    assert best == FakeScheduleEngine.DEFAULT
