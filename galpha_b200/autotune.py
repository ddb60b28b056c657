"""Autotuner: picks the texture density of batches (pixels per point of each
set's cell, galphaSetBatchDensity) and the loop schedule of a handle
(galphaSetSchedule: rounds per counter read of the shifting, missing-site and
flip loops, and the flip-tail hand-over lengths) that minimise the measured
device time of a workload.

Fewer pixels per point mean fewer pixels for the Voronoi colouring; more
points then share a pixel and are inserted afterwards (missing sites), which
costs point location and flips.  Where the balance lies depends on the set
sizes and distributions, so it is measured: each candidate density runs the
sample batch `reps` times through Engine.run_batch and the device time of
the whole pipeline (gpudtStatus.ms[total], CUDA events) is compared.  A set's
result does not depend on the density.

    best, table = tune_batch_density(engine, sample_sets)
    engine.set_batch_density(best)

The schedule changes no result either (a round past the end of a loop does
nothing; the in-block flip rounds run the launched rounds' functors); it
trades counter reads, each a stream synchronisation, against rounds launched
past a loop's end.  tune_schedule walks the five parameters one at a time
(coordinate descent over SCHEDULE_CANDIDATES), timing `run()` -- any callable
that runs the workload on the engine and returns its gpudtStatus -- by the
median device time of `reps` runs, and moves off the value in force only for
a gain above `min_gain`:

    sched, table = tune_schedule(engine, lambda: engine.run_batch(sets))
"""
import json

DEFAULT_CANDIDATES = (3.0, 4.0, 5.0, 6.0, 8.0, 10.0, 14.0)
STAGE_TOTAL = 10  # gpudtStatus.ms index of the whole pipeline


def tune_batch_density(engine, sets, bounds=None, candidates=DEFAULT_CANDIDATES, reps=2, with_alpha=True):
    """Returns (best density, [(density, mean device ms), ...]) and leaves the
    engine set to the best density."""
    if not candidates:
        raise ValueError("no candidate densities")
    table = []
    for d in candidates:
        engine.set_batch_density(d)
        engine.run_batch(sets, bounds=bounds, with_alpha=with_alpha)  # arena growth, first-touch
        ms = []
        for _ in range(max(1, reps)):
            st = engine.run_batch(sets, bounds=bounds, with_alpha=with_alpha)
            ms.append(float(st.ms[STAGE_TOTAL]))
        table.append((float(d), sum(ms) / len(ms)))
    best = min(table, key=lambda t: (t[1], t[0]))[0]
    engine.set_batch_density(best)
    return best, table


SCHEDULE_KEYS = ("shift_group", "missing_group", "flip_sync", "flip_tail_enter", "flip_tail_leave")
SCHEDULE_CANDIDATES = {
    "shift_group": (1, 2, 4, 8),
    "missing_group": (1, 2, 4),
    "flip_sync": (2, 4, 8, 16),
    "flip_tail_enter": (0, 1024, 4096, 16384),
    "flip_tail_leave": (8192, 32768, 131072),
}


def _valid(s):
    return s["flip_tail_leave"] >= s["flip_tail_enter"]


def tune_schedule(engine, run, candidates=None, reps=3, min_gain=0.01):
    """Returns (best schedule dict, [(schedule, median device ms), ...]) and
    leaves the engine set to the best schedule."""
    cand = dict(SCHEDULE_CANDIDATES)
    if candidates:
        cand.update(candidates)
    cur = dict(engine.schedule())
    table = []
    cache = {}

    def measure(s):
        key = tuple(s[k] for k in SCHEDULE_KEYS)
        if key not in cache:
            engine.set_schedule(*key)
            run()  # first run of a schedule: untimed
            ms = sorted(float(run().ms[STAGE_TOTAL]) for _ in range(max(1, reps)))
            cache[key] = ms[len(ms) // 2]
            table.append((dict(s), cache[key]))
        return cache[key]

    best_ms = measure(cur)
    for k in SCHEDULE_KEYS:
        for v in cand[k]:
            trial = dict(cur)
            trial[k] = v
            if trial == cur or not _valid(trial):
                continue
            ms = measure(trial)
            if ms < best_ms * (1.0 - min_gain):
                cur, best_ms = trial, ms
    engine.set_schedule(*(cur[k] for k in SCHEDULE_KEYS))
    return cur, table


def save(path, best, table, workload=""):
    with open(path, "w") as f:
        json.dump({"batch_density": best, "table": table, "workload": workload}, f, indent=1)


def load(path):
    with open(path) as f:
        return json.load(f)["batch_density"]
