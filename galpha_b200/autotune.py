"""Autotuner for the batched pipeline: picks the texture density (pixels per
point of each set's cell, galphaSetBatchDensity) that minimises the device
time of a batch.

Fewer pixels per point mean fewer pixels for the Voronoi colouring; more
points then share a pixel and are inserted afterwards (missing sites), which
costs point location and flips.  Where the balance lies depends on the set
sizes and distributions, so it is measured: each candidate density runs the
sample batch `reps` times through Engine.run_batch and the device time of
the whole pipeline (gpudtStatus.ms[total], CUDA events) is compared.  A set's
result does not depend on the density.

    best, table = tune_batch_density(engine, sample_sets)
    engine.set_batch_density(best)
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


def save(path, best, table, workload=""):
    with open(path, "w") as f:
        json.dump({"batch_density": best, "table": table, "workload": workload}, f, indent=1)


def load(path):
    with open(path) as f:
        return json.load(f)["batch_density"]
