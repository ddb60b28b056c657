"""Request loop for DT + alpha-spectrum requests (the serving form of the engine).

Requests arrive over time, each a point set followed by alpha queries at
spectrum quantiles.  The server owns one or more slots: an Engine each (one
library handle = one CUDA stream + one device arena).  Whenever a slot is
free, every request that has arrived is admitted into one micro-batch for it,
bounded by the slot's share of the device-memory budget; the batch runs
through one batched pipeline pass (``Engine.run_batch``: DT + spectrum of
every set at once) and its queries are answered on the meshes while they are
still resident (``Engine.batch_query``, all sets at once per query).  With
two or more slots this is continuous batching: requests that arrive while
batches are on the GPU go to the next slot that frees up, and the slots'
batches overlap on the device (separate streams) and on the host (staging of
one batch while another computes).  Each request's latency runs from its
arrival to the end of its batch.

The reference has no serving path: it computes one set per
gpudtComputeDT / Alpha_Shapes_2D call on the default stream.
"""
import collections
import threading
import time

import numpy as np

# Device bytes per point of a batched run with alpha: texture cells (about 10
# to 40 pixels per point at 10 B per pixel), triangle slots (2 per vertex with
# their links, free lists and relink records) and the alpha arrays.
BYTES_PER_POINT = 2048


class Request:
    """A DT + alpha-spectrum request: points, their bounds (minX, minY, maxX,
    maxY, as the caller fills GPUDTPARAMS; computed if not given) and the
    spectrum quantiles to query on the resulting mesh."""
    __slots__ = ("rid", "arrival", "points", "bounds", "quantiles", "start", "done", "results")

    def __init__(self, rid, arrival, points, quantiles=(0.1, 0.5, 0.9), bounds=None):
        self.rid = rid
        self.arrival = float(arrival)
        self.points = points
        if bounds is None and len(points):
            x, y = points[:, 0], points[:, 1]
            bounds = (x.min(), y.min(), x.max(), y.max())
        self.bounds = bounds if bounds is not None else (0.0, 0.0, 1.0, 1.0)
        self.quantiles = tuple(quantiles)
        self.start = None
        self.done = None
        self.results = None

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


def poisson_arrivals(rate, duration, seed):
    """Arrival times of a Poisson stream (rate per second) over [0, duration)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.array(out)
        out.append(t)


class Server:
    """Continuous-batching request loop on one device.

    slots: an Engine or a list of Engines (each its own stream and arena);
    hbm_budget: device bytes all slots together may use -- each slot admits
    batches of at most hbm_budget / len(slots) / bytes_per_point points (an
    arena keeps the size of the largest batch it ran, so the per-slot share
    bounds the total); max_batch_points: an additional cap that bounds the
    latency of a batch.  A request larger than the cap runs alone.
    """

    def __init__(self, slots, hbm_budget=120e9, max_batch_points=1 << 25, bytes_per_point=BYTES_PER_POINT):
        self.slots = list(slots) if isinstance(slots, (list, tuple)) else [slots]
        if not self.slots:
            raise ValueError("Server needs at least one engine")
        self.engine = self.slots[0]
        share = hbm_budget // (len(self.slots) * bytes_per_point)
        self.max_points = int(min(max_batch_points, share))
        self.batches = []  # (start, done, requests, points, slot)

    def warm(self, sets, bounds=None):
        """Runs a representative batch (the largest expected) on every slot, so
        that device arenas and pinned staging buffers are grown before the
        first request rather than inside its latency."""
        for e in self.slots:
            e.run_batch(sets, bounds=bounds)
            e.batch_query([0.5] * len(sets), by_quantile=True)

    def _admit(self, queue):
        batch, pts = [], 0
        while queue:
            n = len(queue[0].points)
            if batch and pts + n > self.max_points:
                break
            batch.append(queue.popleft())
            pts += n
        return batch, pts

    def _execute(self, slot, batch, pts, t0, clock):
        eng = self.slots[slot]
        start = clock() - t0
        eng.run_batch([r.points for r in batch], bounds=np.array([r.bounds for r in batch], np.float64))
        nq = max(len(r.quantiles) for r in batch)
        answers = []
        for k in range(nq):
            qs = [r.quantiles[k] if k < len(r.quantiles) else r.quantiles[-1] for r in batch]
            answers.append(eng.batch_query(qs, by_quantile=True))
        done = clock() - t0
        for i, r in enumerate(batch):
            r.start = start
            r.done = done
            r.results = [answers[k][i] for k in range(len(r.quantiles))]
        self.batches.append((start, done, len(batch), pts, slot))

    def run(self, requests, clock=time.perf_counter, sleep=time.sleep):
        """Serve requests (sorted by arrival, times in seconds from the start of
        the run) in real time; returns them with start/done/results filled."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue = collections.deque()
        t0 = clock()
        if len(self.slots) == 1:
            while pending or queue:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.popleft())
                if not queue:
                    sleep(max(0.0, pending[0].arrival - now))
                    continue
                batch, pts = self._admit(queue)
                self._execute(0, batch, pts, t0, clock)
            return requests
        return self._run_slots(requests, pending, queue, t0, clock)

    def _run_slots(self, requests, pending, queue, t0, clock):
        cv = threading.Condition()
        idle = list(range(len(self.slots)))
        failures, workers = [], []

        def work(slot, batch, pts):
            try:
                self._execute(slot, batch, pts, t0, clock)
            except BaseException as e:  # reported by run() once every slot is idle
                failures.append(e)
            finally:
                with cv:
                    idle.append(slot)
                    cv.notify_all()

        with cv:
            while True:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.popleft())
                if queue and idle and not failures:
                    slot = min(idle)
                    idle.remove(slot)
                    batch, pts = self._admit(queue)
                    th = threading.Thread(target=work, args=(slot, batch, pts), daemon=True)
                    th.start()
                    workers.append(th)
                    continue
                if len(idle) == len(self.slots) and (failures or not (pending or queue)):
                    break
                # wake on the next arrival (when there is nothing to admit yet) or a freed slot
                timeout = max(0.0, pending[0].arrival - now) if pending and not queue else None
                cv.wait(timeout)
        for th in workers:
            th.join()
        if failures:
            raise failures[0]
        return requests


def summary(requests, batches=None):
    """p50 / p99 latency (ms), served requests and points per second."""
    lat = np.array([r.latency for r in requests if r.latency is not None])
    pts = sum(len(r.points) for r in requests if r.done is not None)
    span = max(r.done for r in requests) - min(r.arrival for r in requests) if len(lat) else 0.0
    out = {
        "requests": int(len(lat)),
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
        "mean_ms": float(lat.mean() * 1e3) if len(lat) else None,
        "requests_per_s": float(len(lat) / span) if span > 0 else None,
        "mpoints_per_s": float(pts / span / 1e6) if span > 0 else None,
    }
    if batches:
        out["batches"] = len(batches)
        out["mean_batch_requests"] = float(np.mean([b[2] for b in batches]))
    return out
