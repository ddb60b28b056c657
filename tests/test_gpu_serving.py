"""GPU test of the serving loop: a request stream served by continuous batching
on two slots (two handles, two streams); every request's quantile queries
agree with a separate run of its set alone (integer counts and spectrum
values: zero tolerance)."""
import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from galpha_b200 import serving as S

pytestmark = pytest.mark.gpu


def _alone(engine, r):
    fbo = 256
    while fbo < 4096 and fbo * fbo < 16 * len(r.points):
        fbo *= 2
    engine.triangulate(G.GPUDTParams(r.points, fboSize=fbo))
    engine.alpha_resident()
    return [engine.query(quantile=q) for q in r.quantiles]


def test_serving_stream_matches_single_runs(engine):
    rng = np.random.default_rng(5)
    # a burst at t = 0 (several batches at once: both slots busy) then a Poisson stream
    arrivals = np.concatenate([np.zeros(8), 0.02 + S.poisson_arrivals(400.0, 0.08, 7)])
    reqs = []
    for i, t in enumerate(arrivals):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(20000))))
        pts = D.uniform_points(n, 100 + i) if i % 2 == 0 else D.gaussian_blobs(n, 100 + i)
        qs = (0.1, 0.5, 0.9) if i % 3 else (0.0, 0.25, 1.0)
        reqs.append(S.Request(i, t, pts, quantiles=qs))
    slots = [G.Engine(), G.Engine()]
    try:
        srv = S.Server(slots, max_batch_points=40000)
        srv.run(reqs)
    finally:
        for e in slots:
            e.close()
    s = S.summary(reqs, srv.batches)
    assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0
    # both slots ran batches, and batches of different slots were in flight together
    assert {b[4] for b in srv.batches} == {0, 1}
    iv = sorted((b[0], b[1], b[4]) for b in srv.batches)
    assert any(a[2] != b[2] and b[0] < a[1] for a, b in zip(iv, iv[1:]))
    # each result in the mix equals the result of the set run alone
    for r in reqs:
        for got, want in zip(r.results, _alone(engine, r)):
            assert got.alpha == want.alpha and got.rank == want.rank
            assert list(got.nTris) == list(want.nTris) and list(got.nEdges) == list(want.nEdges)
            assert list(got.nPoints) == list(want.nPoints)
