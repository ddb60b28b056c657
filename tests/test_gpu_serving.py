"""GPU test of the serving loop: a short request stream served by micro-batches;
every request's quantile queries agree with a separate single-set run."""
import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from galpha_b200 import serving as S

pytestmark = pytest.mark.gpu


def test_serving_stream_matches_single_runs(engine):
    rng = np.random.default_rng(5)
    arrivals = S.poisson_arrivals(400.0, 0.1, 7)
    reqs = []
    for i, t in enumerate(arrivals):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(20000))))
        pts = D.uniform_points(n, 100 + i) if i % 2 == 0 else D.gaussian_blobs(n, 100 + i)
        reqs.append(S.Request(i, t, pts))
    seng = G.Engine()
    try:
        srv = S.Server(seng, max_batch_points=60000)
        srv.run(reqs)
    finally:
        seng.close()
    s = S.summary(reqs, srv.batches)
    assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0
    for r in reqs[:6]:
        fbo = 256
        while fbo < 4096 and fbo * fbo < 16 * len(r.points):
            fbo *= 2
        engine.triangulate(G.GPUDTParams(r.points, fboSize=fbo))
        engine.alpha_resident()
        for q, got in zip(r.quantiles, r.results):
            want = engine.query(quantile=q)
            assert got.alpha == want.alpha and got.rank == want.rank
            assert list(got.nTris) == list(want.nTris) and list(got.nEdges) == list(want.nEdges)
            assert list(got.nPoints) == list(want.nPoints)
