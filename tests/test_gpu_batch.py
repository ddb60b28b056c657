"""GPU tests of the batched pipeline (galphaRunBatch): every set's result
equals a separate single-set run of the same points -- identical triangle set,
spectrum, per-simplex ranks and intervals (order-free comparison, since the
triangle order depends on the texture size) -- and, for inputs in general
position, the oracle's Delaunay triangulation."""
import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from alphacheck import canonical_alpha
from dtcheck import canon_set
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mixed_sets(seed):
    rng = np.random.default_rng(seed)
    sets = []
    for k, n in enumerate([64, 100, 700, 3000, 9000, 25000, 200, 1500]):
        sets.append(rng.random((n, 2)) * (1 + k))
    r = np.sqrt(rng.random(2000)); a = 2 * np.pi * rng.random(2000)
    sets.append(np.stack([r * np.cos(a), r * np.sin(a)], 1))                      # disk
    r = np.sqrt(0.64 + 0.36 * rng.random(3000)); a = 2 * np.pi * rng.random(3000)
    sets.append(np.stack([r * np.cos(a), r * np.sin(a)], 1) + 5.0)                # annulus
    c = rng.random((6, 2)); sets.append(c[rng.integers(0, 6, 4000)] + rng.normal(0, 0.01, (4000, 2)))
    lat = np.floor(rng.random((2500, 2)) * 24) / 24; sets.append(lat)             # lattice + duplicates
    sets.append(np.stack([np.linspace(0, 1, 50), np.linspace(0, 2, 50)], 1))     # collinear
    sets.append(np.array([[0.5, 0.5], [0.25, 0.75]]))                             # two points
    sets.append(np.zeros((0, 2)))                                                 # empty
    sets.append(np.repeat([[0.3, 0.3]], 10, axis=0))                              # one distinct point
    sets.append(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]))                   # one triangle
    return sets


def _single(engine, pts):
    fbo = 256
    while fbo < 4096 and fbo * fbo < 16 * len(pts):
        fbo *= 2
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=fbo))
    return dt, engine.alpha_resident()


def _compare(engine, sets, results):
    for k, (pts, res) in enumerate(zip(sets, results)):
        dt, ref = _single(engine, pts)
        assert canon_set(res["triangles"]["vtx"]) == canon_set(dt.vtx), "set %d triangles" % k
        # neighbour links are consistent and set-local
        tri = res["triangles"]["tri"]
        for t in range(len(tri)):
            for i in range(3):
                nb = tri[t][i]
                if nb >= 0:
                    assert tri[nb >> 2][nb & 3] == (t << 2) | i, "set %d links" % k
        s1, t1, e1, p1 = canonical_alpha(res["triangles"]["vtx"], res)
        s2, t2, e2, p2 = canonical_alpha(dt.vtx, ref)
        np.testing.assert_array_equal(s1, s2, err_msg="set %d spectrum" % k)
        assert t1 == t2, "set %d triangle ranks" % k
        assert e1 == e2, "set %d edge intervals" % k
        np.testing.assert_array_equal(p1, p2, err_msg="set %d point intervals" % k)


def test_batch_matches_single_runs(engine):
    sets = _mixed_sets(1)
    beng = G.Engine()
    try:
        st = beng.run_batch(sets)
        res = beng.batch_results()
    finally:
        beng.close()
    assert len(res) == len(sets)
    # the annulus and the clusters leave most of their cells empty: envelope path
    assert st.nEnvelopeCells >= 1
    _compare(engine, sets, res)


def test_batch_reuse_and_oracle(engine):
    beng = G.Engine()
    try:
        a = _mixed_sets(2)[:6]
        beng.run_batch(a)
        beng.run_batch(a[::-1])          # a second batch on the same handle
        res = beng.batch_results()
    finally:
        beng.close()
    for pts, r in zip(a[::-1], res):
        v, nb, _ = O.dt(pts)
        assert canon_set(r["triangles"]["vtx"]) == canon_set(v)


def test_batch_c4_sample(engine):
    sets = D.c4_sets()[:48]
    beng = G.Engine()
    try:
        st = beng.run_batch(sets)
        res = beng.batch_results()
    finally:
        beng.close()
    for pts, r in zip(sets, res):
        v, nb, _ = O.dt(pts)
        assert canon_set(r["triangles"]["vtx"]) == canon_set(v)
        assert r["spectrum"][0] == 0.0 and np.all(np.diff(r["spectrum"]) > 0)


def test_batch_query_matches_interval_rule(engine):
    from alphacheck import classify_intervals

    sets = _mixed_sets(3)[:10] + _mixed_sets(3)[-4:]
    beng = G.Engine()
    try:
        beng.run_batch(sets)
        res = beng.batch_results()
        info = beng.batch_sets()
        rng = np.random.default_rng(0)
        for mode, vals in (("q", [0.1] * len(sets)), ("q", [0.9] * len(sets)),
                           ("q", rng.random(len(sets)).tolist()),
                           ("a", [float(r["spectrum"][len(r["spectrum"]) // 2]) for r in res])):
            qr = beng.batch_query(vals, by_quantile=(mode == "q"))
            pc, ec, tc = beng.classes()
            for k, r in enumerate(res):
                wp, we, wt, R = classify_intervals(r, qr[k].alpha)
                assert qr[k].rank == R, k
                si = info[k]
                np.testing.assert_array_equal(pc[si.pointBase:si.pointBase + si.nPoints], wp)
                np.testing.assert_array_equal(ec[si.edgeBase:si.edgeBase + si.nEdges], we)
                np.testing.assert_array_equal(tc[si.triBase:si.triBase + si.nTris], wt)
                assert list(qr[k].nTris) == np.bincount(wt, minlength=4).tolist()
                assert list(qr[k].nEdges) == np.bincount(we, minlength=4).tolist()
                assert list(qr[k].nPoints) == np.bincount(wp, minlength=4).tolist()
    finally:
        beng.close()


@pytest.mark.parametrize("density", [3.0, 24.0])
def test_batch_density_keeps_results(engine, density):
    """The texture density (pixels per point of a set's cell) changes how
    many sites share a pixel, not the result."""
    sets = _mixed_sets(4)[:12]
    beng = G.Engine()
    try:
        beng.set_batch_density(density)
        beng.run_batch(sets)
        res = beng.batch_results()
        with pytest.raises(G.GpudtError):
            beng.set_batch_density(0.5)
    finally:
        beng.close()
    _compare(engine, sets, res)


@pytest.mark.parametrize("sched", [(1, 1, 1, 0, 1), (8, 8, 64, 1 << 20, 1 << 22)])
def test_batch_schedule_keeps_results(engine, sched):
    """The loop schedule (rounds per counter read, flip-tail hand-over)
    changes when the host reads counters, not the result of a batch."""
    sets = _mixed_sets(5)[:12]
    beng = G.Engine()
    try:
        beng.set_schedule(*sched)
        beng.run_batch(sets)
        res = beng.batch_results()
    finally:
        beng.close()
    _compare(engine, sets, res)
