"""GPU tests of the alpha-complex query (galphaQuery / galphaQueryQuantile).

Two checks of every class array: against the numpy restatement of the
interval rule (tests/alphacheck.classify_intervals) on the engine's own
interval output, and -- at small sizes -- against a first-principles
classification in exact rational arithmetic, where a simplex is in the
complex when the correctly rounded FP64 value of its exact squared radius is
<= alpha (the spectrum holds those rounded values).
"""
from fractions import Fraction

import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from alphacheck import classify_intervals
from fraction_alpha import attached, rho_edge, rho_tri

pytestmark = pytest.mark.gpu


def _run(engine, pts, fbo):
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=fbo))
    return dt, engine.alpha_resident()


def _check_query(engine, res, alpha=None, quantile=None):
    q = engine.query(alpha=alpha, quantile=quantile)
    pc, ec, tc = engine.classes()
    a = q.alpha
    if quantile is not None:
        k = int(np.rint(min(max(quantile, 0.0), 1.0) * (len(res["spectrum"]) - 1)))
        assert a == res["spectrum"][k]
    else:
        assert a == alpha
    wp, we, wt, R = classify_intervals(res, a)
    assert q.rank == R
    np.testing.assert_array_equal(pc, wp)
    np.testing.assert_array_equal(ec, we)
    np.testing.assert_array_equal(tc, wt)
    assert list(q.nPoints) == np.bincount(pc, minlength=4).tolist()
    assert list(q.nEdges) == np.bincount(ec, minlength=4).tolist()
    assert list(q.nTris) == np.bincount(tc, minlength=4).tolist()
    return q, pc, ec, tc


@pytest.mark.parametrize("seed", [1, 2])
def test_query_matches_interval_rule(engine, seed):
    pts = D.uniform_points(20000, seed)
    dt, res = _run(engine, pts, 1024)
    spec = res["spectrum"]
    alphas = [-1.0, 0.0, float(spec[1]), float(spec[len(spec) // 3]),
              float(np.nextafter(spec[len(spec) // 2], 0)), float(spec[-1]), 1e30]
    for a in alphas:
        _check_query(engine, res, alpha=a)
    for q in (0.0, 0.1, 0.5, 0.9, 1.0):
        _check_query(engine, res, quantile=q)


def test_query_extremes(engine):
    pts = D.uniform_points(5000, 3)
    dt, res = _run(engine, pts, 512)
    q, pc, ec, tc = _check_query(engine, res, alpha=-0.5)
    assert q.rank == -1 and not pc.any() and not ec.any() and not tc.any()
    q, pc, ec, tc = _check_query(engine, res, alpha=1e300)
    assert (tc == G.api.INTERIOR).all()
    hull = res["edge_list"]["nu_max_rank"] == 0
    assert (ec[hull] == G.api.REGULAR).all() and (ec[~hull] == G.api.INTERIOR).all()


def _first_principles(pts, vtx, nbr, edge_list, alpha):
    P = [(Fraction(float(x)), Fraction(float(y))) for x, y in pts]
    A = Fraction(alpha)

    def inside(rho):  # the spectrum compares correctly rounded values
        return Fraction(float(rho)) <= A

    rt = [rho_tri(P, *[int(v) for v in t]) for t in vtx]
    tc = np.array([3 if inside(r) else 0 for r in rt], np.uint8)
    ec = np.zeros(len(edge_list), np.uint8)
    n = len(pts)
    entry = [None] * n       # earliest value at which a vertex gets an edge
    last = [None] * n        # latest adjacent-triangle value over non-hull edges
    for e, E in enumerate(edge_list):
        t, i = int(E["tIndex"]), int(E["vOpp"])
        a, b = int(vtx[t][(i + 1) % 3]), int(vtx[t][(i + 2) % 3])
        nb = int(nbr[t][i])
        adj = [rt[t]] + ([rt[nb >> 2]] if nb != -1 else [])
        att = attached(P, a, b, int(vtx[t][i])) or (nb != -1 and attached(P, a, b, int(vtx[nb >> 2][nb & 3])))
        if nb != -1 and inside(max(adj)):
            ec[e] = 3
        elif inside(min(adj)):
            ec[e] = 2
        elif not att and inside(rho_edge(P, a, b)):
            ec[e] = 1
        first = min(adj) if att else rho_edge(P, a, b)
        for v in (a, b):
            entry[v] = first if entry[v] is None else min(entry[v], first)
            if nb != -1:
                last[v] = max(adj) if last[v] is None else max(last[v], max(adj))
    pc = np.zeros(n, np.uint8)
    for v in range(n):
        if entry[v] is None or A < 0:
            continue
        if last[v] is not None and inside(last[v]):
            pc[v] = 3
        elif inside(entry[v]):
            pc[v] = 2
        else:
            pc[v] = 1
    return pc, ec, tc


@pytest.mark.parametrize("seed", [5, 6])
def test_query_first_principles(engine, seed):
    rng = np.random.default_rng(seed)
    pts = rng.random((120, 2))
    dt, res = _run(engine, pts, 512)
    spec = res["spectrum"]
    for a in (float(spec[len(spec) // 4]), float(spec[len(spec) // 2]) * 1.0000001, float(spec[-1]) * 0.5):
        q, pc, ec, tc = _check_query(engine, res, alpha=a)
        wp, we, wt = _first_principles(pts, dt.vtx, dt.tri, res["edge_list"], a)
        np.testing.assert_array_equal(tc, wt)
        np.testing.assert_array_equal(ec, we)
        np.testing.assert_array_equal(pc, wp)


def test_query_duplicates_exterior(engine):
    pts = D.uniform_points(3000, 7)
    pts = np.concatenate([pts, pts[:50]])
    dt, res = _run(engine, pts, 512)
    q, pc, ec, tc = _check_query(engine, res, alpha=1e300)
    dropped = res["point_list"]["nu_min_rank"] < 0
    assert dropped.sum() == 50
    assert (pc[dropped] == 0).all() and (pc[~dropped] > 0).all()


def test_query_needs_alpha():
    eng = G.Engine()
    try:
        with pytest.raises(G.GpudtError):
            eng.query(alpha=1.0)
    finally:
        eng.close()
