"""GPU parity tests of the alpha spectrum and intervals (Alpha_Shapes_2D).

The CUDA result is compared with the CPU oracle on the same triangle array
(edge numbering follows triangle order, kernel.cu:138-217): ranks and
intervals identical, spectrum values within 4 ulp of the exact-then-rounded
FP64 oracle.
"""
import os

import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from alphacheck import compare_alpha

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ULP_TOL = 4


def both(engine, pts, fbo):
    p = G.GPUDTParams(pts, fboSize=fbo)
    dt = engine.triangulate(p)
    return p, dt, engine.alpha_resident()


def test_c1_alpha(engine):
    pts, fbo = D.make("c1")
    p, dt, a = both(engine, pts, fbo)
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep
    g = np.load(os.path.join(GOLD, "golden_c1.npz"))
    assert np.array_equal(a["spectrum"], g["spectrum"])


@pytest.mark.parametrize("name,fbo", [("bird", 512), ("alpha", 512), ("1000_1", 2048), ("10000_1", 2048)])
def test_reference_fixtures_alpha(engine, name, fbo):
    pts = np.load(os.path.join(GOLD, "golden_ref_%s.npz" % name))["points"]
    p, dt, a = both(engine, pts, fbo)
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep


@pytest.mark.parametrize("seed", range(4))
def test_random_alpha(engine, seed):
    rng = np.random.default_rng(300 + seed)
    for pts in (rng.random((8000, 2)), D.degenerate_mix(8000, seed), np.floor(rng.random((4000, 2)) * 32) / 32):
        p, dt, a = both(engine, pts, 1024)
        ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
        assert ok, rep


@pytest.mark.parametrize("side", [60, 100])
def test_long_key_group(engine, side):
    """A lattice whose unit edges share one spectrum value, with a few points
    moved by about 1e-12 so that some edge keys agree with it in their top 40
    bits but not below: a group of equal top bits far longer than one thread
    fixes up, out of order, sorted as a sub-array (fewer passes than a full
    64-bit sort).  Moving a vertex along its triangle's circumcircle changes
    the radius only at second order, so the triangle values form a run of
    keys within 2 ulp with exact order violations: at side 100 the run has
    about 19,600 entries and is merge-sorted by one block with the exact
    comparator.  The spectrum and intervals match the oracle."""
    rng = np.random.default_rng(77)
    g = np.arange(side) / 128.0
    pts = np.stack(np.meshgrid(g, g), -1).reshape(-1, 2).copy()
    moved = rng.choice(len(pts), 60, replace=False)
    pts[moved, 0] += rng.choice([-1.0, 1.0], 60) * rng.uniform(1e-12, 3e-12, 60)
    dt, a = engine.compute_all(G.GPUDTParams(pts, fboSize=1024))
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep
    assert dt.status.sortPasses > 5, dt.status.sortPasses  # the top-40 passes plus long-group passes


def test_alpha_of_host_mesh_matches_resident(engine):
    pts = np.random.default_rng(11).random((5000, 2))
    p, dt, a = both(engine, pts, 1024)
    b = engine.alpha_of(p, dt)
    for k in ("spectrum", "point_list", "edge_list", "tri_list"):
        assert np.array_equal(a[k], b[k]), k
    shapes = G.AlphaShapes2D(p, dt, engine=engine).compute_alpha_shapes()
    assert np.array_equal(shapes.spectrum, a["spectrum"])


def test_alpha_empty_and_tiny(engine):
    p, dt, a = both(engine, np.array([[0, 0], [1, 1.0]]), 256)
    assert dt.nTris == 0 and list(a["spectrum"]) == [0.0]
    assert (a["point_list"]["nu_min_rank"] == -1).all()
    pts = np.array([[0, 0], [1, 0], [0, 1.0]])
    p, dt, a = both(engine, pts, 256)
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep
    assert list(a["spectrum"]) == [0.0, 0.25, 0.5]


def test_c2_alpha_matches_oracle(engine):
    """c2 size (4,194,304 uniform points, texture 8192): every triangle, edge
    and vertex interval and every rank identical to the CPU oracle's on the
    GPU's own triangle array, and every spectrum value within 4 ulp of the
    exactly rounded FP64 value (the oracle takes about 30 s on one core)."""
    pts, fbo = D.make("c2")
    p, dt, a = both(engine, pts, fbo)
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep
    print("c2 alpha vs oracle: %r" % rep)


@pytest.mark.parametrize("n,seed", [(20000, 21), (300000, 22)])
def test_compute_all_matches_two_calls(engine, n, seed):
    """galphaComputeAll (triangles downloaded while the alpha stage runs) gives
    the mesh of galphaTriangulate and, for its own triangle order, exactly the
    alpha arrays of galphaCompute on that mesh.  (Triangle slots are handed
    out by atomics, so the order of the triangles, and with it the edge
    numbering, may differ between runs; the triangle set may not.)"""
    from alphacheck import canonical_alpha
    from dtcheck import canon_set

    pts = np.random.default_rng(seed).random((n, 2)) if seed % 2 else D.gaussian_blobs(n, seed)
    p = G.GPUDTParams(pts, fboSize=2048)
    dt1 = engine.triangulate(p)
    a1 = engine.alpha_resident()
    dt2, a2 = engine.compute_all(p)
    assert dt2.nTris == dt1.nTris and canon_set(dt2.vtx) == canon_set(dt1.vtx)
    b = engine.alpha_of(p, dt2)
    for k in ("spectrum", "point_list", "edge_list", "tri_list"):
        assert np.array_equal(a2[k], b[k]), k
    c1, c2 = canonical_alpha(dt1.vtx, a1), canonical_alpha(dt2.vtx, a2)
    assert np.array_equal(c1[0], c2[0]) and np.array_equal(c1[3], c2[3])
    assert c1[1] == c2[1] and c1[2] == c2[2]
    if n <= 20000:
        ok, rep = compare_alpha(pts, dt2.vtx, dt2.tri, a2, ULP_TOL)
        assert ok, rep
    # pinned views (copy=False) hold a complete result until the next call
    dt3, a3 = engine.compute_all(p, copy=False)
    assert canon_set(dt3.vtx) == canon_set(dt1.vtx)
    assert np.array_equal(a3["spectrum"], a1["spectrum"])


def _set_block_run(engine, entries):
    import ctypes

    L = G.load()
    L.galphaSetBlockRun.argtypes = [ctypes.c_void_p, ctypes.c_int]
    assert L.galphaSetBlockRun(engine._h, entries) == 0


def _lattice(side, spacing_den):
    g = np.arange(side) / float(spacing_den)
    return np.stack(np.meshgrid(g, g), -1).reshape(-1, 2).copy()


def test_multi_block_exact_runs(engine):
    """Runs of near-equal spectrum keys longer than one block takes are
    merge-sorted with the exact comparator by many blocks.  A 200 x 200
    lattice of spacing 1/1500 (not representable: its squared lengths differ
    in the last bits) gives runs of about 79,000 triangle values and 79,000
    edge values, above the 65,536 default; the perturbed 100 x 100 lattice of
    test_long_key_group takes the multi-block path with the threshold lowered
    to 512.  Both match the oracle."""
    pts = _lattice(200, 1500)
    dt, a = engine.compute_all(G.GPUDTParams(pts, fboSize=1024))
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep
    rng = np.random.default_rng(77)
    g = np.arange(100) / 128.0
    pts = np.stack(np.meshgrid(g, g), -1).reshape(-1, 2).copy()
    moved = rng.choice(len(pts), 60, replace=False)
    pts[moved, 0] += rng.choice([-1.0, 1.0], 60) * rng.uniform(1e-12, 3e-12, 60)
    try:
        _set_block_run(engine, 512)
        dt, a = engine.compute_all(G.GPUDTParams(pts, fboSize=1024))
    finally:
        _set_block_run(engine, 0)
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, ULP_TOL)
    assert ok, rep


def test_lattice_1500_runs_above_four_million(engine):
    """A 1500 x 1500 lattice of spacing 1/1500: about 4.5 M triangle values and
    4.5 M edge values, each set within a few ulp of one value, forming runs of
    more than 2^22 entries that the exact comparator must order (the
    reference orders them in its odd-even rounds; nothing is refused).  Too
    large for the oracle; checked instead: the spectrum does not decrease
    (distinct exact values may round to the same double), every rank is in
    range, and a sample of entry pairs is ordered as exact rational
    arithmetic orders their values."""
    from fractions import Fraction

    from fraction_alpha import rho_edge, rho_tri

    pts = _lattice(1500, 1500)
    dt, a = engine.compute_all(G.GPUDTParams(pts, fboSize=4096))
    s = a["spectrum"]
    assert s[0] == 0.0 and np.all(np.diff(s[1:]) >= 0)
    tri_ro = a["tri_list"]["ro_rank"]
    e = a["edge_list"]
    assert dt.nTris == 2 * 1499 * 1499
    assert tri_ro.min() >= 1 and tri_ro.max() < len(s) and e["ro_rank"].max() < len(s)
    P = [(Fraction(float(x)), Fraction(float(y))) for x, y in pts]
    vtx = dt.vtx
    rng = np.random.default_rng(5)
    unatt = np.nonzero(e["ro_rank"] > 0)[0]
    for _ in range(400):
        t1, t2 = (int(x) for x in rng.integers(0, dt.nTris, 2))
        r1, r2 = rho_tri(P, *map(int, vtx[t1])), rho_tri(P, *map(int, vtx[t2]))
        assert (r1 < r2) == (tri_ro[t1] < tri_ro[t2]) and (r1 == r2) == (tri_ro[t1] == tri_ro[t2])
        k = int(unatt[int(rng.integers(0, len(unatt)))])
        t, i = int(e["tIndex"][k]), int(e["vOpp"][k])
        re = rho_edge(P, int(vtx[t][(i + 1) % 3]), int(vtx[t][(i + 2) % 3]))
        assert (re < r1) == (e["ro_rank"][k] < tri_ro[t1]) and (re == r1) == (e["ro_rank"][k] == tri_ro[t1])
