"""Constrained Delaunay triangulation (GPUDTPARAMS.nConstraints > 0;
gpudt.cpp:860 cudaConstraint, gpudt/Cuda/cudaConstraint.cu:828-939, and the
flipping that never flips a marked edge, cudaFlipping.cu:111-220).

Constraints are drawn so that the input is valid: edges of another
triangulation of the same points (the Delaunay triangulation of a sheared
copy), which neither cross each other nor pass through a point, minus the
edges the Delaunay triangulation already has; and long chords between the
left and right strips, matched in order of height so that they do not cross.
For points in general position the constrained Delaunay triangulation is
unique, so the GPU result must equal the oracle's triangle for triangle.

CPU tests: the oracle's own invariants.  GPU tests (marked gpu): parity with
the oracle through the C ABI, and the errors the reference leaves undefined
(crossing constraints, a point on a constraint) returned as GPUDT_ERR_ARG
with the handle still usable.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from dtcheck import canon_set


def edges_of(vtx):
    v = np.asarray(vtx).reshape(-1, 3)
    e = set()
    for i in range(3):
        a, b = v[:, i], v[:, (i + 1) % 3]
        e |= set(zip(np.minimum(a, b).tolist(), np.maximum(a, b).tolist()))
    return e


def sheared_constraints(pts, count, seed, shear=6.0):
    """Edges of the Delaunay triangulation of a sheared copy of the points that
    the Delaunay triangulation of the points lacks: valid, non-crossing."""
    v1, _, _ = O.dt(pts)
    v2, _, _ = O.dt(pts * np.array([1.0, shear]))
    extra = sorted(edges_of(v2) - edges_of(v1))
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(extra), min(count, len(extra)), replace=False)
    return np.array([extra[i] for i in sorted(pick)], np.int32)


def chord_constraints(pts, count):
    """Long chords from the left strip to the right strip, paired in order of
    height (non-crossing); each crosses many Delaunay edges."""
    left = np.nonzero(pts[:, 0] < 0.08)[0]
    right = np.nonzero(pts[:, 0] > 0.92)[0]
    left = left[np.argsort(pts[left, 1])]
    right = right[np.argsort(pts[right, 1])]
    k = min(count, len(left), len(right))
    li = np.linspace(0, len(left) - 1, k).astype(int)
    ri = np.linspace(0, len(right) - 1, k).astype(int)
    return np.stack([left[li], right[ri]], axis=1).astype(np.int32)


def without_crossings(pts, cons, chords):
    """The constraints of `cons` that cross none of `chords` (proper crossings
    by exact orientation, oracle predicates), followed by the chords."""
    L = O.lib()
    P = np.ascontiguousarray(pts, np.float64)
    dp = ctypes.POINTER(ctypes.c_double)

    def o(i, j, k):
        return L.oracle_orient2d(ctypes.cast(P.ctypes.data + 16 * int(i), dp), ctypes.cast(P.ctypes.data + 16 * int(j), dp),
                                 ctypes.cast(P.ctypes.data + 16 * int(k), dp))

    keep = []
    for a, b in np.asarray(cons).tolist():
        ok = True
        for c, d in np.asarray(chords).tolist():
            if len({a, b, c, d}) < 4:
                continue
            if o(a, b, c) * o(a, b, d) < 0 and o(c, d, a) * o(c, d, b) < 0:
                ok = False
                break
        if ok:
            keep.append((a, b))
    return np.concatenate([np.array(keep, np.int32).reshape(-1, 2), np.asarray(chords, np.int32)])


def lattice_case(seed, side=64, draws=1200, nchords=8):
    """Points of a side x side lattice (collinear and cocircular sets) and
    non-crossing left-to-right chords between lattice points with coprime
    offsets (no lattice point lies on them).  Vertices inside the crossed
    regions then often lie on an edge of the re-triangulated cavity."""
    import math

    rng = np.random.default_rng(seed)
    gi = np.unique(rng.integers(0, side, size=(draws, 2)), axis=0)
    rng.shuffle(gi)
    pts = gi.astype(np.float64) / side
    left = sorted((i for i in range(len(gi)) if gi[i, 0] < 4), key=lambda i: gi[i, 1])
    right = sorted((i for i in range(len(gi)) if gi[i, 0] > side - 5), key=lambda i: gi[i, 1])
    keep = np.zeros((0, 2), np.int32)
    for k in range(nchords):
        a = left[k * (len(left) - 1) // (nchords - 1)]
        for b in right[k * (len(right) - 1) // (nchords - 1):]:
            d = gi[b] - gi[a]
            if math.gcd(int(abs(d[0])), int(abs(d[1]))) == 1:
                c = np.array([[a, b]], np.int32)
                if len(without_crossings(pts, c, keep)) == len(keep) + 1:
                    keep = np.concatenate([keep, c])
                break
    return pts, keep


def check_cdt(pts, vtx, nbr, cons):
    """Constrained Delaunay invariants: every constraint is an edge, links and
    orientation valid, and every interior edge that breaks the exact empty
    circle is a constraint."""
    chk = O.check_mesh(pts, vtx, nbr)
    have = edges_of(vtx)
    cset = {(min(a, b), max(a, b)) for a, b in np.asarray(cons).tolist()}
    missing = len(cset - have)
    L = O.lib()
    P = np.ascontiguousarray(pts, np.float64)
    dp = ctypes.POINTER(ctypes.c_double)

    def pt(i):
        return ctypes.cast(P.ctypes.data + 16 * int(i), dp)

    bad = 0
    v = np.asarray(vtx).reshape(-1, 3)
    n = np.asarray(nbr).reshape(-1, 3)
    for t in range(len(v)):
        for i in range(3):
            e = int(n[t, i])
            if e < 0:
                continue
            a, b = int(v[t, (i + 1) % 3]), int(v[t, (i + 2) % 3])
            if (min(a, b), max(a, b)) in cset:
                continue
            d = int(v[e >> 2, e & 3])
            if L.oracle_incircle(pt(a), pt(b), pt(v[t, i]), pt(d)) > 0:
                bad += 1
    return dict(links=chk["links"], ccw=chk["ccw"], missing=missing, non_delaunay_free=bad)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_cdt_invariants(seed):
    rng = np.random.default_rng(seed)
    pts = rng.random((3000, 2))
    cons = without_crossings(pts, sheared_constraints(pts, 300, seed), chord_constraints(pts, 6))
    vtx, nbr, _ = O.cdt(pts, cons)
    rep = check_cdt(pts, vtx, nbr, cons)
    assert rep == dict(links=0, ccw=0, missing=0, non_delaunay_free=0), rep
    assert len(vtx) == len(O.dt(pts)[0])  # same vertex set and hull: same triangle count


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_cdt_lattice(seed):
    pts, cons = lattice_case(seed)
    vtx, nbr, _ = O.cdt(pts, cons)
    rep = check_cdt(pts, vtx, nbr, cons)
    assert rep == dict(links=0, ccw=0, missing=0, non_delaunay_free=0), rep
    assert len(vtx) == len(O.dt(pts)[0])


@pytest.mark.gpu
@pytest.mark.parametrize("n,kind,seed", [(3000, "uniform", 0), (20000, "uniform", 1), (20000, "clusters", 2)])
def test_gpu_cdt_matches_oracle(engine, n, kind, seed):
    import galpha_b200 as G
    from galpha_b200 import datasets as D

    pts = D.uniform_points(n, 600 + seed) if kind == "uniform" else D.gaussian_blobs(n, 600 + seed)
    cons = without_crossings(pts, sheared_constraints(pts, n // 10, seed), chord_constraints(pts, 12))
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024 if n <= 5000 else 2048, constraints=cons))
    rep = check_cdt(pts, dt.vtx, dt.tri, cons)
    assert rep == dict(links=0, ccw=0, missing=0, non_delaunay_free=0), rep
    assert 1 <= dt.status.constraintRounds < len(cons), dt.status.constraintRounds
    ov, _, _ = O.cdt(pts, cons)
    assert canon_set(dt.vtx) == canon_set(ov)
    # the alpha stage runs on the constrained mesh as on any triangulation
    from alphacheck import compare_alpha

    a = engine.alpha_resident()
    ok, arep = compare_alpha(pts, dt.vtx, dt.tri, a, 4)
    assert ok, arep


@pytest.mark.gpu
def test_gpu_cdt_errors_and_recovery(engine):
    import galpha_b200 as G
    from galpha_b200 import datasets as D

    pts = D.uniform_points(4000, 611)
    chords = chord_constraints(pts, 4)
    crossing = np.array([[chords[0, 0], chords[3, 1]], [chords[3, 0], chords[0, 1]]], np.int32)
    with pytest.raises(G.GpudtError) as ei:
        engine.triangulate(G.GPUDTParams(pts, fboSize=1024, constraints=crossing))
    assert ei.value.code == -1  # GPUDT_ERR_ARG
    # a point exactly on the segment between two others (dyadic coordinates:
    # the midpoint is exact)
    q = pts.copy()
    q[0], q[1], q[2] = (0.25, 0.25), (0.5, 0.375), (0.75, 0.5)
    with pytest.raises(G.GpudtError) as ei:
        engine.triangulate(G.GPUDTParams(q, fboSize=1024, constraints=np.array([[0, 2]], np.int32)))
    assert ei.value.code == -1
    with pytest.raises(G.GpudtError):
        engine.triangulate(G.GPUDTParams(pts, fboSize=1024, constraints=np.array([[0, 0]], np.int32)))
    # the handle still triangulates, with and without constraints
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024, constraints=chords))
    rep = check_cdt(pts, dt.vtx, dt.tri, chords)
    assert rep == dict(links=0, ccw=0, missing=0, non_delaunay_free=0), rep
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024))
    assert canon_set(dt.vtx) == canon_set(O.dt(pts)[0])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 8, 11])
def test_gpu_cdt_lattice(engine, seed):
    """Cocircular and collinear points: the constrained Delaunay triangulation
    is not unique, so the invariants and the triangle count are checked."""
    import galpha_b200 as G

    pts, cons = lattice_case(seed)
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024, constraints=cons))
    rep = check_cdt(pts, dt.vtx, dt.tri, cons)
    assert rep == dict(links=0, ccw=0, missing=0, non_delaunay_free=0), rep
    assert len(dt.vtx) == len(O.cdt(pts, cons)[0])


@pytest.mark.gpu
def test_gpu_cdt_through_compute_all(engine):
    """Constraints through galphaComputeAll (DT + alpha with host buffers):
    the same triangles as galphaTriangulate, and the alpha result of that
    constrained mesh."""
    import galpha_b200 as G
    from galpha_b200 import datasets as D
    from alphacheck import compare_alpha

    pts = D.uniform_points(5000, 621)
    cons = without_crossings(pts, sheared_constraints(pts, 500, 3), chord_constraints(pts, 8))
    p = G.GPUDTParams(pts, fboSize=1024, constraints=cons)
    ref = engine.triangulate(p)
    dt, al = engine.compute_all(p)
    assert canon_set(dt.vtx) == canon_set(ref.vtx) == canon_set(O.cdt(pts, cons)[0])
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, al, 4)
    assert ok, rep
    # the next call without constraints is the plain Delaunay triangulation again
    dt2, _ = engine.compute_all(G.GPUDTParams(pts, fboSize=1024))
    assert canon_set(dt2.vtx) == canon_set(O.dt(pts)[0])
