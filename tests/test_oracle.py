"""CPU tests that pin the oracle before it is trusted as the checker.

* the reference ships no golden outputs, so the pins are: its own predicates
  (gpudt/predicates.cpp and gpudt/AlphaShape/predicates.h, compiled from the
  reference tree into oracle/_ref by oracle/ref.mk), the exact checkResult
  invariants (main.cu:163-343) on its own input fixtures, an independent exact
  rational restatement of the alpha semantics (tests/fraction_alpha.py) and
  scipy's Qhull on general-position inputs;
* the committed golden fixtures (tests/golden/make_golden.py) are re-derived
  and compared, so an oracle change cannot pass silently.
"""
import ctypes
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as O
from dtcheck import canon_set, compare_dt
from fraction_alpha import alpha_exact, attached, rho_edge, rho_tri

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
REFLIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref.so")


def F(p):
    return [(Fraction(float(x)), Fraction(float(y))) for x, y in p]


# ----------------------------------------------------------------- DT
@pytest.mark.parametrize("n,seed", [(3, 1), (4, 2), (50, 3), (1000, 4), (20000, 5)])
def test_dt_matches_qhull_general_position(n, seed):
    from scipy.spatial import Delaunay

    pts = np.random.default_rng(seed).random((n, 2))
    v, nb, kept = O.dt(pts)
    d = Delaunay(pts)
    ccw = []
    for a, b, c in d.simplices:
        ccw.append((a, b, c) if O.orient2d(pts[a], pts[b], pts[c]) > 0 else (b, a, c))
    assert canon_set(v) == canon_set(ccw)
    ok, rep = compare_dt(pts, v, nb, (v, nb, kept))
    assert ok, rep


@pytest.mark.parametrize("name", ["ref_bird", "ref_alpha", "ref_1000_1", "ref_10000_1", "c1"])
def test_dt_checkresult_invariants_and_golden(name):
    g = np.load(os.path.join(GOLD, "golden_%s.npz" % name))
    pts = g["points"]
    v, nb, kept = O.dt(pts)
    chk = O.check_mesh(pts, v, nb)
    assert chk["links"] == 0 and chk["ccw"] == 0 and chk["delaunay"] == 0 and chk["nonconvex"] == 0, chk
    # Euler characteristic as main.cu:330-337 counts it, over the distinct vertices
    edges = (3 * len(v) + chk["hull_edges"]) // 2
    assert kept - edges + len(v) + 1 == 2
    assert canon_set(v) == canon_set(g["triangles"])
    assert kept == int(g["nkept"])


def test_dt_degenerate_inputs():
    g = np.stack(np.meshgrid(np.arange(20), np.arange(20)), -1).reshape(-1, 2).astype(float)
    pts = np.concatenate([g, g[::3]])
    v, nb, kept = O.dt(pts)
    assert kept == 400 and len(v) == 2 * 19 * 19
    chk = O.check_mesh(pts, v, nb)
    assert chk["delaunay"] == 0 and chk["ccw"] == 0 and chk["links"] == 0
    assert set(np.unique(v)) == set(range(400))  # lowest index of each duplicate kept
    v, nb, kept = O.dt(np.array([[0, 0], [1, 1], [2, 2.0]]))
    assert len(v) == 0


def test_dt_long_degenerate_runs():
    # exactly collinear (dyadic coordinates), and two distinct points with
    # the second one last: no triangle either way
    t = np.arange(5000, dtype=np.float64) / 8192
    assert len(O.dt(np.stack([t, 0.25 + 0.5 * t], 1))[0]) == 0
    dup = np.full((5000, 2), 0.375)
    dup[-1] = (0.625, 0.125)
    assert len(O.dt(dup)[0]) == 0
    # a long run of copies of point 0 ahead of the other points: the mesh is
    # that of the distinct points, with point 0 standing for its copies
    rng = np.random.default_rng(21)
    rest = rng.random((500, 2))
    late = np.concatenate([np.full((4000, 2), 0.5), rest])
    v, nb, kept = O.dt(late)
    assert kept == 501
    v0, _, _ = O.dt(np.concatenate([[[0.5, 0.5]], rest]))
    remap = np.concatenate([[0], np.arange(4000, 4500)])  # distinct set index -> input index
    assert canon_set(v) == canon_set(remap[v0])


def test_dt_rejects_nan():
    with pytest.raises(RuntimeError):
        O.dt(np.array([[0, 0], [1, np.nan], [0, 1.0]]))


# --------------------------------------------------------- predicates
def _adversarial(rng, n):
    """Near-degenerate orientation / in-circle cases: points on a line or circle,
    perturbed by a few ulps."""
    out = []
    for _ in range(n):
        a = rng.random(2)
        d = rng.random(2) - 0.5
        t = rng.random(2)
        pts = [a, a + t[0] * d, a + t[1] * d]
        ang = rng.random(4) * 2 * np.pi
        r = rng.random() + 0.1
        c = rng.random(2)
        circ = [c + r * np.array([np.cos(x), np.sin(x)]) for x in ang]
        k = rng.integers(0, 5)
        pts = [np.nextafter(p, p + (rng.random(2) - 0.5)) if k else p for p in pts]
        out.append((pts, circ))
    return out


def _orient_exact(a, b, c):
    (ax, ay), (bx, by), (cx, cy) = F([a, b, c])
    d = (ax - cx) * (by - cy) - (ay - cy) * (bx - cx)
    return (d > 0) - (d < 0)


def _incircle_exact(a, b, c, d):
    P = F([a, b, c, d])
    (dx, dy) = P[3]
    rows = [(x - dx, y - dy) for x, y in P[:3]]
    m = [(x, y, x * x + y * y) for x, y in rows]
    det = (m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[0][1] * (m[1][0] * m[2][2] - m[2][0] * m[1][2])
           + m[0][2] * (m[1][0] * m[2][1] - m[2][0] * m[1][1]))
    return (det > 0) - (det < 0)


def test_predicates_exact_against_rationals():
    rng = np.random.default_rng(42)
    for line, circ in _adversarial(rng, 400):
        assert O.orient2d(*line) == _orient_exact(*line)
        a, b, c, d = circ
        if _orient_exact(a, b, c) < 0:
            a, b = b, a
        assert O.incircle(a, b, c, d) == _incircle_exact(a, b, c, d)
    assert O.oracle_exact_counts if hasattr(O, "oracle_exact_counts") else True


@pytest.mark.skipif(not os.path.exists(REFLIB), reason="oracle/_ref not built (needs the reference tree)")
def test_predicates_match_reference_predicates_cpp():
    L = ctypes.CDLL(REFLIB)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_counterclockwise.argtypes = [dp, dp, dp]
    L.ref_counterclockwise.restype = ctypes.c_double
    L.ref_incircle.argtypes = [dp, dp, dp, dp]
    L.ref_incircle.restype = ctypes.c_double
    L.ref_exactinit()

    def P(x):
        return np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(dp)

    rng = np.random.default_rng(7)
    for line, circ in _adversarial(rng, 400):
        r = L.ref_counterclockwise(P(line[0]), P(line[1]), P(line[2]))
        assert O.orient2d(*line) == (r > 0) - (r < 0)
        r = L.ref_incircle(*(P(x) for x in circ))
        assert O.incircle(*circ) == (r > 0) - (r < 0)


# -------------------------------------------------------------- alpha
@pytest.mark.parametrize("seed,kind", [(1, "uniform"), (2, "uniform"), (3, "lattice"), (4, "lattice"), (5, "mixed")])
def test_alpha_matches_rational_restatement(seed, kind):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        pts = rng.random((120, 2))
    elif kind == "lattice":
        pts = rng.integers(0, 7, (80, 2)) / 8.0
    else:
        m = rng.random((100, 2))
        pts = np.where(rng.random((100, 1)) < 0.5, np.floor(m * 8) / 8, m)
    v, nb, _ = O.dt(pts)
    a = O.alpha(pts, v, nb)
    b = alpha_exact(pts, v, nb)
    assert a["tri_ro"].tolist() == b["tri_ro"]
    assert a["edge"].tolist() == b["edge"]
    assert a["point"].tolist() == b["point"]
    assert len(a["spectrum"]) == len(b["spectrum"])
    # exact-then-rounded: every value is the double nearest the rational (<= 0.5 ulp)
    for x, q in zip(a["spectrum"], b["spectrum"]):
        assert abs(Fraction(float(x)) - q) <= abs(Fraction(np.spacing(float(x)))) / 2


def test_alpha_predicates_against_rationals():
    rng = np.random.default_rng(9)
    for _ in range(300):
        p = rng.random((6, 2))
        if rng.random() < 0.3:
            p = np.floor(p * 16) / 16
        P = F(p)
        flat1 = (P[1][0] - P[0][0]) * (P[2][1] - P[0][1]) == (P[2][0] - P[0][0]) * (P[1][1] - P[0][1])
        flat2 = (P[4][0] - P[3][0]) * (P[5][1] - P[3][1]) == (P[5][0] - P[3][0]) * (P[4][1] - P[3][1])
        for k1, k2 in ((3, 3), (3, 2), (2, 3), (2, 2)):
            if (k1 == 3 and flat1) or (k2 == 3 and flat2) or (k2 == 2 and P[3] == P[4]) or (k1 == 2 and P[0] == P[1]):
                continue
            r1 = rho_tri(P, 0, 1, 2) if k1 == 3 else rho_edge(P, 0, 1)
            r2 = rho_tri(P, 3, 4, 5) if k2 == 3 else rho_edge(P, 3, 4)
            q1 = p[:3] if k1 == 3 else p[:2]
            q2 = p[3:] if k2 == 3 else p[3:5]
            assert O.compare_rho(k1, q1, k2, q2) == (r1 > r2) - (r1 < r2)
        assert O.is_attached(p[0], p[1], p[2]) == int(attached(P, 0, 1, 2))


@pytest.mark.skipif(not os.path.exists(REFLIB), reason="oracle/_ref not built (needs the reference tree)")
def test_alpha_predicates_match_reference_predicates_h():
    L = ctypes.CDLL(REFLIB)
    dp = ctypes.POINTER(ctypes.c_double)
    for f in ("ref_compare_slow", "ref_compare_cpu"):
        getattr(L, f).argtypes = [ctypes.c_int, dp, ctypes.c_int, dp]
    L.ref_is_attached.argtypes = [dp, dp, dp]
    L.ref_birth_time3.argtypes = [dp]
    L.ref_birth_time3.restype = ctypes.c_double
    L.ref_birth_time2.argtypes = [dp]
    L.ref_birth_time2.restype = ctypes.c_double

    def P(x):
        return np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(dp)

    rng = np.random.default_rng(11)
    mismatches_ee_cpu = 0
    for it in range(300):
        p = rng.random((6, 2))
        if it % 3 == 0:
            p = np.floor(p * 16) / 16
        for k1, k2 in ((3, 3), (3, 2), (2, 3), (2, 2)):
            q1 = p[:3] if k1 == 3 else p[:2]
            q2 = p[3:] if k2 == 3 else p[3:5]
            if (k1 == 3 and O.orient2d(*q1) == 0) or (k2 == 3 and O.orient2d(*q2) == 0):
                continue
            mine = O.compare_rho(k1, q1, k2, q2)
            dev = L.ref_compare_slow(k1, P(q1), k2, P(q2))
            if dev >= -1:  # -2..-4: the reference's 200-double scratch overflowed
                assert dev == mine, (k1, k2, p)
            cpu = L.ref_compare_cpu(k1, P(q1), k2, P(q2))
            if k1 == 2 and k2 == 2:
                mismatches_ee_cpu += cpu != mine  # stale-buffer bug of predicates.h:3064-3080
            else:
                assert cpu == mine, (k1, k2, p)
        assert L.ref_is_attached(P(p[0]), P(p[1]), P(p[2])) == O.is_attached(p[0], p[1], p[2])
    # the reference's FP64 birth-time formulas are what spectrum_ref reports
    pts = rng.random((200, 2))
    v, nb, _ = O.dt(pts)
    a = O.alpha(pts, v, nb)
    ref_vals = set()
    for t in v:
        ref_vals.add(L.ref_birth_time3(P(pts[t].ravel())))
    for e in a["edge"]:
        ref_vals.add(L.ref_birth_time2(P(pts[[e[0], e[1]]].ravel())))
    assert set(a["spectrum_ref"][1:].tolist()) <= ref_vals


@pytest.mark.parametrize("name", ["ref_bird", "ref_alpha", "ref_1000_1", "c1"])
def test_alpha_golden(name):
    g = np.load(os.path.join(GOLD, "golden_%s.npz" % name))
    pts = g["points"]
    v, nb, _ = O.dt(pts)
    a = O.alpha(pts, v, nb)
    assert np.array_equal(a["spectrum"], g["spectrum"])
    assert np.array_equal(a["point"], g["point"])


def test_master_list_restatement_matches_loop():
    """oracle.master_list (numpy) against a direct loop over the reference's
    steps: stable sort by rank, drop rank 0, first index of each run, -1 first."""
    g = np.load(os.path.join(GOLD, "golden_c1.npz"))
    pts = np.concatenate([g["points"], g["points"][:5]])  # duplicates give rank -1 vertices
    v, nb, _ = O.dt(pts)
    a = O.alpha(pts, v, nb)
    e = a["edge"]
    idx, st, at, sp = O.master_list(a["point"], e[:, 2], e[:, 3], e[:, 4], a["tri_ro"])
    n, ne, nt = len(a["point"]), len(e), len(a["tri_ro"])
    entries = []
    for k in range(2 * n + 3 * ne + nt):
        if k < 2 * n:
            r, ent = int(a["point"][k // 2][k % 2]), (k // 2, 2, 1 + k % 2)
        elif k < 2 * n + 3 * ne:
            q = k - 2 * n
            r, ent = int(e[q // 3][2 + q % 3]), (q // 3, 0, q % 3)
        else:
            r, ent = int(a["tri_ro"][k - 2 * n - 3 * ne]), (k - 2 * n - 3 * ne, 1, 0)
        entries.append((r, k, ent))
    entries.sort()
    kept = [(r, ent) for r, k, ent in entries if r != 0]
    assert [x[1] for x in kept] == list(zip(idx.tolist(), st.tolist(), at.tolist()))
    firsts = [-1] + [i for i in range(len(kept)) if i == 0 or kept[i][0] != kept[i - 1][0]]
    assert firsts == sp.tolist()
