"""CPU oracle loader -- TEST INFRASTRUCTURE, not product code.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline /
reference arm may import this module, and only as the checker.  It wraps
``oracle/_build/liboracle.so`` (built from oracle/*.c by oracle/Makefile):

* ``dt(points)``            exact Delaunay triangulation (oracle/dt.c), the
                            output contract of gpudtComputeDT (gpudt/gpudt.h:131)
* ``alpha(points, v, n)``   alpha spectrum + intervals (oracle/alpha.c), the
                            output of Alpha_Shapes_2D::computeAlphaShapes
                            (gpudt/AlphaShape/Alpha_Shapes_2D.cu:206-727)
* ``master_list(...)``      master list + spec pointers (numpy restatement of
                            compute_master_list, Alpha_Shapes_2D.cu:641-727)
* exact predicates for cross-checks.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class _AlphaOut(ctypes.Structure):
    _fields_ = [
        ("nspec", ctypes.c_int),
        ("spectrum", _dp),
        ("spectrum_ref", _dp),
        ("tri_ro", _ip),
        ("edge", _ip),
        ("point", _ip),
        ("exact_compares", ctypes.c_longlong),
        ("exact_ties", ctypes.c_longlong),
    ]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.oracle_dt.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip]
        L.oracle_cdt.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip, _ip, _ip]
        L.oracle_dt.restype = ctypes.c_int
        L.oracle_cdt.restype = ctypes.c_int
        L.oracle_orient2d.argtypes = [_dp, _dp, _dp]
        L.oracle_incircle.argtypes = [_dp, _dp, _dp, _dp]
        L.oracle_exact_counts.argtypes = [ctypes.c_int]
        L.oracle_exact_counts.restype = ctypes.c_longlong
        L.oracle_check_mesh.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_alpha_count_edges.argtypes = [ctypes.c_int, _ip, _ip]
        L.oracle_alpha.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, ctypes.POINTER(_AlphaOut)]
        L.oracle_compare_rho.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp]
        L.oracle_is_attached.argtypes = [_dp, _dp, _dp]
        L.oracle_rho_rounded.argtypes = [ctypes.c_int, _dp]
        L.oracle_rho_rounded.restype = ctypes.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def dt(points):
    """Exact DT.  Returns (vtx[T,3] int32, nbr[T,3] int32, n_distinct)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    n = pts.shape[0]
    cap = max(2 * n, 8)
    vtx = np.empty((cap, 3), dtype=np.int32)
    nbr = np.empty((cap, 3), dtype=np.int32)
    kept = np.zeros(1, dtype=np.int32)
    nt = lib().oracle_dt(n, _d(pts), cap, _i(vtx), _i(nbr), _i(kept))
    if nt < 0:
        raise RuntimeError("oracle_dt failed with status %d" % nt)
    return vtx[:nt].copy(), nbr[:nt].copy(), int(kept[0])


def cdt(points, constraints):
    """Exact constrained DT (oracle_cdt).  constraints: (M, 2) point indices.
    Returns (vtx[T,3] int32, nbr[T,3] int32, n_distinct)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    cons = np.ascontiguousarray(constraints, dtype=np.int32).reshape(-1, 2)
    n = pts.shape[0]
    cap = max(2 * n, 8)
    vtx = np.empty((cap, 3), dtype=np.int32)
    nbr = np.empty((cap, 3), dtype=np.int32)
    kept = np.zeros(1, dtype=np.int32)
    nt = lib().oracle_cdt(n, _d(pts), cons.shape[0], _i(cons), cap, _i(vtx), _i(nbr), _i(kept))
    if nt < 0:
        raise RuntimeError("oracle_cdt failed with status %d" % nt)
    return vtx[:nt].copy(), nbr[:nt].copy(), int(kept[0])


def check_mesh(points, vtx, nbr):
    """Exact validation of a triangle mesh (checkResult invariants, main.cu:163-343).

    Returns dict: links, ccw, delaunay, hull_edges, nonconvex, bad_index."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    vtx = np.ascontiguousarray(vtx, dtype=np.int32).reshape(-1, 3)
    nbr = np.ascontiguousarray(nbr, dtype=np.int32).reshape(-1, 3)
    out = (ctypes.c_longlong * 6)()
    lib().oracle_check_mesh(pts.shape[0], _d(pts), vtx.shape[0], _i(vtx), _i(nbr), out)
    keys = ["links", "ccw", "delaunay", "hull_edges", "nonconvex", "bad_index"]
    return {k: int(out[i]) for i, k in enumerate(keys)}


def alpha(points, vtx, nbr):
    """Alpha spectrum and intervals of triangulation (vtx, nbr)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    vtx = np.ascontiguousarray(vtx, dtype=np.int32)
    nbr = np.ascontiguousarray(nbr, dtype=np.int32)
    n, nt = pts.shape[0], vtx.shape[0]
    L = lib()
    ne = L.oracle_alpha_count_edges(nt, _i(vtx), _i(nbr))
    spec = np.zeros(1 + nt + ne, dtype=np.float64)
    spec_ref = np.zeros(1 + nt + ne, dtype=np.float64)
    tri_ro = np.zeros(nt, dtype=np.int32)
    edge = np.zeros((ne, 7), dtype=np.int32)
    point = np.zeros((n, 2), dtype=np.int32)
    out = _AlphaOut(0, _d(spec), _d(spec_ref), _i(tri_ro), _i(edge), _i(point), 0, 0)
    st = L.oracle_alpha(n, _d(pts), nt, _i(vtx), _i(nbr), ctypes.byref(out))
    if st != 0:
        raise RuntimeError("oracle_alpha failed with status %d" % st)
    k = out.nspec
    return {
        "spectrum": spec[:k].copy(),
        "spectrum_ref": spec_ref[:k].copy(),
        "tri_ro": tri_ro,
        "edge": edge,  # p1, p2, ro, nu_min, nu_max, tIndex, vOpp
        "point": point,
        "exact_compares": out.exact_compares,
        "exact_ties": out.exact_ties,
    }


def master_list(point_nu, edge_ro, edge_nu_min, edge_nu_max, tri_ro):
    """Master list of Alpha_Shapes_2D::compute_master_list (Alpha_Shapes_2D.cu:
    641-727) from the intervals.  Entry k of the unsorted list follows the kernel
    computeMasterList (kernel.cu:626-690): 2 per vertex (nu_min, nu_max), 3 per
    edge (ro, nu_min, nu_max), 1 per triangle (ro); each is keyed by its rank.
    thrust::sort_by_key on int keys is a stable radix sort, remove_if drops rank
    0 keeping order, unique_by_key over a sequence keeps the first index of each
    rank run, and -1 is prepended.  Returns (simplex_index, st, at, spec_pointers)
    with st 0 edge / 1 triangle / 2 vertex and at 0 ro / 1 nu_min / 2 nu_max."""
    point_nu = np.asarray(point_nu, dtype=np.int64).reshape(-1, 2)
    n, ne, nt = len(point_nu), len(edge_ro), len(tri_ro)
    ranks = np.concatenate([
        point_nu.reshape(-1),
        np.stack([np.asarray(edge_ro), np.asarray(edge_nu_min), np.asarray(edge_nu_max)], axis=1).reshape(-1),
        np.asarray(tri_ro),
    ]).astype(np.int64)
    k = np.arange(len(ranks), dtype=np.int64)
    st = np.concatenate([np.full(2 * n, 2), np.full(3 * ne, 0), np.full(nt, 1)])
    at = np.concatenate([np.tile([1, 2], n), np.tile([0, 1, 2], ne), np.zeros(nt, np.int64)])
    idx = np.concatenate([np.repeat(np.arange(n), 2), np.repeat(np.arange(ne), 3), np.arange(nt)])
    order = np.argsort(ranks, kind="stable")
    order = order[ranks[order] != 0]
    r = ranks[order]
    first = np.flatnonzero(np.concatenate([[True], r[1:] != r[:-1]])) if len(r) else np.zeros(0, np.int64)
    spec_pointers = np.concatenate([[-1], first]).astype(np.int32)
    return (idx[order].astype(np.int32), st[order].astype(np.int32), at[order].astype(np.int32), spec_pointers)


def orient2d(a, b, c):
    a, b, c = (np.asarray(x, dtype=np.float64) for x in (a, b, c))
    return lib().oracle_orient2d(_d(a), _d(b), _d(c))


def incircle(a, b, c, d):
    a, b, c, d = (np.asarray(x, dtype=np.float64) for x in (a, b, c, d))
    return lib().oracle_incircle(_d(a), _d(b), _d(c), _d(d))


def compare_rho(kind1, p1, kind2, p2):
    p1 = np.ascontiguousarray(p1, dtype=np.float64).ravel()
    p2 = np.ascontiguousarray(p2, dtype=np.float64).ravel()
    return lib().oracle_compare_rho(kind1, _d(p1), kind2, _d(p2))


def is_attached(i, j, k):
    i, j, k = (np.asarray(x, dtype=np.float64) for x in (i, j, k))
    return lib().oracle_is_attached(_d(i), _d(j), _d(k))


def rho_rounded(kind, p):
    p = np.ascontiguousarray(p, dtype=np.float64).ravel()
    return lib().oracle_rho_rounded(kind, _d(p))
