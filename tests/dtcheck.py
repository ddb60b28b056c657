"""Parity helpers: compare a triangulation against the CPU oracle.

A Delaunay triangulation is unique for points in general position, so there
the canonical triangle sets must be identical.  For degenerate input
(cocircular quads) any diagonal is valid (a flip needs incircle > 0,
gpudt.cpp:179,187), so the criterion is the reference's own: exact local
Delaunay on every edge, exact counterclockwise triangles, consistent links,
convex hull boundary, and the same triangle count and vertex set as the oracle.
"""
import numpy as np

from oracle import oracle as O


def canon_set(vtx):
    v = np.asarray(vtx, dtype=np.int64).reshape(-1, 3)
    if len(v) == 0:
        return set()
    r = np.argmin(v, axis=1)
    rows = np.arange(len(v))
    c = np.stack([v[rows, (r + k) % 3] for k in range(3)], axis=1)
    return set(map(tuple, c.tolist()))


def hull_edges(vtx, nbr):
    v = np.asarray(vtx).reshape(-1, 3)
    n = np.asarray(nbr).reshape(-1, 3)
    out = set()
    for i in range(3):
        m = n[:, i] < 0
        out |= set(zip(v[m, (i + 1) % 3].tolist(), v[m, (i + 2) % 3].tolist()))
    return out


def compare_dt(points, vtx, nbr, oracle_result=None):
    """Returns (ok, report).  ok requires every exact invariant; 'identical'
    in the report says whether the canonical triangle sets are equal."""
    ov, on, kept = oracle_result if oracle_result is not None else O.dt(points)
    chk = O.check_mesh(points, vtx, nbr)
    same_count = len(vtx) == len(ov)
    verts = set(np.unique(np.asarray(vtx)).tolist())
    overts = set(np.unique(np.asarray(ov)).tolist())
    identical = canon_set(vtx) == canon_set(ov)
    same_hull = hull_edges(vtx, nbr) == hull_edges(ov, on)
    ok = (chk["links"] == 0 and chk["ccw"] == 0 and chk["delaunay"] == 0 and chk["nonconvex"] == 0
          and chk["bad_index"] == 0 and same_count and verts == overts and same_hull)
    report = dict(chk, same_count=same_count, same_vertices=verts == overts, same_hull=same_hull,
                  identical=identical, ntri=len(vtx), oracle_ntri=len(ov))
    return ok, report
