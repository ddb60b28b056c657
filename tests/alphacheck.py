"""Parity helpers for the alpha stage: compare engine output with oracle.alpha
on the same triangle array (edge numbering follows triangle order,
kernel.cu:138-217, so both sides must see identical triangles)."""
import numpy as np

from oracle import oracle as O


def ulp_diff(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def compare_alpha(points, vtx, nbr, res, ulp_tol=4):
    """res: dict from Engine.alpha_*().  Returns (ok, report)."""
    ref = O.alpha(points, vtx, nbr)
    rep = {}
    spec, rspec = res["spectrum"], ref["spectrum"]
    rep["nspec"] = (len(spec), len(rspec))
    same_len = len(spec) == len(rspec)
    maxulp = int(ulp_diff(spec, rspec).max()) if same_len and len(spec) else -1
    rep["spectrum_max_ulp"] = maxulp
    rep["ref_formula_max_ulp"] = int(ulp_diff(ref["spectrum_ref"], rspec).max()) if len(rspec) else 0
    tri_ok = np.array_equal(res["tri_list"]["ro_rank"], ref["tri_ro"])
    e = res["edge_list"]
    E = ref["edge"]
    edge_ok = (len(e) == len(E) and np.array_equal(e["ro_rank"], E[:, 2]) and np.array_equal(e["nu_min_rank"], E[:, 3])
               and np.array_equal(e["nu_max_rank"], E[:, 4]) and np.array_equal(e["tIndex"], E[:, 5])
               and np.array_equal(e["vOpp"], E[:, 6]))
    p = res["point_list"]
    pt_ok = np.array_equal(p["nu_min_rank"], ref["point"][:, 0]) and np.array_equal(p["nu_max_rank"], ref["point"][:, 1])
    rep.update(tri_ok=tri_ok, edge_ok=edge_ok, point_ok=pt_ok)
    ok = same_len and 0 <= maxulp <= ulp_tol and tri_ok and edge_ok and pt_ok
    if len(spec) == 1 and same_len:
        ok = tri_ok and edge_ok and pt_ok
    return ok, rep


def classify_intervals(res, alpha):
    """Alpha-complex classes (0 exterior, 1 singular, 2 regular, 3 interior)
    of points, edges and triangles at ``alpha``, from the interval output
    alone (numpy restatement of the rule documented for galphaQuery)."""
    spec = np.asarray(res["spectrum"], dtype=np.float64)
    R = -1 if alpha < 0 else int(np.searchsorted(spec, alpha, side="right") - 1)
    pt, ed, tr = res["point_list"], res["edge_list"], res["tri_list"]

    def interval(ro, nmin, nmax):
        c = np.zeros(len(nmin), np.uint8)
        c[(ro >= 0) & (ro <= R)] = 1
        c[nmin <= R] = 2
        c[(nmax > 0) & (nmax <= R)] = 3
        return c

    if R < 0:
        return np.zeros(len(pt), np.uint8), np.zeros(len(ed), np.uint8), np.zeros(len(tr), np.uint8), R
    pc = interval(np.zeros(len(pt), np.int64), pt["nu_min_rank"], pt["nu_max_rank"])
    pc[pt["nu_min_rank"] < 0] = 0
    ro = np.where(ed["ro_rank"] != 0, ed["ro_rank"], -1)
    ec = interval(ro, ed["nu_min_rank"], ed["nu_max_rank"])
    tc = np.where(tr["ro_rank"] <= R, 3, 0).astype(np.uint8)
    return pc, ec, tc, R


def canonical_alpha(vtx, res):
    """Order-free view of an alpha result: triangle -> ro, edge -> (ro, nu_min,
    nu_max) keyed by sorted vertex pair, plus the spectrum and point_list as
    they are (both independent of triangle order)."""
    vtx = np.asarray(vtx)
    tri = {}
    for t, r in zip(vtx.tolist(), res["tri_list"]["ro_rank"].tolist()):
        k = t.index(min(t))
        tri[tuple(t[k:] + t[:k])] = r
    edge = {}
    for E in res["edge_list"]:
        t, i = int(E["tIndex"]), int(E["vOpp"])
        a, b = int(vtx[t][(i + 1) % 3]), int(vtx[t][(i + 2) % 3])
        edge[(min(a, b), max(a, b))] = (int(E["ro_rank"]), int(E["nu_min_rank"]), int(E["nu_max_rank"]))
    return np.asarray(res["spectrum"]), tri, edge, np.asarray(res["point_list"])
