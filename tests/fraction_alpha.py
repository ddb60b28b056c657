"""Independent exact (rational) restatement of the GAlpha interval semantics.

Used by the CPU tests to pin the C oracle (oracle/alpha.c) at small sizes with
Python's exact ``fractions.Fraction`` arithmetic -- a different exact method
from the oracle's floating-point expansions.  The semantics follow
gpudt/AlphaShape/kernel.cu:160-624 (edge ownership, birth times, attached test,
intervals) and Alpha_Shapes_2D.cu:308-639 (exact sort, tie merging, ranks).
"""
from fractions import Fraction


def rho_tri(P, a, b, c):
    (x1, y1), (x2, y2), (x3, y3) = P[a], P[b], P[c]
    la = (x1 - x2) ** 2 + (y1 - y2) ** 2
    lb = (x2 - x3) ** 2 + (y2 - y3) ** 2
    lc = (x3 - x1) ** 2 + (y3 - y1) ** 2
    ar = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    return la * lb * lc / (4 * ar * ar)


def rho_edge(P, a, b):
    (x1, y1), (x2, y2) = P[a], P[b]
    return ((x1 - x2) ** 2 + (y1 - y2) ** 2) / 4


def attached(P, i, j, k):
    (xi, yi), (xj, yj), (xk, yk) = P[i], P[j], P[k]
    d1 = (xi - xj) ** 2 + (yi - yj) ** 2
    d2 = (xi + xj - 2 * xk) ** 2 + (yi + yj - 2 * yk) ** 2
    return d1 - d2 >= 0


def alpha_exact(points, vtx, nbr):
    P = [(Fraction(float(x)), Fraction(float(y))) for x, y in points]
    nt = len(vtx)
    edges = []
    for t in range(nt):
        for i in range(3):
            p1, p2 = int(vtx[t][(i + 1) % 3]), int(vtx[t][(i + 2) % 3])
            if p1 < p2 or nbr[t][i] == -1:
                edges.append([p1, p2, -1, 0, 0, t, i])
    entries = []
    for t in range(nt):
        entries.append((rho_tri(P, *[int(v) for v in vtx[t]]), 3, t))
    for e, E in enumerate(edges):
        p1, p2, _, _, _, t, i = E
        att = attached(P, p1, p2, int(vtx[t][i]))
        nb = int(nbr[t][i])
        if not att and nb != -1:
            att = attached(P, p1, p2, int(vtx[nb >> 2][nb & 3]))
        if att:
            E[2] = 0
        else:
            entries.append((rho_edge(P, p1, p2), 2, e))
    entries.sort(key=lambda s: s[0])
    spectrum = [Fraction(0)]
    tri_ro = [0] * nt
    prev = None
    for val, kind, idx in entries:
        if prev is None or val != prev:
            spectrum.append(val)
        prev = val
        r = len(spectrum) - 1
        if kind == 3:
            tri_ro[idx] = r
        else:
            edges[idx][2] = r
    for E in edges:
        t, i = E[5], E[6]
        nb = int(nbr[t][i])
        tr = tri_ro[t]
        if nb == -1:
            E[3], E[4] = tr, 0
        else:
            o = tri_ro[nb >> 2]
            E[3], E[4] = min(tr, o), max(tr, o)
    point = [[-1, -1] for _ in range(len(points))]
    seen = [False] * len(points)
    for E in edges:
        vmin = E[2] if E[2] != 0 else E[3]
        for v in (E[0], E[1]):
            if not seen[v]:
                seen[v] = True
                point[v] = [vmin, E[4]]
            else:
                point[v][0] = min(point[v][0], vmin)
                point[v][1] = max(point[v][1], E[4])
    return {"spectrum": spectrum, "tri_ro": tri_ro, "edge": edges, "point": point}
