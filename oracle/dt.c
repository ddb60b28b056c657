/*
 * oracle/dt.c -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU oracle for the Delaunay triangulation that gpudtComputeDT returns
 * (gpudt/gpudt.h:131, gpudt/gpudt.cpp:771-924).  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may use
 * it, and only as the checker.
 *
 * What the reference's path guarantees about its output, and what this oracle
 * therefore reproduces:
 *   - exact duplicates are dropped; the survivor is the lowest input index
 *     (the racy survivor of kernelVoronoi.h:72-73 / cudaMissing.cu:285-289,
 *     canonicalised);
 *   - triangles are counterclockwise under exact orientation (main.cu:205-216);
 *   - every interior edge is locally Delaunay under the exact in-circle test,
 *     i.e. the opposite apex is not strictly inside (main.cu:292-326,
 *     gpudt.cpp:160-189: a flip needs incircle > 0);
 *   - the triangulation covers the convex hull, collinear hull points stay
 *     vertices (cudaBoundary.cu:278 patches with ccw > 0 only);
 *   - neighbour links follow gpudt.h:97-102: tri[i] = (t << 2) | j is the
 *     neighbour across the edge opposite vtx[i], j the index of the apex of the
 *     neighbour opposite that edge; -1 on the hull.
 *
 * Algorithm: lexicographic sweep (each new point is outside the hull of the
 * previous ones; the visible hull edges are fanned to it), followed by Lawson
 * legalisation with the exact in-circle test.  The flip itself restates the
 * reference's flip() (gpudt.cpp:88-155) and recursive legalisation
 * (gpudtRecursiveFlip, gpudt.cpp:191-304).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "pred.h"
#include "oracle.h"

_Thread_local long long oracle_exact_orient_calls = 0;
_Thread_local long long oracle_exact_incircle_calls = 0;

typedef struct {
    const double *xy;
    int *v;   /* 3 per triangle */
    int *n;   /* 3 per triangle */
    int nt, cap;
    int *hnext, *hprev, *htri; /* hull cycle, htri[u] = (t<<2)|j: edge u->hnext[u] */
    int *stack;
    int stack_cap;
} dtctx;

#define P(i) (c->xy + 2 * (size_t)(i))

static int new_tri(dtctx *c, int a, int b, int d)
{
    int t = c->nt++;
    c->v[3 * t] = a; c->v[3 * t + 1] = b; c->v[3 * t + 2] = d;
    c->n[3 * t] = c->n[3 * t + 1] = c->n[3 * t + 2] = -1;
    return t;
}

static void bond(dtctx *c, int t, int i, int u, int j)
{
    if (t >= 0) c->n[3 * t + i] = (u >= 0) ? ((u << 2) | j) : -1;
    if (u >= 0) c->n[3 * u + j] = (t >= 0) ? ((t << 2) | i) : -1;
}

/* Flip the edge of t opposite vtx[i] (cf. gpudt.cpp:88-155).  t becomes
 * (a, b, d), the neighbour u becomes (d, c, a), a = apex of t, d = apex of u. */
static void flip(dtctx *c, int t, int i)
{
    int e = c->n[3 * t + i];
    int u = e >> 2, j = e & 3;
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    int a = c->v[3 * t + i], b = c->v[3 * t + i1], cc = c->v[3 * t + i2], d = c->v[3 * u + j];
    int nti1 = c->n[3 * t + i1], nti2 = c->n[3 * t + i2];
    int nuj1 = c->n[3 * u + j1], nuj2 = c->n[3 * u + j2];
    c->v[3 * t] = a; c->v[3 * t + 1] = b; c->v[3 * t + 2] = d;
    c->v[3 * u] = d; c->v[3 * u + 1] = cc; c->v[3 * u + 2] = a;
    /* t: opp a = (b,d) <- u's old edge b->d (opp c, index j1); opp b = (d,a) <- u;
     *    opp d = (a,b) <- t's old edge (opp c, index i2)
     * u: opp d = (c,a) <- t's old edge (opp b, index i1); opp c = (a,d) <- t;
     *    opp a = (d,c) <- u's old edge (opp b, index j2) */
    bond(c, t, 0, nuj1 >= 0 ? nuj1 >> 2 : -1, nuj1 & 3);
    bond(c, t, 2, nti2 >= 0 ? nti2 >> 2 : -1, nti2 & 3);
    bond(c, u, 0, nti1 >= 0 ? nti1 >> 2 : -1, nti1 & 3);
    bond(c, u, 2, nuj2 >= 0 ? nuj2 >> 2 : -1, nuj2 & 3);
    bond(c, t, 1, u, 1);
    /* keep hull records valid: a hull edge that moved changes (t, index) */
    if (nuj1 < 0) c->htri[b] = (t << 2) | 0;
    if (nti2 < 0) c->htri[a] = (t << 2) | 2;
    if (nti1 < 0) c->htri[cc] = (u << 2) | 0;
    if (nuj2 < 0) c->htri[d] = (u << 2) | 2;
}

/* Legalise the edge of t opposite vtx[i], and recursively the edges it exposes
 * (cf. gpudtRecursiveFlip, gpudt.cpp:191-304).  Explicit stack of (t,i). */
static int legalize(dtctx *c, int t0, int i0)
{
    int sp = 0;
    c->stack[sp++] = (t0 << 2) | i0;
    while (sp > 0) {
        int e = c->stack[--sp], t = e >> 2, i = e & 3;
        int ne = c->n[3 * t + i];
        if (ne < 0) continue;
        int u = ne >> 2, j = ne & 3;
        int a = c->v[3 * t + i], b = c->v[3 * t + (i + 1) % 3], cc = c->v[3 * t + (i + 2) % 3];
        int d = c->v[3 * u + j];
        if (orx_incircle(P(b), P(cc), P(a), P(d)) > 0) {
            flip(c, t, i);
            /* new t = (a,b,d): edge (b,d) opposite a (index 0);
             * new u = (d,c,a): edge (d,c) opposite a (index 2) */
            if (sp + 2 > c->stack_cap) return -1;
            c->stack[sp++] = (t << 2) | 0;
            c->stack[sp++] = (u << 2) | 2;
        }
    }
    return 0;
}

static const double *g_sort_xy;
static int cmp_lex(const void *pa, const void *pb)
{
    int a = *(const int *)pa, b = *(const int *)pb;
    const double *A = g_sort_xy + 2 * (size_t)a, *B = g_sort_xy + 2 * (size_t)b;
    if (A[0] < B[0]) return -1;
    if (A[0] > B[0]) return 1;
    if (A[1] < B[1]) return -1;
    if (A[1] > B[1]) return 1;
    return (a > b) - (a < b);
}

int oracle_dt(int npts, const double *xy, int cap, int *out_vtx, int *out_nbr, int *out_nkept)
{
    dtctx C, *c = &C;
    int *ord, m = 0, k, i, status = 0;
    if (npts < 0) return ORACLE_ERR_ARG;
    for (i = 0; i < npts; i++)
        if (!isfinite(xy[2 * i]) || !isfinite(xy[2 * i + 1])) return ORACLE_ERR_ARG;
    memset(c, 0, sizeof(*c));
    c->xy = xy;
    c->v = out_vtx;
    c->n = out_nbr;
    c->cap = cap;
    ord = (int *)malloc(sizeof(int) * (size_t)(npts > 0 ? npts : 1));
    c->hnext = (int *)malloc(sizeof(int) * (size_t)(npts + 1));
    c->hprev = (int *)malloc(sizeof(int) * (size_t)(npts + 1));
    c->htri = (int *)malloc(sizeof(int) * (size_t)(npts + 1));
    c->stack_cap = 4 * npts + 64;
    c->stack = (int *)malloc(sizeof(int) * (size_t)c->stack_cap);
    for (i = 0; i < npts; i++) ord[i] = i;
    g_sort_xy = xy;
    qsort(ord, (size_t)npts, sizeof(int), cmp_lex);
    /* drop exact duplicates, keep the lowest index (first after the index tie-break) */
    for (i = 0; i < npts; i++) {
        if (m > 0) {
            const double *A = P(ord[m - 1]), *B = P(ord[i]);
            if (A[0] == B[0] && A[1] == B[1]) continue;
        }
        ord[m++] = ord[i];
    }
    if (out_nkept) *out_nkept = m;
    /* collinear prefix */
    k = 2;
    while (k < m && orx_orient2d(P(ord[0]), P(ord[1]), P(ord[k])) == 0) k++;
    if (m < 3 || k >= m) {
        status = 0; /* all collinear (or < 3 points): no triangle */
        goto done;
    }
    if ((size_t)(k - 1) > (size_t)cap) { status = ORACLE_ERR_CAP; goto done; }
    {
        int p = ord[k];
        int left = orx_orient2d(P(ord[0]), P(ord[1]), P(p)) > 0;
        int prev = -1;
        for (i = 0; i + 1 < k; i++) {
            int ci = ord[i], cj = ord[i + 1], t;
            if (left) {
                t = new_tri(c, ci, cj, p);           /* edge ci->cj opp p (2) */
                if (prev >= 0) bond(c, t, 1, prev, 0); /* (p,ci) opp cj  <->  prev's (cj',p) opp ci' */
                c->htri[ci] = (t << 2) | 2;
                c->hnext[ci] = cj; c->hprev[cj] = ci;
            } else {
                t = new_tri(c, cj, ci, p);           /* edge cj->ci opp p (2) */
                if (prev >= 0) bond(c, t, 0, prev, 1); /* (ci,p) opp cj  <->  prev's (p,ci') opp... */
                c->htri[cj] = (t << 2) | 2;
                c->hnext[cj] = ci; c->hprev[ci] = cj;
            }
            prev = t;
        }
        {
            int c0 = ord[0], cl = ord[k - 1];
            int t0 = 0, tl = c->nt - 1;
            if (left) {
                /* cycle c0 -> ... -> cl -> p -> c0 */
                c->hnext[cl] = p; c->hprev[p] = cl; c->htri[cl] = (tl << 2) | 0;
                c->hnext[p] = c0; c->hprev[c0] = p; c->htri[p] = (t0 << 2) | 1;
            } else {
                /* cycle c0 -> p -> cl -> ... -> c0 */
                c->hnext[c0] = p; c->hprev[p] = c0; c->htri[c0] = (t0 << 2) | 0;
                c->hnext[p] = cl; c->hprev[cl] = p; c->htri[p] = (tl << 2) | 1;
            }
        }
        for (i = 0; i < c->nt; i++)
            if (legalize(c, i, 2) < 0) { status = ORACLE_ERR_CAP; goto done; }
    }
    for (int s = k + 1; s < m; s++) {
        int p = ord[s], v0 = ord[s - 1];
        int a, b, u;
        /* visible edges u->hnext[u]: orient(u, hnext[u], p) < 0 */
        a = v0;
        if (orx_orient2d(P(a), P(c->hnext[a]), P(p)) >= 0 && orx_orient2d(P(c->hprev[a]), P(a), P(p)) >= 0) {
            /* defensive: scan the whole hull for a visible edge */
            int w = v0, found = -1;
            do {
                if (orx_orient2d(P(w), P(c->hnext[w]), P(p)) < 0) { found = w; break; }
                w = c->hnext[w];
            } while (w != v0);
            if (found < 0) { status = ORACLE_ERR_TOPOLOGY; goto done; }
            a = found;
        }
        /* extend backwards and forwards */
        if (orx_orient2d(P(a), P(c->hnext[a]), P(p)) >= 0) a = c->hprev[a];
        while (orx_orient2d(P(c->hprev[a]), P(a), P(p)) < 0) a = c->hprev[a];
        b = a;
        while (orx_orient2d(P(b), P(c->hnext[b]), P(p)) < 0) b = c->hnext[b];
        /* fan p to edges a -> ... -> b */
        {
            int prev = -1, first = -1, t;
            for (u = a; u != b; ) {
                int w = c->hnext[u];
                int he = c->htri[u];
                if (c->nt + 1 > cap) { status = ORACLE_ERR_CAP; goto done; }
                t = new_tri(c, w, u, p);             /* edge w->u opp p (2) */
                bond(c, t, 2, he >> 2, he & 3);
                if (prev >= 0) bond(c, t, 0, prev, 1); /* t.(u,p) <-> prev.(p,u) */
                if (first < 0) first = t;
                prev = t;
                u = w;
            }
            /* consecutive visible edges u0->u1, u1->u2 give t1 = (u1,u0,p) and
             * t2 = (u2,u1,p); they share (u1,p): index 1 of t1, index 0 of t2. */
            c->hnext[a] = p; c->hprev[p] = a; c->htri[a] = (first << 2) | 0;
            c->hnext[p] = b; c->hprev[b] = p; c->htri[p] = (prev << 2) | 1;
            for (t = first; t <= prev; t++)
                if (legalize(c, t, 2) < 0) { status = ORACLE_ERR_CAP; goto done; }
        }
    }
done:
    free(ord);
    free(c->hnext);
    free(c->hprev);
    free(c->htri);
    free(c->stack);
    if (status < 0) return status;
    return c->nt;
}

/*
 * Mesh validator: the invariants of the reference's checkResult (main.cu:163-343)
 * with exact predicates, plus link symmetry and the convex-hull boundary.
 * out[0] link errors, out[1] non-counterclockwise triangles, out[2] interior
 * edges failing the exact empty-circle test (incircle > 0), out[3] hull edges,
 * out[4] hull edges with some point strictly outside (non-convex hull),
 * out[5] vertex indices out of range.
 */
int oracle_check_mesh(int npts, const double *xy, int ntri, const int *vtx, const int *nbr, long long *out)
{
    int t, i;
    for (i = 0; i < 6; i++) out[i] = 0;
    for (t = 0; t < ntri; t++)
        for (i = 0; i < 3; i++)
            if (vtx[3 * t + i] < 0 || vtx[3 * t + i] >= npts) out[5]++;
    if (out[5]) return -1;
    for (t = 0; t < ntri; t++) {
        const int *v = vtx + 3 * t;
        if (orx_orient2d(xy + 2 * v[0], xy + 2 * v[1], xy + 2 * v[2]) <= 0) out[1]++;
        for (i = 0; i < 3; i++) {
            int e = nbr[3 * t + i];
            int a = v[(i + 1) % 3], b = v[(i + 2) % 3];
            if (e < 0) {
                out[3]++;
                continue;
            }
            int u = e >> 2, j = e & 3;
            if (u < 0 || u >= ntri || j > 2 || nbr[3 * u + j] != ((t << 2) | i) || vtx[3 * u + (j + 1) % 3] != b ||
                vtx[3 * u + (j + 2) % 3] != a) {
                out[0]++;
                continue;
            }
            if (orx_incircle(xy + 2 * a, xy + 2 * b, xy + 2 * v[i], xy + 2 * vtx[3 * u + j]) > 0) out[2]++;
        }
    }
    /* hull edges: no input point strictly to the right of a -> b */
    {
        int *ha = (int *)malloc(sizeof(int) * (size_t)(out[3] + 1)), *hb = (int *)malloc(sizeof(int) * (size_t)(out[3] + 1));
        int nh = 0, k;
        for (t = 0; t < ntri; t++)
            for (i = 0; i < 3; i++)
                if (nbr[3 * t + i] < 0) {
                    ha[nh] = vtx[3 * t + (i + 1) % 3];
                    hb[nh] = vtx[3 * t + (i + 2) % 3];
                    nh++;
                }
        if (nh <= 4096)
            for (k = 0; k < nh; k++)
                for (i = 0; i < npts; i++)
                    if (orx_orient2d(xy + 2 * ha[k], xy + 2 * hb[k], xy + 2 * i) < 0) {
                        out[4]++;
                        break;
                    }
        free(ha);
        free(hb);
    }
    return 0;
}
