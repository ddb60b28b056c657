/*
 * oracle/alpha.c -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU oracle for the GAlpha alpha-shape stage (Alpha_Shapes_2D::
 * computeAlphaShapes, gpudt/AlphaShape/Alpha_Shapes_2D.cu:206-233).  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
 * may use it, and only as the checker.
 *
 * Restated, step by step, from the reference:
 *   edge ownership and numbering  computeTriEdgeCount / exclusive_scan /
 *                                 computeEdgeTriMap (kernel.cu:138-217,
 *                                 Alpha_Shapes_2D.cu:127-154): triangle t owns
 *                                 its edge i (opposite vtx[i]) when
 *                                 vtx[i+1] < vtx[i+2] or tri[i] == -1; edges are
 *                                 numbered by triangle, then by i.
 *   birth times                   computeTriangleRo / computeEdgeRo
 *                                 (kernel.cu:219-308): triangle rho = R^2 =
 *                                 abc / (4 ar^2), edge rho = |pq|^2 / 4, the
 *                                 spectrum holds squared radii; entry 0 is the
 *                                 sentinel 0.
 *   attached edges                processAttached + isAttached(Slow)
 *                                 (kernel.cu:310-358, predicates.h:1359-1444):
 *                                 an edge is attached when an opposite apex lies
 *                                 in the closed diametral disc (exact sign of
 *                                 |pq|^2 - |p+q-2k|^2 >= 0); its ro_rank is 0 and
 *                                 it leaves the spectrum.
 *   sort and ranks                sort_spectrum + CPU_insertion_sort +
 *                                 processSpectrum + UpdateBackRefs
 *                                 (Alpha_Shapes_2D.cu:308-610, kernel.cu:360-401,
 *                                 kernel.cu:1016-1102): the exact order of the
 *                                 squared radii; exactly equal values share one
 *                                 rank; rank r indexes the deduplicated spectrum.
 *                                 The reference's own edge-edge CPU comparison
 *                                 reads stale buffers (predicates.h:3064-3080);
 *                                 the oracle uses the correct exact comparison.
 *   intervals                     edgeIntervals / computeVertexIntervals
 *                                 (kernel.cu:427-624): edge nu_min/nu_max are the
 *                                 min/max rank of its two triangles (hull edge:
 *                                 nu_min = its triangle's rank, nu_max = 0);
 *                                 vertex nu_min = min over incident edges of
 *                                 (ro_rank, or nu_min_rank when attached),
 *                                 vertex nu_max = max over incident edges of
 *                                 nu_max_rank; a vertex in no triangle keeps
 *                                 (-1, -1).
 * Spectrum values are exact-then-rounded (numerator and denominator as exact
 * expansions, quotient refined once); spectrum_ref carries the value of the
 * reference's own FP64 formula for the same rank.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "pred.h"
#include "oracle.h"

static _Thread_local double g_t1[ORX_CAP], g_t2[ORX_CAP];

/* |p - q|^2 exactly */
static int sqdist(const double *p, const double *q, double *h)
{
    double dx[2], dy[2], sx[64], sy[64];
    int ndx = orx_diff2(p[0], q[0], dx), ndy = orx_diff2(p[1], q[1], dy);
    int nsx = orx_mul(ndx, dx, ndx, dx, sx, g_t1, g_t2);
    int nsy = orx_mul(ndy, dy, ndy, dy, sy, g_t1, g_t2);
    return orx_compress(orx_sum(nsx, sx, nsy, sy, h), h);
}

/* rho = N / D as exact expansions.  kind 3: triangle p[0..5]; kind 2: edge p[0..3]. */
static int rho_nd(int kind, const double *p, double *N, int *nN, double *D, int *nD)
{
    if (kind == 2) {
        *nN = sqdist(p, p + 2, N);
        D[0] = 4.0;
        *nD = 1;
        return 0;
    } else {
        double la[128], lb[128], lc[128], ab[512];
        double ux[2], uy[2], vx[2], vy[2], m1[64], m2[64], ar[128], ar2[512];
        int na = sqdist(p, p + 2, la), nb = sqdist(p + 2, p + 4, lb), nc = sqdist(p + 4, p, lc);
        int nab = orx_mul(na, la, nb, lb, ab, g_t1, g_t2);
        if (nab < 0) return -1;
        *nN = orx_mul(nab, ab, nc, lc, N, g_t1, g_t2);
        if (*nN < 0) return -1;
        /* ar = (x2-x1)(y3-y1) - (x3-x1)(y2-y1) */
        int nux = orx_diff2(p[2], p[0], ux), nvy = orx_diff2(p[5], p[1], vy);
        int nvx = orx_diff2(p[4], p[0], vx), nuy = orx_diff2(p[3], p[1], uy);
        int n1 = orx_mul(nux, ux, nvy, vy, m1, g_t1, g_t2);
        int n2 = orx_mul(nvx, vx, nuy, uy, m2, g_t1, g_t2);
        orx_negate(n2, m2, m2);
        int nar = orx_compress(orx_sum(n1, m1, n2, m2, ar), ar);
        int nar2 = orx_mul(nar, ar, nar, ar, ar2, g_t1, g_t2);
        if (nar2 < 0) return -1;
        *nD = orx_scale(nar2, ar2, 4.0, D);
        return 0;
    }
}

static _Thread_local double g_N1[ORX_CAP], g_D1[ORX_CAP], g_N2[ORX_CAP], g_D2[ORX_CAP];
static _Thread_local double g_A[ORX_CAP], g_B[ORX_CAP], g_C[2 * ORX_CAP];
static _Thread_local long long g_exact_compares;

int oracle_compare_rho(int kind1, const double *p1, int kind2, const double *p2)
{
    int nN1, nD1, nN2, nD2, nA, nB, nC;
    g_exact_compares++;
    if (rho_nd(kind1, p1, g_N1, &nN1, g_D1, &nD1) < 0) return ORACLE_ERR_EXACT;
    if (rho_nd(kind2, p2, g_N2, &nN2, g_D2, &nD2) < 0) return ORACLE_ERR_EXACT;
    nA = orx_mul(nN1, g_N1, nD2, g_D2, g_A, g_t1, g_t2);
    nB = orx_mul(nN2, g_N2, nD1, g_D1, g_B, g_t1, g_t2);
    if (nA < 0 || nB < 0) return ORACLE_ERR_EXACT;
    orx_negate(nB, g_B, g_B);
    nC = orx_sum(nA, g_A, nB, g_B, g_C);
    return orx_sign(nC, g_C);
}

double oracle_rho_rounded(int kind, const double *p)
{
    int nN, nD, nq, nR;
    double q0, q1, dD;
    if (rho_nd(kind, p, g_N1, &nN, g_D1, &nD) < 0) return NAN;
    dD = orx_estimate(nD, g_D1);
    if (dD == 0.0) return INFINITY;
    q0 = orx_estimate(nN, g_N1) / dD;
    nq = orx_scale(nD, g_D1, -q0, g_A);
    nR = orx_sum(nN, g_N1, nq, g_A, g_C);
    nR = orx_compress(nR, g_C);
    q1 = orx_estimate(nR, g_C) / dD;
    return q0 + q1;
}

/* Reference FP64 formulas (predicates.h:1297-1357), evaluated as written. */
static double rho_ref(int kind, const double *p)
{
    if (kind == 2) {
        double ax = p[0] - p[2], ay = p[1] - p[3];
        ax = ax * ax;
        ay = ay * ay;
        return (ax + ay) / 4;
    } else {
        double x1 = p[0], y1 = p[1], x2 = p[2], y2 = p[3], x3 = p[4], y3 = p[5];
        double ax = x1 - x2, ay = y1 - y2, bx = x2 - x3, by = y2 - y3, cx = x3 - x1, cy = y3 - y1;
        ax = ax * ax; ay = ay * ay; bx = bx * bx; by = by * by; cx = cx * cx; cy = cy * cy;
        double a = ax + ay, b = bx + by, c = cx + cy;
        double ar1 = x2 * y3 - x3 * y2 - x1 * y3 + x3 * y1 + x1 * y2 - x2 * y1;
        double den = 4 * ar1 * ar1;
        return (a * b * c) / den;
    }
}

int oracle_is_attached(const double *i, const double *j, const double *k)
{
    /* d1 - d2 with d1 = |i-j|^2, d2 = |i + j - 2k|^2 (predicates.h:1359-1444) */
    double d1[128], sx[4], sy[4], ex[8], ey[8], k2x[1], k2y[1], qx[64], qy[64], d2[128], r[256];
    int nd1 = sqdist(i, j, d1);
    double hi, lo;
    int nsx = 0, nsy = 0, nex, ney;
    orx_two_sum(i[0], j[0], &hi, &lo);
    if (lo != 0.0) sx[nsx++] = lo;
    if (hi != 0.0) sx[nsx++] = hi;
    orx_two_sum(i[1], j[1], &hi, &lo);
    if (lo != 0.0) sy[nsy++] = lo;
    if (hi != 0.0) sy[nsy++] = hi;
    k2x[0] = -2.0 * k[0];
    k2y[0] = -2.0 * k[1];
    nex = orx_sum(nsx, sx, k2x[0] != 0.0, k2x, ex);
    ney = orx_sum(nsy, sy, k2y[0] != 0.0, k2y, ey);
    int nqx = orx_mul(nex, ex, nex, ex, qx, g_t1, g_t2);
    int nqy = orx_mul(ney, ey, ney, ey, qy, g_t1, g_t2);
    int nd2 = orx_sum(nqx, qx, nqy, qy, d2);
    orx_negate(nd2, d2, d2);
    int nr = orx_sum(nd1, d1, nd2, d2, r);
    return orx_sign(nr, r) >= 0;
}

int oracle_orient2d(const double *a, const double *b, const double *c) { return orx_orient2d(a, b, c); }
int oracle_incircle(const double *a, const double *b, const double *c, const double *d)
{
    return orx_incircle(a, b, c, d);
}
long long oracle_exact_counts(int which)
{
    if (which == 0) return oracle_exact_orient_calls;
    if (which == 1) return oracle_exact_incircle_calls;
    return g_exact_compares;
}

int oracle_alpha_count_edges(int ntri, const int *vtx, const int *nbr)
{
    int t, i, ne = 0;
    for (t = 0; t < ntri; t++)
        for (i = 0; i < 3; i++)
            if (vtx[3 * t + (i + 1) % 3] < vtx[3 * t + (i + 2) % 3] || nbr[3 * t + i] == -1) ne++;
    return ne;
}

typedef struct {
    double key;
    int kind;  /* 3 triangle, 2 edge */
    int idx;   /* triangle or edge id */
} sentry;

static int cmp_key(const void *pa, const void *pb)
{
    const sentry *a = (const sentry *)pa, *b = (const sentry *)pb;
    if (a->key < b->key) return -1;
    if (a->key > b->key) return 1;
    if (a->kind != b->kind) return a->kind < b->kind ? -1 : 1;
    return (a->idx > b->idx) - (a->idx < b->idx);
}

static void entry_pts(const sentry *s, const double *xy, const int *vtx, const int *edge, double *p)
{
    int k;
    if (s->kind == 3) {
        for (k = 0; k < 3; k++) {
            int v = vtx[3 * s->idx + k];
            p[2 * k] = xy[2 * v];
            p[2 * k + 1] = xy[2 * v + 1];
        }
    } else {
        int a = edge[7 * s->idx], b = edge[7 * s->idx + 1];
        p[0] = xy[2 * a]; p[1] = xy[2 * a + 1];
        p[2] = xy[2 * b]; p[3] = xy[2 * b + 1];
    }
}

static int exact_cmp_entries(const sentry *a, const sentry *b, const double *xy, const int *vtx,
                             const int *edge)
{
    double pa[6], pb[6];
    entry_pts(a, xy, vtx, edge, pa);
    entry_pts(b, xy, vtx, edge, pb);
    return oracle_compare_rho(a->kind, pa, b->kind, pb);
}

static int near_equal(double a, double b)
{
    /* true when b - a <= 4 ulp(b): the keys carry <= 1 ulp of error each */
    double u = nextafter(b, INFINITY) - b;
    return (b - a) <= 4.0 * u;
}

int oracle_alpha(int npts, const double *xy, int ntri, const int *vtx, const int *nbr,
                 oracle_alpha_out *out)
{
    int t, i, e, ne = oracle_alpha_count_edges(ntri, vtx, nbr);
    int *edge = out->edge;
    int nspec_in = 0, status = 0;
    sentry *S = (sentry *)malloc(sizeof(sentry) * (size_t)(1 + ntri + ne));
    int *rank_of = (int *)malloc(sizeof(int) * (size_t)(1 + ntri + ne));
    g_exact_compares = 0;
    out->exact_ties = 0;
    /* edges, in the reference's numbering */
    e = 0;
    for (t = 0; t < ntri; t++)
        for (i = 0; i < 3; i++) {
            int p1 = vtx[3 * t + (i + 1) % 3], p2 = vtx[3 * t + (i + 2) % 3];
            if (p1 < p2 || nbr[3 * t + i] == -1) {
                int *E = edge + 7 * e;
                E[0] = p1; E[1] = p2; E[2] = -1; E[3] = 0; E[4] = 0; E[5] = t; E[6] = i;
                e++;
            }
        }
    /* triangle birth times */
    for (t = 0; t < ntri; t++) {
        double p[6];
        S[nspec_in].kind = 3;
        S[nspec_in].idx = t;
        entry_pts(&S[nspec_in], xy, vtx, edge, p);
        S[nspec_in].key = oracle_rho_rounded(3, p);
        nspec_in++;
    }
    /* edges: attached test, then birth time of the unattached */
    for (e = 0; e < ne; e++) {
        int *E = edge + 7 * e, tt = E[5], vo = E[6];
        const double *pi = xy + 2 * E[0], *pj = xy + 2 * E[1];
        const double *apex = xy + 2 * vtx[3 * tt + vo];
        int att = oracle_is_attached(pi, pj, apex);
        int nb = nbr[3 * tt + vo];
        if (!att && nb != -1) {
            const double *apex2 = xy + 2 * vtx[3 * (nb >> 2) + (nb & 3)];
            att = oracle_is_attached(pi, pj, apex2);
        }
        if (att) {
            E[2] = 0;
        } else {
            double p[4] = {pi[0], pi[1], pj[0], pj[1]};
            S[nspec_in].kind = 2;
            S[nspec_in].idx = e;
            S[nspec_in].key = oracle_rho_rounded(2, p);
            nspec_in++;
        }
    }
    qsort(S, (size_t)nspec_in, sizeof(sentry), cmp_key);
    /* exact resolution of runs of near-equal keys (insertion sort, exact comparator) */
    for (i = 0; i < nspec_in;) {
        int j = i + 1;
        while (j < nspec_in && near_equal(S[j - 1].key, S[j].key)) j++;
        if (j - i > 1) {
            int a, b;
            for (a = i + 1; a < j; a++) {
                sentry cur = S[a];
                for (b = a - 1; b >= i; b--) {
                    int c = exact_cmp_entries(&S[b], &cur, xy, vtx, edge);
                    if (c == ORACLE_ERR_EXACT) { status = ORACLE_ERR_EXACT; goto done; }
                    if (c <= 0) break;
                    S[b + 1] = S[b];
                }
                S[b + 1] = cur;
            }
        }
        i = j;
    }
    /* ranks: exactly equal neighbours share a rank */
    {
        int r = 0;
        out->spectrum[0] = 0.0;
        out->spectrum_ref[0] = 0.0;
        for (i = 0; i < nspec_in; i++) {
            int same = 0;
            if (i > 0 && near_equal(S[i - 1].key, S[i].key)) {
                int c = exact_cmp_entries(&S[i - 1], &S[i], xy, vtx, edge);
                if (c == ORACLE_ERR_EXACT) { status = ORACLE_ERR_EXACT; goto done; }
                same = (c == 0);
            }
            if (!same) {
                double p[6];
                r++;
                out->spectrum[r] = S[i].key;
                entry_pts(&S[i], xy, vtx, edge, p);
                out->spectrum_ref[r] = rho_ref(S[i].kind, p);
            } else {
                out->exact_ties++;
            }
            if (S[i].kind == 3) out->tri_ro[S[i].idx] = r;
            else edge[7 * S[i].idx + 2] = r;
        }
        out->nspec = r + 1;
    }
    /* edge intervals (kernel.cu:427-462) */
    for (e = 0; e < ne; e++) {
        int *E = edge + 7 * e, tt = E[5], vo = E[6];
        int nb = nbr[3 * tt + vo], tr = out->tri_ro[tt];
        if (nb == -1) {
            E[3] = tr;
            E[4] = 0;
        } else {
            int orr = out->tri_ro[nb >> 2];
            E[3] = tr <= orr ? tr : orr;
            E[4] = tr <= orr ? orr : tr;
        }
    }
    /* vertex intervals (kernel.cu:518-624): min/max over incident edges */
    for (i = 0; i < npts; i++) {
        out->point[2 * i] = -1;
        out->point[2 * i + 1] = -1;
    }
    {
        char *seen = (char *)calloc((size_t)(npts > 0 ? npts : 1), 1);
        for (e = 0; e < ne; e++) {
            int *E = edge + 7 * e, k;
            int vmin = E[2] != 0 ? E[2] : E[3];
            for (k = 0; k < 2; k++) {
                int v = E[k];
                if (!seen[v]) {
                    seen[v] = 1;
                    out->point[2 * v] = vmin;
                    out->point[2 * v + 1] = E[4];
                } else {
                    if (vmin < out->point[2 * v]) out->point[2 * v] = vmin;
                    if (E[4] > out->point[2 * v + 1]) out->point[2 * v + 1] = E[4];
                }
            }
        }
        free(seen);
    }
done:
    out->exact_compares = g_exact_compares;
    free(S);
    free(rank_of);
    return status;
}
