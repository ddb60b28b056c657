/*
 * oracle/cdt.c -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU oracle for the constrained Delaunay triangulation that gpudtComputeDT
 * returns when GPUDTPARAMS.nConstraints > 0 (gpudt.cpp:860 cudaConstraint,
 * gpudt/Cuda/cudaConstraint.cu:828-939, and the constraint-aware flipping of
 * gpudt/Cuda/cudaFlipping.cu:111-220 / gpudt.cpp:88-155, where an edge marked
 * as a constraint is never flipped).
 *
 * The result is the constrained Delaunay triangulation: every constraint
 * segment is an edge, and every other interior edge is locally Delaunay under
 * the exact in-circle test.  For points in general position and constraints
 * that neither cross each other nor pass through a point it is unique, which
 * is what the GPU parity tests compare against.
 *
 * Algorithm (sequential, exact predicates):
 *   1. the exact DT (oracle_dt);
 *   2. each constraint (a, b) is inserted by flips: the edges its open segment
 *      crosses are found by walking from a and queued; Sloan's edge insertion
 *      by flipping (FIFO queue, convex quadrilaterals only, a new diagonal
 *      that still crosses goes back in the queue) removes every crossing;
 *   3. Lawson legalisation of every edge with the exact in-circle test, never
 *      flipping a constraint edge.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "pred.h"
#include "oracle.h"

typedef struct {
    const double *xy;
    int *v, *n;
    int nt;
    int *vt;                 /* vertex -> one incident triangle (t<<2 | index) */
    unsigned long long *set; /* open-addressing set of constraint pairs */
    int mask;
} cdt;

#define PT(i) (c->xy + 2 * (size_t)(i))

static unsigned long long pair_key(int a, int b)
{
    unsigned lo = (unsigned)(a < b ? a : b), hi = (unsigned)(a < b ? b : a);
    return ((unsigned long long)lo << 32) | hi;
}

static unsigned mix(unsigned long long k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return (unsigned)k;
}

static void set_add(cdt *c, int a, int b)
{
    unsigned long long k = pair_key(a, b);
    unsigned h = mix(k) & (unsigned)c->mask;
    while (c->set[h] != ~0ull && c->set[h] != k) h = (h + 1) & (unsigned)c->mask;
    c->set[h] = k;
}

static int set_has(const cdt *c, int a, int b)
{
    unsigned long long k = pair_key(a, b);
    unsigned h = mix(k) & (unsigned)c->mask;
    while (c->set[h] != ~0ull) {
        if (c->set[h] == k) return 1;
        h = (h + 1) & (unsigned)c->mask;
    }
    return 0;
}

static void bond(cdt *c, int t, int i, int e)
{
    c->n[3 * t + i] = e;
    if (e >= 0) c->n[3 * (e >> 2) + (e & 3)] = (t << 2) | i;
}

/* Flip the edge of t opposite vtx[i]: t becomes (a, b, d), its neighbour u
 * becomes (d, c, a), a = apex of t, d = apex of u (the gpudt.cpp:88-155 flip). */
static void flip(cdt *c, int t, int i)
{
    int e = c->n[3 * t + i], u = e >> 2, j = e & 3;
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    int a = c->v[3 * t + i], b = c->v[3 * t + i1], cc = c->v[3 * t + i2], d = c->v[3 * u + j];
    int nti1 = c->n[3 * t + i1], nti2 = c->n[3 * t + i2], nuj1 = c->n[3 * u + j1], nuj2 = c->n[3 * u + j2];
    c->v[3 * t] = a; c->v[3 * t + 1] = b; c->v[3 * t + 2] = d;
    c->v[3 * u] = d; c->v[3 * u + 1] = cc; c->v[3 * u + 2] = a;
    bond(c, t, 0, nuj1);
    bond(c, t, 2, nti2);
    bond(c, u, 0, nti1);
    bond(c, u, 2, nuj2);
    c->n[3 * t + 1] = (u << 2) | 1;
    c->n[3 * u + 1] = (t << 2) | 1;
    c->vt[a] = (t << 2) | 0;
    c->vt[b] = (t << 2) | 1;
    c->vt[d] = (t << 2) | 2;
    c->vt[cc] = (u << 2) | 1;
}

/* Edges crossed by the open segment a -> b, found by walking from a:
 * out[k] = (t << 2) | i, the edge of t opposite vtx[i].  Returns their count,
 * 0 if (a, b) is already an edge, or a negative ORACLE_ERR_* when the segment
 * passes through another point (or the walk fails). */
static int crossings(cdt *c, int a, int b, int *out, int cap)
{
    int start = c->vt[a];
    if (start < 0) return ORACLE_ERR_TOPOLOGY;
    int t = start >> 2, j = start & 3, dir = 0, steps = 0, found = 0;
    /* rotate around a: counterclockwise first, clockwise after meeting the hull */
    for (;;) {
        int p = c->v[3 * t + (j + 1) % 3], q = c->v[3 * t + (j + 2) % 3];
        if (p == b || q == b) return 0;
        int o1 = orx_orient2d(PT(a), PT(p), PT(b)), o2 = orx_orient2d(PT(a), PT(q), PT(b));
        if (o1 > 0 && o2 < 0) { found = 1; break; }
        if (o1 == 0) {
            const double *A = PT(a), *P = PT(p), *B = PT(b);
            if ((P[0] - A[0]) * (B[0] - A[0]) + (P[1] - A[1]) * (B[1] - A[1]) > 0) return ORACLE_ERR_ARG;
        }
        int e = dir == 0 ? c->n[3 * t + (j + 1) % 3] : c->n[3 * t + (j + 2) % 3];
        if (e < 0) {
            if (dir == 1) break;
            dir = 1;
            t = start >> 2;
            j = start & 3;
            continue;
        }
        t = e >> 2;
        j = dir == 0 ? ((e & 3) + 1) % 3 : ((e & 3) + 2) % 3;
        if ((t << 2 | j) == start) break;
        if (++steps > 1 << 24) return ORACLE_ERR_TOPOLOGY;
    }
    if (!found) return ORACLE_ERR_TOPOLOGY;
    int p = c->v[3 * t + (j + 1) % 3], q = c->v[3 * t + (j + 2) % 3];
    int k = 0, jt = j;
    for (;;) {
        if (k >= cap) return ORACLE_ERR_CAP;
        out[k++] = (t << 2) | jt;
        int e = c->n[3 * t + jt];
        if (e < 0) return ORACLE_ERR_TOPOLOGY;
        int u = e >> 2, r = c->v[3 * u + (e & 3)];
        if (r == b) break;
        int o = orx_orient2d(PT(a), PT(b), PT(r));
        if (o == 0) return ORACLE_ERR_ARG;
        int other = o > 0 ? q : p; /* the next crossed edge of u is opposite `other` */
        int m;
        for (m = 0; m < 3; m++)
            if (c->v[3 * u + m] == other) break;
        if (o > 0) q = r;
        else p = r;
        t = u;
        jt = m;
    }
    return k;
}

static int convex_flippable(const cdt *c, int t, int i)
{
    int e = c->n[3 * t + i];
    if (e < 0) return 0;
    int u = e >> 2;
    int a = c->v[3 * t + i], b = c->v[3 * t + (i + 1) % 3], cc = c->v[3 * t + (i + 2) % 3], d = c->v[3 * u + (e & 3)];
    return orx_orient2d(PT(a), PT(b), PT(d)) > 0 && orx_orient2d(PT(d), PT(cc), PT(a)) > 0;
}

/* The edge (p, q): a triangle holding it and the index of the vertex opposite,
 * found by rotating around p from vt[p].  Returns -1 if (p, q) is not an edge. */
static int find_edge(const cdt *c, int p, int q)
{
    int start = c->vt[p], t = start >> 2, j = start & 3, dir = 0;
    long long steps = 0;
    for (;;) {
        if (c->v[3 * t + (j + 1) % 3] == q) return (t << 2) | ((j + 2) % 3);
        if (c->v[3 * t + (j + 2) % 3] == q) return (t << 2) | ((j + 1) % 3);
        int e = dir == 0 ? c->n[3 * t + (j + 1) % 3] : c->n[3 * t + (j + 2) % 3];
        if (e < 0) {
            if (dir == 1) return -1;
            dir = 1;
            t = start >> 2;
            j = start & 3;
            continue;
        }
        t = e >> 2;
        j = dir == 0 ? ((e & 3) + 1) % 3 : ((e & 3) + 2) % 3;
        if ((t << 2 | j) == start || ++steps > 1 << 24) return -1;
    }
}

/* Open segments (a, b) and (x, y) cross at one interior point. */
static int crosses(const cdt *c, int a, int b, int x, int y)
{
    if (x == a || x == b || y == a || y == b) return 0;
    int o1 = orx_orient2d(PT(a), PT(b), PT(x)), o2 = orx_orient2d(PT(a), PT(b), PT(y));
    int o3 = orx_orient2d(PT(x), PT(y), PT(a)), o4 = orx_orient2d(PT(x), PT(y), PT(b));
    return o1 * o2 < 0 && o3 * o4 < 0;
}

/* Sloan's insertion of the constraint (a, b) by flips: the crossed edges, as
 * vertex pairs, in a FIFO queue; an edge whose quadrilateral is not strictly
 * convex goes to the back, a flipped edge whose new diagonal still crosses
 * (a, b) is appended (the FIFO order is what makes the process terminate). */
static int insert_constraint(cdt *c, int a, int b, int *x, int xcap)
{
    int m = crossings(c, a, b, x, xcap);
    if (m <= 0) return m;
    int *qa = (int *)malloc(sizeof(int) * (size_t)(2 * m + 2));
    int head = 0, count = m, cap = m + 1, k;
    for (k = 0; k < m; k++) {
        int t = x[k] >> 2, i = x[k] & 3;
        qa[2 * k] = c->v[3 * t + (i + 1) % 3];
        qa[2 * k + 1] = c->v[3 * t + (i + 2) % 3];
    }
    long long guard = 0;
    int status = 0;
    while (count > 0) {
        int p = qa[2 * head], q = qa[2 * head + 1];
        head = (head + 1) % cap;
        count--;
        int e = find_edge(c, p, q);
        if (e < 0) { status = ORACLE_ERR_TOPOLOGY; break; }
        int t = e >> 2, i = e & 3;
        int tail = (head + count) % cap;
        if (!convex_flippable(c, t, i)) {
            qa[2 * tail] = p;
            qa[2 * tail + 1] = q;
            count++;
        } else {
            int ne = c->n[3 * t + i];
            int xa = c->v[3 * t + i], xd = c->v[3 * (ne >> 2) + (ne & 3)];
            flip(c, t, i);
            if (crosses(c, a, b, xa, xd)) {
                qa[2 * tail] = xa;
                qa[2 * tail + 1] = xd;
                count++;
            }
        }
        if (++guard > 100000000ll) { status = ORACLE_ERR_TOPOLOGY; break; }
    }
    free(qa);
    return status;
}

static int legalize_all(cdt *c)
{
    int *stack = (int *)malloc(sizeof(int) * (size_t)(3 * c->nt + 64));
    int sp = 0, cap = 3 * c->nt + 64, t, i;
    long long guard = 0;
    for (t = 0; t < c->nt; t++)
        for (i = 0; i < 3; i++) stack[sp++] = (t << 2) | i;
    while (sp > 0) {
        int e0 = stack[--sp], tt = e0 >> 2, ii = e0 & 3;
        int ne = c->n[3 * tt + ii];
        if (ne < 0) continue;
        int u = ne >> 2, jj = ne & 3;
        int a = c->v[3 * tt + ii], b = c->v[3 * tt + (ii + 1) % 3], cc = c->v[3 * tt + (ii + 2) % 3];
        int d = c->v[3 * u + jj];
        if (set_has(c, b, cc)) continue;
        if (orx_incircle(PT(b), PT(cc), PT(a), PT(d)) > 0) {
            flip(c, tt, ii);
            if (sp + 4 > cap) {
                cap *= 2;
                int *ns = (int *)realloc(stack, sizeof(int) * (size_t)cap);
                if (!ns) { free(stack); return ORACLE_ERR_CAP; }
                stack = ns;
            }
            stack[sp++] = (tt << 2) | 0;
            stack[sp++] = (tt << 2) | 2;
            stack[sp++] = (u << 2) | 0;
            stack[sp++] = (u << 2) | 2;
            if (++guard > 100000000ll) { free(stack); return ORACLE_ERR_TOPOLOGY; }
        }
    }
    free(stack);
    return 0;
}

int oracle_cdt(int npts, const double *xy, int ncons, const int *cons, int cap, int *out_vtx, int *out_nbr,
               int *out_nkept)
{
    int nt = oracle_dt(npts, xy, cap, out_vtx, out_nbr, out_nkept);
    if (nt <= 0 || ncons <= 0) return nt;
    cdt C, *c = &C;
    int k, t, i, status = 0;
    memset(c, 0, sizeof(*c));
    c->xy = xy;
    c->v = out_vtx;
    c->n = out_nbr;
    c->nt = nt;
    c->vt = (int *)malloc(sizeof(int) * (size_t)npts);
    for (i = 0; i < npts; i++) c->vt[i] = -1;
    for (t = 0; t < nt; t++)
        for (i = 0; i < 3; i++) c->vt[c->v[3 * t + i]] = (t << 2) | i;
    int size = 16;
    while (size < 2 * ncons + 2) size <<= 1;
    c->mask = size - 1;
    c->set = (unsigned long long *)malloc(sizeof(unsigned long long) * (size_t)size);
    for (i = 0; i < size; i++) c->set[i] = ~0ull;
    int xcap = 3 * nt + 16;
    int *x = (int *)malloc(sizeof(int) * (size_t)xcap);
    for (k = 0; k < ncons && status == 0; k++) {
        int a = cons[2 * k], b = cons[2 * k + 1];
        if (a < 0 || a >= npts || b < 0 || b >= npts || a == b || c->vt[a] < 0 || c->vt[b] < 0) {
            status = ORACLE_ERR_ARG;
            break;
        }
        set_add(c, a, b);
        status = insert_constraint(c, a, b, x, xcap);
    }
    if (status == 0) status = legalize_all(c);
    free(x);
    free(c->vt);
    free(c->set);
    return status < 0 ? status : nt;
}
