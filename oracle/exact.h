/*
 * oracle/exact.h -- TEST INFRASTRUCTURE, not product code.
 *
 * Exact floating-point expansion arithmetic for the CPU oracle.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may use
 * anything under oracle/, and only as the checker.
 *
 * This restates the published algorithms of J. R. Shewchuk, "Adaptive
 * Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates"
 * (Discrete & Computational Geometry 18, 1997): Two-Sum, Dekker's Two-Product
 * with Veltkamp splitting, Fast-Expansion-Sum with zero elimination,
 * Scale-Expansion with zero elimination and Compress.  The reference uses the
 * same published algorithms through gpudt/predicates.cpp (host) and
 * gpudt/AlphaShape/predicates.h:502-1276 (host + device).
 *
 * Representation: an expansion is an array of doubles, nonoverlapping and
 * ordered by increasing magnitude, zero components removed.  Length 0 means
 * the value zero.  The sign of an expansion is the sign of its last component.
 *
 * Built with -ffp-contract=off: these routines must never be fused into FMAs.
 */
#ifndef GALPHA_ORACLE_EXACT_H
#define GALPHA_ORACLE_EXACT_H

#include <math.h>
#include <string.h>

/* 2^27 + 1: Veltkamp splitter for 53-bit doubles. */
#define ORX_SPLITTER 134217729.0
#define ORX_EPS      1.1102230246251565e-16 /* 2^-53 */

static inline void orx_two_sum(double a, double b, double *x, double *y)
{
    double s = a + b, bv = s - a, av = s - bv;
    *x = s;
    *y = (a - av) + (b - bv);
}

static inline void orx_fast_two_sum(double a, double b, double *x, double *y)
{
    /* requires |a| >= |b| */
    double s = a + b;
    *x = s;
    *y = b - (s - a);
}

static inline void orx_split(double a, double *hi, double *lo)
{
    double c = ORX_SPLITTER * a, big = c - a;
    *hi = c - big;
    *lo = a - *hi;
}

static inline void orx_two_prod(double a, double b, double *x, double *y)
{
    double p = a * b, ahi, alo, bhi, blo, e1, e2, e3;
    orx_split(a, &ahi, &alo);
    orx_split(b, &bhi, &blo);
    e1 = p - ahi * bhi;
    e2 = e1 - alo * bhi;
    e3 = e2 - ahi * blo;
    *x = p;
    *y = alo * blo - e3;
}

/* h = e + f.  h must not alias e or f.  Capacity of h: elen + flen. */
static inline int orx_sum(int elen, const double *e, int flen, const double *f, double *h)
{
    int i = 0, j = 0, m = 0, k, n;
    double Q, hh;
    /* merge by increasing magnitude */
    while (i < elen && j < flen) {
        if (fabs(e[i]) <= fabs(f[j])) h[m++] = e[i++];
        else h[m++] = f[j++];
    }
    while (i < elen) h[m++] = e[i++];
    while (j < flen) h[m++] = f[j++];
    if (m == 0) return 0;
    if (m == 1) return h[0] != 0.0 ? 1 : 0;
    /* in-place accumulation: the write index never overtakes the read index */
    orx_fast_two_sum(h[1], h[0], &Q, &hh);
    n = 0;
    if (hh != 0.0) h[n++] = hh;
    for (k = 2; k < m; k++) {
        double g = h[k];
        orx_two_sum(Q, g, &Q, &hh);
        if (hh != 0.0) h[n++] = hh;
    }
    if (Q != 0.0 || n == 0) h[n++] = Q;
    if (n == 1 && h[0] == 0.0) return 0;
    return n;
}

/* h = b * e.  h must not alias e.  Capacity of h: 2 * elen. */
static inline int orx_scale(int elen, const double *e, double b, double *h)
{
    int i, n = 0;
    double Q, hh, p1, p0, s;
    if (elen == 0 || b == 0.0) return 0;
    orx_two_prod(e[0], b, &Q, &hh);
    if (hh != 0.0) h[n++] = hh;
    for (i = 1; i < elen; i++) {
        orx_two_prod(e[i], b, &p1, &p0);
        orx_two_sum(Q, p0, &s, &hh);
        if (hh != 0.0) h[n++] = hh;
        orx_fast_two_sum(p1, s, &Q, &hh);
        if (hh != 0.0) h[n++] = hh;
    }
    if (Q != 0.0 || n == 0) h[n++] = Q;
    if (n == 1 && h[0] == 0.0) return 0;
    return n;
}

/* Compress in place (Shewchuk's Compress). */
static inline int orx_compress(int elen, double *e)
{
    int bottom, top, i;
    double Q, Qnew, q;
    if (elen <= 1) return elen;
    bottom = elen - 1;
    Q = e[bottom];
    for (i = elen - 2; i >= 0; i--) {
        orx_fast_two_sum(Q, e[i], &Qnew, &q);
        if (q != 0.0) {
            e[bottom--] = Qnew;
            Q = q;
        } else {
            Q = Qnew;
        }
    }
    top = 0;
    for (i = bottom + 1; i < elen; i++) {
        orx_fast_two_sum(e[i], Q, &Qnew, &q);
        if (q != 0.0) e[top++] = q;
        Q = Qnew;
    }
    e[top] = Q;
    if (top == 0 && Q == 0.0) return 0;
    return top + 1;
}

static inline int orx_sign(int elen, const double *e)
{
    if (elen == 0) return 0;
    return e[elen - 1] > 0.0 ? 1 : (e[elen - 1] < 0.0 ? -1 : 0);
}

static inline double orx_estimate(int elen, const double *e)
{
    double s = 0.0;
    int i;
    for (i = 0; i < elen; i++) s += e[i];
    return s;
}

static inline int orx_negate(int elen, const double *e, double *h)
{
    int i;
    for (i = 0; i < elen; i++) h[i] = -e[i];
    return elen;
}

/* Expansion workspace with a fixed capacity per operand. */
#define ORX_CAP 4096

/* h = e * f, compressed.  h must alias neither.  Uses caller scratch t1, t2
 * of capacity ORX_CAP each.  Returns -1 on capacity overflow. */
static inline int orx_mul(int elen, const double *e, int flen, const double *f,
                          double *h, double *t1, double *t2)
{
    int j, hl = 0, tl;
    if (elen == 0 || flen == 0) return 0;
    if (2 * elen > ORX_CAP) return -1;
    for (j = 0; j < flen; j++) {
        tl = orx_scale(elen, e, f[j], t1);
        if (hl + tl > ORX_CAP) return -1;
        memcpy(t2, h, (size_t)hl * sizeof(double));
        hl = orx_sum(hl, t2, tl, t1, h);
        hl = orx_compress(hl, h);
    }
    return hl;
}

/* 2-component exact difference a - b as an expansion (length 0..2). */
static inline int orx_diff2(double a, double b, double *h)
{
    double x, y;
    int n = 0;
    orx_two_sum(a, -b, &x, &y);
    if (y != 0.0) h[n++] = y;
    if (x != 0.0) h[n++] = x;
    return n;
}

#endif
