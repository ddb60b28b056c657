/*
 * oracle/pred.h -- TEST INFRASTRUCTURE, not product code (see oracle/exact.h).
 *
 * Exact orientation and in-circle signs for the CPU oracle.  Restates the
 * semantics of the reference's host predicates gpudt/predicates.cpp:322
 * (counterclockwise) and :942 (incircle): a floating-point filter with
 * Shewchuk's error bound ccwerrboundA / iccerrboundA (predicates.cpp:28,
 * gpudt_exactinit), and an exact expansion evaluation when the filter cannot
 * decide.  Only the sign is returned, which is all the reference's callers use
 * (gpudt.cpp:160-189, :395, main.cu:313).
 */
#ifndef GALPHA_ORACLE_PRED_H
#define GALPHA_ORACLE_PRED_H

#include "exact.h"

static const double ORX_CCWERRA = (3.0 + 16.0 * ORX_EPS) * ORX_EPS;
static const double ORX_ICCERRA = (10.0 + 96.0 * ORX_EPS) * ORX_EPS;

/* Exact counters (how often the filter fell through), for reporting. */
extern _Thread_local long long oracle_exact_orient_calls;
extern _Thread_local long long oracle_exact_incircle_calls;

static inline int orx_orient2d_exact(const double *a, const double *b, const double *c)
{
    static _Thread_local double t1[ORX_CAP], t2[ORX_CAP];
    double acx[2], acy[2], bcx[2], bcy[2];
    double l[64], r[64], nr[64], d[128];
    int nacx = orx_diff2(a[0], c[0], acx), nacy = orx_diff2(a[1], c[1], acy);
    int nbcx = orx_diff2(b[0], c[0], bcx), nbcy = orx_diff2(b[1], c[1], bcy);
    int nl = orx_mul(nacx, acx, nbcy, bcy, l, t1, t2);
    int nrr = orx_mul(nacy, acy, nbcx, bcx, r, t1, t2);
    orx_negate(nrr, r, nr);
    int nd = orx_sum(nl, l, nrr, nr, d);
    return orx_sign(nd, d);
}

/* >0: a, b, c counterclockwise; <0 clockwise; 0 collinear. */
static inline int orx_orient2d(const double *a, const double *b, const double *c)
{
    double detleft = (a[0] - c[0]) * (b[1] - c[1]);
    double detright = (a[1] - c[1]) * (b[0] - c[0]);
    double det = detleft - detright, detsum;
    if (detleft > 0.0) {
        if (detright <= 0.0) return det > 0.0 ? 1 : (det < 0.0 ? -1 : 0);
        detsum = detleft + detright;
    } else if (detleft < 0.0) {
        if (detright >= 0.0) return det > 0.0 ? 1 : (det < 0.0 ? -1 : 0);
        detsum = -detleft - detright;
    } else {
        return det > 0.0 ? 1 : (det < 0.0 ? -1 : 0);
    }
    double errbound = ORX_CCWERRA * detsum;
    if (det >= errbound || -det >= errbound) return det > 0.0 ? 1 : -1;
    oracle_exact_orient_calls++;
    return orx_orient2d_exact(a, b, c);
}

static inline int orx_incircle_exact(const double *a, const double *b, const double *c, const double *d)
{
    static _Thread_local double t1[ORX_CAP], t2[ORX_CAP];
    double adx[2], ady[2], bdx[2], bdy[2], cdx[2], cdy[2];
    double s1[64], s2[64], lift[3][128], m1[64], m2[64], mm[64], cr[3][128], term[3][512];
    double acc[1024], acc2[1536];
    int nadx = orx_diff2(a[0], d[0], adx), nady = orx_diff2(a[1], d[1], ady);
    int nbdx = orx_diff2(b[0], d[0], bdx), nbdy = orx_diff2(b[1], d[1], bdy);
    int ncdx = orx_diff2(c[0], d[0], cdx), ncdy = orx_diff2(c[1], d[1], cdy);
    const double *X[3] = {adx, bdx, cdx}, *Y[3] = {ady, bdy, cdy};
    int nX[3] = {nadx, nbdx, ncdx}, nY[3] = {nady, nbdy, ncdy};
    int nlift[3], ncr[3], nterm[3], i;
    for (i = 0; i < 3; i++) {
        int n1 = orx_mul(nX[i], X[i], nX[i], X[i], s1, t1, t2);
        int n2 = orx_mul(nY[i], Y[i], nY[i], Y[i], s2, t1, t2);
        nlift[i] = orx_compress(orx_sum(n1, s1, n2, s2, lift[i]), lift[i]);
    }
    /* cr[0] = bdx*cdy - bdy*cdx ; cr[1] = cdx*ady - cdy*adx ; cr[2] = adx*bdy - ady*bdx */
    for (i = 0; i < 3; i++) {
        int j = (i + 1) % 3, k = (i + 2) % 3;
        int n1 = orx_mul(nX[j], X[j], nY[k], Y[k], m1, t1, t2);
        int n2 = orx_mul(nY[j], Y[j], nX[k], X[k], m2, t1, t2);
        orx_negate(n2, m2, mm);
        ncr[i] = orx_compress(orx_sum(n1, m1, n2, mm, cr[i]), cr[i]);
    }
    for (i = 0; i < 3; i++) nterm[i] = orx_mul(nlift[i], lift[i], ncr[i], cr[i], term[i], t1, t2);
    int na = orx_sum(nterm[0], term[0], nterm[1], term[1], acc);
    int nb = orx_sum(na, acc, nterm[2], term[2], acc2);
    return orx_sign(nb, acc2);
}

/* >0: d inside the circle through counterclockwise a, b, c. */
static inline int orx_incircle(const double *a, const double *b, const double *c, const double *d)
{
    double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
    double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
    double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    double alift = adx * adx + ady * ady;
    double cdxady = cdx * ady, adxcdy = adx * cdy;
    double blift = bdx * bdx + bdy * bdy;
    double adxbdy = adx * bdy, bdxady = bdx * ady;
    double clift = cdx * cdx + cdy * cdy;
    double det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
    double permanent = (fabs(bdxcdy) + fabs(cdxbdy)) * alift + (fabs(cdxady) + fabs(adxcdy)) * blift +
                       (fabs(adxbdy) + fabs(bdxady)) * clift;
    double errbound = ORX_ICCERRA * permanent;
    if (det > errbound || -det > errbound) return det > 0.0 ? 1 : -1;
    oracle_exact_incircle_calls++;
    return orx_incircle_exact(a, b, c, d);
}

#endif
