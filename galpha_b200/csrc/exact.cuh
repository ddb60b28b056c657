// exact.cuh -- staged exact geometric predicates for the galpha-b200 kernels.
//
// Each mesh predicate is staged: an FP32 evaluation with a certified error
// bound (orient2d_filter32, incircle_filter32) decides almost every call; an
// undecided call goes to the FP64 evaluation with Shewchuk's certified error
// bound; the rare call that is still undecided falls through to an exact
// evaluation in floating-point expansion arithmetic (Shewchuk, "Adaptive
// Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates",
// 1997).  The reference's device predicates stop at the filter
// for in-circle (gpudt/Cuda/cudaCCW.h:484-524 returns "unsure") and hand the
// edge to the host (gpudt.cpp:879-914); here the exact stage runs on the
// device, so no host hand-off exists.
//
// Two-Product uses the hardware FMA (exact on sm_100: fma(a,b,-a*b) is the
// rounding error of a*b).  Expansions are fixed-capacity local arrays; an
// operation that would overflow its capacity returns EXACT_OVERFLOW and the
// caller records GPUDT_ERR_EXACT.
#pragma once
#include <math.h>

#ifndef GALPHA_HD
#define GALPHA_HD __host__ __device__ __forceinline__
#endif

namespace galpha {

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr double kCcwErrA = (3.0 + 16.0 * kEps) * kEps;
constexpr double kIccErrA = (10.0 + 96.0 * kEps) * kEps;
constexpr int EXACT_OVERFLOW = 0x7fff;

// FP32 stage.  Its inputs are the FP64 coordinate differences rounded to
// FP32, so each carries a relative error u <= 2^-24 + 2^-53 (two roundings)
// where Shewchuk's analysis assumes 2^-24; every later operation rounds once
// (an FMA contraction only removes roundings).  Shewchuk's relative bounds
// for the same expression trees are 3 eps (orient2d) and 10 eps (in-circle);
// the constants below are at least twice those.  Underflow adds an absolute
// error below 2^-126 per FP32 operation or conversion (2^-150 with gradual
// underflow; 2^-126 also covers flush-to-zero).  Weighted by the largest
// factor each error is later multiplied by, with every difference at most
// M = 2^10 in magnitude, those terms total below (4M + 3) 2^-126 < 2^-113 for
// orient2d and (48 M^3 + 36 M^2 + 5) 2^-126 < 2^-90 for in-circle; the
// absolute allowances below are 8 and 16 times those.  A call with a larger
// difference, a NaN or an infinity starts at the FP64 stage.
constexpr float kEps32 = 5.9604644775390625e-08f;  // 2^-24
constexpr float kCcwErrF = 8.0f * kEps32;
constexpr float kIccErrF = 20.0f * kEps32;
constexpr float kCcwAbsF = 0x1p-110f;
constexpr float kIccAbsF = 0x1p-86f;
constexpr double kF32Span = 1024.0;  // largest coordinate difference the FP32 stage takes

GALPHA_HD void two_sum(double a, double b, double &x, double &y)
{
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    x = s;
    y = (a - av) + (b - bv);
}

GALPHA_HD void fast_two_sum(double a, double b, double &x, double &y)
{
    double s = a + b;
    x = s;
    y = b - (s - a);
}

GALPHA_HD void two_prod(double a, double b, double &x, double &y)
{
    double p = a * b;
    x = p;
    y = fma(a, b, -p);
}

// h = e + f (merge by magnitude, then accumulate); h must not alias e or f.
GALPHA_HD int xsum(int elen, const double *e, int flen, const double *f, double *h, int hcap)
{
    if (elen + flen > hcap) return -1;
    int i = 0, j = 0, m = 0;
    while (i < elen && j < flen) {
        if (fabs(e[i]) <= fabs(f[j])) h[m++] = e[i++];
        else h[m++] = f[j++];
    }
    while (i < elen) h[m++] = e[i++];
    while (j < flen) h[m++] = f[j++];
    if (m == 0) return 0;
    if (m == 1) return h[0] != 0.0 ? 1 : 0;
    double Q, hh;
    fast_two_sum(h[1], h[0], Q, hh);
    int n = 0;
    if (hh != 0.0) h[n++] = hh;
    for (int k = 2; k < m; k++) {
        double g = h[k];
        two_sum(Q, g, Q, hh);
        if (hh != 0.0) h[n++] = hh;
    }
    if (Q != 0.0 || n == 0) h[n++] = Q;
    if (n == 1 && h[0] == 0.0) return 0;
    return n;
}

// h = b * e; h must not alias e.
GALPHA_HD int xscale(int elen, const double *e, double b, double *h, int hcap)
{
    if (elen == 0 || b == 0.0) return 0;
    if (2 * elen > hcap) return -1;
    double Q, hh, p1, p0, s;
    int n = 0;
    two_prod(e[0], b, Q, hh);
    if (hh != 0.0) h[n++] = hh;
    for (int i = 1; i < elen; i++) {
        two_prod(e[i], b, p1, p0);
        two_sum(Q, p0, s, hh);
        if (hh != 0.0) h[n++] = hh;
        fast_two_sum(p1, s, Q, hh);
        if (hh != 0.0) h[n++] = hh;
    }
    if (Q != 0.0 || n == 0) h[n++] = Q;
    if (n == 1 && h[0] == 0.0) return 0;
    return n;
}

// Compress in place.
GALPHA_HD int xcompress(int elen, double *e)
{
    if (elen <= 1) return elen;
    int bottom = elen - 1;
    double Q = e[bottom], Qnew, q;
    for (int i = elen - 2; i >= 0; i--) {
        fast_two_sum(Q, e[i], Qnew, q);
        if (q != 0.0) {
            e[bottom--] = Qnew;
            Q = q;
        } else {
            Q = Qnew;
        }
    }
    int top = 0;
    for (int i = bottom + 1; i < elen; i++) {
        fast_two_sum(e[i], Q, Qnew, q);
        if (q != 0.0) e[top++] = q;
        Q = Qnew;
    }
    e[top] = Q;
    if (top == 0 && Q == 0.0) return 0;
    return top + 1;
}

GALPHA_HD int xsign(int n, const double *e)
{
    if (n <= 0) return 0;
    return e[n - 1] > 0.0 ? 1 : (e[n - 1] < 0.0 ? -1 : 0);
}

GALPHA_HD double xestimate(int n, const double *e)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += e[i];
    return s;
}

GALPHA_HD int xneg(int n, double *e)
{
    for (int i = 0; i < n; i++) e[i] = -e[i];
    return n;
}

GALPHA_HD int xdiff2(double a, double b, double *h)
{
    double x, y;
    two_sum(a, -b, x, y);
    int n = 0;
    if (y != 0.0) h[n++] = y;
    if (x != 0.0) h[n++] = x;
    return n;
}

// Small product scratch: h = e * f (compressed), lengths bounded by the caps.
template <int CAP>
GALPHA_HD int xmul(int elen, const double *e, int flen, const double *f, double *h)
{
    double t1[CAP], t2[CAP];
    int hl = 0;
    if (elen < 0 || flen < 0) return -1;
    for (int j = 0; j < flen; j++) {
        int tl = xscale(elen, e, f[j], t1, CAP);
        if (tl < 0) return -1;
        for (int k = 0; k < hl; k++) t2[k] = h[k];
        hl = xsum(hl, t2, tl, t1, h, CAP);
        if (hl < 0) return -1;
        hl = xcompress(hl, h);
    }
    return hl;
}

// ---------------------------------------------------------------- orient2d
// Exact sign of det[[ax-cx, ay-cy], [bx-cx, by-cy]].
__host__ __device__ __noinline__ inline int orient2d_exact(double ax, double ay, double bx, double by,
                                                            double cx, double cy)
{
    double acx[2], acy[2], bcx[2], bcy[2], l[16], r[16], d[32];
    int nacx = xdiff2(ax, cx, acx), nacy = xdiff2(ay, cy, acy);
    int nbcx = xdiff2(bx, cx, bcx), nbcy = xdiff2(by, cy, bcy);
    int nl = xmul<16>(nacx, acx, nbcy, bcy, l);
    int nr = xmul<16>(nacy, acy, nbcx, bcx, r);
    if (nl < 0 || nr < 0) return EXACT_OVERFLOW;
    xneg(nr, r);
    int nd = xsum(nl, l, nr, r, d, 32);
    if (nd < 0) return EXACT_OVERFLOW;
    return xsign(nd, d);
}

// Filter; returns 2 when undecided.
GALPHA_HD int orient2d_filter(double ax, double ay, double bx, double by, double cx, double cy)
{
    double detleft = (ax - cx) * (by - cy);
    double detright = (ay - cy) * (bx - cx);
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
    double errbound = kCcwErrA * detsum;
    if (det >= errbound || -det >= errbound) return det > 0.0 ? 1 : -1;
    return 2;
}

// FP32 stage of orient2d; returns 2 when undecided (a zero determinant is
// always left to the FP64 stage).
GALPHA_HD int orient2d_filter32(double ax, double ay, double bx, double by, double cx, double cy)
{
    const double dax = ax - cx, day = ay - cy, dbx = bx - cx, dby = by - cy;
    if (!(fabs(dax) <= kF32Span && fabs(day) <= kF32Span && fabs(dbx) <= kF32Span && fabs(dby) <= kF32Span))
        return 2;
    const float acx = (float)dax, acy = (float)day, bcx = (float)dbx, bcy = (float)dby;
    const float l = acx * bcy, r = acy * bcx;
    const float det = l - r;
    const float bound = kCcwErrF * (fabsf(l) + fabsf(r)) + kCcwAbsF;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return 2;
}

// Orientation sign (>0 counterclockwise).  *nexact counts exact fall-throughs.
GALPHA_HD int orient2d(double ax, double ay, double bx, double by, double cx, double cy, int *nexact)
{
    int s = orient2d_filter32(ax, ay, bx, by, cx, cy);
    if (s != 2) return s;
    s = orient2d_filter(ax, ay, bx, by, cx, cy);
    if (s != 2) return s;
    if (nexact) (*nexact)++;
    return orient2d_exact(ax, ay, bx, by, cx, cy);
}

// ---------------------------------------------------------------- incircle
__host__ __device__ __noinline__ inline int incircle_exact(const double *a, const double *b, const double *c,
                                                            const double *d)
{
    double X[3][2], Y[3][2];
    int nX[3], nY[3];
    const double *P[3] = {a, b, c};
    for (int i = 0; i < 3; i++) {
        nX[i] = xdiff2(P[i][0], d[0], X[i]);
        nY[i] = xdiff2(P[i][1], d[1], Y[i]);
    }
    double lift[3][24], cr[3][24];
    int nlift[3], ncr[3];
    for (int i = 0; i < 3; i++) {
        double s1[12], s2[12];
        int n1 = xmul<12>(nX[i], X[i], nX[i], X[i], s1);
        int n2 = xmul<12>(nY[i], Y[i], nY[i], Y[i], s2);
        if (n1 < 0 || n2 < 0) return EXACT_OVERFLOW;
        int n = xsum(n1, s1, n2, s2, lift[i], 24);
        if (n < 0) return EXACT_OVERFLOW;
        nlift[i] = xcompress(n, lift[i]);
    }
    for (int i = 0; i < 3; i++) {
        int j = (i + 1) % 3, k = (i + 2) % 3;
        double m1[12], m2[12];
        int n1 = xmul<12>(nX[j], X[j], nY[k], Y[k], m1);
        int n2 = xmul<12>(nY[j], Y[j], nX[k], X[k], m2);
        if (n1 < 0 || n2 < 0) return EXACT_OVERFLOW;
        xneg(n2, m2);
        int n = xsum(n1, m1, n2, m2, cr[i], 24);
        if (n < 0) return EXACT_OVERFLOW;
        ncr[i] = xcompress(n, cr[i]);
    }
    double term[3][48], acc[96], acc2[144];
    int nterm[3];
    for (int i = 0; i < 3; i++) {
        nterm[i] = xmul<48>(nlift[i], lift[i], ncr[i], cr[i], term[i]);
        if (nterm[i] < 0) return EXACT_OVERFLOW;
    }
    int na = xsum(nterm[0], term[0], nterm[1], term[1], acc, 96);
    if (na < 0) return EXACT_OVERFLOW;
    int nb = xsum(na, acc, nterm[2], term[2], acc2, 144);
    if (nb < 0) return EXACT_OVERFLOW;
    return xsign(nb, acc2);
}

// Filter; returns 2 when undecided.  (a, b, c counterclockwise; >0: d inside.)
GALPHA_HD int incircle_filter(const double *a, const double *b, const double *c, const double *d)
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
    double errbound = kIccErrA * permanent;
    if (det > errbound || -det > errbound) return det > 0.0 ? 1 : -1;
    return 2;
}

// FP32 stage of the in-circle test (same expression tree as incircle_filter);
// returns 2 when undecided.
GALPHA_HD int incircle_filter32(const double *a, const double *b, const double *c, const double *d)
{
    const double ex = a[0] - d[0], ey = a[1] - d[1], fx = b[0] - d[0], fy = b[1] - d[1];
    const double gx = c[0] - d[0], gy = c[1] - d[1];
    if (!(fabs(ex) <= kF32Span && fabs(ey) <= kF32Span && fabs(fx) <= kF32Span && fabs(fy) <= kF32Span &&
          fabs(gx) <= kF32Span && fabs(gy) <= kF32Span))
        return 2;
    const float adx = (float)ex, ady = (float)ey, bdx = (float)fx, bdy = (float)fy, cdx = (float)gx, cdy = (float)gy;
    const float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const float alift = adx * adx + ady * ady;
    const float cdxady = cdx * ady, adxcdy = adx * cdy;
    const float blift = bdx * bdx + bdy * bdy;
    const float adxbdy = adx * bdy, bdxady = bdx * ady;
    const float clift = cdx * cdx + cdy * cdy;
    const float det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
    const float permanent = (fabsf(bdxcdy) + fabsf(cdxbdy)) * alift + (fabsf(cdxady) + fabsf(adxcdy)) * blift +
                            (fabsf(adxbdy) + fabsf(bdxady)) * clift;
    const float bound = kIccErrF * permanent + kIccAbsF;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return 2;
}

GALPHA_HD int incircle(const double *a, const double *b, const double *c, const double *d, int *nexact)
{
    int s = incircle_filter32(a, b, c, d);
    if (s != 2) return s;
    s = incircle_filter(a, b, c, d);
    if (s != 2) return s;
    if (nexact) (*nexact)++;
    return incircle_exact(a, b, c, d);
}

// ------------------------------------------------------- alpha predicates
// |p - q|^2 exactly.
GALPHA_HD int xsqdist(const double *p, const double *q, double *h /*24*/)
{
    double dx[2], dy[2], sx[12], sy[12];
    int ndx = xdiff2(p[0], q[0], dx), ndy = xdiff2(p[1], q[1], dy);
    int nsx = xmul<12>(ndx, dx, ndx, dx, sx);
    int nsy = xmul<12>(ndy, dy, ndy, dy, sy);
    if (nsx < 0 || nsy < 0) return -1;
    int n = xsum(nsx, sx, nsy, sy, h, 24);
    if (n < 0) return -1;
    return xcompress(n, h);
}

// Birth time rho = N / D as exact expansions (kind 3 triangle p[0..5], kind 2 edge p[0..3]).
// Capacities: N, D 96 each.
__host__ __device__ __noinline__ inline int rho_nd(int kind, const double *p, double *N, int *nN, double *D,
                                                    int *nD)
{
    if (kind == 2) {
        int n = xsqdist(p, p + 2, N);
        if (n < 0) return -1;
        *nN = n;
        D[0] = 4.0;
        *nD = 1;
        return 0;
    }
    double la[24], lb[24], lc[24], ab[48];
    int na = xsqdist(p, p + 2, la), nb = xsqdist(p + 2, p + 4, lb), nc = xsqdist(p + 4, p, lc);
    if (na < 0 || nb < 0 || nc < 0) return -1;
    int nab = xmul<48>(na, la, nb, lb, ab);
    if (nab < 0) return -1;
    int nN_ = xmul<96>(nab, ab, nc, lc, N);
    if (nN_ < 0) return -1;
    *nN = nN_;
    double ux[2], uy[2], vx[2], vy[2], m1[12], m2[12], ar[24], ar2[48];
    int nux = xdiff2(p[2], p[0], ux), nvy = xdiff2(p[5], p[1], vy);
    int nvx = xdiff2(p[4], p[0], vx), nuy = xdiff2(p[3], p[1], uy);
    int n1 = xmul<12>(nux, ux, nvy, vy, m1);
    int n2 = xmul<12>(nvx, vx, nuy, uy, m2);
    if (n1 < 0 || n2 < 0) return -1;
    xneg(n2, m2);
    int nar = xsum(n1, m1, n2, m2, ar, 24);
    if (nar < 0) return -1;
    nar = xcompress(nar, ar);
    int nar2 = xmul<48>(nar, ar, nar, ar, ar2);
    if (nar2 < 0) return -1;
    int nd = xscale(nar2, ar2, 4.0, D, 96);
    if (nd < 0) return -1;
    *nD = nd;
    return 0;
}

// Exact sign(rho1 - rho2); EXACT_OVERFLOW on capacity overflow.
__host__ __device__ __noinline__ inline int compare_rho_exact(int kind1, const double *p1, int kind2,
                                                               const double *p2)
{
    double N1[96], D1[96], N2[96], D2[96];
    int nN1, nD1, nN2, nD2;
    if (rho_nd(kind1, p1, N1, &nN1, D1, &nD1) < 0) return EXACT_OVERFLOW;
    if (rho_nd(kind2, p2, N2, &nN2, D2, &nD2) < 0) return EXACT_OVERFLOW;
    double A[192], B[192], C[384];
    int nA = xmul<192>(nN1, N1, nD2, D2, A);
    int nB = xmul<192>(nN2, N2, nD1, D1, B);
    if (nA < 0 || nB < 0) return EXACT_OVERFLOW;
    xneg(nB, B);
    int nC = xsum(nA, A, nB, B, C, 384);
    if (nC < 0) return EXACT_OVERFLOW;
    return xsign(nC, C);
}

// Exact-then-rounded rho (one refinement of the quotient); NaN on overflow.
__host__ __device__ __noinline__ inline double rho_rounded_exact(int kind, const double *p)
{
    double N[96], D[96];
    int nN, nD;
    if (rho_nd(kind, p, N, &nN, D, &nD) < 0) return NAN;
    double dD = xestimate(nD, D);
    double q0 = xestimate(nN, N) / dD;
    double S[192], R[288];
    int nS = xscale(nD, D, -q0, S, 192);
    if (nS < 0) return NAN;
    int nR = xsum(nN, N, nS, S, R, 288);
    if (nR < 0) return NAN;
    nR = xcompress(nR, R);
    return q0 + xestimate(nR, R) / dD;
}

// Attached test (predicates.h:1359-1444): 1 if k lies in the closed diametral
// disc of (i, j), i.e. |i-j|^2 - |i+j-2k|^2 >= 0.  Filter then exact.
__host__ __device__ __noinline__ inline int attached_exact(const double *i, const double *j, const double *k)
{
    double d1[24];
    int nd1 = xsqdist(i, j, d1);
    if (nd1 < 0) return EXACT_OVERFLOW;
    double sx[3], sy[3], hi, lo;
    int nsx = 0, nsy = 0;
    two_sum(i[0], j[0], hi, lo);
    if (lo != 0.0) sx[nsx++] = lo;
    if (hi != 0.0) sx[nsx++] = hi;
    two_sum(i[1], j[1], hi, lo);
    if (lo != 0.0) sy[nsy++] = lo;
    if (hi != 0.0) sy[nsy++] = hi;
    double kx = -2.0 * k[0], ky = -2.0 * k[1];
    double ex[4], ey[4];
    int nex = xsum(nsx, sx, kx != 0.0 ? 1 : 0, &kx, ex, 4);
    int ney = xsum(nsy, sy, ky != 0.0 ? 1 : 0, &ky, ey, 4);
    double qx[24], qy[24], d2[48], r[72];
    int nqx = xmul<24>(nex, ex, nex, ex, qx);
    int nqy = xmul<24>(ney, ey, ney, ey, qy);
    if (nqx < 0 || nqy < 0) return EXACT_OVERFLOW;
    int nd2 = xsum(nqx, qx, nqy, qy, d2, 48);
    if (nd2 < 0) return EXACT_OVERFLOW;
    xneg(nd2, d2);
    int nr = xsum(nd1, d1, nd2, d2, r, 72);
    if (nr < 0) return EXACT_OVERFLOW;
    return xsign(nr, r) >= 0 ? 1 : 0;
}

// Filtered attached test; returns 2 when undecided.
GALPHA_HD int attached_filter(const double *i, const double *j, const double *k)
{
    double ax = i[0] - j[0], ay = i[1] - j[1];
    double d1 = ax * ax + ay * ay;
    double sx = i[0] + j[0] - 2.0 * k[0], sy = i[1] + j[1] - 2.0 * k[1];
    double d2 = sx * sx + sy * sy;
    double diff = d1 - d2;
    double ex = fabs(i[0] + j[0]) + 2.0 * fabs(k[0]), ey = fabs(i[1] + j[1]) + 2.0 * fabs(k[1]);
    double permanent = d1 + ex * ex + ey * ey;
    // every term carries at most ~6 roundings of relative 2^-53 of the permanent
    double errbound = 8.0 * kEps * permanent;
    if (diff > errbound) return 1;
    if (-diff > errbound) return 0;
    return 2;
}

}  // namespace galpha
