// Host check of the staged predicates in galpha_b200/csrc/exact.cuh: the FP32
// and FP64 filters must never return a sign that differs from the exact
// expansion's.  Built and run by tests/test_predicates_host.py.
//
//   pred_stages_check count <cases>   adversarial families, one summary line each:
//                                     "<family> <pred> cases decided32 decided64 wrong32 wrong64"
//   pred_stages_check dump <cases>    near-degenerate cases as hex floats with both filters'
//                                     answers, for an independent rational check
#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#include "exact.cuh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cstdint>

using namespace galpha;

static uint64_t g_state = 0x9e3779b97f4a7c15ull;
static uint64_t next_u64()
{
    uint64_t z = (g_state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static double unif() { return (double)(next_u64() >> 11) * 0x1p-53; }
static int irange(int lo, int hi) { return lo + (int)(next_u64() % (uint64_t)(hi - lo + 1)); }
static double nudge(double x, int ulps)
{
    for (; ulps > 0; ulps--) x = nextafter(x, INFINITY);
    for (; ulps < 0; ulps++) x = nextafter(x, -INFINITY);
    return x;
}

// One generated case: four points (orient2d uses the first three).
struct Case {
    double p[4][2];
};

// family ids
enum { F_UNIFORM, F_NEAR_LINE, F_LATTICE, F_NEAR_CIRCLE, F_TINY, F_SUBNORMAL32, F_WIDE, F_MIXED, F_COUNT };
static const char *kNames[F_COUNT] = {"uniform",  "near_line", "lattice", "near_circle",
                                      "tiny",     "subnormal32", "wide",  "mixed"};

static void gen(int fam, Case &c)
{
    switch (fam) {
    case F_UNIFORM:
        for (auto &q : c.p) q[0] = unif(), q[1] = unif();
        break;
    case F_NEAR_LINE: {
        // c on the segment ab up to rounding, then a few ulps off; d near the same line
        double ax = unif(), ay = unif(), bx = unif(), by = unif();
        c.p[0][0] = ax, c.p[0][1] = ay, c.p[1][0] = bx, c.p[1][1] = by;
        for (int k = 2; k < 4; k++) {
            double t = unif() * 3.0 - 1.0;
            c.p[k][0] = nudge(ax + t * (bx - ax), irange(-3, 3));
            c.p[k][1] = nudge(ay + t * (by - ay), irange(-3, 3));
        }
        break;
    }
    case F_LATTICE:
        // 1024 x 1024 lattice: exact collinear triples and cocircular quads are common
        for (auto &q : c.p) q[0] = irange(0, 7) / 1024.0 + 0.5, q[1] = irange(0, 7) / 1024.0 + 0.25;
        break;
    case F_NEAR_CIRCLE: {
        double cx = unif(), cy = unif(), r = 1e-6 + unif() * 0.5;
        double th0 = unif() * 6.283185307179586;
        for (int k = 0; k < 4; k++) {
            double th = th0 + k * 1.5 + unif() * 0.5;  // counterclockwise a, b, c
            c.p[k][0] = nudge(cx + r * cos(th), k == 3 ? irange(-2, 2) : 0);
            c.p[k][1] = nudge(cy + r * sin(th), k == 3 ? irange(-2, 2) : 0);
        }
        break;
    }
    case F_TINY: {
        // differences around 1e-12 .. 1e-20 near a point of the unit square
        double s = pow(10.0, -12.0 - 8.0 * unif());
        double bx = unif(), by = unif();
        for (auto &q : c.p) q[0] = bx + s * (unif() - 0.5), q[1] = by + s * (unif() - 0.5);
        break;
    }
    case F_SUBNORMAL32: {
        // coordinates near the origin whose differences are FP32 subnormals or smaller
        double s = pow(2.0, -120.0 - 40.0 * unif());
        for (auto &q : c.p) q[0] = s * (unif() - 0.5), q[1] = s * (unif() - 0.5);
        if (next_u64() & 1) c.p[3][0] = c.p[0][0], c.p[3][1] = c.p[1][1];
        break;
    }
    case F_WIDE: {
        // differences up to 2^11: above 2^10 the FP32 stage must pass the call on
        double s = 2048.0;
        for (auto &q : c.p) q[0] = s * (unif() - 0.5), q[1] = s * (unif() - 0.5);
        break;
    }
    case F_MIXED: {
        // one far point, three within 2^-60 .. 2^-20 of each other
        double s = pow(2.0, -60.0 + 40.0 * unif());
        double bx = unif(), by = unif();
        for (int k = 0; k < 4; k++) c.p[k][0] = bx + s * (unif() - 0.5), c.p[k][1] = by + s * (unif() - 0.5);
        int far = irange(0, 3);
        c.p[far][0] = 1000.0 * (unif() - 0.5), c.p[far][1] = 1000.0 * (unif() - 0.5);
        break;
    }
    }
}

static int orient_of(const Case &c, int &s32, int &s64)
{
    const double *a = c.p[0], *b = c.p[1], *q = c.p[2];
    s32 = orient2d_filter32(a[0], a[1], b[0], b[1], q[0], q[1]);
    s64 = orient2d_filter(a[0], a[1], b[0], b[1], q[0], q[1]);
    return orient2d_exact(a[0], a[1], b[0], b[1], q[0], q[1]);
}

static int incircle_of(Case &c, int &s32, int &s64)
{
    // the in-circle convention wants a, b, c counterclockwise
    int o = orient2d_exact(c.p[0][0], c.p[0][1], c.p[1][0], c.p[1][1], c.p[2][0], c.p[2][1]);
    if (o < 0)
        for (int k = 0; k < 2; k++) {
            double t = c.p[0][k];
            c.p[0][k] = c.p[1][k];
            c.p[1][k] = t;
        }
    s32 = incircle_filter32(c.p[0], c.p[1], c.p[2], c.p[3]);
    s64 = incircle_filter(c.p[0], c.p[1], c.p[2], c.p[3]);
    return incircle_exact(c.p[0], c.p[1], c.p[2], c.p[3]);
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s count|dump <cases>\n", argv[0]);
        return 2;
    }
    const bool dump = strcmp(argv[1], "dump") == 0;
    const long long n = atoll(argv[2]);
    for (int fam = 0; fam < F_COUNT; fam++) {
        for (int pred = 0; pred < 2; pred++) {
            long long dec32 = 0, dec64 = 0, bad32 = 0, bad64 = 0, overflow = 0;
            for (long long i = 0; i < n; i++) {
                Case c;
                gen(fam, c);
                int s32, s64;
                const int se = pred == 0 ? orient_of(c, s32, s64) : incircle_of(c, s32, s64);
                if (se == EXACT_OVERFLOW) {
                    overflow++;
                    continue;
                }
                if (s32 != 2) {
                    dec32++;
                    if (s32 != se) bad32++;
                }
                if (s64 != 2) {
                    dec64++;
                    if (s64 != se) bad64++;
                }
                if (dump)
                    printf("case %s %s %a %a %a %a %a %a %a %a %d %d\n", kNames[fam], pred ? "incircle" : "orient",
                           c.p[0][0], c.p[0][1], c.p[1][0], c.p[1][1], c.p[2][0], c.p[2][1], c.p[3][0], c.p[3][1],
                           s32, s64);
            }
            printf("%s %s %lld %lld %lld %lld %lld %lld\n", kNames[fam], pred ? "incircle" : "orient", n, dec32,
                   dec64, bad32, bad64, overflow);
        }
    }
    return 0;
}
