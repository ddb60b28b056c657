// oracle/ref_alpha.cpp -- TEST INFRASTRUCTURE: C entry points over the
// reference's alpha predicates (gpudt/AlphaShape/predicates.h:402-3107),
// host-compiled from the reference tree by oracle/ref.mk.  The two container
// types that header expects from kernel.h are given minimal definitions here.
#include <cstdlib>
#define __device__
#define __host__
#include "gpudt.h"

template <typename T>
struct KernelArray {
    T *_array;
    int _size;
};

struct PrecisionData {
    KernelArray<double> P1, P2, temp2a, temp2b, runningSum1, runningSum2;
};

#include "AlphaShape/predicates.h"

static Predicates *g_ps = nullptr;
static PrecisionData g_pd;

static Predicates *ps()
{
    if (!g_ps) {
        g_ps = new Predicates;
        g_ps->exactinit();
        // host buffers as Alpha_Shapes_2D.cu:545-551 sizes them
        g_ps->CPUtemp2a = new double[136130];
        g_ps->CPUtemp2b = new double[136130];
        g_ps->CPUtemp2 = new double[272260];
        g_ps->CPUrunningSum1 = new double[1633536];
        g_ps->CPUrunningSum2 = new double[1633536];
        g_ps->CPUP1 = new double[1633536];
        g_ps->CPUP2 = new double[1633536];
        // device-path scratch: 200 doubles per thread (Alpha_Shapes_2D.cu:370-375)
        KernelArray<double> *arrs[6] = {&g_pd.P1, &g_pd.P2, &g_pd.temp2a, &g_pd.temp2b, &g_pd.runningSum1,
                                        &g_pd.runningSum2};
        for (auto *k : arrs) {
            k->_array = new double[200];
            k->_size = 200;
        }
    }
    return g_ps;
}

static gpudtVertex V(const double *p) { return gpudtVertex{p[0], p[1]}; }

extern "C" {
double ref_birth_time3(const double *p)
{
    gpudtVertex a = V(p), b = V(p + 2), c = V(p + 4);
    return ps()->birth_time(a, b, c);
}

double ref_birth_time2(const double *p)
{
    gpudtVertex a = V(p), b = V(p + 2);
    return ps()->birth_time(a, b);
}

int ref_is_attached(const double *i, const double *j, const double *k)
{
    gpudtVertex a = V(i), b = V(j), c = V(k);
    return ps()->isAttached(a, b, c, false) ? 1 : 0;
}

// The device comparison path (compareSlow, predicates.h:2443-2560) run on the
// host; kind 3 = triangle (6 coordinates), kind 2 = edge (4).  Negative
// values below -1 are the reference's overflow codes (-2, -3, -4).
int ref_compare_slow(int k1, const double *p1, int k2, const double *p2)
{
    Predicates *P = ps();
    gpudtVertex a = V(p1), b = V(p1 + 2), c = V(p1 + 4), d = V(p2), e = V(p2 + 2), f = V(p2 + 4);
    if (k1 == 2 && k2 == 2) return P->compareSlow(a, b, d, e, g_pd, 0);
    if (k1 == 2 && k2 == 3) return P->compareSlow(a, b, d, e, f, 1, g_pd, 0);
    if (k1 == 3 && k2 == 2) return P->compareSlow(a, b, c, d, e, g_pd, 0);
    return P->compareSlow(a, b, c, d, e, f, g_pd, 0);
}

// The host comparison path (CPUcompareSlow, predicates.h:2934-3106) with the
// dispatch of exactCompare (kernel.cu:1143-1153).
int ref_compare_cpu(int k1, const double *p1, int k2, const double *p2)
{
    Predicates *P = ps();
    gpudtVertex a = V(p1), b = V(p1 + 2), c = V(p1 + 4), d = V(p2), e = V(p2 + 2), f = V(p2 + 4);
    if (k1 == 2 && k2 == 2) return P->CPUcompareSlow(a, b, d, e);
    if (k1 == 2 && k2 == 3) return P->CPUcompareSlow(a, b, d, e, f, 1);
    if (k1 == 3 && k2 == 2) return P->CPUcompareSlow(a, b, c, d, e);
    return P->CPUcompareSlow(a, b, c, d, e, f);
}
}
