// oracle/ref_pred.cpp -- TEST INFRASTRUCTURE: C entry points over the
// reference's host predicates (gpudt/predicates.cpp:28, :322, :942), compiled
// from the reference tree by oracle/ref.mk.
#include "gpudt.h"
#include "predicates.h"

extern "C" {
void ref_exactinit(void) { gpudt_exactinit(); }

double ref_counterclockwise(const double *a, const double *b, const double *c)
{
    gpudtVertex A{a[0], a[1]}, B{b[0], b[1]}, C{c[0], c[1]};
    return counterclockwise(&A, &B, &C);
}

double ref_incircle(const double *a, const double *b, const double *c, const double *d)
{
    gpudtVertex A{a[0], a[1]}, B{b[0], b[1]}, C{c[0], c[1]}, D{d[0], d[1]};
    return incircle(&A, &B, &C, &D);
}
}
