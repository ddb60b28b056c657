// oracle/ref_alpha_gpu.cu -- TEST INFRASTRUCTURE: a C entry point that runs the
// reference's own GPU alpha-shape engine, unmodified, on a given triangulation.
//
// oracle/ref.mk compiles the reference's gpudt/AlphaShape/{Alpha_Shapes_2D.cu,
// kernel.cu, headers.cu} from the reference tree (never copied here) with nvcc
// for sm_100a and links this file into oracle/_ref/librefalpha.so.  Only the
// GPU parity tests load it, as the checker of galphaCompute: it is never linked
// into libgalpha.so and no product path calls it.
//
// The engine is driven exactly as the reference's main.cu:392-395 does:
// Alpha_Shapes_2D(pInput, pDT) then computeAlphaShapes()
// (Alpha_Shapes_2D.cu:206-233, which ends in compute_master_list,
// :641-727).  Its results are host vectors; spectrum and master_list are
// public, point_list / edge_list / tri_list / spec_pointers are private and
// read by the class's friend `Visualizer` (Alpha_Shapes_2D.h:117).  The
// reference's own Visualizer (an OpenGL viewer) is not built, so the
// `Visualizer` below is the only class of that name in the library: a reader
// of those members, nothing else.
#include <cstdio>
#include <cstring>
#include <vector>

#include "Alpha_Shapes_2D.h"

class Visualizer {
public:
    static void sizes(Alpha_Shapes_2D &a, int *out)
    {
        out[0] = (int)a.spectrum.size();
        out[1] = (int)a.point_list.size();
        out[2] = (int)a.edge_list.size();
        out[3] = (int)a.tri_list.size();
        out[4] = (int)a.master_list.size();
        out[5] = (int)a.spec_pointers.size();
    }

    template <typename T>
    static void put(const thrust::host_vector<T> &v, void *dst)
    {
        if (dst && v.size()) memcpy(dst, thrust::raw_pointer_cast(v.data()), v.size() * sizeof(T));
    }

    static void copy(Alpha_Shapes_2D &a, double *spectrum, int *point_list, int *edge_list, int *tri_list,
                     int *master_list, int *spec_pointers)
    {
        put(a.spectrum, spectrum);
        put(a.point_list, point_list);
        put(a.edge_list, edge_list);
        put(a.tri_list, tri_list);
        put(a.master_list, master_list);
        put(a.spec_pointers, spec_pointers);
    }
};

namespace {

struct RefRun {
    std::vector<gpudtVertex> pts;
    std::vector<gpudtTriangle> tris;
    GPUDTPARAMS in;
    GPUDTOUTPUT dt;
    Alpha_Shapes_2D *engine = nullptr;
};

}  // namespace

// Element layouts the caller reads (headers.h:48-90): point_interval 2 ints,
// edge_interval 6 ints (ro, nu_min, nu_max, sc, tIndex, vOpp), triangle_interval
// 1 int, Alpha 3 ints (simplex_index, st, at).
static_assert(sizeof(point_interval) == 8, "point_interval layout");
static_assert(sizeof(edge_interval) == 24, "edge_interval layout");
static_assert(sizeof(triangle_interval) == 4, "triangle_interval layout");
static_assert(sizeof(Alpha) == 12, "Alpha layout");
static_assert(sizeof(gpudtTriangle) == 36, "gpudtTriangle layout");

// Runs the reference engine on n points (xy: 2n doubles) and the triangle
// array tris (nTris records of 9 ints, gpudtTriangle).  Returns a handle, or
// NULL after a CUDA error (message on stderr).
extern "C" void *refalpha_run(const double *xy, int n, const int *tris, int nTris)
{
    if (n <= 0 || nTris <= 0 || !xy || !tris) return nullptr;
    RefRun *r = new RefRun;
    r->pts.resize(n);
    memcpy(r->pts.data(), xy, sizeof(gpudtVertex) * (size_t)n);
    r->tris.resize(nTris);
    memcpy(r->tris.data(), tris, sizeof(gpudtTriangle) * (size_t)nTris);
    double x0 = xy[0], x1 = xy[0], y0 = xy[1], y1 = xy[1];
    for (int i = 1; i < n; i++) {
        x0 = xy[2 * i] < x0 ? xy[2 * i] : x0;
        x1 = xy[2 * i] > x1 ? xy[2 * i] : x1;
        y0 = xy[2 * i + 1] < y0 ? xy[2 * i + 1] : y0;
        y1 = xy[2 * i + 1] > y1 ? xy[2 * i + 1] : y1;
    }
    memset(&r->in, 0, sizeof(r->in));
    r->in.minX = x0;
    r->in.minY = y0;
    r->in.maxX = x1;
    r->in.maxY = y1;
    r->in.nPoints = n;
    r->in.points = r->pts.data();
    r->in.fboSize = 512;
    r->dt.triangles = r->tris.data();
    r->dt.nTris = nTris;
    cudaGetLastError();
    r->engine = new Alpha_Shapes_2D(&r->in, &r->dt);
    r->engine->computeAlphaShapes();
    fflush(stdout);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "refalpha_run: CUDA error %s\n", cudaGetErrorString(e));
        delete r->engine;
        delete r;
        return nullptr;
    }
    return r;
}

// sizes[0..5] = spectrum, point_list, edge_list, tri_list, master_list, spec_pointers
extern "C" void refalpha_sizes(void *h, int *sizes)
{
    Visualizer::sizes(*((RefRun *)h)->engine, sizes);
}

extern "C" void refalpha_copy(void *h, double *spectrum, int *point_list, int *edge_list, int *tri_list,
                              int *master_list, int *spec_pointers)
{
    Visualizer::copy(*((RefRun *)h)->engine, spectrum, point_list, edge_list, tri_list, master_list,
                     spec_pointers);
}

extern "C" void refalpha_free(void *h)
{
    RefRun *r = (RefRun *)h;
    if (!r) return;
    delete r->engine;
    delete r;
}
