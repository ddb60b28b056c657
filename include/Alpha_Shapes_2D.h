/*
 * Alpha_Shapes_2D.h -- source-compatible replacement of the reference's
 * alpha-shape class (gpudt/AlphaShape/Alpha_Shapes_2D.h:43-121), header-only,
 * over the C ABI of galpha.h (libgalpha.so).
 *
 * A caller of the reference recompiles unchanged against this header:
 *
 *     pOutput = gpudtComputeDT(pInput);            // main.cu:392
 *     Alpha_Shapes_2D as(pInput, pOutput);         // main.cu:394
 *     as.computeAlphaShapes();                     // main.cu:395
 *     for (MasterList_iterator it = as.Master_begin(); it != as.Master_end(); ++it) ...
 *
 * Kept from the reference: the class name, both constructors,
 * computeAlphaShapes(), Master_begin() / Master_end(), setAlpha() /
 * getAlpha(), dumpValues(), the public members spectrum, alpha, alpha_index
 * and master_list, the private point_list / edge_list / tri_list /
 * spec_pointers read by the friend class Visualizer, and the element types
 * and enums of headers.h:36-90 (point_interval, edge_interval,
 * triangle_interval, Alpha, simplex_type, alpha_type, simplex_category).
 *
 * Changed on purpose:
 *   - the host vectors are std::vector (define GALPHA_THRUST_HOST_VECTORS
 *     before including this header to get thrust::host_vector, as the
 *     reference declares them); both have size(), operator[], begin()/end();
 *   - computeAlphaShapes() reports a failure through status() and
 *     lastError() (and prints it, as the reference prints its errors) instead
 *     of continuing on broken state; the vectors are then empty;
 *   - dumpValues(fname) writes "<fname>out.txt" in the working directory
 *     (the reference writes under a fixed Windows path, Alpha_Shapes_2D.cu:755);
 *   - the class owns a galpha handle (one CUDA stream + device arena) and
 *     releases it in its destructor; it is movable, not copyable.
 * Values: spectrum holds the exactly rounded squared radii (the reference
 * stores its plain FP64 formula, which differs on slivers); ranks, intervals,
 * master_list and spec_pointers are those of the reference.
 */
#ifndef GALPHA_ALPHA_SHAPES_2D_H
#define GALPHA_ALPHA_SHAPES_2D_H

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gpudt.h"
#include "galpha.h"

#ifdef GALPHA_THRUST_HOST_VECTORS
#include <thrust/host_vector.h>
#define GALPHA_HVEC thrust::host_vector
#else
#define GALPHA_HVEC std::vector
#endif

/* headers.h:36-90 */
enum simplex_type { EDGE = 0, TRIANGLE = 1, VERTEX = 2 };
enum alpha_type { ro = 0, nu_min = 1, nu_max = 2 };
enum simplex_category { ATTACHED = 0, UNATTACHED };

struct point_interval {
    int nu_min_rank, nu_max_rank;
};

struct edge_interval {
    int ro_rank, nu_min_rank, nu_max_rank;
    simplex_category sc;
    int tIndex, vOpp;
};

struct triangle_interval {
    int ro_rank;
};

struct Alpha {
    int simplex_index;
    simplex_type st;
    alpha_type at;
};

static_assert(sizeof(point_interval) == sizeof(galphaPointInterval), "point_interval layout");
static_assert(sizeof(edge_interval) == sizeof(galphaEdgeInterval), "edge_interval layout");
static_assert(sizeof(triangle_interval) == sizeof(galphaTriangleInterval), "triangle_interval layout");
static_assert(sizeof(Alpha) == sizeof(galphaAlpha), "Alpha layout");

typedef GALPHA_HVEC<double> DoubleHVec;
typedef GALPHA_HVEC<Alpha> AlphaHVec;
typedef GALPHA_HVEC<point_interval> PointIntervalHVec;
typedef GALPHA_HVEC<edge_interval> EdgeIntervalHVec;
typedef GALPHA_HVEC<triangle_interval> TriangleIntervalHVec;
typedef GALPHA_HVEC<int> IntHVec;
typedef AlphaHVec::iterator MasterList_iterator;

class Alpha_Shapes_2D {
private:
    PGPUDTOUTPUT pDT;
    PGPUDTPARAMS pInput;

    PointIntervalHVec point_list;
    EdgeIntervalHVec edge_list;
    TriangleIntervalHVec tri_list;
    IntHVec spec_pointers;

    galphaHandle handle_;
    int status_;
    std::string error_;

    template <typename T, typename S>
    static void fill(GALPHA_HVEC<T> &dst, const S *src, int n)
    {
        dst.resize(n > 0 ? (size_t)n : 0);
        if (n > 0) memcpy(&dst[0], src, sizeof(T) * (size_t)n);
    }

    void fail(int code, const char *where)
    {
        status_ = code;
        const char *txt = galphaLastError();
        error_ = std::string(where) + " failed (" + std::to_string(code) + ")";
        if (txt && *txt) error_ += ": " + std::string(txt);
        fprintf(stderr, "Alpha_Shapes_2D: %s\n", error_.c_str());
    }

    void clear_all()
    {
        point_list.clear();
        edge_list.clear();
        tri_list.clear();
        spec_pointers.clear();
        spectrum.clear();
        master_list.clear();
    }

public:
    DoubleHVec spectrum;
    REAL alpha;
    int alpha_index;
    AlphaHVec master_list;

    Alpha_Shapes_2D() : pDT(NULL), pInput(NULL), handle_(NULL), status_(GPUDT_OK), alpha(0), alpha_index(0) {}

    Alpha_Shapes_2D(PGPUDTPARAMS pIpt, PGPUDTOUTPUT pDelaunay)
        : pDT(pDelaunay), pInput(pIpt), handle_(NULL), status_(GPUDT_OK), alpha(0), alpha_index(0)
    {
    }

    ~Alpha_Shapes_2D()
    {
        if (handle_) galphaDestroy(handle_);
    }

    Alpha_Shapes_2D(const Alpha_Shapes_2D &) = delete;
    Alpha_Shapes_2D &operator=(const Alpha_Shapes_2D &) = delete;
    Alpha_Shapes_2D(Alpha_Shapes_2D &&o) noexcept
        : pDT(o.pDT), pInput(o.pInput), point_list(std::move(o.point_list)), edge_list(std::move(o.edge_list)),
          tri_list(std::move(o.tri_list)), spec_pointers(std::move(o.spec_pointers)), handle_(o.handle_),
          status_(o.status_), error_(std::move(o.error_)), spectrum(std::move(o.spectrum)), alpha(o.alpha),
          alpha_index(o.alpha_index), master_list(std::move(o.master_list))
    {
        o.handle_ = NULL;
    }

    /* Alpha_Shapes_2D.cu:206-233: spectrum, intervals and master list of the
     * triangulation pDT of pInput's points. */
    void computeAlphaShapes()
    {
        clear_all();
        alpha = 0;
        alpha_index = 0;
        status_ = GPUDT_OK;
        error_.clear();
        if (!pInput || !pDT) {
            fail(GPUDT_ERR_ARG, "computeAlphaShapes (no input)");
            return;
        }
        if (!handle_) {
            int r = galphaCreate(-1, 0, &handle_);
            if (r) {
                handle_ = NULL;
                fail(r, "galphaCreate");
                return;
            }
        }
        GAlphaOutput out;
        memset(&out, 0, sizeof(out));
        int r = galphaCompute(handle_, pInput, pDT, &out);
        if (r) {
            galphaReleaseOutput(&out);
            fail(r, "galphaCompute");
            return;
        }
        fill(spectrum, out.spectrum, out.nSpectrum);
        fill(point_list, out.point_list, out.nPoints);
        fill(edge_list, out.edge_list, out.nEdges);
        fill(tri_list, out.tri_list, out.nTris);
        galphaReleaseOutput(&out);
        GAlphaMasterList ml;
        memset(&ml, 0, sizeof(ml));
        r = galphaMasterList(handle_, &ml);
        if (r) {
            galphaReleaseMasterList(&ml);
            clear_all();
            fail(r, "galphaMasterList");
            return;
        }
        fill(master_list, ml.master_list, ml.nMaster);
        fill(spec_pointers, ml.spec_pointers, ml.nSpecPointers);
        galphaReleaseMasterList(&ml);
    }

    MasterList_iterator Master_begin() { return master_list.begin(); }
    MasterList_iterator Master_end() { return master_list.end(); }
    void setAlpha(REAL val) { alpha = val; }
    REAL getAlpha() { return alpha; }

    /* Writes the spectrum size, as the reference's dumpValues does. */
    void dumpValues(std::string fname)
    {
        FILE *f = fopen((fname + "out.txt").c_str(), "w");
        if (!f) return;
        fprintf(f, "%d\n", (int)spectrum.size());
        fclose(f);
    }

    /* Extensions: GPUDT_OK or the GPUDT_ERR_* code of the last
     * computeAlphaShapes(), with its message. */
    int status() const { return status_; }
    const std::string &lastError() const { return error_; }

    friend class Visualizer;
};

#endif
