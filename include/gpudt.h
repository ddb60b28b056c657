/*
 * gpudt.h -- drop-in C/C++ boundary of the galpha-b200 Delaunay engine.
 *
 * Types are laid out exactly as the reference's gpudt/gpudt.h:81-128 (REAL is
 * double; SINGLE_PRECISION is not supported), so a caller compiled against the
 * reference header links against libgalpha.so unchanged.
 *
 *   reference interface                          replaced by
 *   -------------------------------------------  -----------------------------------
 *   PGPUDTOUTPUT gpudtComputeDT(PGPUDTPARAMS)    gpudtComputeDT (same C++ symbol,
 *     gpudt/gpudt.h:131, gpudt.cpp:771-924         _Z14gpudtComputeDTP11GPUDTPARAMS)
 *   void gpudtReleaseDTOutput(PGPUDTOUTPUT)      gpudtReleaseDTOutput (same C++ symbol,
 *     gpudt/gpudt.h:132, gpudt.cpp:926-929         _Z20gpudtReleaseDTOutputP11GPUDTOUTPUT)
 *   (none: the reference exits on error)         gpudtComputeDTEx, status-returning,
 *                                                 re-entrant per handle
 *
 * Semantics kept from the reference:
 *   - points are read from pParam->points[0..nPoints); minX..maxY must bound them
 *     (they fix the grid mapping, gpudt.cpp:722-769);
 *   - fboSize is the discrete Voronoi texture edge, a power of two in [256, 16384];
 *   - the output owns triangles = new gpudtTriangle[2 * nVerts] (capacity), nTris
 *     of them valid, counterclockwise, vtx[] are input indices; tri[i] =
 *     (t << 2) | j is the neighbour across the edge opposite vtx[i], -1 on the hull;
 *   - exact duplicates are dropped (the lowest input index survives);
 *   - constraints[0..2*nConstraints) are pairs of input indices that become
 *     edges of the result, which is then the constrained Delaunay triangulation
 *     (gpudt.cpp:860 cudaConstraint).
 * Differences from the reference: errors are returned, not exit(-1); tmp[3]
 * is zero-filled instead of internal chain garbage; constraints that cross
 * each other or pass through a point are GPUDT_ERR_ARG (undefined there).
 */
#ifndef GALPHA_GPUDT_H
#define GALPHA_GPUDT_H

#define REAL double
#define MARKER -32768

typedef struct {
    REAL x, y;
} gpudtVertex;

typedef struct gpudtTriangle {
    int tri[3]; /* 3 neighbour triangles, encoded oriented triangles */
    int vtx[3]; /* 3 vertices, counterclockwise */
    int tmp[3]; /* zero */
} gpudtTriangle;

typedef struct {
    REAL minX, minY;
    REAL maxX, maxY;
    int nPoints;
    gpudtVertex *points;
    int nConstraints;
    int *constraints;
    int fboSize;
} GPUDTPARAMS, *PGPUDTPARAMS;

typedef struct {
    gpudtTriangle *triangles;
    int nTris;
} GPUDTOUTPUT, *PGPUDTOUTPUT;

/* Status codes returned by the Ex / handle entry points. */
#define GPUDT_OK               0
#define GPUDT_ERR_ARG         -1 /* bad parameters (fboSize, nPoints, NaN/Inf, constraints) */
#define GPUDT_ERR_CUDA        -2 /* a CUDA runtime call failed */
#define GPUDT_ERR_NOMEM       -3 /* device or host allocation failed / over budget */
#define GPUDT_ERR_TOPOLOGY    -4 /* an internal mesh invariant did not hold */
#define GPUDT_ERR_NOCONVERGE  -5 /* an iterative stage hit its iteration cap */
#define GPUDT_ERR_EXACT       -6 /* exact-arithmetic scratch overflow */
#define GPUDT_ERR_NODEVICE    -7 /* no usable sm_100 device */

/* Per-call statistics (all counts are for the last call on the handle). */
typedef struct {
    int status;
    int nVerts;              /* nPoints + fake ring sites */
    int nFake;               /* fake ring sites added and removed */
    int nDuplicates;         /* exact duplicates dropped */
    int nMissing;            /* sites inserted by point location */
    int nBadShift;           /* sites that could not be shifted (removed, re-inserted) */
    int nIslandPixels;       /* island pixels recoloured on the envelope (global) path */
    int nFlips;              /* Lawson flips performed */
    int flipRounds;          /* flip rounds */
    int shiftRounds;         /* shifting rounds */
    int missingRounds;       /* insertion rounds */
    int nRepairTiles;        /* fused-path tiles with islands, repaired locally */
    int nEscalated;          /* textures (point sets) redone on the envelope path */
    int nEnvelopeCells;      /* textures (point sets) coloured on the envelope path */
    /* Predicate stages (FP32 filter -> FP64 filter -> exact expansion).  A test
     * decided by the FP32 filter is counted in the total only. */
    long long exactOrient;   /* orientation tests that needed exact arithmetic */
    long long exactIncircle; /* in-circle tests that needed exact arithmetic */
    long long filteredIncircle; /* in-circle tests decided by the FP64 filter */
    long long incircleTests;    /* in-circle tests (flip stage), all stages */
    long long orientTests;      /* orientation tests of the mesh stages, all stages */
    long long filteredOrient;   /* orientation tests decided by the FP64 filter */
    float ms[12];            /* stage times (CUDA events), see galpha.h GALPHA_STAGE_* */
    float kernelMs[4];       /* single-kernel times (CUDA events on the launch stream):
                                [0] colour + dual-triangle kernel (k_vd_tri; k_row_pass on
                                the envelope path), [1] column pass,
                                [2] triangle emission (count + write),
                                [3] spectrum key sort (all radix passes, alpha stage) */
    long long sortKeys;      /* keys of the spectrum sort */
    int sortPasses;          /* radix passes it took (8-bit digits) */
    int hostReads;           /* device -> host reads of the call, each one stream synchronisation
                                (the host reads work-list sizes between stages) */
    int constraintRounds;    /* segment-insertion rounds (0 without constraints) */
    int reserved0;
    int hostReadsStage[12];  /* hostReads per stage, indexed like ms[] */
} gpudtStatus;

#ifdef __cplusplus
/* C++ linkage, as the reference's gpudt.h:131-132. */
PGPUDTOUTPUT gpudtComputeDT(PGPUDTPARAMS pParam);
void gpudtReleaseDTOutput(PGPUDTOUTPUT pGpudtOutput);
extern "C" {
#endif

/* extern "C" twins of the two reference entry points (for C, ctypes, cgo). */
PGPUDTOUTPUT gpudt_compute_dt(PGPUDTPARAMS pParam);
void gpudt_release_dt_output(PGPUDTOUTPUT pGpudtOutput);

/* Status-returning form.  Fills *pOutput (triangles allocated with new[] as the
 * reference does; release with gpudt_release_dt_output / gpudtReleaseDTOutput,
 * which also frees the struct only if it was returned by gpudt_compute_dt).
 * status may be NULL.  Uses an internal default handle (not re-entrant); the
 * handle API in galpha.h is re-entrant per handle. */
int gpudtComputeDTEx(const GPUDTPARAMS *pParam, GPUDTOUTPUT *pOutput, gpudtStatus *status);

#ifdef __cplusplus
}
#endif
#endif
