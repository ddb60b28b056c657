/*
 * galpha.h -- alpha-shape (GAlpha) boundary of the galpha-b200 engine, plus the
 * re-entrant handle API used by the DT + alpha-spectrum hot path.
 *
 *   reference interface                                  replaced by
 *   ---------------------------------------------------  -------------------------------
 *   Alpha_Shapes_2D(PGPUDTPARAMS, PGPUDTOUTPUT)          galphaCompute(h, params, dt, out)
 *     + computeAlphaShapes()                              (alpha of a host triangulation)
 *     gpudt/AlphaShape/Alpha_Shapes_2D.h:43-121,
 *     Alpha_Shapes_2D.cu:206-727
 *   public members spectrum / private point_list,        GAlphaOutput arrays (same element
 *     edge_list, tri_list (Alpha_Shapes_2D.h:100-117,      layouts as headers.h:48-90)
 *     headers.h:48-64)
 *   gpudtComputeDT then Alpha_Shapes_2D (main.cu:392-395) galphaTriangulate +
 *                                                         galphaComputeResident (mesh stays in
 *                                                         device memory between the two)
 *
 * Interval semantics (kernel.cu:219-624): the spectrum holds squared radii in
 * increasing order, spectrum[0] = 0 is the sentinel "attached / not applicable";
 * exactly equal values share one rank; every *_rank indexes the spectrum;
 * nu_max_rank 0 on a hull edge means "infinity".  Edges are numbered as the
 * reference numbers them: triangle t owns its edge i (opposite vtx[i]) when
 * vtx[i+1] < vtx[i+2] or tri[i] == -1, edges ordered by t then i.
 */
#ifndef GALPHA_GALPHA_H
#define GALPHA_GALPHA_H

#include "gpudt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* headers.h:48-64 element layouts */
typedef struct { int nu_min_rank, nu_max_rank; } galphaPointInterval;
typedef struct {
    int ro_rank, nu_min_rank, nu_max_rank;
    int sc; /* simplex_category: 0 ATTACHED, 1 UNATTACHED */
    int tIndex, vOpp;
} galphaEdgeInterval;
typedef struct { int ro_rank; } galphaTriangleInterval;

typedef struct {
    int nSpectrum;                    /* distinct values incl. the 0 sentinel */
    double *spectrum;                 /* [nSpectrum] */
    int nPoints;
    galphaPointInterval *point_list;  /* [nPoints] */
    int nEdges;
    galphaEdgeInterval *edge_list;    /* [nEdges] */
    int nTris;
    galphaTriangleInterval *tri_list; /* [nTris] */
    long long exactCompares;          /* spectrum comparisons resolved exactly */
    long long exactTies;              /* exactly equal neighbours merged */
    long long exactAttached;          /* attached tests resolved exactly */
} GAlphaOutput;

typedef struct galpha_ctx *galphaHandle;

/* Stage indices of gpudtStatus.ms */
#define GALPHA_STAGE_UPLOAD    0
#define GALPHA_STAGE_VORONOI   1  /* scatter + column pass + row pass + islands */
#define GALPHA_STAGE_TRIANGLES 2  /* Voronoi vertices -> triangles + links */
#define GALPHA_STAGE_SHIFT     3  /* shifting + bad-case removal */
#define GALPHA_STAGE_MISSING   4  /* missing-site insertion */
#define GALPHA_STAGE_BOUNDARY  5  /* fake ring removal + hull */
#define GALPHA_STAGE_FLIP      6  /* Lawson flipping */
#define GALPHA_STAGE_COMPACT   7  /* compaction / output layout */
#define GALPHA_STAGE_ALPHA     8  /* birth times + attached + sort + ranks + intervals */
#define GALPHA_STAGE_DOWNLOAD  9
#define GALPHA_STAGE_TOTAL     10
#define GALPHA_STAGE_MASTER    11  /* master list (galphaRunDevice with withAlpha = 2) */

/* Create a handle on CUDA device `device` (-1: current device).  Device memory
 * is reserved lazily and grown on demand; budgetBytes (0: no limit) caps it. */
int galphaCreate(int device, long long budgetBytes, galphaHandle *out);
int galphaDestroy(galphaHandle h);
/* Work on a caller stream (a cudaStream_t passed as void*; NULL: the handle's own). */
int galphaSetStream(galphaHandle h, void *stream);

/* Delaunay triangulation.  If out != NULL the triangles are copied to host:
 * into out->triangles when the caller sets it (capacity in out->nTris; pinned
 * memory makes it one DMA copy), else into a new[] array of capacity
 * 2 * nVerts as gpudtComputeDT allocates it.  The mesh also stays resident on
 * the device for galphaComputeResident. */
int galphaTriangulate(galphaHandle h, const GPUDTPARAMS *params, GPUDTOUTPUT *out, gpudtStatus *st);

/* Alpha spectrum + intervals of the handle's resident mesh.  Output arrays:
 * caller buffers when all four pointers are set (capacities in the count
 * fields; GPUDT_ERR_NOMEM if too small), else malloc'd arrays released by
 * galphaReleaseOutput. */
int galphaComputeResident(galphaHandle h, GAlphaOutput *out);

/* gpudtComputeDT followed by Alpha_Shapes_2D + computeAlphaShapes
 * (main.cu:392-395) in one call: dt receives the triangles (same rules as
 * galphaTriangulate's out), out the alpha arrays (same rules as
 * galphaComputeResident).  The triangles travel to the host while the alpha
 * stage runs. */
int galphaComputeAll(galphaHandle h, const GPUDTPARAMS *params, GPUDTOUTPUT *dt, GAlphaOutput *out,
                     gpudtStatus *st);

/* Alpha spectrum + intervals of a host triangulation (Alpha_Shapes_2D(pInput, pDT)). */
int galphaCompute(galphaHandle h, const GPUDTPARAMS *params, const GPUDTOUTPUT *dt, GAlphaOutput *out);

/* Device-resident hot path: points already in device memory (d_xy: 2*n doubles).
 * Runs DT (+ alpha when withAlpha & 3 is 1; + the master list when it is 2) and
 * leaves every result on the device.  With GALPHA_RUN_TRIANGLES set in
 * withAlpha the gpudtTriangle records are built on the device too (otherwise
 * they are built by the first call that copies them out).
 * Returns the status; counts through galphaGetCounts. */
#define GALPHA_RUN_TRIANGLES 4
int galphaRunDevice(galphaHandle h, const double *d_xy, int n, double minX, double minY,
                    double maxX, double maxY, int fboSize, int withAlpha, gpudtStatus *st);

/* Sizes of the last result: nTris, nEdges, nSpectrum (any pointer may be NULL). */
int galphaGetCounts(galphaHandle h, int *nTris, int *nEdges, int *nSpectrum);

/* Copy the resident triangles (gpudtTriangle layout) to host memory. */
int galphaCopyTriangles(galphaHandle h, gpudtTriangle *dst, int cap);

void galphaReleaseOutput(GAlphaOutput *out);

/* ------------------------------------------------------------ batches
 * Many independent point sets in one pipeline run (no reference
 * counterpart: the reference computes one set per gpudtComputeDT /
 * Alpha_Shapes_2D call).  Set s has setSizes[s] points, stored after the
 * points of sets 0..s-1 in one interleaved xy array, and the bounds
 * bounds[4s .. 4s+3] = minX, minY, maxX, maxY (the GPUDTPARAMS fields, which
 * must contain every point of the set).  Each set's result is exactly what a
 * separate galphaRunDevice call gives (the texture size is chosen per set);
 * the results are stored set after set: */
typedef struct {
    int nPoints, pointBase;  /* point_list rows of the set */
    int nTris, triBase;      /* triangles and tri_list rows of the set */
    int nEdges, edgeBase;    /* edge_list rows of the set */
    int nSpectrum, specBase; /* spectrum values of the set, [specBase] = 0 (its rank 0) */
} galphaBatchSet;

/* d_xy: device memory.  withAlpha: 0 DT only, 1 DT + alpha. */
int galphaRunBatch(galphaHandle h, int nSets, const int *setSizes, const double *d_xy, const double *bounds,
                   int withAlpha, gpudtStatus *st);
/* The same from host memory (copied to the device inside the call). */
int galphaRunBatchHost(galphaHandle h, int nSets, const int *setSizes, const double *xy, const double *bounds,
                       int withAlpha, gpudtStatus *st);
/* Texture pixels per point of each set's cell in later batches (1 to 64;
 * default 10).  The cell is the smallest power of two, at least 128, whose
 * area inside the fake-site margin holds that many pixels per point; the
 * result of a set does not depend on it, the speed does (see
 * galpha_b200/autotune.py). */
int galphaSetBatchDensity(galphaHandle h, double pixelsPerPoint);
/* Per-set counts and bases of the last batch (host array of nSets). */
int galphaBatchSets(galphaHandle h, galphaBatchSet *sets);
/* Copy the last batch's results to host buffers sized by galphaBatchSets
 * (any pointer may be NULL).  Vertex, triangle and neighbour indices are local
 * to each set, as a per-set gpudtComputeDT would return them; ranks are per
 * set; spectrum holds every set's spectrum at its specBase. */
int galphaBatchCopy(galphaHandle h, gpudtTriangle *tris, galphaPointInterval *points,
                    galphaEdgeInterval *edges, int *triRanks, double *spectrum);

/* Alpha (headers.h:80-86): one master-list entry.  st: 0 edge, 1 triangle,
 * 2 vertex (simplex_type); at: 0 ro, 1 nu_min, 2 nu_max (alpha_type). */
typedef struct {
    int simplex_index;
    int st;
    int at;
} galphaAlpha;

/* master_list and spec_pointers of Alpha_Shapes_2D (compute_master_list,
 * Alpha_Shapes_2D.cu:641-727): every interval end point (2 per vertex, 3 per
 * edge, 1 per triangle) sorted stably by rank, rank-0 entries removed;
 * spec_pointers = -1 followed by the first master-list index of each distinct
 * rank.  When both pointers are set they are caller buffers (capacities in
 * nMaster / nSpecPointers on input), else the arrays are malloc'd and freed by
 * galphaReleaseMasterList. */
typedef struct {
    int nMaster;
    galphaAlpha *master_list;
    int nSpecPointers;
    int *spec_pointers;
} GAlphaMasterList;

/* Master list of the resident alpha result (after galphaCompute,
 * galphaComputeResident or galphaRunDevice with alpha). */
int galphaMasterList(galphaHandle h, GAlphaMasterList *out);
void galphaReleaseMasterList(GAlphaMasterList *out);

/* Alpha-complex query on the resident result (after galphaCompute,
 * galphaComputeResident or galphaRunDevice with alpha).  alpha is a squared
 * radius (the unit of the spectrum).  With R the largest rank whose spectrum
 * value is <= alpha, every simplex is classified from its interval
 * (headers.h:48-64 ranks; interval meaning as kernel.cu:427-624):
 *   GALPHA_INTERIOR  nu_max finite (!= 0) and <= R   (triangles: ro <= R)
 *   GALPHA_REGULAR   nu_min <= R
 *   GALPHA_SINGULAR  unattached edge with ro <= R; a vertex below nu_min
 *   GALPHA_EXTERIOR  otherwise, every simplex when alpha < 0, and input
 *                    points dropped as duplicates.
 * The classes stay on the device (galphaCopyClasses) and the per-class counts
 * are returned.  The reference exposes this only through its viewer
 * (Visualizer.cu:296-337). */
#define GALPHA_EXTERIOR 0
#define GALPHA_SINGULAR 1
#define GALPHA_REGULAR 2
#define GALPHA_INTERIOR 3

typedef struct {
    double alpha;    /* the value classified (for a quantile query, the spectrum value chosen) */
    int rank;        /* largest rank with spectrum[rank] <= alpha; -1 when alpha < 0 */
    int nPoints[4];  /* counts per class, indexed by GALPHA_* */
    int nEdges[4];
    int nTris[4];
} galphaQueryResult;

int galphaQuery(galphaHandle h, double alpha, galphaQueryResult *res);

/* The same at alpha = spectrum[round(q * (nSpectrum - 1))], q in [0, 1]. */
int galphaQueryQuantile(galphaHandle h, double q, galphaQueryResult *res);

/* Copy the classes of the last query (one byte per point / edge / triangle,
 * in point, edge_list and tri_list order); any pointer may be NULL. */
int galphaCopyClasses(galphaHandle h, unsigned char *pointClass, unsigned char *edgeClass,
                      unsigned char *triClass);

/* Alpha-complex query (as galphaQuery) on every set of the last batch at
 * once: values[s] is set s's alpha, or its spectrum quantile when byQuantile
 * is set; res[s] receives set s's counts.  The per-simplex classes, in batch
 * order, are then available through galphaCopyClasses. */
int galphaBatchQuery(galphaHandle h, const double *values, int byQuantile, galphaQueryResult *res);

/* Edge numbering of a triangle-neighbour mesh that is already in device
 * memory, for callers that cannot allocate: a serving or rendering loop that
 * has reserved its device memory up front and cannot give any to a library
 * mid-stream, or code that must not call cudaMalloc/cudaFree because those
 * can synchronise the whole device while other streams have work in flight.
 * This call allocates nothing (no device or pinned memory, no handle, no
 * events); it runs one kernel on `stream` and returns without waiting.
 *
 * In:  d_tris[0..nTris), gpudtTriangle layout, device memory.
 * Out: d_edges[2*k], d_edges[2*k+1] = (tIndex, vOpp) of edge k, in the order
 *      and with the owner rule of GAlphaOutput.edge_list (an edge belongs to
 *      the triangle in which its first vertex has the smaller index, or that
 *      has no neighbour across it); at most edgeCapacity pairs are written.
 *      *d_nEdges = the number of edges (may exceed edgeCapacity), or a
 *      negative GPUDT_ERR_* code written by the kernel.
 * Limit: nTris <= 67,108,864; larger meshes are rejected with GPUDT_ERR_ARG
 * (the kernel's scratch is a fixed 512 KB device array inside the library,
 * held by every device that loads it until the process exits).
 * Every call on a device shares that array: calls on one device must be
 * ordered (one stream, or synchronised); two calls in flight at once race.
 * The first call on each device (and the first after a cudaDeviceReset)
 * zeroes the array on `stream`; make that call before any stream capture.
 * No counterpart in the reference: there the edge list is built inside
 * Alpha_Shapes_2D (Alpha_Shapes_2D.cu:170-199) in thrust-allocated memory. */
int galphaEdgeListNoAlloc(const gpudtTriangle *d_tris, int nTris, int *d_edges, int edgeCapacity,
                          int *d_nEdges, void *stream);

/* Failure-detection limits, for tests of the error paths.  On a handle:
 * maxRounds caps every iterative stage (shifting, insertion, fake removal,
 * flipping, island recolouring; default 100,000), after which the call
 * returns GPUDT_ERR_NOCONVERGE; spinLimit bounds each wait of the spectrum
 * sort's single-pass look-back (default 2^22 polls), after which the call
 * returns GPUDT_ERR_NOCONVERGE with detail 98; holdFirstTile != 0 makes the
 * first tile of that look-back withhold its counts, so that the next tile's
 * wait runs out.  With h == NULL, spinLimit and holdFirstTile apply in the
 * same way to galphaEdgeListNoAlloc (process-wide; its *d_nEdges then reads
 * GPUDT_ERR_NOCONVERGE).  Values <= 0 restore the defaults.  Every wait stays
 * bounded, a failed call leaves the handle usable, and the next call with
 * the defaults restored computes the full result.
 * No counterpart in the reference, whose stages loop until done and whose
 * CUDA failures exit the process (common.h:55-93). */
int galphaSetLimits(galphaHandle h, int maxRounds, int spinLimit, int holdFirstTile);

/* Spectrum entries whose keys lie within 2 ulp of their neighbours form runs
 * that are ordered with exact arithmetic.  A run of more than `entries`
 * entries (default 65,536; <= 0 restores it) is merge-sorted by many blocks,
 * one launch per merge level, instead of by one block; there is no upper
 * limit on a run's length (a lattice of non-dyadic spacing gives runs of
 * millions).  No counterpart in the reference, whose odd-even rounds and
 * host insertion sort (kernel.cu:962-1102, Alpha_Shapes_2D.cu:524-610)
 * order such runs without a size limit. */
int galphaSetBlockRun(galphaHandle h, int entries);

/* Loop schedule of the handle's later calls.  shiftGroup and missingGroup
 * (1..8; defaults 4 and 2): rounds of the shifting loops and of missing-site
 * insertion run between two device-to-host counter reads; flipSync (1..64,
 * default 4): the same for the flip rounds; flipTailEnter (0..2^20, default
 * 4,096): the active flip list length at or below which the remaining rounds
 * run inside one block; flipTailLeave (>= flipTailEnter, up to 2^22, default
 * 32,768): the length above which that block hands them back.  A round past
 * the end of a loop does nothing and the in-block rounds are the launched
 * rounds' functors, so no value changes a result, only the time and
 * gpudtStatus.hostReads; 0 (-1 for flipTailEnter) restores a default, values
 * out of range return GPUDT_ERR_ARG.  galphaGetSchedule fills out5 with the
 * five values in force.  The autotuner (galpha_b200.autotune) picks them per
 * workload.  No counterpart in the reference. */
int galphaSetSchedule(galphaHandle h, int shiftGroup, int missingGroup, int flipSync, int flipTailEnter,
                      int flipTailLeave);
int galphaGetSchedule(galphaHandle h, int *out5);

/* Text of the last error on the calling thread (cleared when a compute call
 * -- RunDevice, Triangulate, Compute*, RunBatch*, gpudtComputeDTEx -- starts). */
const char *galphaLastError(void);

/* Number of CUDA kernels this library has launched since it was loaded. */
unsigned long long galphaLaunchCount(void);

/* Version / build information string. */
const char *galphaVersion(void);

#ifdef __cplusplus
}
#endif
#endif
