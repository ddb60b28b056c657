/*
 * oracle/oracle.h -- TEST INFRASTRUCTURE, not product code.
 *
 * C entry points of the CPU oracle (liboracle.so).  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load
 * this library, and only as the checker.
 */
#ifndef GALPHA_ORACLE_H
#define GALPHA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_ERR_ARG      -1
#define ORACLE_ERR_CAP      -2
#define ORACLE_ERR_TOPOLOGY -3
#define ORACLE_ERR_EXACT    -4

/* Exact Delaunay triangulation of npts points (xy interleaved).  Writes up to
 * cap triangles: out_vtx[3t+i] vertices (counterclockwise), out_nbr[3t+i] the
 * encoded neighbour across the edge opposite vtx[i] (gpudt.h:97-102).
 * Returns the triangle count or a negative ORACLE_ERR_*. */
int oracle_dt(int npts, const double *xy, int cap, int *out_vtx, int *out_nbr, int *out_nkept);

/* Constrained Delaunay triangulation: cons holds ncons pairs of point
 * indices (non-crossing segments through no other point).  Same outputs as
 * oracle_dt; every constraint is an edge, every other edge locally Delaunay. */
int oracle_cdt(int npts, const double *xy, int ncons, const int *cons, int cap, int *out_vtx, int *out_nbr,
               int *out_nkept);

/* Validates a mesh; out[6]: link errors, non-CCW, non-Delaunay edges, hull
 * edges, non-convex hull edges, bad indices. */
int oracle_check_mesh(int npts, const double *xy, int ntri, const int *vtx, const int *nbr, long long *out);

/* Exact sign predicates (for cross-checks of the product's predicates). */
int oracle_orient2d(const double *a, const double *b, const double *c);
int oracle_incircle(const double *a, const double *b, const double *c, const double *d);
long long oracle_exact_counts(int which);

/* Alpha-shape spectrum and intervals of a triangulation (Alpha_Shapes_2D,
 * gpudt/AlphaShape/Alpha_Shapes_2D.cu:206-727).  Sizes: nedges is returned by
 * oracle_alpha_count_edges; spectrum capacity 1 + ntri + nedges. */
int oracle_alpha_count_edges(int ntri, const int *vtx, const int *nbr);

typedef struct {
    int nspec;              /* distinct spectrum values incl. the 0 sentinel */
    double *spectrum;       /* [1 + ntri + nedges] exact-then-rounded squared radii, by rank */
    double *spectrum_ref;   /* same ranks, value of the reference's FP64 formula (predicates.h:1297-1357) */
    int *tri_ro;            /* [ntri] */
    int *edge;              /* [nedges * 7]: p1, p2, ro, nu_min, nu_max, tIndex, vOpp */
    int *point;             /* [npts * 2]: nu_min, nu_max */
    long long exact_compares;
    long long exact_ties;
} oracle_alpha_out;

int oracle_alpha(int npts, const double *xy, int ntri, const int *vtx, const int *nbr,
                 oracle_alpha_out *out);

/* Exact comparison of two birth times: kind 3 = triangle (a,b,c), kind 2 = edge (a,b).
 * Returns sign(rho1 - rho2), or ORACLE_ERR_EXACT on overflow of the scratch. */
int oracle_compare_rho(int kind1, const double *p1, int kind2, const double *p2);
/* Exact attached test: 1 if k lies in the closed diametral disc of (i, j). */
int oracle_is_attached(const double *i, const double *j, const double *k);
/* Exact-then-rounded squared radius of a triangle (kind 3) or half-edge (kind 2). */
double oracle_rho_rounded(int kind, const double *p);

#ifdef __cplusplus
}
#endif
#endif
