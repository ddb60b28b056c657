// internal.cuh -- device context, buffers and launch helpers of galpha-b200.
//
// One handle owns one CUDA stream and one set of device buffers, grown on
// demand and reused across calls, so repeated calls allocate nothing.  All
// kernels of the pipeline are launched on that stream; the few host decisions
// between stages read a small pinned counter block.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include <stdint.h>
#include <stddef.h>
#include "../../include/gpudt.h"
#include "../../include/galpha.h"

#ifndef GALPHA_HD
#define GALPHA_HD __host__ __device__ __forceinline__
#endif

namespace galpha {

// ------------------------------------------------------------- constants
constexpr int kFakeSpacing = 16;                 // fake ring site every <= 16 pixels
constexpr int kMargin = kFakeSpacing / 2 + 1;    // real sites stay >= 9 pixels from the border
constexpr int kMaxFan = 64;                      // star holes / fans handled per thread
constexpr int kMaxRounds = 100000;               // cap of every iterative stage (default)
constexpr int kSpinLimit = 1 << 22;              // bound of every look-back wait (default)
constexpr int kBlockRun = 1 << 16;
constexpr int kShiftGroupDefault = 4, kMissingGroupDefault = 2, kFlipSyncDefault = 4;
constexpr int kTailEnterDefault = 4096, kTailLeaveDefault = 32768;
constexpr int kMaxGroup = 8;  // Counters::grp holds one group's per-round counts               // longest exact-sort run for one block (default)

// vertex states
enum : int8_t {
    VS_UNDECIDED = 0,  // present in the texture, not yet shifted
    VS_SHIFTED = 1,    // in the mesh at its true coordinates
    VS_BAD = 2,        // cannot be shifted: to be removed and re-inserted
    VS_MISSING = 3,    // not in the mesh, to be inserted by point location
    VS_FAKE = 4,       // fake ring site in the mesh
    VS_DUP = 5,        // exact duplicate of a lower index: dropped
    VS_GONE = 6,       // fake ring site removed
};

// Device counter block (one per handle, mapped to host through a pinned copy).
struct Counters {
    int ntris;      // triangle slots in use (tail of the slot array)
    int nfree;      // entries of the free-slot stack
    int nlist;      // generic work-list length
    int nlist2;     // second work list
    int nrec;       // relink records this round
    int changed;    // generic progress flag / count
    int err;        // first error code (GPUDT_ERR_*), 0 if none
    int errinfo;    // stage-specific detail of the first error
    int nisland;    // island pixels
    int nflips;     // flips this round
    int nties;      // exact spectrum ties merged
    int act[2];     // flip: active-list lengths (ping-pong)
    int cand;       // flip: candidates this round
    int flips_total;
    int escalate;   // island repair could not stay local: redo the Voronoi stage globally
    unsigned long long exact_compares;
    unsigned long long exact_orient;
    unsigned long long exact_incircle;
    unsigned long long exact_attached;
    // predicate stage counts, each spread over 64 counters (one per warp id mod 64)
    unsigned long long filt_spread[64];  // in-circle tests decided by the FP64 filter
    unsigned long long icc_spread[64];   // in-circle tests, all stages
    unsigned long long ori_spread[64];   // orientation tests of the mesh stages, all stages
    unsigned long long ori64_spread[64]; // orientation tests decided by the FP64 filter
    int qcount[12];  // alpha query: [type*4 + class], type 0 points, 1 edges, 2 triangles
    int qrank;       // alpha query: largest spectrum rank <= alpha (-1 if alpha < 0)
    int qpad;
    double qalpha;   // alpha query: the alpha value classified
    int tail_rounds; // flip: rounds run by the last in-block tail launch
    int runstage;    // fake runs: staged fan entries
    int nlong;       // key sort: out-of-order pairs recorded in groups too long for one thread
    int nhuge;       // alpha ranks: runs too long for one block, listed for the multi-block merge
    int sh_n[2];     // shift: sites dropped by the current / previous optimistic iteration
    int sh_total;    // shift: all dropped sites listed so far
    int grp[8];      // per-round counts of a group of rounds run between two counter reads
    int ndup;        // missing sites found to be exact duplicates
};

// Relink record: an edge of a triangle created this round (loc = (t<<2)|i, or -1
// when the edge became a hull edge) and the encoded outer neighbour it had
// before the round (old = (u<<2)|j, or -1).
struct Relink {
    int loc;
    int old;
};

// A grown-on-demand device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    long long budget = 0;
    long long reserved = 0;
    int sm_count = 148;

    // problem
    int N = 0, F = 0, V = 0, T = 0, logT = 0;
    double scale = 1, shiftX = 0, shiftY = 0;
    int cap_tris = 0;

    // device arrays (pointers into bufs)
    double2 *opos = nullptr;   // [V] true coordinates
    double2 *pos = nullptr;    // [V] current coordinates
    short2 *gpix = nullptr;    // [V] texture pixel of each site
    int *idmap = nullptr;      // [T*T] site id of each occupied pixel (lowest index)
    uint32_t *occ = nullptr;   // [T * T/32] column-major occupancy bits
    uint32_t *bandocc = nullptr;  // [T * W2] per-column 64-row band occupancy
    int16_t *ycol = nullptr;   // [T*T] row of the nearest site in the pixel's column
    int *colour = nullptr;     // [T*T] discrete Voronoi diagram (site id per pixel)
    int *list = nullptr;       // [max(T*T/?, V, cap)] work list
    int *list2 = nullptr;
    int *aux = nullptr;        // [cap] generic int scratch
    int *aux2 = nullptr;
    int4 *tv = nullptr;        // [cap] triangle vertices (x,y,z; w = flags)
    int4 *tn = nullptr;        // [cap] triangle neighbours (x,y,z; w unused)
    int4 *fwd = nullptr;       // [cap] forwarding of consumed triangles' edges
    int *epoch = nullptr;      // [cap] round that consumed the slot
    int *vote = nullptr;       // [cap]
    int *stamp = nullptr;      // [cap]
    int4 *cv = nullptr;        // [cap] compacted triangle vertices
    int4 *cn = nullptr;        // [cap] compacted triangle neighbours
    int *freelist = nullptr;   // [cap]
    Relink *rec = nullptr;     // [3*cap]
    int *vtri = nullptr;       // [V] one incident oriented triangle
    int8_t *eflag = nullptr;   // [cap] flip: edges of a triangle still to be tested (bit i: edge opposite vtx[i])
    int *perm = nullptr;       // [V] single-set path: internal (spatially sorted) vertex -> input index
    bool renumbered = false;   // the mesh stages ran on spatially sorted ids (perm); outputs use input ids
    int8_t *vstate = nullptr;  // [V]
    int *vround = nullptr;     // [V]
    int *anchor = nullptr;     // [V]
    int *deg = nullptr;        // [V+1]
    int *inc = nullptr;        // [3*cap]
    int *tilecount = nullptr;  // [ntiles + 1]
    Counters *ctr = nullptr;   // device counters
    Counters *hctr = nullptr;  // pinned, device-mapped host mirror of ctr (written by a kernel)
    Counters *hctr_dev = nullptr;  // the device address of hctr
    char *hmail = nullptr, *hmail_dev = nullptr;  // mapped mailbox for other small reads

    // alpha arrays
    int nT_out = 0, nE = 0, nSpecIn = 0, nSpec = 0;
    int *e_off = nullptr;      // [nT+1] first edge of each triangle
    int4 *edges = nullptr;     // [nE] p1, p2, tIndex | vOpp<<30? (see alpha.cu)
    int *edge_ro = nullptr;    // [nE]
    int2 *edge_nu = nullptr;   // [nE]
    int *tri_ro = nullptr;     // [nT]
    int2 *pt_nu = nullptr;     // [N]
    unsigned long long *keys = nullptr, *keys2 = nullptr;  // [nSpecIn]
    int *vals = nullptr, *vals2 = nullptr;                 // [nSpecIn]
    int *rank = nullptr;       // [nSpecIn]
    double *spectrum = nullptr;  // [nSpecIn + 1]
    uint8_t *qclass = nullptr;   // alpha query classes: points [V], edges [2 cap], triangles [cap]
    // master list (own allocation, made on first use)
    char *ml_buf = nullptr;
    size_t ml_bytes = 0;
    galphaAlpha *ml_out = nullptr;  // [nMaster]
    int *ml_sp = nullptr;           // [nSpecPtr]
    int nMaster = 0, nSpecPtr = 0;
    bool have_master = false;
    int *hist = nullptr;       // scan scratch
    int *rhist = nullptr;      // radix sort histograms
    long long rhist_ints = 0;  // its size
    gpudtTriangle *outtri = nullptr;  // [cap] AoS output staging
    bool outtri_ready = false;          // outtri holds the current mesh (built on the first download)
    bool want_outtri = false;           // this call needs outtri: compaction writes it directly
    galphaEdgeInterval *edge_aos = nullptr;  // [2*cap] edge records for download

    DevBuf bufs[64];
    int nbufs = 0;

    // events for stage timing
    cudaEvent_t ev[GALPHA_STAGE_TOTAL + 2];
    int reads_at[GALPHA_STAGE_TOTAL + 2] = {};  // host_reads when event k was recorded
    cudaEvent_t kev[10];  // [2k, 2k+1] bracket single kernel k (see gpudtStatus.kernelMs)
    bool kev_rec[10];     // recorded during the current call
    bool events = false;
    gpudtStatus st;
    bool have_mesh = false, have_alpha = false;
    int sort_passes = 0;  // radix passes of the last radix_sort call
    bool fused_done = false;  // triangles came from the fused colour + dual kernel
    int round_counter = 1;    // ids of operation rounds (per handle: stamps live in its arena)
    int host_reads = 0;       // device -> host reads (each a stream synchronisation) of the current call

    // constrained edges of the current call (GPUDTPARAMS.nConstraints > 0)
    int n_cons = 0;
    const int *h_cons = nullptr;       // host pairs of input indices
    char *cons_buf = nullptr;          // own allocation: constraint state + hash set
    size_t cons_bytes = 0;
    int *cons_pool = nullptr;          // own allocation: per-round walk records
    long long cons_pool_ints = 0;
    const unsigned long long *chash = nullptr;  // set of constrained vertex pairs (internal ids), or null
    unsigned cmask = 0;                // its size - 1 (a power of two)
    int cons_rounds = 0;               // insertion rounds of the last call

    // failure-detection limits (galphaSetLimits): the round cap of every
    // iterative stage, the spin bound of the single-pass look-back waits, and
    // a test switch under which tile 0 of each look-back kernel withholds its
    // status so that the next tile's bounded wait runs out
    int max_rounds = kMaxRounds;
    int spin_limit = kSpinLimit;
    int hold_first = 0;
    // runs of near-equal spectrum keys longer than this are merge-sorted with
    // the exact comparator by many blocks (one launch per merge level)
    // instead of by one block
    int block_run = kBlockRun;
    // loop schedule (galphaSetSchedule): rounds per counter read of the
    // shifting and missing-site loops and of the flip stage, and the active
    // list lengths at which the flip stage hands its rounds to one block and
    // takes them back.  None of them changes a result.
    int shift_group = kShiftGroupDefault;
    int missing_group = kMissingGroupDefault;
    int flip_sync = kFlipSyncDefault;
    int tail_enter = kTailEnterDefault;
    int tail_leave = kTailLeaveDefault;
};

// ------------------------------------------------------------- error helpers
#define GALPHA_CUDA(call)                                               \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return galpha::cuda_fail(e_, #call);     \
    } while (0)

int cuda_fail(cudaError_t e, const char *what);
const char *last_error_text();
void set_last_error(const char *text);

// Reserve device buffers for V vertices, T texture, cap triangles.
int reserve(Ctx &c, int V, int T, int cap_tris, bool alpha);
int read_counters(Ctx &c);
// Small device -> host read (bytes a multiple of 4, src 4-byte aligned): a
// kernel writes into mapped pinned memory, so the read never queues behind
// large copies on the copy engines; synchronises the handle's stream.
int read_small(Ctx &c, void *host_dst, const void *dev_src, size_t bytes);
// Records the failing stage and the device-side detail code (galphaLastError).
int stage_fail(Ctx &c, int r, const char *stage);
constexpr size_t kMailBytes = 65536;

// Limits of galphaEdgeListNoAlloc (noalloc.cu), set by galphaSetLimits(NULL, ...).
void noalloc_set_limits(int spin_limit, int hold_first);

// Kernel launches issued by this library (all handles, all threads).
extern unsigned long long g_launches;
inline void count_launch(unsigned long long k = 1) { __atomic_fetch_add(&g_launches, k, __ATOMIC_RELAXED); }

#ifdef __CUDACC__
// Grid-stride launch of a device functor over [0, n).
template <class F>
__global__ void __launch_bounds__(256) k_for_each(F f, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) f(i);
}

// The same with at least MINB resident blocks of 256 threads per SM asked of
// the register allocator (for latency-bound functors whose rare exact paths
// would otherwise set the register count of the common one).
template <class F, int MINB>
__global__ void __launch_bounds__(256, MINB) k_for_each_occ(F f, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) f(i);
}

// Grid-stride launch over [0, *n) with the count read on the device, so a
// round of kernels can run without the host learning its size.
template <class F>
__global__ void __launch_bounds__(256) k_for_each_dev(F f, const int *n)
{
    long long nn = *n;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < nn; i += stride) f(i);
}

template <class F>
inline void launch_dev(const Ctx &c, F f, const int *n_dev, long long max_n)
{
    if (max_n <= 0) return;
    long long blocks = (max_n + 255) / 256;
    long long maxb = (long long)c.sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    k_for_each_dev<<<(unsigned)blocks, 256, 0, c.stream>>>(f, n_dev);
    count_launch();
}

template <int MINB, class F>
inline void launch_occ(const Ctx &c, F f, long long n)
{
    if (n <= 0) return;
    long long blocks = (n + 255) / 256;
    long long maxb = (long long)c.sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    k_for_each_occ<F, MINB><<<(unsigned)blocks, 256, 0, c.stream>>>(f, n);
    count_launch();
}

template <class F>
inline void launch_n(const Ctx &c, F f, long long n)
{
    if (n <= 0) return;
    long long blocks = (n + 255) / 256;
    long long maxb = (long long)c.sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    k_for_each<<<(unsigned)blocks, 256, 0, c.stream>>>(f, n);
    count_launch();
}
#endif

// Element copies and single-word stores as kernels: on the handle's stream
// they never wait behind downloads that the copy engines are busy with.
template <typename T>
struct CopyElems {
    T *dst;
    const T *src;
    __device__ void operator()(long long i) const { dst[i] = src[i]; }
};

struct SetInt {
    int *p;
    int v;
    __device__ void operator()(long long) const { *p = v; }
};

// Report the first error from device code.
__device__ __forceinline__ void set_err(Counters *ct, int code, int info)
{
    if (atomicCAS(&ct->err, 0, code) == 0) ct->errinfo = info;
}

// Counts one event per calling thread with one atomic per warp.
__device__ __forceinline__ void warp_count(unsigned long long *c)
{
    unsigned m = __activemask();
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(c, (unsigned long long)__popc(m));
}

// Adds every calling thread's cnt with one atomic per warp, into one of 64
// counters chosen by warp (a single hot counter serialises on the L2 atomics).
__device__ __forceinline__ void warp_add_spread(unsigned long long *arr, int cnt)
{
    const unsigned m = __activemask();
    const int tot = __reduce_add_sync(m, cnt);
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && tot)
        atomicAdd(&arr[((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & 63], (unsigned long long)tot);
}

// Counts one event per calling lane (one atomic per converged group of lanes).
__device__ __forceinline__ void warp_count_spread(unsigned long long *arr)
{
    const unsigned m = __activemask();
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1)
        atomicAdd(&arr[((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & 63], (unsigned long long)__popc(m));
}

// Reserves cnt consecutive slots of *counter for every calling thread with one
// atomic per warp; returns the thread's first slot.  The calling lanes are a
// prefix of the warp in grid-stride loops; any other set falls back to one
// atomic per thread.
__device__ __forceinline__ int warp_reserve(int *counter, int cnt)
{
    const unsigned m = __activemask();
    if (m & (m + 1u)) return cnt ? atomicAdd(counter, cnt) : 0;
    const int lane = threadIdx.x & 31;
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(m, incl, o);
        if (lane >= o) incl += v;
    }
    const int last = 31 - __clz(m);
    const int tot = __shfl_sync(m, incl, last);
    int base = 0;
    if (lane == last && tot) base = atomicAdd(counter, tot);
    base = __shfl_sync(m, base, last);
    return base + incl - cnt;
}

// 32-bit invertible mix (murmur3 finaliser): a random-looking priority per id.
GALPHA_HD uint32_t prio(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

GALPHA_HD int enc(int t, int i) { return (t << 2) | i; }
GALPHA_HD int dtri(int e) { return e >> 2; }
GALPHA_HD int dori(int e) { return e & 3; }
GALPHA_HD int p1(int i) { return i == 2 ? 0 : i + 1; }
GALPHA_HD int m1(int i) { return i == 0 ? 2 : i - 1; }
GALPHA_HD int geti(const int4 &v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
GALPHA_HD void seti(int4 &v, int i, int x)
{
    if (i == 0) v.x = x;
    else if (i == 1) v.y = x;
    else v.z = x;
}

// Stage entry points (dt_grid.cu, dt_mesh.cu, alpha.cu)
int has_triangles(Ctx &c, const double *d_xy, int n);
int stage_setup(Ctx &c, const double *d_xy, int n, double minX, double minY, double maxX, double maxY, int T);
int stage_voronoi(Ctx &c);
int stage_triangles(Ctx &c);
int stage_links(Ctx &c);
int stage_shift(Ctx &c);
int stage_missing(Ctx &c);
int stage_boundary(Ctx &c);
int stage_flip(Ctx &c);
int stage_constraints(Ctx &c);
int stage_compact(Ctx &c);
// ------------------------------------------------------------------ batches
// One point set of a batch: its grid scaling, its texture cell and its
// vertex / fake ranges (batch.cu).
struct SetDesc {
    double scale, sx, sy, minX, minY, maxX, maxY;
    long long tex;   // first pixel of the set's cell in ycol / idmap
    long long occw;  // first word of the cell in occ
    long long band;  // first word of the cell in bandocc
    int n, vbase, fbase, nfake, nside, T, logT, W2, live;
};

struct BatchClass {   // cells of one texture size, stacked
    int T, logT, W2, cells;
    long long tex, occw, band;  // first pixel / words of the class
    int tile0;                  // first fused tile of the class
    std::vector<int> sets;      // set of each cell
};

struct BatchHost {
    std::vector<SetDesc> sets;
    std::vector<BatchClass> classes;
    std::vector<int> tbase, ebase, nd, specoff;  // per set after a run (K + 1 entries for bases)
    int K = 0, N = 0, Fmax = 0;
    long long T2 = 0, occw = 0, band = 0;
    int ntiles = 0;
    bool alpha = false, valid = false;
    double density = 10.0;  // texture pixels per point of a set (galphaSetBatchDensity)
};

struct BatchDev {
    char *buf = nullptr;
    size_t bytes = 0;
    SetDesc *sets = nullptr;
    int *vbases = nullptr, *fbases = nullptr, *vset = nullptr, *vsetall = nullptr, *first = nullptr,
        *offline = nullptr, *esc = nullptr, *tset = nullptr, *tbase = nullptr, *seg = nullptr,
        *firstexcl = nullptr, *nd = nullptr, *spec_off = nullptr, *ebase = nullptr;
    gpudtTriangle *otri = nullptr;  // [cap] set-local output triangles
    double *qparam = nullptr, *qalpha = nullptr;  // [K] per-set query values
    int *qR = nullptr, *qcounts = nullptr;        // [K], [12 K]
    int *cellmap = nullptr;                       // [K] launch cell -> cell of a class
    int2 *chunk = nullptr;                        // [fused tiles] (first slot, count) per tile
};

void grid_scaling(double minX, double minY, double maxX, double maxY, int T, double &scale, double &sx, double &sy);
// Compaction in the new order: new triangle j is slot order[j], j < nalive
// (cv / cn only).
void launch_compact_gather(Ctx &c, const int *order, const int *newidx, int nalive);
int batch_plan(BatchHost &bh, int K, const int *sizes, const double *bounds);
int fused_tiles(int T);  // tiles of the fused colouring kernel per T x T cell
// The mesh in the gpudtTriangle layout (outtri), built from cv / cn when a
// host download first needs it.
int ensure_outtri(Ctx &c);
int batch_buffers(Ctx &c, BatchDev &B, int K, int N, int V, int cap, int nspec, int ntiles);
int batch_setup(Ctx &c, BatchDev &B, BatchHost &bh, const double *d_xy);
int batch_voronoi(Ctx &c, BatchDev &B, BatchHost &bh);
int batch_compact(Ctx &c, BatchDev &B, BatchHost &bh);
int batch_local_outputs(Ctx &c, BatchDev &B, gpudtTriangle *tris, galphaEdgeInterval *edges);

// Segments of a batched alpha stage: entries are ranked per point set (set of
// a compacted triangle: tset), each set with its own rank 0 sentinel.
struct AlphaSegs {
    const int *tset;  // [nT] set of each compacted triangle
    int K;            // number of sets
    int *seg;         // [nSpecIn] scratch: set of each sorted entry
    int *firstexcl;   // [K] global rank count before the set's first entry
    int *nd;          // [K] distinct values of the set
    int *spec_off;    // [K + 1] first spectrum slot of the set (its rank 0)
    const int *tbase; // [K + 1] first compacted triangle of each set (non-decreasing; [K] = nT)
    int *ebase;       // [K + 1] scratch: first edge of each set
};
int stage_alpha(Ctx &c, AlphaSegs *segs = nullptr);
int alpha_query(Ctx &c, double alpha, double q, bool by_quantile);
int alpha_query_sets(Ctx &c, int K, const int *vset, const int *tset, const int *spec_off, const int *nd,
                     const double *param, int by_quantile, int *R, double *alpha, int *counts);
int master_list(Ctx &c);
int alpha_from_host_mesh(Ctx &c, const double *h_xy, int n, const gpudtTriangle *tris, int nt);

// Block-level kernels of the Voronoi stage (voronoi_kernels.cu)
constexpr int kEmitThreads = 256;
constexpr int kEmitTile = kEmitThreads;
int launch_column_pass(Ctx &c, int W2);
int launch_row_pass(Ctx &c);
int launch_emit(Ctx &c, int ntiles, long long nwin, bool write, int4 *tv_out);
int voronoi_global(Ctx &c, int cells, const int *cellmap);
int cell_occupancy(Ctx &c, const uint32_t *bandocc, int T, int W2, int cells, int *dev, int *host);
bool occupancy_ok(int T, int occupied);
int emit_global(Ctx &c, int base, int cells, const int *cellmap);
int launch_vd_tri(Ctx &c);
int launch_vd_repair(Ctx &c, int nflag);
int launch_vd_repair_cells(Ctx &c, int nflag, int T, int logT, int cells, const int16_t *ycol, const int *idmap,
                           int *esc_cells, const int *cellmap, const int2 *chunk);
int launch_vd_tri_cells(Ctx &c, int T, int logT, int cells, const int16_t *ycol, const int *idmap, int2 *chunk,
                        int *flagged, const int *cellmap);
int launch_row_pass_cells(Ctx &c, int cells, const int *cellmap);
int launch_emit_cells(Ctx &c, int ntiles, long long nwin, bool write, int4 *tv_out, int cells, const int *cellmap);
int launch_column_pass_cells(Ctx &c, int T, int W2, int cells, const uint32_t *occ, const uint32_t *bandocc,
                             int16_t *ycol);
// LSD radix sort of (keys, vals) ascending (sort.cu)
int radix_sort(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *keys2, int *vals2, int n,
               bool *in_second);
int radix_sort32(Ctx &c, unsigned int *keys, int *vals, unsigned int *keys2, int *vals2, int n, int *scratch,
                 int key_bits = 0);
// Stable sort by the low nbits of 32-bit set ids, moving (keys, vals) along;
// the result ends in (skey, keys, vals).
int radix_sort_set_kv(Ctx &c, unsigned *skey, unsigned *skey2, unsigned long long *keys, int *vals,
                      unsigned long long *keys2, int *vals2, int n, int nbits);
// Geometry of the compacted mesh for the alpha stage: triangles with the
// mesh stages' vertex ids (cv holds input ids, which decide edge ownership
// and index the point intervals; after a spatial numbering the internal ids
// are kept in fwd, idle once the flips are done) and the positions by those
// ids (opos).
inline const int4 *alpha_geom_tris(const Ctx &c) { return c.renumbered ? c.fwd : c.cv; }
long long radix_scratch_ints(long long n);
long long radix_sort_scratch_ints(long long n);  // radix_sort and radix_sort32 of n keys

// Prefix sums (scan.cu)
int exclusive_scan_int(Ctx &c, const int *in, int *out, int n, int *total_dev);
size_t scan_scratch_bytes(int n);

}  // namespace galpha
