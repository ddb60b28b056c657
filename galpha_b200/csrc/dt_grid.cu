// dt_grid.cu -- discrete Voronoi diagram and its dual triangles.
//
// Stage map (reference -> here):
//   computeScalingFactors (gpudt.cpp:722-769)      grid_scaling: power-of-two aligned
//                                                  scale/shift so every snapped
//                                                  coordinate shift + g*scale is exact
//   fake boundary circle (gpudt.cpp:810-832) and   fake ring: sites every <= 16 pixels on
//   gpudtFixConvexHull (gpudt.cpp:349-647)          the texture border, inside the texture,
//                                                  so the dual is closed by construction
//                                                  and no host hull walk is needed
//   kernelMapping / kernelMapPointsToTexture       SetupSites: snap, scatter the
//   (cudaMain.cu:160-176, kernelVoronoi.h:56-74)    lowest index into an id map and a
//                                                  column-major occupancy bitmap
//   PBA phase 1 (pba2DKernel.h:90-206)             k_column_pass: nearest site per
//                                                  column from 64-bit band masks
//   PBA phases 2+3 + transposes                    k_row_pass: one CTA per row builds the
//   (pba2DKernel.h:48-88, 209-478)                  lower envelope of the column candidates
//                                                  in shared memory (exact integer
//                                                  dominance) and colours the row
//   cudaIslandDetection (cudaVoronoi.cu:220-307,   k_island_*: isolated pixels, iterated
//   kernelVoronoi.h:82-191)                         on a work list, recoloured on device
//   kernelFindRealVoronoiVertices + kernelFlood1D  k_emit_*: 2x2 windows with 3-4 colours
//   + kernelCountRow/GenerateTriangles               give 1-2 counterclockwise triangles,
//   (kernelVoronoi.h:196-270,                        written in window order through a
//    cudaReconstruction.cu:134-208)                  tile-count scan (no host prefix sum)
#include <cstdio>
#include <cmath>
#include <algorithm>
#include "internal.cuh"
#include "exact.cuh"

namespace galpha {

// ---------------------------------------------------------------- scaling
// scale and shift are multiples of u = 2^e with scale/u < 2^37 and
// |coordinate|/u < 2^51, so shift + g*scale is exact for |g| < 2^15.
void grid_scaling(double minX, double minY, double maxX, double maxY, int T, double &scale,
                         double &sx, double &sy)
{
    int D = T - 2 * kMargin;  // usable pixels [kMargin, T-1-kMargin]
    double range = std::max(maxX - minX, maxY - minY);
    if (!(range > 0.0)) range = std::max(1.0, std::fabs(minX) + std::fabs(minY));
    double scale0 = range / (D - 2);
    double maxabs = std::max(std::max(std::fabs(minX), std::fabs(minY)), std::max(std::fabs(maxX), std::fabs(maxY)));
    int es = std::ilogb(scale0) - 36;
    int eb = maxabs > 0.0 ? std::ilogb(maxabs) - 50 : es;
    int e = std::max(es, eb);
    double u = std::ldexp(1.0, e);
    scale = std::ceil(scale0 / u) * u;
    sx = std::floor(minX / u) * u;
    sy = std::floor(minY / u) * u;
}

struct RingPix {
    int T, nside;
    __host__ __device__ short2 operator()(int k) const
    {
        int side = k / nside, i = k % nside;
        int off = (int)(((long long)i * (T - 1)) / nside);
        switch (side) {
        case 0: return make_short2((short)off, 0);
        case 1: return make_short2((short)(T - 1), (short)off);
        case 2: return make_short2((short)(T - 1 - off), (short)(T - 1));
        default: return make_short2(0, (short)(T - 1 - off));
        }
    }
};

// Pixel of input point v inside the margin (the snap SetupSites makes).
__device__ __forceinline__ void snap_pixel(double x, double y, double sx, double sy, double scale, int D, int *ix,
                                           int *iy)
{
    const double gx = floor((x - sx) / scale), gy = floor((y - sy) / scale);
    *ix = (int)fmin(fmax(gx, 0.0), (double)(D - 1));
    *iy = (int)fmin(fmax(gy, 0.0), (double)(D - 1));
}

__device__ __forceinline__ unsigned spread_bits14(unsigned v)
{
    v &= 0x3fffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Morton code of each input point's pixel, with its input index as payload.
// Sorted stably, it numbers the vertices so that neighbours in the plane
// have nearby ids (their positions, states and incidence share cache lines),
// and points that share a pixel keep their input order, so the lowest input
// index still owns the pixel.
struct SpatialKeys {
    const double *xy;
    unsigned *keys;
    int *vals;
    double scale, sx, sy;
    int D;
    __device__ void operator()(long long i) const
    {
        int ix, iy;
        snap_pixel(xy[2 * i], xy[2 * i + 1], sx, sy, scale, D, &ix, &iy);
        keys[i] = spread_bits14((unsigned)ix) | (spread_bits14((unsigned)iy) << 1);
        vals[i] = (int)i;
    }
};

struct SetupSites {
    const double *xy;
    const int *perm;  // internal vertex -> input index (nullptr: identity)
    double2 *opos, *pos;
    short2 *gpix;
    int *idmap;
    uint32_t *occ, *bandocc;
    int8_t *vstate;
    int *vtri, *vround, *anchor;
    int N, F, T, logT, W2;
    double scale, sx, sy, minX, minY, maxX, maxY;
    RingPix ring;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        double2 o, p;
        int px, py;
        if (v < N) {
            const int src = perm ? perm[v] : v;
            o = make_double2(xy[2 * src], xy[2 * src + 1]);
            if (!(o.x >= minX && o.x <= maxX && o.y >= minY && o.y <= maxY)) set_err(ct, GPUDT_ERR_ARG, src);
            int D = T - 2 * kMargin;
            int ix, iy;
            snap_pixel(o.x, o.y, sx, sy, scale, D, &ix, &iy);
            p = make_double2(sx + ix * scale, sy + iy * scale);
            px = ix + kMargin;
            py = iy + kMargin;
            vstate[v] = VS_UNDECIDED;
        } else {
            short2 q = ring(v - N);
            px = q.x;
            py = q.y;
            p = make_double2(sx + (px - kMargin) * scale, sy + (py - kMargin) * scale);
            o = p;
            vstate[v] = VS_FAKE;
        }
        opos[v] = o;
        pos[v] = p;
        gpix[v] = make_short2((short)px, (short)py);
        vtri[v] = -1;
        vround[v] = v < N ? 0 : 1;  // fake ring sites never move: decided before the first priority round (id 2)
        anchor[v] = -1;
        size_t pix = ((size_t)py << logT) + px;
        idmap[pix] = v;
        atomicOr(&occ[(size_t)px * (T >> 5) + (py >> 5)], 1u << (py & 31));
        atomicOr(&bandocc[(size_t)px * W2 + (py >> 11)], 1u << ((py >> 6) & 31));
    }
};

struct MinId {
    const short2 *gpix;
    int *idmap;
    int logT;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        short2 g = gpix[v];
        int *slot = &idmap[((size_t)g.y << logT) + g.x];
        if (*slot > v) atomicMin(slot, v);
    }
};

struct ClassifySites {
    const short2 *gpix;
    const int *idmap;
    int8_t *vstate;
    int *anchor;
    int logT;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        short2 g = gpix[v];
        int w = idmap[((size_t)g.y << logT) + g.x];
        if (w != v) {
            vstate[v] = VS_MISSING;
            anchor[v] = w;
        }
    }
};

// ----------------------------------------------------------------- islands
// A pixel is isolated when none of the (up to three) neighbours in the
// direction of its site carries its colour (kernelVoronoi.h:133-191).
__device__ __forceinline__ bool isolated(const int *colour, const short2 *gpix, int T, int logT, int x, int y)
{
    int c = colour[((size_t)y << logT) + x];
    if (c < 0) return false;
    short2 s = gpix[c];
    int dx = (s.x > x) - (s.x < x), dy = (s.y > y) - (s.y < y);
    if (dx == 0 && dy == 0) return false;
    if (dx != 0 && colour[((size_t)y << logT) + x + dx] == c) return false;
    if (dy != 0) {
        if (colour[((size_t)(y + dy) << logT) + x] == c) return false;
        if (dx != 0 && colour[((size_t)(y + dy) << logT) + x + dx] == c) return false;
    }
    return true;
}

// Pixel indices of the island lists are cell-major over a stack of T x T
// cells: p = (cell << 2 logT) + (y << logT) + x (cell 0 for a single texture).
struct IslandDetectAll {
    const int *colour;
    const short2 *gpix;
    int *list;
    Counters *ct;
    int T, logT, cap;
    const int *cellmap;  // launch cell -> texture cell (nullptr: identity)
    __device__ void operator()(long long i) const
    {
        const int z = (int)(i >> (2 * logT));
        const long long local = i & (((long long)1 << (2 * logT)) - 1);
        const long long cell = cellmap ? cellmap[z] : z;
        int x = (int)(local & (T - 1)), y = (int)(local >> logT);
        if (isolated(colour + (cell << (2 * logT)), gpix, T, logT, x, y)) {
            int k = atomicAdd(&ct->nlist, 1);
            if (k < cap) list[k] = (int)((cell << (2 * logT)) + local);
            else set_err(ct, GPUDT_ERR_NOMEM, 1);
        }
    }
};

struct IslandMark {
    int *colour;
    const int *list;
    int from;
    __device__ void operator()(long long i) const { colour[list[from + i]] = -1; }
};

// Neighbours of newly marked pixels may now be isolated.
struct IslandDetectNear {
    const int *colour;
    const short2 *gpix;
    int *list;
    Counters *ct;
    int T, logT, from, cap;
    __device__ void operator()(long long i) const
    {
        int p = list[from + i];
        const int cell = p >> (2 * logT), local = p & ((1 << (2 * logT)) - 1);
        const int *col = colour + ((size_t)cell << (2 * logT));
        int x = local & (T - 1), y = local >> logT;
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int xx = x + dx, yy = y + dy;
                if ((dx == 0 && dy == 0) || xx < 0 || yy < 0 || xx >= T || yy >= T) continue;
                if (isolated(col, gpix, T, logT, xx, yy)) {
                    // a pixel next to several new islands is listed once per
                    // neighbour; the set (not the multiplicity) is what matters
                    int q = (cell << (2 * logT)) + (yy << logT) + xx;
                    int k = atomicAdd(&ct->nlist, 1);
                    if (k < cap) list[k] = q;
                    else set_err(ct, GPUDT_ERR_NOMEM, 2);
                }
            }
    }
};

// Recolour: an unassigned pixel takes, among its assigned 8-neighbours, the
// colour whose site is nearest to it (ties: lower id).  Jacobi rounds.
struct IslandPropose {
    const int *colour;
    const short2 *gpix;
    const int *list;
    int *cand;
    Counters *ct;
    int T, logT;
    __device__ void operator()(long long i) const
    {
        int p = list[i];
        if (colour[p] >= 0) {
            cand[i] = colour[p];
            return;
        }
        const int cell = p >> (2 * logT), local = p & ((1 << (2 * logT)) - 1);
        const int *col = colour + ((size_t)cell << (2 * logT));
        int x = local & (T - 1), y = local >> logT;
        long long best = -1;
        int bestc = -1;
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int xx = x + dx, yy = y + dy;
                if ((dx == 0 && dy == 0) || xx < 0 || yy < 0 || xx >= T || yy >= T) continue;
                int c = col[((size_t)yy << logT) + xx];
                if (c < 0) continue;
                short2 s = gpix[c];
                long long d = (long long)(s.x - x) * (s.x - x) + (long long)(s.y - y) * (s.y - y);
                if (bestc < 0 || d < best || (d == best && c < bestc)) {
                    best = d;
                    bestc = c;
                }
            }
        cand[i] = bestc;
        if (bestc < 0) atomicAdd(&ct->changed, 1);
    }
};

struct IslandApply {
    int *colour;
    const int *list;
    const int *cand;
    __device__ void operator()(long long i) const { colour[list[i]] = cand[i]; }
};

// ------------------------------------------------- degenerate input check
// An input with fewer than 3 distinct points, or with all points collinear,
// has no triangle; the pipeline is skipped for it.
constexpr int kPrecheckPrefix = 1024;

// The first kPrecheckPrefix points in one block, with no shared-address
// traffic: the smallest index of a point distinct from point 0 into *first
// (left alone when there is none) and ct->changed = 1 when one of them is
// off the line through point 0 and that point. This decides general input;
// the grid-wide scans below then return at once.
__global__ void __launch_bounds__(kPrecheckPrefix) k_precheck_prefix(const double *xy, int n, int *first, Counters *ct)
{
    __shared__ int wmin[kPrecheckPrefix / 32];
    __shared__ int jsh;
    const int i = threadIdx.x, lane = i & 31, w = i >> 5;
    const bool in = i < n;
    const double x0 = xy[0], y0 = xy[1];
    double xi = x0, yi = y0;
    if (in) {
        xi = xy[2 * i];
        yi = xy[2 * i + 1];
    }
    const int cand = __reduce_min_sync(0xffffffffu, (xi != x0 || yi != y0) ? i : 0x7fffffff);
    if (lane == 0) wmin[w] = cand;
    __syncthreads();
    if (w == 0) {
        const int v = __reduce_min_sync(0xffffffffu, lane < kPrecheckPrefix / 32 ? wmin[lane] : 0x7fffffff);
        if (lane == 0) jsh = v;
    }
    __syncthreads();
    const int j = jsh;
    if (j == 0x7fffffff) return;  // the prefix is all point 0: the grid scans decide
    if (i == 0) *first = j;
    int s = 0;
    if (in) {
        const double xj = xy[2 * j], yj = xy[2 * j + 1];
        s = orient2d_filter(x0, y0, xj, yj, xi, yi);
        if (s == 2) s = orient2d_exact(x0, y0, xj, yj, xi, yi);
    }
    if (__syncthreads_or(s != 0) && i == 0) ct->changed = 1;
}

// The smallest index of a point distinct from point 0 into *first, over all
// points, when the prefix found none (*first still above every index). One
// atomic per point below the smallest index found so far (a plain read
// filters the rest).
__global__ void __launch_bounds__(256) k_first_distinct(const double *xy, long long n, int *first)
{
    if (*first < n) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if ((xy[2 * i] != xy[0] || xy[2 * i + 1] != xy[1]) && (int)i < *(volatile int *)first) atomicMin(first, (int)i);
}

// ct->changed = 1 when some point is off the line through point 0 and point
// *first, over all points, when the prefix found none (*first >= n: every
// point equals point 0 and nothing is off the line).
__global__ void __launch_bounds__(256) k_count_off_line(const double *xy, const int *first, long long n, Counters *ct)
{
    if (ct->changed) return;
    const int j = *first;
    if (j >= n) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int s = orient2d_filter(xy[0], xy[1], xy[2 * j], xy[2 * j + 1], xy[2 * i], xy[2 * i + 1]);
        if (s == 2) s = orient2d_exact(xy[0], xy[1], xy[2 * j], xy[2 * j + 1], xy[2 * i], xy[2 * i + 1]);
        if (s != 0 && *(volatile int *)&ct->changed == 0) ct->changed = 1;
    }
}

// Returns 1 when the input has at least one triangle.
int has_triangles(Ctx &c, const double *d_xy, int n)
{
    if (n < 3) return 0;
    int *first = c.aux;
    GALPHA_CUDA(cudaMemsetAsync(first, 0x7f, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    k_precheck_prefix<<<1, kPrecheckPrefix, 0, c.stream>>>(d_xy, n, first, c.ctr);
    count_launch();
    long long blocks = ((long long)n + 255) / 256;
    if (blocks > (long long)c.sm_count * 8) blocks = (long long)c.sm_count * 8;
    k_first_distinct<<<(unsigned)blocks, 256, 0, c.stream>>>(d_xy, n, first);
    count_launch();
    // the line through point 0 and the first point distinct from it (none:
    // `first` stays above every index and no point counts), one host read
    k_count_off_line<<<(unsigned)blocks, 256, 0, c.stream>>>(d_xy, first, n, c.ctr);
    count_launch();
    int r = read_counters(c);
    if (r) return r;
    return c.hctr->changed > 0 ? 1 : 0;
}

// Occupied 64 x 64 blocks of each cell, counted away from the ring of fake
// sites (interior blocks only) from the per-column band bitmaps.
struct CellOccupancy {
    const uint32_t *bandocc;
    int T, W2, nb;  // nb = T / 64 blocks per side
    int *count;     // [cells]
    __device__ void operator()(long long i) const
    {
        const int inner = nb - 2;
        const int z = (int)(i / ((long long)inner * inner));
        const int rem = (int)(i - (long long)z * inner * inner);
        const int bx = 1 + rem / inner, by = 1 + rem % inner;
        const uint32_t *b = bandocc + (size_t)z * T * W2;
        uint32_t any = 0;
        for (int x = 64 * bx; x < 64 * bx + 64; x++) any |= b[(size_t)x * W2 + (by >> 5)];
        if ((any >> (by & 31)) & 1u) atomicAdd(&count[z], 1);
    }
};

// Interior-block occupancy of `cells` stacked T x T cells into host[cells]
// (dev: cells ints of device scratch).
int cell_occupancy(Ctx &c, const uint32_t *bandocc, int T, int W2, int cells, int *dev, int *host)
{
    const int nb = T / 64;
    for (int z = 0; z < cells; z++) host[z] = 0;
    if (nb <= 2) return GPUDT_OK;
    GALPHA_CUDA(cudaMemsetAsync(dev, 0, sizeof(int) * (size_t)cells, c.stream));
    launch_n(c, CellOccupancy{bandocc, T, W2, nb, dev}, (long long)cells * (nb - 2) * (nb - 2));
    return read_small(c, host, dev, sizeof(int) * (size_t)cells);
}

// The fused path pays a window scan as long as the distance to the nearest
// site, so it is used only when at least 60 % of the interior 64 x 64 blocks
// hold a site.
bool occupancy_ok(int T, int occupied)
{
    const int nb = T / 64;
    return nb <= 2 || occupied >= 0.6 * (nb - 2) * (nb - 2);
}

// ------------------------------------------------------------------ stages
int stage_setup(Ctx &c, const double *d_xy, int n, double minX, double minY, double maxX, double maxY, int T)
{
    c.N = n;
    c.T = T;
    c.logT = 0;
    while ((1 << c.logT) < T) c.logT++;
    int nside = (T - 1 + kFakeSpacing - 1) / kFakeSpacing;
    c.F = 4 * nside;
    c.V = c.N + c.F;
    grid_scaling(minX, minY, maxX, maxY, T, c.scale, c.shiftX, c.shiftY);
    int W2 = ((T >> 6) + 31) / 32;
    GALPHA_CUDA(cudaMemsetAsync(c.occ, 0, sizeof(uint32_t) * (size_t)T * (T >> 5), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.bandocc, 0, sizeof(uint32_t) * (size_t)T * W2, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.ctr, 0, sizeof(Counters), c.stream));
    // spatial numbering of the input points (stable radix sort of pixel Morton codes)
    c.renumbered = n > 1;
    if (c.renumbered) {
        unsigned *k1 = (unsigned *)c.keys, *k2 = (unsigned *)c.keys2;
        launch_n(c, SpatialKeys{d_xy, k1, c.perm, c.scale, c.shiftX, c.shiftY, T - 2 * kMargin}, n);
        // pixel coordinates below T: Morton codes of 2 logT bits
        int r = radix_sort32(c, k1, c.perm, k2, c.vals2, n, c.rhist, 2 * c.logT);
        if (r) return r;
    }
    SetupSites s;
    s.xy = d_xy;
    s.perm = c.renumbered ? c.perm : nullptr;
    s.opos = c.opos;
    s.pos = c.pos;
    s.gpix = c.gpix;
    s.idmap = c.idmap;
    s.occ = c.occ;
    s.bandocc = c.bandocc;
    s.vstate = c.vstate;
    s.vtri = c.vtri;
    s.vround = c.vround;
    s.anchor = c.anchor;
    s.N = c.N;
    s.F = c.F;
    s.T = T;
    s.logT = c.logT;
    s.W2 = W2;
    s.scale = c.scale;
    s.sx = c.shiftX;
    s.sy = c.shiftY;
    s.minX = minX;
    s.minY = minY;
    s.maxX = maxX;
    s.maxY = maxY;
    s.ring = RingPix{T, nside};
    s.ct = c.ctr;
    launch_n(c, s, c.V);
    launch_n(c, MinId{c.gpix, c.idmap, c.logT}, c.N);
    launch_n(c, ClassifySites{c.gpix, c.idmap, c.vstate, c.anchor, c.logT}, c.N);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int stage_voronoi(Ctx &c)
{
    const int T = c.T;
    int W2 = ((T >> 6) + 31) / 32;
    int r0 = launch_column_pass(c, W2);
    if (r0) return r0;
    // Fused path: colours stay in shared memory and the dual triangles are
    // emitted directly.  Sparse inputs (mean site spacing above 16 pixels)
    // make the per-pixel window scan long, so they take the envelope path.
    c.fused_done = false;
    long long D = T - 2 * kMargin;
    int occupied = 0;
    r0 = cell_occupancy(c, c.bandocc, T, W2, 1, c.aux, &occupied);
    if (r0) return r0;
    if ((long long)c.N * 256 >= D * D && occupancy_ok(T, occupied)) {
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->ntris, 0, sizeof(int), c.stream));
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nisland, 0, sizeof(int), c.stream));
        r0 = launch_vd_tri(c);
        if (r0) return r0;
        r0 = read_counters(c);
        if (r0) return r0;
        if (c.hctr->err) return c.hctr->err;
        int nflag = c.hctr->nisland;
        c.st.nRepairTiles = nflag;
        bool local_ok = true;
        if (nflag > 0) {
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->escalate, 0, sizeof(int), c.stream));
            r0 = launch_vd_repair(c, nflag);
            if (r0) return r0;
            r0 = read_counters(c);
            if (r0) return r0;
            if (c.hctr->err) return c.hctr->err;
            local_ok = c.hctr->escalate == 0;
        }
        if (local_ok) {
            c.fused_done = true;
            return GPUDT_OK;
        }
        // an island component too large for a local repair: global path
        c.st.nEscalated = 1;
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->ntris, 0, 2 * sizeof(int), c.stream));  // ntris, nfree
    }
    c.st.nEnvelopeCells = 1;
    return voronoi_global(c, 1, nullptr);
}

// Envelope colouring of `cells` textures of size c.T x c.T (cell cellmap[z],
// or z, of the stack at c.ycol / c.idmap / c.colour), then the global island
// repair over all of them.
int voronoi_global(Ctx &c, int cells, const int *cellmap)
{
    const int T = c.T;
    int r0 = launch_row_pass_cells(c, cells, cellmap);
    if (r0) return r0;
    GALPHA_CUDA(cudaGetLastError());
    // islands
    long long npix = (long long)T * T * cells;
    int cap = (int)std::min<long long>(npix, (long long)c.cap_tris * 3);
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
    launch_n(c, IslandDetectAll{c.colour, c.gpix, c.list, c.ctr, T, c.logT, cap, cellmap}, npix);
    int r = read_counters(c);
    if (r) return r;
    int total = c.hctr->nlist;
    c.st.nIslandPixels += total;
    if (total == 0) return GPUDT_OK;
    // iterate detection around newly marked pixels
    int from = 0, to = total, guard = 0;
    while (from < to) {
        if (to > cap) return GPUDT_ERR_NOMEM;
        launch_n(c, IslandMark{c.colour, c.list, from}, to - from);
        launch_n(c, IslandDetectNear{c.colour, c.gpix, c.list, c.ctr, T, c.logT, from, cap}, to - from);
        r = read_counters(c);
        if (r) return r;
        from = to;
        to = c.hctr->nlist;
        if (++guard > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
    }
    total = to;
    // recolour
    guard = 0;
    while (true) {
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
        launch_n(c, IslandPropose{c.colour, c.gpix, c.list, c.list2, c.ctr, T, c.logT}, total);
        launch_n(c, IslandApply{c.colour, c.list, c.list2}, total);
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->changed == 0) break;
        if (++guard > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
    }
    return GPUDT_OK;
}

// Dual triangles of the coloured cells appended at slot `base`
// (c.ctr->ntris = base + count).
int emit_global(Ctx &c, int base, int cells, const int *cellmap)
{
    const int T = c.T;
    long long nwin = (long long)(T - 1) * (T - 1);
    int ntiles = (int)((nwin + kEmitTile - 1) / kEmitTile);
    int r0 = launch_emit_cells(c, ntiles, nwin, false, nullptr, cells, cellmap);
    if (r0) return r0;
    int r = exclusive_scan_int(c, c.tilecount, c.tilecount, ntiles * cells, &c.ctr->nlist2);
    if (r) return r;
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return c.hctr->err;
    const int total = c.hctr->nlist2;
    if ((long long)base + total > c.cap_tris) return GPUDT_ERR_NOMEM;
    r = launch_emit_cells(c, ntiles, nwin, true, c.tv + base, cells, cellmap);
    if (r) return r;
    launch_n(c, SetInt{&c.ctr->ntris, base + total}, 1);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int stage_triangles(Ctx &c)
{
    if (c.fused_done) return GPUDT_OK;  // emitted by the fused kernel
    return emit_global(c, 0, 1, nullptr);
}

}  // namespace galpha
