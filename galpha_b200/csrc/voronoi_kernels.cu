// voronoi_kernels.cu -- block-level kernels of the discrete Voronoi stage:
// the column pass, the per-row lower envelope + colouring, and the 2x2-window
// triangle emission.  Launchers are called from dt_grid.cu.
#include <mutex>
#include "internal.cuh"

namespace galpha {

static inline void kev_record(Ctx &c, int k)
{
    if (!c.events) return;
    cudaEventRecord(c.kev[k], c.stream);
    c.kev_rec[k] = true;
}

// ------------------------------------------------------------ column pass
// Thread (x, band): ycol[y][x] = row of the nearest occupied pixel of column x
// (ties: the upper one, i.e. smaller y), -1 for an empty column.
__global__ void __launch_bounds__(256) k_column_pass(const uint32_t *__restrict__ occ,
                                                     const uint32_t *__restrict__ bandocc,
                                                     int16_t *__restrict__ ycol, int T, int W2)
{
    // blockIdx.z: texture cell of a batch (cells are stacked T x T textures)
    occ += (size_t)blockIdx.z * T * (T >> 5);
    bandocc += (size_t)blockIdx.z * T * W2;
    ycol += (size_t)blockIdx.z * T * T;
    int x = blockIdx.x * 32 + threadIdx.x;
    int b = blockIdx.y * blockDim.y + threadIdx.y;
    int nb = T >> 6;
    if (x >= T || b >= nb) return;
    const uint32_t *col = occ + (size_t)x * (T >> 5);
    const uint32_t *bo = bandocc + (size_t)x * W2;
    unsigned long long m = (unsigned long long)col[2 * b] | ((unsigned long long)col[2 * b + 1] << 32);
    // previous non-empty band
    int yabove = -1, ybelow = -1;
    {
        int w = b >> 5;
        uint32_t bits = bo[w] & ((b & 31) ? (0xffffffffu >> (32 - (b & 31))) : 0u);
        while (true) {
            if (bits) {
                int pb = w * 32 + 31 - __clz(bits);
                unsigned long long pm =
                    (unsigned long long)col[2 * pb] | ((unsigned long long)col[2 * pb + 1] << 32);
                yabove = pb * 64 + 63 - __clzll(pm);
                break;
            }
            if (--w < 0) break;
            bits = bo[w];
        }
    }
    {
        int w = b >> 5;
        int sh = (b & 31) + 1;
        uint32_t bits = sh >= 32 ? 0u : (bo[w] & (0xffffffffu << sh));
        while (true) {
            if (bits) {
                int nb2 = w * 32 + __ffs(bits) - 1;
                unsigned long long nm =
                    (unsigned long long)col[2 * nb2] | ((unsigned long long)col[2 * nb2 + 1] << 32);
                ybelow = nb2 * 64 + __ffsll((long long)nm) - 1;
                break;
            }
            if (++w >= W2) break;
            bits = bo[w];
        }
    }
    int y0 = b * 64;
    int16_t *out = ycol + (size_t)y0 * T + x;
    for (int r = 0; r < 64; r++) {
        unsigned long long lowmask = (r == 63) ? ~0ull : ((2ull << r) - 1ull);
        unsigned long long lo = m & lowmask;
        unsigned long long hi = m & ~((1ull << r) - 1ull);
        int y = y0 + r;
        int yp = lo ? (y0 + 63 - __clzll(lo)) : yabove;
        int yn = hi ? (y0 + __ffsll((long long)hi) - 1) : ybelow;
        int best;
        if (yp < 0) best = yn;
        else if (yn < 0) best = yp;
        else best = (y - yp <= yn - y) ? yp : yn;
        out[(size_t)r * T] = (int16_t)best;
    }
}

// --------------------------------------------------------------- row pass
// Exact-integer lower envelope of the parabolas f_x(p) = (p - x)^2 + (y - yc[x])^2.
struct Par {
    int x;
    int c;  // x^2 + h
};

__device__ __forceinline__ int par_c(int x, int yc, int y)
{
    int h = y - yc;
    return x * x + h * h;
}

// true if b is hidden between a and c: s(a,b) >= s(b,c) with s(a,b) = (cb - ca) / (2 (xb - xa)).
__device__ __forceinline__ bool dominated(Par a, Par b, Par c)
{
    long long n1 = (long long)(b.c - a.c), d1 = 2LL * (b.x - a.x);
    long long n2 = (long long)(c.c - b.c), d2 = 2LL * (c.x - b.x);
    return n1 * d2 >= n2 * d1;
}

// last integer pixel owned by a (a left of b, ties go left): floor((cb - ca) / (2 (xb - xa)))
__device__ __forceinline__ int boundary(Par a, Par b)
{
    int num = b.c - a.c, den = 2 * (b.x - a.x);
    int q = num / den;
    if ((num % den != 0) && ((num < 0) != (den < 0))) q--;
    return q;
}

constexpr int kRowThreads = 256;
constexpr int16_t kDead = -2;  // nxt[] marker of an element popped from the envelope

__global__ void __launch_bounds__(kRowThreads) k_row_pass(const int16_t *__restrict__ ycol,
                                                          const int *__restrict__ idmap,
                                                          int *__restrict__ colour, int T, int logT,
                                                          const int *__restrict__ cellmap)
{
    // blockIdx.y: texture cell (cellmap[z], or z) of a batch
    {
        const size_t off = (size_t)(cellmap ? cellmap[blockIdx.y] : blockIdx.y) << (2 * logT);
        ycol += off;
        idmap += off;
        colour += off;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    int16_t *ys = (int16_t *)smem;       // [T]
    int16_t *nxt = ys + T;               // [T]
    int16_t *prv = nxt + T;              // [T]
    int *row = (int *)(prv + T + (T & 1));  // [T] colour staging
    __shared__ int16_t segHead[kRowThreads], segTail[kRowThreads];

    const int y = blockIdx.x;
    const int tid = threadIdx.x;
    const int S = T >= kRowThreads ? T / kRowThreads : 1;  // columns per thread (T < 256: one, or none)
    // 1. load the row of column candidates (16-byte vectors)
    {
        const int4 *src = (const int4 *)(ycol + (size_t)y * T);
        int4 *dst = (int4 *)ys;
        for (int k = tid; k < T / 8; k += kRowThreads) dst[k] = src[k];
    }
    __syncthreads();
    // 2. local envelope of each thread's segment
    {
        int head = -1, tail = -1;
        int x0 = tid * S;
        for (int x = x0; x < x0 + S && x < T; x++) {
            int yc = ys[x];
            if (yc < 0) continue;
            Par cur{x, par_c(x, yc, y)};
            while (tail >= 0 && prv[tail] >= 0) {
                int pt = prv[tail];
                Par a{pt, par_c(pt, ys[pt], y)}, b{tail, par_c(tail, ys[tail], y)};
                if (!dominated(a, b, cur)) break;
                nxt[tail] = kDead;
                tail = pt;
            }
            prv[x] = (int16_t)tail;
            nxt[x] = -1;
            if (tail >= 0) nxt[tail] = (int16_t)x;
            else head = x;
            tail = x;
        }
        segHead[tid] = (int16_t)head;
        segTail[tid] = (int16_t)tail;
    }
    __syncthreads();
    // 3. pairwise merges
    for (int w = 1; w < kRowThreads; w <<= 1) {
        if ((tid & (2 * w - 1)) == 0) {
            int lh = segHead[tid], lt = segTail[tid];
            int rh = segHead[tid + w], rt = segTail[tid + w];
            if (lh < 0) {
                lh = rh;
                lt = rt;
            } else if (rh >= 0) {
                while (true) {
                    int plt = prv[lt];
                    if (plt >= 0) {
                        Par a{plt, par_c(plt, ys[plt], y)}, b{lt, par_c(lt, ys[lt], y)},
                            c{rh, par_c(rh, ys[rh], y)};
                        if (dominated(a, b, c)) {
                            nxt[lt] = kDead;
                            lt = plt;
                            continue;
                        }
                    }
                    int nrh = nxt[rh];
                    if (nrh >= 0) {
                        Par a{lt, par_c(lt, ys[lt], y)}, b{rh, par_c(rh, ys[rh], y)},
                            c{nrh, par_c(nrh, ys[nrh], y)};
                        if (dominated(a, b, c)) {
                            nxt[rh] = kDead;
                            prv[nrh] = -1;
                            rh = nrh;
                            continue;
                        }
                    }
                    break;
                }
                nxt[lt] = (int16_t)rh;
                prv[rh] = (int16_t)lt;
                lt = rt;
            }
            segHead[tid] = (int16_t)lh;
            segTail[tid] = (int16_t)lt;
        }
        __syncthreads();
    }
    // 4. colour: every live element paints its own interval
    {
        int x0 = tid * S;
        for (int x = x0; x < x0 + S && x < T; x++) {
            int yc = ys[x];
            if (yc < 0) continue;
            int nx = nxt[x];
            if (nx == kDead) continue;  // popped from the envelope
            int pv = prv[x];
            Par me{x, par_c(x, yc, y)};
            int lo = 0, hi = T - 1;
            if (pv >= 0) {
                Par a{pv, par_c(pv, ys[pv], y)};
                lo = boundary(a, me) + 1;
            }
            if (nx >= 0) {
                Par b{nx, par_c(nx, ys[nx], y)};
                hi = boundary(me, b);
            }
            if (lo < 0) lo = 0;
            if (hi > T - 1) hi = T - 1;
            if (lo > hi) continue;
            int id = idmap[((size_t)yc << logT) + x];
            for (int p = lo; p <= hi; p++) row[p] = id;
        }
    }
    __syncthreads();
    {
        const int4 *src = (const int4 *)row;
        int4 *dst = (int4 *)(colour + (size_t)y * T);
        for (int k = tid; k < T / 4; k += kRowThreads) dst[k] = src[k];
    }
}

// ------------------------------------------------------ dual triangles
// 2x2 window at (x, y): corners c0 (x,y), c1 (x+1,y), c2 (x+1,y+1), c3 (x,y+1),
// counterclockwise.  Returns the triangle count and the triangles.
__device__ __forceinline__ long long orient_pix(short2 a, short2 b, short2 c)
{
    return (long long)(a.x - c.x) * (b.y - c.y) - (long long)(a.y - c.y) * (b.x - c.x);
}

__device__ __forceinline__ int window_tris(const int *colour, const short2 *gpix, int logT, int x, int y,
                                           int3 *t, int *bad)
{
    size_t r0 = ((size_t)y << logT) + x, r1 = r0 + ((size_t)1 << logT);
    int c[4] = {colour[r0], colour[r0 + 1], colour[r1 + 1], colour[r1]};
    if (c[0] == c[2] || c[1] == c[3]) return 0;
    int L[4], n = 0;
    for (int k = 0; k < 4; k++)
        if (c[k] != c[(k + 3) & 3]) L[n++] = c[k];
    if (n == 3) {
        t[0] = make_int3(L[0], L[1], L[2]);
        if (orient_pix(gpix[L[0]], gpix[L[1]], gpix[L[2]]) <= 0) *bad = 1;
        return 1;
    }
    if (n == 4) {
        short2 g0 = gpix[L[0]], g1 = gpix[L[1]], g2 = gpix[L[2]], g3 = gpix[L[3]];
        if (orient_pix(g0, g1, g2) > 0 && orient_pix(g0, g2, g3) > 0) {
            t[0] = make_int3(L[0], L[1], L[2]);
            t[1] = make_int3(L[0], L[2], L[3]);
        } else {
            t[0] = make_int3(L[1], L[2], L[3]);
            t[1] = make_int3(L[1], L[3], L[0]);
            if (orient_pix(g1, g2, g3) <= 0 || orient_pix(g1, g3, g0) <= 0) *bad = 1;
        }
        return 2;
    }
    return 0;
}


__device__ __forceinline__ int block_exclusive_scan(int v, int *total)
{
    __shared__ int warpsum[kEmitThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warpsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int s = lane < kEmitThreads / 32 ? warpsum[lane] : 0;
        int si = s;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < kEmitThreads / 32) warpsum[lane] = si - s;
    }
    __syncthreads();
    int excl = incl - v + warpsum[w];
    if (total) {
        __shared__ int tot;
        if (threadIdx.x == kEmitThreads - 1) tot = excl + v;
        __syncthreads();
        *total = tot;
    }
    return excl;
}

// Blocks are numbered cell-major: tiles_per_cell consecutive blocks per cell.
__global__ void __launch_bounds__(kEmitThreads) k_emit_count(const int *__restrict__ colour,
                                                             const short2 *__restrict__ gpix, int *tilecount,
                                                             int T, int logT, long long nwin, Counters *ct,
                                                             const int *__restrict__ cellmap, int tiles_per_cell)
{
    const int z = blockIdx.x / tiles_per_cell;
    colour += (size_t)(cellmap ? cellmap[z] : z) << (2 * logT);
    long long w = (long long)(blockIdx.x - z * tiles_per_cell) * kEmitThreads + threadIdx.x;
    int n = 0, bad = 0;
    if (w < nwin) {
        int x = (int)(w % (T - 1)), y = (int)(w / (T - 1));
        int3 t[2];
        n = window_tris(colour, gpix, logT, x, y, t, &bad);
        if (bad) set_err(ct, GPUDT_ERR_TOPOLOGY, 10);
    }
    int total;
    block_exclusive_scan(n, &total);
    if (threadIdx.x == 0) tilecount[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kEmitThreads) k_emit_write(const int *__restrict__ colour,
                                                             const short2 *__restrict__ gpix,
                                                             const int *__restrict__ tileoff, int4 *tv, int T,
                                                             int logT, long long nwin,
                                                             const int *__restrict__ cellmap, int tiles_per_cell)
{
    const int z = blockIdx.x / tiles_per_cell;
    colour += (size_t)(cellmap ? cellmap[z] : z) << (2 * logT);
    long long w = (long long)(blockIdx.x - z * tiles_per_cell) * kEmitThreads + threadIdx.x;
    int n = 0, bad = 0;
    int3 t[2];
    if (w < nwin) {
        int x = (int)(w % (T - 1)), y = (int)(w / (T - 1));
        n = window_tris(colour, gpix, logT, x, y, t, &bad);
    }
    int off = block_exclusive_scan(n, nullptr) + tileoff[blockIdx.x];
    for (int k = 0; k < n; k++) tv[off + k] = make_int4(t[k].x, t[k].y, t[k].z, 0);
}


// ------------------------------------------------- fused colour + dual
// One CTA owns a tile of KT_W x KT_H windows.  It colours the tile's pixels plus
// a one-pixel halo (rows y0-1 .. y0+KT_H+1) by an exact window scan over the
// column candidates, keeps the colours as packed site pixel coordinates in
// shared memory, checks the island property on every pixel the windows use,
// and emits the dual triangles of the tile -- the colour texture never goes
// to HBM.  A tile with an island pixel emits nothing and raises a flag; the
// host then runs the envelope path (k_row_pass + island repair + k_emit_*).
//
// Window scan: owner(x, y) = argmin over columns cx of (d, cx) with
// d = (x - cx)^2 + (y - ycol[y][cx])^2 (ties: smaller column; within a column
// the column pass already kept the upper site).  Columns are visited at
// growing distance k from x; the scan stops once k^2 exceeds the best d, which
// no further column can beat.  This is the same assignment k_row_pass makes.
constexpr int KT_W = 128, KT_H = 16;  // 16 rows: the one-pixel halo adds 21 % to the coloured pixels, not 41 %
constexpr int KT_CW = KT_W + 3, KT_CH = KT_H + 3;  // coloured pixels incl. halo
constexpr int kFusedThreads = 512;

// 32-bit arithmetic throughout: T <= 16384, so k^2 + dy^2 < 2^30.  Scanning
// outwards, a left candidate at distance k has a smaller column than every
// earlier best (all lie within k - 1 of x), so it wins ties; a right one never
// does -- the (d, column) order without a column compare.
__device__ __forceinline__ unsigned owner_scan(const int16_t *__restrict__ row, int x, int y, int T)
{
    int bestd = 0x7fffffff, bx = -1;
    const int yc = row[x];
    if (yc >= 0) {
        bestd = (y - yc) * (y - yc);
        bx = x;
    }
    for (int k = 1; k < T && k * k <= bestd; k++) {
        const int kk = k * k, xl = x - k, xr = x + k;
        if (xl >= 0) {
            const int c = row[xl];
            if (c >= 0) {
                const int d = kk + (y - c) * (y - c);
                if (d <= bestd) {
                    bestd = d;
                    bx = xl;
                }
            }
        }
        if (xr < T) {
            const int c = row[xr];
            if (c >= 0) {
                const int d = kk + (y - c) * (y - c);
                if (d < bestd) {
                    bestd = d;
                    bx = xr;
                }
            }
        }
    }
    const int sy = row[bx];
    return ((unsigned)sy << 16) | (unsigned)bx;
}

__device__ __forceinline__ long long orient_pk(unsigned a, unsigned b, unsigned c)
{
    int ax = a & 0xffff, ay = a >> 16, bx = b & 0xffff, by = b >> 16, cx = c & 0xffff, cy = c >> 16;
    return (long long)(ax - cx) * (by - cy) - (long long)(ay - cy) * (bx - cx);
}

__global__ void __launch_bounds__(kFusedThreads) k_vd_tri(const int16_t *__restrict__ ycol,
                                                          const int *__restrict__ idmap, int4 *__restrict__ tv,
                                                          int2 *__restrict__ chunk, int *__restrict__ flagged,
                                                          int T, int logT, int cap, Counters *ct,
                                                          const int *__restrict__ cellmap)
{
    // blockIdx.z: texture cell (cellmap[z], or z) of a batch; tiles are
    // numbered over the launched cells
    const int tile = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    {
        const size_t off = (size_t)(cellmap ? cellmap[blockIdx.z] : blockIdx.z) << (2 * logT);
        ycol += off;
        idmap += off;
    }
    __shared__ unsigned col[KT_CH][KT_CW];
    __shared__ int tile_island;
    const int x0 = blockIdx.x * KT_W, y0 = blockIdx.y * KT_H;
    if (threadIdx.x == 0) tile_island = 0;
    // 1. colours of pixels (x0-1 .. x0+KT_W+1) x (y0-1 .. y0+KT_H+1), clamped
    for (int k = threadIdx.x; k < KT_CH * KT_CW; k += kFusedThreads) {
        int ly = k / KT_CW, lx = k - ly * KT_CW;
        int x = x0 - 1 + lx, y = y0 - 1 + ly;
        unsigned o = 0xffffffffu;
        if (x >= 0 && y >= 0 && x < T && y < T) o = owner_scan(ycol + ((size_t)y << logT), x, y, T);
        col[ly][lx] = o;
    }
    __syncthreads();
    // 2. island test on every pixel a window of this tile uses
    for (int k = threadIdx.x; k < (KT_H + 1) * (KT_W + 1); k += kFusedThreads) {
        int ly = k / (KT_W + 1), lx = k - ly * (KT_W + 1);
        int x = x0 + lx, y = y0 + ly;
        if (x >= T || y >= T) continue;
        unsigned c = col[ly + 1][lx + 1];
        int sx = c & 0xffff, sy = c >> 16;
        int dx = (sx > x) - (sx < x), dy = (sy > y) - (sy < y);
        if (dx == 0 && dy == 0) continue;
        bool ok = (dx != 0 && col[ly + 1][lx + 1 + dx] == c) || (dy != 0 && col[ly + 1 + dy][lx + 1] == c) ||
                  (dx != 0 && dy != 0 && col[ly + 1 + dy][lx + 1 + dx] == c);
        if (!ok) tile_island = 1;
    }
    __syncthreads();
    if (tile_island) {
        if (threadIdx.x == 0) {
            chunk[tile] = make_int2(0, 0);
            flagged[atomicAdd(&ct->nisland, 1)] = tile;
        }
        return;
    }
    // 3. dual triangles of the tile's windows (x, y) .. (x+1, y+1)
    int n = 0;
    unsigned tri[2 * (KT_H * KT_W / kFusedThreads)][3];
    for (int k = threadIdx.x; k < KT_H * KT_W; k += kFusedThreads) {
        int ly = k / KT_W, lx = k - ly * KT_W;
        int x = x0 + lx, y = y0 + ly;
        if (x >= T - 1 || y >= T - 1) continue;
        unsigned c[4] = {col[ly + 1][lx + 1], col[ly + 1][lx + 2], col[ly + 2][lx + 2], col[ly + 2][lx + 1]};
        if (c[0] == c[2] || c[1] == c[3]) continue;
        unsigned L[4];
        int m = 0;
        for (int q = 0; q < 4; q++)
            if (c[q] != c[(q + 3) & 3]) L[m++] = c[q];
        if (m == 3) {
            if (orient_pk(L[0], L[1], L[2]) <= 0) set_err(ct, GPUDT_ERR_TOPOLOGY, 11);
            tri[n][0] = L[0];
            tri[n][1] = L[1];
            tri[n][2] = L[2];
            n++;
        } else if (m == 4) {
            if (orient_pk(L[0], L[1], L[2]) > 0 && orient_pk(L[0], L[2], L[3]) > 0) {
                tri[n][0] = L[0]; tri[n][1] = L[1]; tri[n][2] = L[2]; n++;
                tri[n][0] = L[0]; tri[n][1] = L[2]; tri[n][2] = L[3]; n++;
            } else {
                if (orient_pk(L[1], L[2], L[3]) <= 0 || orient_pk(L[1], L[3], L[0]) <= 0)
                    set_err(ct, GPUDT_ERR_TOPOLOGY, 12);
                tri[n][0] = L[1]; tri[n][1] = L[2]; tri[n][2] = L[3]; n++;
                tri[n][0] = L[1]; tri[n][1] = L[3]; tri[n][2] = L[0]; n++;
            }
        }
    }
    // block-wide offsets, one atomic per block
    __shared__ int warpsum[kFusedThreads / 32];
    __shared__ int base;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warpsum[w] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int q = 0; q < kFusedThreads / 32; q++) {
            int v = warpsum[q];
            warpsum[q] = s;
            s += v;
        }
        base = s ? atomicAdd(&ct->ntris, s) : 0;
        if (base + s > cap) set_err(ct, GPUDT_ERR_NOMEM, 13);
        chunk[tile] = make_int2(base, s);
    }
    __syncthreads();
    int off = base + warpsum[w] + incl - n;
    if (off + n > cap) return;
    for (int q = 0; q < n; q++) {
        int a = idmap[((size_t)(tri[q][0] >> 16) << logT) + (tri[q][0] & 0xffff)];
        int b = idmap[((size_t)(tri[q][1] >> 16) << logT) + (tri[q][1] & 0xffff)];
        int c = idmap[((size_t)(tri[q][2] >> 16) << logT) + (tri[q][2] & 0xffff)];
        tv[off + q] = make_int4(a, b, c, 0);
    }
}

// Island repair for one tile: colours the tile with an 8-pixel margin, marks
// island components (iterated isolation test, the repeat loop of
// cudaIslandDetection, cudaVoronoi.cu:220-247), recolours them from their
// non-island neighbours (each island pixel takes, among its 8 neighbours
// already coloured, the site nearest to it; ties: smaller packed coordinate;
// Jacobi rounds), and emits the tile's triangles.  Neighbouring tiles see the
// same small components and make the same decisions.
constexpr int KS_M = 8;
constexpr int KS_W = KT_W + 1 + 2 * KS_M, KS_H = KT_H + 1 + 2 * KS_M;

__global__ void __launch_bounds__(kFusedThreads) k_vd_tri_repair(const int16_t *__restrict__ ycol,
                                                                 const int *__restrict__ idmap,
                                                                 int4 *__restrict__ tv, const int *__restrict__ tiles,
                                                                 const int *__restrict__ freelist, int tiles_x, int T,
                                                                 int logT, int cap, int *esc_cells, Counters *ct,
                                                                 const int *__restrict__ cellmap)
{
    __shared__ unsigned col[KS_H][KS_W];
    __shared__ unsigned nxt[KS_H][KS_W];

    const int gtile = tiles[blockIdx.x];
    const int tiles_y = (T - 1 + KT_H - 1) / KT_H;
    const int cell = gtile / (tiles_x * tiles_y), tile = gtile - cell * tiles_x * tiles_y;
    {
        const size_t off = (size_t)(cellmap ? cellmap[cell] : cell) << (2 * logT);
        ycol += off;
        idmap += off;
    }
    const int x0 = (tile % tiles_x) * KT_W, y0 = (tile / tiles_x) * KT_H;
    const int gx = x0 - KS_M, gy = y0 - KS_M;  // pixel of col[0][0]
    const unsigned NONE = 0xffffffffu, ISL = 0xfffffffeu;
    for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
        int ly = k / KS_W, lx = k - ly * KS_W;
        int x = gx + lx, y = gy + ly;
        col[ly][lx] = (x >= 0 && y >= 0 && x < T && y < T) ? owner_scan(ycol + ((size_t)y << logT), x, y, T) : NONE;
    }
    __syncthreads();
    // mark island components: a pixel whose toward-site neighbours (all inside
    // the region) carry neither its colour is marked; repeat
    // (the round flags are block-wide reductions, __syncthreads_or, so every
    // thread leaves a loop after the same round)
    for (int round = 0; round < KS_M; round++) {
        int mine = 0;
        for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
            int ly = k / KS_W, lx = k - ly * KS_W;
            unsigned c = col[ly][lx];
            nxt[ly][lx] = c;
            if (c >= ISL || ly == 0 || lx == 0 || ly == KS_H - 1 || lx == KS_W - 1) continue;
            int x = gx + lx, y = gy + ly;
            int sx = c & 0xffff, sy = c >> 16;
            int dx = (sx > x) - (sx < x), dy = (sy > y) - (sy < y);
            if (dx == 0 && dy == 0) continue;
            bool ok = (dx != 0 && col[ly][lx + dx] == c) || (dy != 0 && col[ly + dy][lx] == c) ||
                      (dx != 0 && dy != 0 && col[ly + dy][lx + dx] == c);
            if (!ok) {
                nxt[ly][lx] = ISL;
                mine = 1;
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
            int ly = k / KS_W, lx = k - ly * KS_W;
            col[ly][lx] = nxt[ly][lx];
        }
        if (!__syncthreads_or(mine)) break;
    }
    // components that reach the region border may extend past the redo set:
    // flood the island pixels from the border zone; if one of the tile's own
    // pixels is reached, the repair cannot stay local
    {
        for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
            int ly = k / KS_W, lx = k - ly * KS_W;
            bool border = ly <= 1 || lx <= 1 || ly >= KS_H - 2 || lx >= KS_W - 2;
            nxt[ly][lx] = (col[ly][lx] == ISL && border) ? 1u : 0u;
        }
        __syncthreads();
        for (int round = 0; round < KS_W + KS_H; round++) {
            int mine = 0;
            for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
                int ly = k / KS_W, lx = k - ly * KS_W;
                if (col[ly][lx] != ISL || nxt[ly][lx]) continue;
                bool hit = false;
                for (int dy = -1; dy <= 1 && !hit; dy++)
                    for (int dx = -1; dx <= 1 && !hit; dx++) {
                        int yy = ly + dy, xx = lx + dx;
                        if (yy >= 0 && xx >= 0 && yy < KS_H && xx < KS_W && nxt[yy][xx] == 1u) hit = true;
                    }
                if (hit) {
                    nxt[ly][lx] = 1u;
                    mine = 1;
                }
            }
            if (!__syncthreads_or(mine)) break;
        }
        for (int k = threadIdx.x; k < (KT_H + 1) * (KT_W + 1); k += kFusedThreads) {
            int ly = k / (KT_W + 1) + KS_M, lx = k % (KT_W + 1) + KS_M;
            if (nxt[ly][lx] == 1u) {
                ct->escalate = 1;
                if (esc_cells) esc_cells[cell] = 1;
            }
        }
        __syncthreads();
    }
    // recolour
    for (int round = 0; round < 4 * KS_M; round++) {
        int mine = 0;
        for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
            int ly = k / KS_W, lx = k - ly * KS_W;
            unsigned c = col[ly][lx];
            nxt[ly][lx] = c;
            if (c != ISL) continue;
            int x = gx + lx, y = gy + ly;
            long long bd = -1;
            unsigned bc = ISL;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    int yy = ly + dy, xx = lx + dx;
                    if ((!dx && !dy) || yy < 0 || xx < 0 || yy >= KS_H || xx >= KS_W) continue;
                    unsigned q = col[yy][xx];
                    if (q >= ISL) continue;
                    int sx = q & 0xffff, sy = q >> 16;
                    long long d = (long long)(sx - x) * (sx - x) + (long long)(sy - y) * (sy - y);
                    if (bd < 0 || d < bd || (d == bd && q < bc)) {
                        bd = d;
                        bc = q;
                    }
                }
            nxt[ly][lx] = bc;
            if (bc == ISL) mine = 1;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < KS_H * KS_W; k += kFusedThreads) {
            int ly = k / KS_W, lx = k - ly * KS_W;
            col[ly][lx] = nxt[ly][lx];
        }
        if (!__syncthreads_or(mine)) break;
    }
    // emit the tile's windows; a recolouring that leaves a window without a
    // consistent dual (an unresolved island, or three colours not in
    // counterclockwise order) sends the texture to the envelope path instead
    int mybad = 0;
    int n = 0;
    unsigned tri[2 * (KT_H * KT_W / kFusedThreads)][3];
    for (int k = threadIdx.x; k < KT_H * KT_W; k += kFusedThreads) {
        int ly = k / KT_W, lx = k - ly * KT_W;
        int x = x0 + lx, y = y0 + ly;
        if (x >= T - 1 || y >= T - 1) continue;
        int py = ly + KS_M, px = lx + KS_M;
        unsigned c[4] = {col[py][px], col[py][px + 1], col[py + 1][px + 1], col[py + 1][px]};
        if (c[0] >= ISL || c[1] >= ISL || c[2] >= ISL || c[3] >= ISL) {
            mybad = 1;
            continue;
        }
        if (c[0] == c[2] || c[1] == c[3]) continue;
        unsigned L[4];
        int m = 0;
        for (int q = 0; q < 4; q++)
            if (c[q] != c[(q + 3) & 3]) L[m++] = c[q];
        if (m == 3) {
            if (orient_pk(L[0], L[1], L[2]) <= 0) mybad = 1;
            tri[n][0] = L[0]; tri[n][1] = L[1]; tri[n][2] = L[2]; n++;
        } else if (m == 4) {
            if (orient_pk(L[0], L[1], L[2]) > 0 && orient_pk(L[0], L[2], L[3]) > 0) {
                tri[n][0] = L[0]; tri[n][1] = L[1]; tri[n][2] = L[2]; n++;
                tri[n][0] = L[0]; tri[n][1] = L[2]; tri[n][2] = L[3]; n++;
            } else {
                if (orient_pk(L[1], L[2], L[3]) <= 0 || orient_pk(L[1], L[3], L[0]) <= 0) mybad = 1;
                tri[n][0] = L[1]; tri[n][1] = L[2]; tri[n][2] = L[3]; n++;
                tri[n][0] = L[1]; tri[n][1] = L[3]; tri[n][2] = L[0]; n++;
            }
        }
    }
    if (__syncthreads_or(mybad)) {
        if (threadIdx.x == 0) {
            ct->escalate = 1;
            if (esc_cells) esc_cells[cell] = 1;
        }
        return;
    }
    for (int q = 0; q < n; q++) {
        // reuse the slots released by the redo set first, then the tail
        int k = atomicSub(&ct->nfree, 1) - 1;
        int s = k >= 0 ? freelist[k] : atomicAdd(&ct->ntris, 1);
        if (s >= cap) {
            set_err(ct, GPUDT_ERR_NOMEM, 18);
            return;
        }
        int a = idmap[((size_t)(tri[q][0] >> 16) << logT) + (tri[q][0] & 0xffff)];
        int b = idmap[((size_t)(tri[q][1] >> 16) << logT) + (tri[q][1] & 0xffff)];
        int cc = idmap[((size_t)(tri[q][2] >> 16) << logT) + (tri[q][2] & 0xffff)];
        tv[s] = make_int4(a, b, cc, 0);
    }
}

// Redo set = flagged tiles and their 8 neighbours; their fast-path triangles
// are released (dead slots: vertex 0 = -1, pushed on the free list).
__global__ void k_redo_mark(const int *flagged, int nflag, unsigned char *redo, int tiles_x, int tiles_y)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nflag) return;
    const int per = tiles_x * tiles_y;
    int g = flagged[i], cell = g / per, t = g - cell * per, tx = t % tiles_x, ty = t / tiles_x;
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
            int x = tx + dx, y = ty + dy;
            if (x >= 0 && y >= 0 && x < tiles_x && y < tiles_y) redo[(size_t)cell * per + y * tiles_x + x] = 1;
        }
}

__global__ void k_redo_collect(const unsigned char *redo, int ntiles, const int2 *chunk, int4 *tv, int *list,
                               int *freelist, Counters *ct)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles || !redo[t]) return;
    list[atomicAdd(&ct->nlist, 1)] = t;
    const int2 ch = chunk[t];
    // the tile's triangles go to the free list in one reservation (one atomic
    // per tile on the shared counter, not one per triangle)
    const int base = ch.y > 0 ? atomicAdd(&ct->nfree, ch.y) : 0;
    for (int q = 0; q < ch.y; q++) {
        tv[ch.x + q] = make_int4(-1, -1, -1, 0);
        freelist[base + q] = ch.x + q;
    }
}

__global__ void k_clamp_free(Counters *ct)
{
    if (ct->nfree < 0) ct->nfree = 0;
}

int launch_vd_repair(Ctx &c, int nflag)
{
    return launch_vd_repair_cells(c, nflag, c.T, c.logT, 1, c.ycol, c.idmap, nullptr, nullptr, (const int2 *)c.colour);
}

int launch_vd_repair_cells(Ctx &c, int nflag, int T, int logT, int cells, const int16_t *ycol, const int *idmap,
                           int *esc_cells, const int *cellmap, const int2 *chunk)
{
    int tiles_x = (T - 1 + KT_W - 1) / KT_W, tiles_y = (T - 1 + KT_H - 1) / KT_H;
    int ntiles = tiles_x * tiles_y * cells;
    unsigned char *redo = (unsigned char *)c.aux;
    GALPHA_CUDA(cudaMemsetAsync(redo, 0, (size_t)ntiles, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
    k_redo_mark<<<(nflag + 127) / 128, 128, 0, c.stream>>>(c.list2, nflag, redo, tiles_x, tiles_y);
    count_launch();
    k_redo_collect<<<(ntiles + 255) / 256, 256, 0, c.stream>>>(redo, ntiles, chunk, c.tv, c.list, c.freelist, c.ctr);
    count_launch();
    int r = read_counters(c);
    if (r) return r;
    int nredo = c.hctr->nlist;
    k_vd_tri_repair<<<nredo, kFusedThreads, 0, c.stream>>>(ycol, idmap, c.tv, c.list, c.freelist, tiles_x, T, logT,
                                                           c.cap_tris, esc_cells, c.ctr, cellmap);
    count_launch();
    k_clamp_free<<<1, 1, 0, c.stream>>>(c.ctr);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int launch_vd_tri(Ctx &c)
{
    return launch_vd_tri_cells(c, c.T, c.logT, 1, c.ycol, c.idmap, (int2 *)c.colour, c.list2, nullptr);
}

// Tiles of all launched cells, numbered cell-major; chunk / flagged use that
// numbering.  cellmap (or identity) gives the texture cell of launch cell z.
int launch_vd_tri_cells(Ctx &c, int T, int logT, int cells, const int16_t *ycol, const int *idmap, int2 *chunk,
                        int *flagged, const int *cellmap)
{
    dim3 grid((T - 1 + KT_W - 1) / KT_W, (T - 1 + KT_H - 1) / KT_H, cells);
    kev_record(c, 0);
    k_vd_tri<<<grid, kFusedThreads, 0, c.stream>>>(ycol, idmap, c.tv, chunk, flagged, T, logT, c.cap_tris, c.ctr,
                                                    cellmap);
    count_launch();
    kev_record(c, 1);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

// Tiles of the fused kernel per T x T cell.
int fused_tiles(int T)
{
    return ((T - 1 + KT_W - 1) / KT_W) * ((T - 1 + KT_H - 1) / KT_H);
}

// ---------------------------------------------------------------- launchers
int launch_column_pass(Ctx &c, int W2)
{
    return launch_column_pass_cells(c, c.T, W2, 1, c.occ, c.bandocc, c.ycol);
}

int launch_column_pass_cells(Ctx &c, int T, int W2, int cells, const uint32_t *occ, const uint32_t *bandocc,
                             int16_t *ycol)
{
    dim3 block(32, 8), grid(T / 32, ((T >> 6) + 7) / 8, cells);
    kev_record(c, 2);
    k_column_pass<<<grid, block, 0, c.stream>>>(occ, bandocc, ycol, T, W2);
    kev_record(c, 3);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int launch_row_pass(Ctx &c)
{
    return launch_row_pass_cells(c, 1, nullptr);
}

// Rows of `cells` texture cells of size c.T at c.ycol / c.idmap / c.colour
// (cell cellmap[z], or z).
int launch_row_pass_cells(Ctx &c, int cells, const int *cellmap)
{
    const int T = c.T;
    size_t sm = sizeof(int16_t) * (3 * (size_t)T + (T & 1)) + sizeof(int) * (size_t)T;
    {
        // once per device, for the largest texture (16384): a per-size setting
        // would race between handles driven from different threads
        static std::mutex mu;
        static bool configured[64];
        const size_t smax = sizeof(int16_t) * 3 * 16384 + sizeof(int) * 16384;
        const int dv = c.device >= 0 && c.device < 64 ? c.device : 0;
        std::lock_guard<std::mutex> lk(mu);
        if (!configured[dv]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_row_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
            configured[dv] = true;
        }
    }
    kev_record(c, 0);
    k_row_pass<<<dim3(T, cells), kRowThreads, sm, c.stream>>>(c.ycol, c.idmap, c.colour, T, c.logT, cellmap);
    kev_record(c, 1);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int launch_emit(Ctx &c, int ntiles, long long nwin, bool write, int4 *tv_out)
{
    return launch_emit_cells(c, ntiles, nwin, write, tv_out, 1, nullptr);
}

// ntiles blocks per cell; `cells` cells of size c.T at c.colour (cellmap[z], or z).
int launch_emit_cells(Ctx &c, int ntiles, long long nwin, bool write, int4 *tv_out, int cells, const int *cellmap)
{
    kev_record(c, write ? 6 : 4);
    const long long blocks = (long long)ntiles * cells;
    if (!write)
        k_emit_count<<<(unsigned)blocks, kEmitThreads, 0, c.stream>>>(c.colour, c.gpix, c.tilecount, c.T, c.logT, nwin,
                                                                      c.ctr, cellmap, ntiles);
    else
        k_emit_write<<<(unsigned)blocks, kEmitThreads, 0, c.stream>>>(c.colour, c.gpix, c.tilecount, tv_out, c.T,
                                                                      c.logT, nwin, cellmap, ntiles);
    count_launch();
    kev_record(c, write ? 7 : 5);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

}  // namespace galpha
