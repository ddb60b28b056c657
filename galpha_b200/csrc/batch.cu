// batch.cu -- many independent point sets in one pipeline run.
//
// The reference triangulates one point set per gpudtComputeDT call
// (gpudt.cpp:771-929) and computes one Alpha_Shapes_2D per call.  Here a batch
// of K sets runs the same stages once over the disjoint union of the sets:
//
//  * every set gets its own square texture cell (a power-of-two T chosen from
//    its size), its own grid scaling and its own fake ring, so the Voronoi
//    stage never relates sites of different sets; cells of equal T are stacked
//    and coloured by one launch per size (blockIdx.z = cell);
//  * the mesh stages (links, shifting, missing sites, fake removal, flipping)
//    are local operations and run unchanged on the union mesh, whose
//    connected components are the sets;
//  * compaction groups the triangles by set (a stable radix sort on the set
//    id), so each set's triangles, edges and spectrum are contiguous;
//  * the alpha stage sorts its entries by (set, value) and ranks every set
//    separately, each with its own rank-0 sentinel.
//
// Vertex numbering: real vertices are the sets' points concatenated in set
// order; fake ring sites follow, set by set (4 * nside per set, so each ring
// starts at a multiple of 4 and the ring classes of fake removal stay apart).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include "internal.cuh"
#include "exact.cuh"

namespace galpha {

namespace {

// power-of-two texture cell for n points: at least `density` pixels per point
// inside the ring margin (10 by default; a tuned value from the autotuner),
// at least 128 (the fused tile width), so the dense (fused) colouring path
// applies.  Fewer pixels per point mean fewer pixels to colour and more
// points sharing a pixel (missing sites, inserted later).
int cell_size(int n, double density)
{
    int T = 128;
    while (T < 16384 && (double)(T - 2 * kMargin) * (T - 2 * kMargin) < density * n) T *= 2;
    return T;
}

__device__ __forceinline__ int find_set(const int *base, int K, int v)
{
    // last set whose base is <= v
    int lo = 0, hi = K - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct BFirstDistinct {
    const double *xy;
    const int *vset;
    const SetDesc *sets;
    int *first;
    __device__ void operator()(long long i) const
    {
        int v = (int)i, s = vset[v], b = sets[s].vbase;
        const int cand = (xy[2 * v] != xy[2 * b] || xy[2 * v + 1] != xy[2 * b + 1]) ? v : 0x7fffffff;
        // sets are contiguous: the lanes of a warp share one or two sets, so
        // one atomic per set and warp instead of one per point
        const unsigned same = __match_any_sync(__activemask(), s);
        const int mn = (int)__reduce_min_sync(same, (unsigned)cand);
        if ((int)(threadIdx.x & 31) == __ffs(same) - 1 && mn != 0x7fffffff && mn < first[s]) atomicMin(&first[s], mn);
    }
};

struct BCountOffLine {
    const double *xy;
    const int *vset;
    const SetDesc *sets;
    const int *first;
    int *offline;
    __device__ void operator()(long long i) const
    {
        int v = (int)i, s = vset[v], b = sets[s].vbase, j = first[s];
        if (j == 0x7fffffff) return;
        int o = orient2d_filter(xy[2 * b], xy[2 * b + 1], xy[2 * j], xy[2 * j + 1], xy[2 * v], xy[2 * v + 1]);
        if (o == 2) o = orient2d_exact(xy[2 * b], xy[2 * b + 1], xy[2 * j], xy[2 * j + 1], xy[2 * v], xy[2 * v + 1]);
        if (o != 0 && !offline[s]) offline[s] = 1;  // any point off the line: the set is not collinear
    }
};

struct NoneToMax {
    int *a;
    __device__ void operator()(long long i) const
    {
        if (a[i] == 0x7f7f7f7f) a[i] = 0x7fffffff;
    }
};

struct VertexSets {
    const int *vbases;
    int K;
    int *vset;
    __device__ void operator()(long long i) const { vset[i] = find_set(vbases, K, (int)i); }
};

// Morton code of each point's pixel in its set's cell (payload: the input
// index), and the set of the point at a sorted position: two stable sorts,
// by code then by set, number each set's vertices spatially inside the set's
// own id range.
struct BSpatialKeys {
    const double *xy;
    const SetDesc *sets;
    const int *vset;
    unsigned *keys;
    int *vals;
    __device__ void operator()(long long i) const
    {
        const SetDesc &S = sets[vset[i]];
        const int D = S.T - 2 * kMargin;
        const double gx = floor((xy[2 * i] - S.sx) / S.scale), gy = floor((xy[2 * i + 1] - S.sy) / S.scale);
        const unsigned ix = (unsigned)fmin(fmax(gx, 0.0), (double)(D - 1));
        const unsigned iy = (unsigned)fmin(fmax(gy, 0.0), (double)(D - 1));
        unsigned m = 0;
        for (int b = 0; b < 14; b++) m |= ((ix >> b) & 1u) << (2 * b) | ((iy >> b) & 1u) << (2 * b + 1);
        keys[i] = m;
        vals[i] = (int)i;
    }
};

struct SetOfPerm {
    const int *vset, *perm;
    unsigned *keys;
    __device__ void operator()(long long i) const { keys[i] = (unsigned)vset[perm[i]]; }
};

struct BSetupSites {
    const double *xy;
    const int *perm;  // internal vertex -> input index (nullptr: identity)
    const SetDesc *sets;
    const int *vset;
    const int *fbases;  // [K] fake bases (relative to N)
    double2 *opos, *pos;
    short2 *gpix;
    int *idmap;
    uint32_t *occ, *bandocc;
    int8_t *vstate;
    int *vtri, *vround, *anchor, *vsetall;
    int N, K;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        int s = v < N ? vset[v] : find_set(fbases, K, v - N);
        const SetDesc S = sets[s];
        vsetall[v] = s;
        vtri[v] = -1;
        anchor[v] = -1;
        vround[v] = v < N ? 0 : 1;
        double2 o, p;
        int px, py;
        if (v < N) {
            const int src = perm ? perm[v] : v;
            o = make_double2(xy[2 * src], xy[2 * src + 1]);
            if (!S.live) {
                opos[v] = o;
                pos[v] = o;
                gpix[v] = make_short2(0, 0);
                vstate[v] = VS_GONE;  // a set without triangles stays out of the mesh
                return;
            }
            if (!(o.x >= S.minX && o.x <= S.maxX && o.y >= S.minY && o.y <= S.maxY)) set_err(ct, GPUDT_ERR_ARG, src);
            int D = S.T - 2 * kMargin;
            double gx = floor((o.x - S.sx) / S.scale), gy = floor((o.y - S.sy) / S.scale);
            int ix = (int)fmin(fmax(gx, 0.0), (double)(D - 1));
            int iy = (int)fmin(fmax(gy, 0.0), (double)(D - 1));
            p = make_double2(S.sx + ix * S.scale, S.sy + iy * S.scale);
            px = ix + kMargin;
            py = iy + kMargin;
            vstate[v] = VS_UNDECIDED;
        } else {
            const int k = v - N - S.fbase;
            short2 q = RingPixB{S.T, S.nside}(k);
            px = q.x;
            py = q.y;
            p = make_double2(S.sx + (px - kMargin) * S.scale, S.sy + (py - kMargin) * S.scale);
            o = p;
            vstate[v] = VS_FAKE;
        }
        opos[v] = o;
        pos[v] = p;
        gpix[v] = make_short2((short)px, (short)py);
        idmap[S.tex + ((long long)py << S.logT) + px] = v;
        atomicOr(&occ[S.occw + (long long)px * (S.T >> 5) + (py >> 5)], 1u << (py & 31));
        atomicOr(&bandocc[S.band + (long long)px * S.W2 + (py >> 11)], 1u << ((py >> 6) & 31));
    }
    struct RingPixB {
        int T, nside;
        __device__ short2 operator()(int k) const
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
};

struct BMinId {
    const short2 *gpix;
    const SetDesc *sets;
    const int *vset;
    int *idmap;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        const SetDesc &S = sets[vset[v]];
        if (!S.live) return;
        short2 g = gpix[v];
        int *slot = &idmap[S.tex + ((long long)g.y << S.logT) + g.x];
        if (*slot > v) atomicMin(slot, v);
    }
};

struct BClassify {
    const short2 *gpix;
    const SetDesc *sets;
    const int *vset;
    const int *idmap;
    int8_t *vstate;
    int *anchor;
    __device__ void operator()(long long i) const
    {
        int v = (int)i;
        const SetDesc &S = sets[vset[v]];
        if (!S.live) return;
        short2 g = gpix[v];
        int w = idmap[S.tex + ((long long)g.y << S.logT) + g.x];
        if (w != v) {
            vstate[v] = VS_MISSING;
            anchor[v] = w;
        }
    }
};

// triangles whose first vertex belongs to an escalated set are released
struct KillSetTris {
    int4 *tv;
    const int *vsetall, *esc;
    int *freelist;
    Counters *ct;
    __device__ void operator()(long long t) const
    {
        int4 v = tv[t];
        if (v.x < 0 || !esc[vsetall[v.x]]) return;
        tv[t] = make_int4(-1, -1, -1, 0);
        freelist[atomicAdd(&ct->nfree, 1)] = (int)t;
    }
};

// Before the links exist the triangle list is plain vertex triples, so the
// slots released by KillSetTris are reclaimed by compacting the list.
struct AliveFlag {
    const int4 *tv;
    int *flag;
    __device__ void operator()(long long t) const { flag[t] = tv[t].x >= 0 ? 1 : 0; }
};

struct ScatterAlive {
    const int4 *tv;
    const int *flag, *pos;
    int4 *out;
    __device__ void operator()(long long t) const
    {
        if (flag[t]) out[pos[t]] = tv[t];
    }
};

// ------------------------------------------------------- grouped compaction
struct AliveBySet {
    const int4 *tv;
    const int *vsetall;
    unsigned *key;
    int *val;
    Counters *ct;
    __device__ void operator()(long long t) const
    {
        int4 v = tv[t];
        bool alive = v.x >= 0;
        key[t] = alive ? (unsigned)vsetall[v.x] : 0xffffffffu;
        val[t] = (int)t;
        warp_reserve(&ct->nlist, alive ? 1 : 0);  // one atomic per warp on the shared count
    }
};

struct NewIndex {
    const unsigned *key;
    const int *val;
    int *newidx, *tset, *tbase;
    int nalive, nslots, K;
    __device__ void operator()(long long jj) const
    {
        int j = (int)jj;
        int t = val[j];
        if (j < nalive) {
            newidx[t] = j;
            int s = (int)key[j];
            tset[j] = s;
            if (j == 0 || key[j - 1] != key[j]) tbase[s] = j;
        } else {
            newidx[t] = -1;
        }
    }
};

struct FillEmptyBases {
    int *tbase;  // sets without triangles point at the next set's base
    int K, total;
    __device__ void operator()(long long) const
    {
        int next = total;
        for (int s = K - 1; s >= 0; s--) {
            if (tbase[s] < 0) tbase[s] = next;
            next = tbase[s];
        }
        tbase[K] = total;
    }
};

// --------------------------------------------------------------- outputs
// gpudtTriangle records with set-local indices, straight from the compacted
// mesh (cv / cn), so compaction writes no record array of its own.
struct LocalTriangles {
    const int4 *cv, *cn;
    const int *tset, *tbase;
    const SetDesc *sets;
    gpudtTriangle *out;
    __device__ void operator()(long long t) const
    {
        const int4 v = cv[t], n = cn[t];
        const int s = tset[t], tb = tbase[s], vb = sets[s].vbase;
        gpudtTriangle g;
        g.vtx[0] = v.x - vb;
        g.vtx[1] = v.y - vb;
        g.vtx[2] = v.z - vb;
        g.tri[0] = n.x >= 0 ? n.x - (tb << 2) : n.x;
        g.tri[1] = n.y >= 0 ? n.y - (tb << 2) : n.y;
        g.tri[2] = n.z >= 0 ? n.z - (tb << 2) : n.z;
        g.tmp[0] = g.tmp[1] = g.tmp[2] = 0;
        out[t] = g;
    }
};

struct LocalEdges {
    const int4 *edges;
    const int *ero;
    const int2 *enu;
    const int *tset, *tbase;
    galphaEdgeInterval *out;
    __device__ void operator()(long long e) const
    {
        int4 q = edges[e];
        galphaEdgeInterval E;
        E.ro_rank = ero[e];
        E.nu_min_rank = enu[e].x;
        E.nu_max_rank = enu[e].y;
        E.sc = E.ro_rank == 0 ? 0 : 1;
        E.tIndex = q.z - tbase[tset[q.z]];
        E.vOpp = q.w;
        out[e] = E;
    }
};

}  // namespace

int batch_buffers(Ctx &c, BatchDev &B, int K, int N, int V, int cap, int nspec, int ntiles)
{
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t need = al(sizeof(SetDesc) * (size_t)K) + 2 * al(4 * (size_t)(K + 1)) + al(4 * (size_t)N + 4) +
                  al(4 * (size_t)V + 4) + 3 * al(4 * (size_t)(K + 1)) + al(4 * (size_t)cap + 4) +
                  al(4 * (size_t)(K + 1)) + al(4 * (size_t)nspec + 4) + 4 * al(4 * (size_t)(K + 1)) +
                  al(sizeof(gpudtTriangle) * (size_t)cap) + 2 * al(8 * (size_t)(K + 1)) + al(4 * (size_t)(K + 1)) +
                  al(48 * (size_t)(K + 1)) + al(4 * (size_t)(K + 1)) + al(8 * (size_t)(ntiles + 1));
    if (need > B.bytes) {
        if (B.buf) cudaFree(B.buf);
        B.buf = nullptr;
        B.bytes = 0;
        GALPHA_CUDA(cudaMalloc(&B.buf, need));
        B.bytes = need;
    }
    char *p = B.buf;
    auto take = [&](size_t b) {
        char *q = p;
        p += al(b);
        return q;
    };
    B.sets = (SetDesc *)take(sizeof(SetDesc) * (size_t)K);
    B.vbases = (int *)take(4 * (size_t)(K + 1));
    B.fbases = (int *)take(4 * (size_t)(K + 1));
    B.vset = (int *)take(4 * (size_t)N + 4);
    B.vsetall = (int *)take(4 * (size_t)V + 4);
    B.first = (int *)take(4 * (size_t)(K + 1));
    B.offline = (int *)take(4 * (size_t)(K + 1));
    B.esc = (int *)take(4 * (size_t)(K + 1));
    B.tset = (int *)take(4 * (size_t)cap + 4);
    B.tbase = (int *)take(4 * (size_t)(K + 1));
    B.seg = (int *)take(4 * (size_t)nspec + 4);
    B.firstexcl = (int *)take(4 * (size_t)(K + 1));
    B.nd = (int *)take(4 * (size_t)(K + 1));
    B.spec_off = (int *)take(4 * (size_t)(K + 1));
    B.ebase = (int *)take(4 * (size_t)(K + 1));
    B.otri = (gpudtTriangle *)take(sizeof(gpudtTriangle) * (size_t)cap);
    B.qparam = (double *)take(8 * (size_t)(K + 1));
    B.qalpha = (double *)take(8 * (size_t)(K + 1));
    B.qR = (int *)take(4 * (size_t)(K + 1));
    B.qcounts = (int *)take(48 * (size_t)(K + 1));
    B.cellmap = (int *)take(4 * (size_t)(K + 1));
    B.chunk = (int2 *)take(8 * (size_t)(ntiles + 1));
    (void)c;
    return GPUDT_OK;
}

// ------------------------------------------------------------------ driver
// Host plan: texture cell of every set, cells grouped by size, vertex bases.
// Fake ranges are provisional (every set gets a ring) until batch_setup knows
// which sets are degenerate.
int batch_plan(BatchHost &bh, int K, const int *sizes, const double *bounds)
{
    const double density = bh.density;  // a handle setting, kept across batches
    bh = BatchHost();
    bh.density = density;
    bh.K = K;
    bh.sets.resize(K);
    long long N = 0, F = 0;
    for (int s = 0; s < K; s++) {
        if (sizes[s] < 0) return GPUDT_ERR_ARG;
        SetDesc &S = bh.sets[s];
        memset(&S, 0, sizeof(S));
        S.n = sizes[s];
        S.vbase = (int)N;
        N += sizes[s];
        S.minX = bounds[4 * s];
        S.minY = bounds[4 * s + 1];
        S.maxX = bounds[4 * s + 2];
        S.maxY = bounds[4 * s + 3];
        if (!(S.minX <= S.maxX && S.minY <= S.maxY)) return GPUDT_ERR_ARG;
        S.T = cell_size(S.n, bh.density);
        S.logT = 0;
        while ((1 << S.logT) < S.T) S.logT++;
        S.W2 = ((S.T >> 6) + 31) / 32;
        S.nside = (S.T - 1 + kFakeSpacing - 1) / kFakeSpacing;
        S.nfake = 4 * S.nside;
        S.fbase = (int)F;
        F += S.nfake;
        S.live = 1;
        grid_scaling(S.minX, S.minY, S.maxX, S.maxY, S.T, S.scale, S.sx, S.sy);
    }
    if (N + F > 0x3fffffffLL) return GPUDT_ERR_NOMEM;
    bh.N = (int)N;
    bh.Fmax = (int)F;
    // classes in increasing size; cells in set order
    std::vector<int> Ts;
    for (auto &S : bh.sets) Ts.push_back(S.T);
    std::sort(Ts.begin(), Ts.end());
    Ts.erase(std::unique(Ts.begin(), Ts.end()), Ts.end());
    long long tex = 0, occw = 0, band = 0;
    int tiles = 0;
    for (int T : Ts) {
        BatchClass C;
        C.T = T;
        C.logT = 0;
        while ((1 << C.logT) < T) C.logT++;
        C.W2 = ((T >> 6) + 31) / 32;
        C.tex = tex;
        C.occw = occw;
        C.band = band;
        C.tile0 = tiles;
        for (int s = 0; s < K; s++)
            if (bh.sets[s].T == T) {
                SetDesc &S = bh.sets[s];
                S.tex = tex;
                S.occw = occw;
                S.band = band;
                tex += (long long)T * T;
                occw += (long long)T * (T >> 5);
                band += (long long)T * C.W2;
                C.sets.push_back(s);
            }
        C.cells = (int)C.sets.size();
        // island pixel lists index a class's cells with 32-bit integers
        if ((long long)C.cells * T * T > 0x7fffffffLL) return GPUDT_ERR_NOMEM;
        tiles += C.cells * fused_tiles(T);
        bh.classes.push_back(C);
    }
    bh.T2 = tex;
    bh.occw = occw;
    bh.band = band;
    bh.ntiles = tiles;
    return GPUDT_OK;
}

// Degenerate sets (fewer than three distinct points, or all collinear) get no
// fake ring and no triangles; then the sites of all other sets are set up.
int batch_setup(Ctx &c, BatchDev &B, BatchHost &bh, const double *d_xy)
{
    const int K = bh.K, N = bh.N;
    std::vector<int> vb(K + 1), fb(K + 1);
    for (int s = 0; s < K; s++) vb[s] = bh.sets[s].vbase;
    vb[K] = N;
    GALPHA_CUDA(cudaMemcpyAsync(B.vbases, vb.data(), sizeof(int) * (size_t)(K + 1), cudaMemcpyHostToDevice, c.stream));
    GALPHA_CUDA(cudaMemcpyAsync(B.sets, bh.sets.data(), sizeof(SetDesc) * (size_t)K, cudaMemcpyHostToDevice, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(B.first, 0x7f, sizeof(int) * (size_t)K, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(B.offline, 0, sizeof(int) * (size_t)K, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.ctr, 0, sizeof(Counters), c.stream));
    launch_n(c, VertexSets{B.vbases, K, B.vset}, N);
    launch_n(c, BFirstDistinct{d_xy, B.vset, B.sets, B.first}, N);
    // atomicMin above starts from 0x7f7f7f7f; mark "none" as 0x7fffffff for the next kernel
    launch_n(c, NoneToMax{B.first}, K);
    launch_n(c, BCountOffLine{d_xy, B.vset, B.sets, B.first, B.offline}, N);
    std::vector<int> off(K);
    GALPHA_CUDA(cudaMemcpyAsync(off.data(), B.offline, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    long long F = 0;
    for (int s = 0; s < K; s++) {
        SetDesc &S = bh.sets[s];
        S.live = (S.n >= 3 && off[s] > 0) ? 1 : 0;
        S.fbase = (int)F;
        if (!S.live) S.nfake = 0;
        F += S.nfake;
        fb[s] = S.fbase;
    }
    fb[K] = (int)F;
    c.N = N;
    c.F = (int)F;
    c.V = N + (int)F;
    c.T = 0;
    c.logT = 0;
    GALPHA_CUDA(cudaMemcpyAsync(B.fbases, fb.data(), sizeof(int) * (size_t)(K + 1), cudaMemcpyHostToDevice, c.stream));
    GALPHA_CUDA(cudaMemcpyAsync(B.sets, bh.sets.data(), sizeof(SetDesc) * (size_t)K, cudaMemcpyHostToDevice, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.occ, 0, sizeof(uint32_t) * (size_t)bh.occw, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.bandocc, 0, sizeof(uint32_t) * (size_t)bh.band, c.stream));
    // spatial numbering inside each set
    c.renumbered = N > 1;
    if (c.renumbered) {
        unsigned *k1 = (unsigned *)c.keys, *k2 = (unsigned *)c.keys2;
        launch_n(c, BSpatialKeys{d_xy, B.sets, B.vset, k1, c.perm}, N);
        int r = radix_sort32(c, k1, c.perm, k2, c.vals2, N, c.rhist);
        if (r) return r;
        launch_n(c, SetOfPerm{B.vset, c.perm, k1}, N);
        r = radix_sort32(c, k1, c.perm, k2, c.vals2, N, c.rhist);
        if (r) return r;
    }
    BSetupSites st;
    st.xy = d_xy;
    st.perm = c.renumbered ? c.perm : nullptr;
    st.sets = B.sets;
    st.vset = B.vset;
    st.fbases = B.fbases;
    st.opos = c.opos;
    st.pos = c.pos;
    st.gpix = c.gpix;
    st.idmap = c.idmap;
    st.occ = c.occ;
    st.bandocc = c.bandocc;
    st.vstate = c.vstate;
    st.vtri = c.vtri;
    st.vround = c.vround;
    st.anchor = c.anchor;
    st.vsetall = B.vsetall;
    st.N = N;
    st.K = K;
    st.ct = c.ctr;
    launch_n(c, st, c.V);
    launch_n(c, BMinId{c.gpix, B.sets, B.vset, c.idmap}, N);
    launch_n(c, BClassify{c.gpix, B.sets, B.vset, c.idmap, c.vstate, c.anchor}, N);
    GALPHA_CUDA(cudaGetLastError());
    int r = read_counters(c);
    if (r) return r;
    return c.hctr->err;
}

// Colouring + dual triangles, per cell size.  Cells whose interior is mostly
// empty (holes, gaps between clusters) make the window scan of the fused
// kernel long and its islands frequent; they take the envelope path
// (per-row lower envelope, cost independent of emptiness).  So does a cell
// whose island repair cannot stay local.
int batch_voronoi(Ctx &c, BatchDev &B, BatchHost &bh)
{
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->ntris, 0, 2 * sizeof(int), c.stream));  // ntris, nfree
    int *const colour0 = c.colour;
    int16_t *const ycol0 = c.ycol;
    int *const idmap0 = c.idmap;
    for (auto &C : bh.classes) {
        std::vector<int> fused, env;  // launch lists of cell indices within the class
        std::vector<int> occ(C.cells, 0);
        int r = launch_column_pass_cells(c, C.T, C.W2, C.cells, c.occ + C.occw, c.bandocc + C.band, c.ycol + C.tex);
        if (r) return r;
        r = cell_occupancy(c, c.bandocc + C.band, C.T, C.W2, C.cells, B.esc, occ.data());
        if (r) return r;
        for (int z = 0; z < C.cells; z++) {
            const SetDesc &S = bh.sets[C.sets[z]];
            if (!S.live) continue;
            const double D = S.T - 2 * kMargin;
            const bool dense = (double)S.n * 256.0 >= D * D;
            const bool filled = occupancy_ok(C.T, occ[z]);
            (dense && filled ? fused : env).push_back(z);
        }
        if (!fused.empty()) {
            const int nf = (int)fused.size();
            GALPHA_CUDA(cudaMemcpyAsync(B.cellmap, fused.data(), sizeof(int) * (size_t)nf, cudaMemcpyHostToDevice,
                                        c.stream));
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nisland, 0, sizeof(int), c.stream));
            r = launch_vd_tri_cells(c, C.T, C.logT, nf, c.ycol + C.tex, c.idmap + C.tex, B.chunk, c.list2, B.cellmap);
            if (r) return r;
            r = read_counters(c);
            if (r) return r;
            if (c.hctr->err) return c.hctr->err;
            const int nflag = c.hctr->nisland;
            c.st.nRepairTiles += nflag;
            if (nflag > 0) {
                GALPHA_CUDA(cudaMemsetAsync(&c.ctr->escalate, 0, sizeof(int), c.stream));
                GALPHA_CUDA(cudaMemsetAsync(B.esc, 0, sizeof(int) * (size_t)nf, c.stream));
                r = launch_vd_repair_cells(c, nflag, C.T, C.logT, nf, c.ycol + C.tex, c.idmap + C.tex, B.esc,
                                           B.cellmap, B.chunk);
                if (r) return r;
                r = read_counters(c);
                if (r) return r;
                if (c.hctr->err) return c.hctr->err;
                if (c.hctr->escalate) {
                    // drop the escalated cells' triangles, reclaim their slots,
                    // and colour those cells on the envelope path below
                    std::vector<int> esc(nf), setesc(bh.K, 0);
                    GALPHA_CUDA(cudaMemcpyAsync(esc.data(), B.esc, sizeof(int) * (size_t)nf, cudaMemcpyDeviceToHost,
                                                c.stream));
                    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
                    for (int k = 0; k < nf; k++)
                        if (esc[k]) {
                            setesc[C.sets[fused[k]]] = 1;
                            env.push_back(fused[k]);
                            c.st.nEscalated++;
                        }
                    GALPHA_CUDA(cudaMemcpyAsync(B.offline, setesc.data(), sizeof(int) * (size_t)bh.K,
                                                cudaMemcpyHostToDevice, c.stream));
                    const int nt = c.hctr->ntris;
                    launch_n(c, KillSetTris{c.tv, B.vsetall, B.offline, c.freelist, c.ctr}, nt);
                    launch_n(c, AliveFlag{c.tv, c.aux}, nt);
                    r = exclusive_scan_int(c, c.aux, c.aux2, nt, &c.ctr->ntris);
                    if (r) return r;
                    launch_n(c, ScatterAlive{c.tv, c.aux, c.aux2, c.tn}, nt);
                    r = read_counters(c);
                    if (r) return r;
                    GALPHA_CUDA(cudaMemcpyAsync(c.tv, c.tn, sizeof(int4) * (size_t)c.hctr->ntris,
                                                cudaMemcpyDeviceToDevice, c.stream));
                    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nfree, 0, sizeof(int), c.stream));
                }
            }
        }
        if (!env.empty()) {
            const int ne = (int)env.size();
            GALPHA_CUDA(cudaMemcpyAsync(B.cellmap, env.data(), sizeof(int) * (size_t)ne, cudaMemcpyHostToDevice,
                                        c.stream));
            c.T = C.T;
            c.logT = C.logT;
            c.ycol = ycol0 + C.tex;
            c.idmap = idmap0 + C.tex;
            c.colour = colour0 + C.tex;
            r = voronoi_global(c, ne, B.cellmap);
            if (!r) {
                r = read_counters(c);
                if (!r) r = emit_global(c, c.hctr->ntris, ne, B.cellmap);
            }
            c.ycol = ycol0;
            c.idmap = idmap0;
            c.colour = colour0;
            c.T = 0;
            c.logT = 0;
            if (r) return r;
            c.st.nEnvelopeCells += ne;
        }
    }
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

// Compaction with the triangles grouped by set (stable: slot order within a set).
int batch_compact(Ctx &c, BatchDev &B, BatchHost &bh)
{
    int r = read_counters(c);
    if (r) return r;
    const int nt = c.hctr->ntris;
    unsigned *ka = (unsigned *)c.keys, *kb = (unsigned *)c.keys2;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
    launch_n(c, AliveBySet{c.tv, B.vsetall, ka, c.vals, c.ctr}, nt);
    r = radix_sort32(c, ka, c.vals, kb, c.vals2, nt, c.rhist);
    if (r) return r;
    r = read_counters(c);
    if (r) return r;
    const int nalive = c.hctr->nlist;
    GALPHA_CUDA(cudaMemsetAsync(B.tbase, 0xff, sizeof(int) * (size_t)(bh.K + 1), c.stream));
    launch_n(c, NewIndex{ka, c.vals, c.aux2, B.tset, B.tbase, nalive, nt, bh.K}, nt);
    launch_n(c, FillEmptyBases{B.tbase, bh.K, nalive}, 1);
    launch_compact_gather(c, c.vals, c.aux2, nalive);
    GALPHA_CUDA(cudaGetLastError());
    c.nT_out = nalive;
    bh.tbase.resize(bh.K + 1);
    GALPHA_CUDA(cudaMemcpyAsync(bh.tbase.data(), B.tbase, sizeof(int) * (size_t)(bh.K + 1), cudaMemcpyDeviceToHost,
                                c.stream));
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    return GPUDT_OK;
}

// Triangles and edge intervals with set-local vertex and triangle indices.
int batch_local_outputs(Ctx &c, BatchDev &B, gpudtTriangle *tris, galphaEdgeInterval *edges)
{
    if (tris && c.nT_out > 0) launch_n(c, LocalTriangles{c.cv, c.cn, B.tset, B.tbase, B.sets, tris}, c.nT_out);
    if (edges && c.nE > 0)
        launch_n(c, LocalEdges{c.edges, c.edge_ro, c.edge_nu, B.tset, B.tbase, edges}, c.nE);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

}  // namespace galpha
