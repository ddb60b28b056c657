// master.cu -- the master list and spectrum pointers of the alpha complex.
//
// Restates compute_master_list (Alpha_Shapes_2D.cu:641-727) and the kernel
// computeMasterList (kernel.cu:626-690): entry k of the unsorted list is
//   k <  2N            vertex k/2, at = nu_min (k even) or nu_max (k odd)
//   k <  2N + 3E       edge (k-2N)/3, at = ro, nu_min, nu_max
//   k <  2N + 3E + T   triangle k-2N-3E, at = ro
// with the rank of that interval end as key.  The reference sorts the keys
// with thrust::sort_by_key (a stable radix sort for int keys), removes rank-0
// entries (remove_if keeps order) and takes the first index of every run of
// equal ranks (unique_by_key on a sequence), with -1 prepended.  Ranks are >= -1
// (-1: a vertex dropped as a duplicate), so key = rank + 1 orders the same way.
//
// The keys are dense (one per spectrum rank), so the stable sort is a
// counting sort: count the entries of every key, scan the counts into run
// starts, move each entry into its run (two levels, see k_ml_partition /
// k_ml_place), then put every run back in entry order (runs are a few entries
// long: an insertion sort per run; the rare long runs -- exact ties on
// lattices, dropped duplicates -- are radix-sorted as sub-arrays).  The
// spectrum pointers are the run starts.  Keys outside [0, nSpec] (a batch's
// segmented ranks) take an LSD sort of the whole list instead.
#include <algorithm>
#include <mutex>

#include "internal.cuh"

namespace galpha {
namespace {

struct MasterKeys {
    const int2 *pt;
    const int *edge_ro;
    const int2 *edge_nu;
    const int *tri_ro;
    unsigned *keys;
    int *vals;
    int N, nE;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int k = (int)ii;
        int r;
        if (k < 2 * N) {
            int2 v = pt[k >> 1];
            r = (k & 1) ? v.y : v.x;
        } else if (k < 2 * N + 3 * nE) {
            int q = k - 2 * N, e = q / 3, at = q - 3 * e;
            r = at == 0 ? edge_ro[e] : (at == 1 ? edge_nu[e].x : edge_nu[e].y);
        } else {
            r = tri_ro[k - 2 * N - 3 * nE];
        }
        keys[k] = (unsigned)(r + 1);
        vals[k] = k;
        // counts of the rank -1 and rank 0 runs (warp-aggregated)
        int bin = r < 0 ? 0 : (r == 0 ? 1 : 2);
        unsigned peers = __match_any_sync(__activemask(), bin);
        if (bin < 2 && (peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0)
            atomicAdd(bin == 0 ? &ct->nlist : &ct->nlist2, __popc(peers));
    }
};

__device__ __forceinline__ galphaAlpha decode_entry(int k, int N, int nE)
{
    galphaAlpha a;
    if (k < 2 * N) {
        a.simplex_index = k >> 1;
        a.st = 2;             // VERTEX
        a.at = 1 + (k & 1);   // nu_min, nu_max
    } else if (k < 2 * N + 3 * nE) {
        int q = k - 2 * N, e = q / 3;
        a.simplex_index = e;
        a.st = 0;             // EDGE
        a.at = q - 3 * e;     // ro, nu_min, nu_max
    } else {
        a.simplex_index = k - 2 * N - 3 * nE;
        a.st = 1;             // TRIANGLE
        a.at = 0;             // ro
    }
    return a;
}

// Output index i reads sorted position i (the rank -1 run) or i + nzero.
struct MasterWrite {
    const unsigned *keys;
    const int *vals;
    galphaAlpha *out;
    int *runstart;
    int nneg, nzero, N, nE;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        int src = i < nneg ? i : i + nzero;
        out[i] = decode_entry(vals[src], N, nE);
        int prev = i - 1 < nneg ? i - 1 : i - 1 + nzero;
        runstart[i] = (i == 0 || keys[src] != keys[prev]) ? 1 : 0;
    }
};

struct SpecPointers {
    const int *runstart, *pos;
    int *sp;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        if (i == 0) sp[0] = -1;
        if (runstart[i]) sp[1 + pos[i]] = i;
    }
};


constexpr int kMaxShortRun = 64;    // runs put in order by one thread
constexpr int kMaxLongRuns = 4096;  // longer runs sorted as sub-arrays, else the LSD path

__device__ __forceinline__ int master_rank(int k, const int2 *pt, const int *edge_ro, const int2 *edge_nu,
                                           const int *tri_ro, int N, int nE)
{
    if (k < 2 * N) {
        const int2 v = pt[k >> 1];
        return (k & 1) ? v.y : v.x;
    }
    if (k < 2 * N + 3 * nE) {
        const int q = k - 2 * N, e = q / 3, at = q - 3 * e;
        return at == 0 ? edge_ro[e] : (at == 1 ? edge_nu[e].x : edge_nu[e].y);
    }
    return tri_ro[k - 2 * N - 3 * nE];
}

// cnt[rank + 1] += 1 for every entry of rank != 0; an out-of-range key sets
// ct->changed (the LSD path then runs instead).
struct MasterCount {
    const int2 *pt;
    const int *edge_ro;
    const int2 *edge_nu;
    const int *tri_ro;
    int *cnt;
    int N, nE, nK;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int r = master_rank((int)ii, pt, edge_ro, edge_nu, tri_ro, N, nE);
        if (r == 0) return;
        const int K = r + 1;
        if (K < 0 || K >= nK) {
            ct->changed = 1;
            return;
        }
        atomicAdd(&cnt[K], 1);
    }
};

// Two-level placement.  Ranks are grouped into buckets of kBucket
// consecutive keys; a bucket's entries occupy one contiguous range of the
// list (its runs' starts come from the count scan).  k_ml_partition moves
// every entry (key, index) into its bucket's range, a tile at a time (block
// histogram, one reservation per bucket and tile), and k_ml_place then
// places one bucket per block in shared memory, puts every run of it in
// entry order and writes the bucket out in one coalesced pass.  The random
// part of the permutation thus happens in shared memory, not as scattered
// 4-byte stores to HBM.
constexpr int kBucketBits = 13, kBucket = 1 << kBucketBits;
constexpr int kPartTile = 8192, kPartThreads = 256;
constexpr int kMaxBuckets = 4096;
constexpr int kPlaceCap = 40960, kPlaceThreads = 512;  // entries of a bucket placed in shared memory

struct BucketCursors {
    const int *start;
    int *gcur;
    int nK;
    __device__ void operator()(long long b) const { gcur[b] = start[min((long long)nK, b * kBucket)]; }
};

__global__ void __launch_bounds__(kPartThreads) k_ml_partition(const int2 *__restrict__ pt,
                                                               const int *__restrict__ edge_ro,
                                                               const int2 *__restrict__ edge_nu,
                                                               const int *__restrict__ tri_ro, int N, int nE,
                                                               long long M, int nK, int nb, int *gcur, int2 *P)
{
    extern __shared__ int ml_part[];
    int *Ks = ml_part, *loc = Ks + kPartTile, *h = loc + kPartTile, *gb = h + nb;
    const long long t0 = (long long)blockIdx.x * kPartTile;
    for (int i = threadIdx.x; i < nb; i += kPartThreads) h[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < kPartTile; i += kPartThreads) {
        const long long k = t0 + i;
        int K = -1;
        if (k < M) {
            const int r = master_rank((int)k, pt, edge_ro, edge_nu, tri_ro, N, nE);
            if (r != 0 && r + 1 >= 0 && r + 1 < nK) K = r + 1;
        }
        Ks[i] = K;
        if (K >= 0) loc[i] = atomicAdd(&h[K >> kBucketBits], 1);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += kPartThreads)
        if (h[b]) gb[b] = atomicAdd(&gcur[b], h[b]);
    __syncthreads();
    for (int i = threadIdx.x; i < kPartTile; i += kPartThreads) {
        const int K = Ks[i];
        if (K >= 0) P[gb[K >> kBucketBits] + loc[i]] = make_int2(K, (int)(t0 + i));
    }
}

// Puts run [bgn, end) of a (shared or global) array in entry order, or lists
// it for a sub-array sort when it is longer than kMaxShortRun.
__device__ __forceinline__ void ml_order_run(int *a, int bgn, int end, int gofs, int *longs, Counters *ct)
{
    if (end - bgn <= 1) return;
    if (end - bgn > kMaxShortRun) {
        const int q = atomicAdd(&ct->nlong, 1);
        if (q < kMaxLongRuns) {
            longs[2 * q] = gofs + bgn;
            longs[2 * q + 1] = gofs + end;
        }
        return;
    }
    for (int i = bgn + 1; i < end; i++) {
        const int x = a[i];
        int j = i - 1;
        while (j >= bgn && a[j] > x) {
            a[j + 1] = a[j];
            j--;
        }
        a[j + 1] = x;
    }
}

__global__ void __launch_bounds__(kPlaceThreads) k_ml_place(const int2 *__restrict__ P, const int *__restrict__ start,
                                                            int nK, int *slot, int *nonempty, int *gcurK,
                                                            int *longs, Counters *ct)
{
    extern __shared__ int ml_place[];
    int *cur = ml_place, *out = cur + kBucket;
    const int K0 = blockIdx.x * kBucket, K1 = min(K0 + kBucket, nK);
    const int s0 = start[K0], n = start[K1] - s0;
    if (n <= kPlaceCap) {
        for (int j = threadIdx.x; j < K1 - K0; j += kPlaceThreads) cur[j] = start[K0 + j] - s0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kPlaceThreads) {
            const int2 e = P[s0 + i];
            out[atomicAdd(&cur[e.x - K0], 1)] = e.y;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < K1 - K0; j += kPlaceThreads) {
            const int bgn = start[K0 + j] - s0, end = cur[j];
            nonempty[K0 + j] = end > bgn ? 1 : 0;
            ml_order_run(out, bgn, end, s0, longs, ct);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kPlaceThreads) slot[s0 + i] = out[i];
    } else {  // a bucket too large for shared memory: the same steps in HBM
        for (int j = threadIdx.x; j < K1 - K0; j += kPlaceThreads) gcurK[K0 + j] = start[K0 + j];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kPlaceThreads) {
            const int2 e = P[s0 + i];
            slot[atomicAdd(&gcurK[e.x], 1)] = e.y;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < K1 - K0; j += kPlaceThreads) {
            const int bgn = start[K0 + j], end = gcurK[K0 + j];
            nonempty[K0 + j] = end > bgn ? 1 : 0;
            ml_order_run(slot, bgn, end, 0, longs, ct);
        }
    }
}

struct MasterDecode {
    const int *slot;
    galphaAlpha *out;
    int N, nE;
    __device__ void operator()(long long i) const { out[i] = decode_entry(slot[i], N, nE); }
};

struct RunPointers {
    const int *start, *nonempty, *pos;
    int *sp;
    __device__ void operator()(long long ii) const
    {
        const int K = (int)ii;
        if (K == 0) sp[0] = -1;
        if (nonempty[K]) sp[1 + pos[K]] = start[K];
    }
};
}  // namespace

static int master_list_radix(Ctx &c)
{
    const long long M = 2LL * c.N + 3LL * c.nE + c.nT_out;
    if (M > 0x7fffffffLL) return GPUDT_ERR_NOMEM;
    const long long scr = radix_scratch_ints(M);
    // keys, keys2 (u32), vals, vals2, runstart, pos (int), out (12 B), sp (int), scratch
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t need = 6 * al(4 * (size_t)(M + 1)) + al(sizeof(galphaAlpha) * (size_t)(M + 1)) +
                        al(4 * (size_t)(M + 2)) + al(4 * (size_t)scr);
    if (need > c.ml_bytes) {
        if (c.ml_buf) cudaFree(c.ml_buf);
        c.ml_buf = nullptr;
        c.ml_bytes = 0;
        GALPHA_CUDA(cudaMalloc(&c.ml_buf, need));
        c.ml_bytes = need;
    }
    char *p = c.ml_buf;
    auto take = [&](size_t b) {
        char *q = p;
        p += al(b);
        return q;
    };
    unsigned *keys = (unsigned *)take(4 * (size_t)(M + 1));
    unsigned *keys2 = (unsigned *)take(4 * (size_t)(M + 1));
    int *vals = (int *)take(4 * (size_t)(M + 1));
    int *vals2 = (int *)take(4 * (size_t)(M + 1));
    int *runstart = (int *)take(4 * (size_t)(M + 1));
    int *pos = (int *)take(4 * (size_t)(M + 1));
    c.ml_out = (galphaAlpha *)take(sizeof(galphaAlpha) * (size_t)(M + 1));
    c.ml_sp = (int *)take(4 * (size_t)(M + 2));
    int *scratch = (int *)take(4 * (size_t)scr);

    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, 2 * sizeof(int), c.stream));  // nlist, nlist2
    launch_n(c, MasterKeys{c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, keys, vals, c.N, c.nE, c.ctr}, M);
    int r = radix_sort32(c, keys, vals, keys2, vals2, (int)M, scratch);
    if (r) return r;
    r = read_counters(c);
    if (r) return r;
    const int nneg = c.hctr->nlist, nzero = c.hctr->nlist2;
    const int nout = (int)M - nzero;
    launch_n(c, MasterWrite{keys, vals, c.ml_out, runstart, nneg, nzero, c.N, c.nE}, nout);
    r = exclusive_scan_int(c, runstart, pos, nout, &c.ctr->nlist);
    if (r) return r;
    launch_n(c, SpecPointers{runstart, pos, c.ml_sp}, nout);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    c.nMaster = nout;
    c.nSpecPtr = 1 + (nout > 0 ? c.hctr->nlist : 0);
    c.have_master = true;
    return GPUDT_OK;
}

int master_list(Ctx &c)
{
    const long long M = 2LL * c.N + 3LL * c.nE + c.nT_out;
    if (M > 0x7fffffffLL) return GPUDT_ERR_NOMEM;
    const long long nK = (long long)c.nSpec + 1;  // keys rank + 1 in [0, nSpec]
    const long long nb = (nK + kBucket - 1) / kBucket;
    if (M == 0 || nb > kMaxBuckets) return master_list_radix(c);
    {
        static std::mutex mu;
        static bool attr_set[64];
        std::lock_guard<std::mutex> lk(mu);
        if (c.device < 0 || c.device >= 64 || !attr_set[c.device]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_ml_partition, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(int) * (2 * kPartTile + 2 * kMaxBuckets)));
            GALPHA_CUDA(cudaFuncSetAttribute(k_ml_place, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(int) * (kBucket + kPlaceCap)));
            if (c.device >= 0 && c.device < 64) attr_set[c.device] = true;
        }
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const long long scr = radix_scratch_ints(M);
    // slot, P (2 ints per entry; later the sub-sorts' second keys and values),
    // sval2 (int); start, nonempty, pos, gcurK (nK + 1 ints each); bucket
    // cursors; long-run extents; out (12 B); sp; sort scratch
    const size_t need = al(4 * (size_t)M) * 4 + al(4 * (size_t)(nK + 1)) * 4 + al(4 * (size_t)nb) +
                        al(8 * (size_t)kMaxLongRuns) + al(sizeof(galphaAlpha) * (size_t)M) +
                        al(4 * (size_t)(nK + 2)) + al(4 * (size_t)scr);
    if (need > c.ml_bytes) {
        if (c.ml_buf) cudaFree(c.ml_buf);
        c.ml_buf = nullptr;
        c.ml_bytes = 0;
        GALPHA_CUDA(cudaMalloc(&c.ml_buf, need));
        c.ml_bytes = need;
    }
    char *p = c.ml_buf;
    auto take = [&](size_t b) {
        char *q = p;
        p += al(b);
        return q;
    };
    int *slot = (int *)take(4 * (size_t)M);
    int2 *P = (int2 *)take(8 * (size_t)M);
    int *sval2 = (int *)take(4 * (size_t)M);
    int *start = (int *)take(4 * (size_t)(nK + 1));
    int *nonempty = (int *)take(4 * (size_t)(nK + 1));
    int *pos = (int *)take(4 * (size_t)(nK + 1));
    int *gcurK = (int *)take(4 * (size_t)(nK + 1));
    int *gcur = (int *)take(4 * (size_t)nb);
    int *longs = (int *)take(8 * (size_t)kMaxLongRuns);
    c.ml_out = (galphaAlpha *)take(sizeof(galphaAlpha) * (size_t)M);
    c.ml_sp = (int *)take(4 * (size_t)(nK + 2));
    int *scratch = (int *)take(4 * (size_t)scr);

    GALPHA_CUDA(cudaMemsetAsync(start, 0, 4 * (size_t)(nK + 1), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlong, 0, sizeof(int), c.stream));
    launch_n(c, MasterCount{c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, start, c.N, c.nE, (int)nK, c.ctr}, M);
    // run starts (start[nK] = entries kept, also in nlist)
    int r = exclusive_scan_int(c, start, start, (int)nK + 1, &c.ctr->nlist);
    if (r) return r;
    launch_n(c, BucketCursors{start, gcur, (int)nK}, nb);
    k_ml_partition<<<(unsigned)((M + kPartTile - 1) / kPartTile), kPartThreads,
                     sizeof(int) * (2 * kPartTile + 2 * (size_t)nb), c.stream>>>(
        c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, c.N, c.nE, M, (int)nK, (int)nb, gcur, P);
    count_launch();
    k_ml_place<<<(unsigned)nb, kPlaceThreads, sizeof(int) * (kBucket + kPlaceCap), c.stream>>>(
        P, start, (int)nK, slot, nonempty, gcurK, longs, c.ctr);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->changed || c.hctr->nlong > kMaxLongRuns) return master_list_radix(c);
    const int nout = c.hctr->nlist, nlong = c.hctr->nlong;
    if (nlong > 0) {
        int *skey2 = (int *)P, *sval = (int *)P + M;  // P is free after the placement
        int hl[2 * 64];
        for (int q0 = 0; q0 < nlong; q0 += 64) {  // the long runs' extents, 64 at a time
            const int qn = std::min(64, nlong - q0);
            r = read_small(c, hl, longs + 2 * q0, sizeof(int) * 2 * (size_t)qn);
            if (r) return r;
            for (int q = 0; q < qn; q++) {
                const int b = hl[2 * q], e = hl[2 * q + 1];
                // entry indices are distinct: sorting them as keys is the stable order
                r = radix_sort32(c, (unsigned *)slot + b, sval + b, (unsigned *)skey2 + b, sval2 + b, e - b,
                                 scratch);
                if (r) return r;
            }
        }
    }
    launch_n(c, MasterDecode{slot, c.ml_out, c.N, c.nE}, nout);
    r = exclusive_scan_int(c, nonempty, pos, (int)nK, &c.ctr->nlist2);
    if (r) return r;
    launch_n(c, RunPointers{start, nonempty, pos, c.ml_sp}, nK);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    c.nMaster = nout;
    c.nSpecPtr = 1 + (nout > 0 ? c.hctr->nlist2 : 0);
    c.have_master = true;
    return GPUDT_OK;
}

}  // namespace galpha
