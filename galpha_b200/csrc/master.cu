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
// starts, drop each entry into its run by an atomic cursor, then put every
// run back in entry order (runs are a few entries long: an insertion sort per
// run; the rare long runs -- exact ties on lattices, dropped duplicates -- are
// radix-sorted as sub-arrays).  The spectrum pointers are the run starts.
// That is one read of the ranks per pass instead of four full passes of an
// LSD sort.  Keys outside [0, nSpec] (a batch's segmented ranks) take the LSD
// sort of the whole list instead.
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

// Entry k goes to the next free place of its run; cur[K] starts at the run's
// start and ends at the next run's start.
struct MasterPlace {
    const int2 *pt;
    const int *edge_ro;
    const int2 *edge_nu;
    const int *tri_ro;
    int *cur, *slot;
    int N, nE, nK;
    __device__ void operator()(long long ii) const
    {
        const int k = (int)ii;
        const int r = master_rank(k, pt, edge_ro, edge_nu, tri_ro, N, nE);
        if (r == 0) return;
        const int K = r + 1;
        if (K < 0 || K >= nK) return;
        slot[atomicAdd(&cur[K], 1)] = k;
    }
};

// Run K is slot[end[K-1] .. end[K]) (end[-1] = 0): short runs are put in entry
// order here; long ones are listed (begin, end) for a sub-array sort.
// nonempty[K] marks the runs that exist (their starts are the spectrum
// pointers).
struct MasterRuns {
    const int *end;
    int *slot, *nonempty, *longs;
    int nK;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int K = (int)ii;
        const int b = K == 0 ? 0 : end[K - 1], e = end[K];
        nonempty[K] = e > b ? 1 : 0;
        if (e - b <= 1) return;
        if (e - b > kMaxShortRun) {
            const int q = atomicAdd(&ct->nlong, 1);
            if (q < kMaxLongRuns) {
                longs[2 * q] = b;
                longs[2 * q + 1] = e;
            }
            return;
        }
        for (int i = b + 1; i < e; i++) {
            const int x = slot[i];
            int j = i - 1;
            while (j >= b && slot[j] > x) {
                slot[j + 1] = slot[j];
                j--;
            }
            slot[j + 1] = x;
        }
    }
};

struct MasterDecode {
    const int *slot;
    galphaAlpha *out;
    int N, nE;
    __device__ void operator()(long long i) const { out[i] = decode_entry(slot[i], N, nE); }
};

struct RunPointers {
    const int *end, *nonempty, *pos;
    int *sp;
    __device__ void operator()(long long ii) const
    {
        const int K = (int)ii;
        if (K == 0) sp[0] = -1;
        if (nonempty[K]) sp[1 + pos[K]] = K == 0 ? 0 : end[K - 1];
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
    if (M == 0 || nK > 0x3fffffffLL) return master_list_radix(c);
    // slot, sub-sort keys2 / vals / vals2 (int), cnt (run starts, then ends),
    // nonempty, pos (int), long-run extents, out (12 B), sp (int), sort scratch
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const long long scr = radix_scratch_ints(M);
    const size_t need = al(4 * (size_t)M) * 4 + al(4 * (size_t)(nK + 1)) * 3 + al(8 * (size_t)kMaxLongRuns) +
                        al(sizeof(galphaAlpha) * (size_t)M) + al(4 * (size_t)(nK + 2)) + al(4 * (size_t)scr);
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
    int *skey2 = (int *)take(4 * (size_t)M);
    int *sval = (int *)take(4 * (size_t)M);
    int *sval2 = (int *)take(4 * (size_t)M);
    int *cnt = (int *)take(4 * (size_t)(nK + 1));
    int *nonempty = (int *)take(4 * (size_t)(nK + 1));
    int *pos = (int *)take(4 * (size_t)(nK + 1));
    int *longs = (int *)take(8 * (size_t)kMaxLongRuns);
    c.ml_out = (galphaAlpha *)take(sizeof(galphaAlpha) * (size_t)M);
    c.ml_sp = (int *)take(4 * (size_t)(nK + 2));
    int *scratch = (int *)take(4 * (size_t)scr);

    GALPHA_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)(nK + 1), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlong, 0, sizeof(int), c.stream));
    launch_n(c, MasterCount{c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, cnt, c.N, c.nE, (int)nK, c.ctr}, M);
    int r = exclusive_scan_int(c, cnt, cnt, (int)nK, &c.ctr->nlist);  // run starts; nlist = entries kept
    if (r) return r;
    launch_n(c, MasterPlace{c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, cnt, slot, c.N, c.nE, (int)nK}, M);
    launch_n(c, MasterRuns{cnt, slot, nonempty, longs, (int)nK, c.ctr}, nK);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->changed || c.hctr->nlong > kMaxLongRuns) return master_list_radix(c);
    const int nout = c.hctr->nlist, nlong = c.hctr->nlong;
    if (nlong > 0) {
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
    launch_n(c, RunPointers{cnt, nonempty, pos, c.ml_sp}, nK);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    c.nMaster = nout;
    c.nSpecPtr = 1 + (nout > 0 ? c.hctr->nlist2 : 0);
    c.have_master = true;
    return GPUDT_OK;
}

}  // namespace galpha
