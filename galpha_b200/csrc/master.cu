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
// (-1: a vertex dropped as a duplicate), so key = rank + 1 as an unsigned
// 32-bit integer sorts in the same order; the stable LSD radix sort of
// sort.cu gives the same permutation, and the rank-0 entries form one
// contiguous run (key 1) that the output pass skips.
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

}  // namespace

int master_list(Ctx &c)
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

}  // namespace galpha
