// alpha.cu -- alpha spectrum and per-simplex intervals on the device.
//
// Stage map (reference -> here):
//   computeTriEdgeCount + exclusive_scan +          k_edge_count + scan: the reference's
//   computeEdgeTriMap (kernel.cu:138-217)           ownership and numbering rule
//   computeTriangleRo / computeEdgeRo /             k_tri_keys / k_edge_keys: birth times in
//   processAttached (kernel.cu:219-358,             double-double (<= 1 ulp, certified),
//   predicates.h:1297-1444)                         slivers recomputed exactly; attached test
//                                                   filtered then exact (closed disc)
//   thrust::remove_if x2 (Alpha_Shapes_2D.cu:       unattached edges compacted by a scan
//   276-281)
//   thrust::sort_by_key (Alpha_Shapes_2D.cu:317)    radix_sort: LSD radix sort of the FP64
//                                                   bit patterns with an int payload
//   markSpectrum + sorT odd-even rounds +           k_mark_runs / k_resolve_runs: every run
//   CPU_insertion_sort (kernel.cu:785-1102,         of keys within 2 ulp is sorted with the
//   Alpha_Shapes_2D.cu:344-610)                     exact comparator on the device; exact
//                                                   ties share a rank
//   processSpectrum / remove_if / UpdateBackRefs    scan of "new rank" flags + k_scatter_ranks
//   (kernel.cu:360-401, Alpha_Shapes_2D.cu:483-512)
//   edgeIntervals / computeVertexIntervals          k_edge_intervals / k_vertex_intervals:
//   (kernel.cu:427-624)                             vertex min/max by atomics over edges
#include <cstdio>
#include <algorithm>
#include <vector>
#include "internal.cuh"
#include "exact.cuh"

namespace galpha {

// ------------------------------------------------------------ double-double
struct dd {
    double h, l;
};

__device__ __forceinline__ dd dd_from_diff(double a, double b)
{
    dd r;
    two_sum(a, -b, r.h, r.l);
    return r;
}

__device__ __forceinline__ dd dd_mul(dd a, dd b)
{
    double p, e;
    two_prod(a.h, b.h, p, e);
    e = fma(a.h, b.l, e);
    e = fma(a.l, b.h, e);
    dd r;
    fast_two_sum(p, e, r.h, r.l);
    return r;
}

__device__ __forceinline__ dd dd_add(dd a, dd b)
{
    double s, e;
    two_sum(a.h, b.h, s, e);
    e += a.l + b.l;
    dd r;
    fast_two_sum(s, e, r.h, r.l);
    return r;
}

__device__ __forceinline__ dd dd_sub(dd a, dd b)
{
    b.h = -b.h;
    b.l = -b.l;
    return dd_add(a, b);
}

__device__ __forceinline__ double dd_div_to_double(dd a, dd b)
{
    double q1 = a.h / b.h;
    dd qb = dd_mul(dd{q1, 0.0}, b);
    dd r = dd_sub(a, qb);
    double q2 = r.h / b.h;
    return q1 + q2;
}

__device__ __forceinline__ dd dd_sqdist(double2 p, double2 q)
{
    dd dx = dd_from_diff(p.x, q.x), dy = dd_from_diff(p.y, q.y);
    return dd_add(dd_mul(dx, dx), dd_mul(dy, dy));
}

// Edge birth time (|pq|/2)^2.
__device__ __forceinline__ double rho_edge(double2 p, double2 q)
{
    dd s = dd_sqdist(p, q);
    return (s.h + s.l) * 0.25;
}

// Triangle birth time R^2 = abc / (4 ar^2); *sliver set when ar is too
// cancelled for the double-double evaluation to certify 1 ulp.
__device__ __forceinline__ double rho_tri(double2 A, double2 B, double2 C, bool *sliver)
{
    dd a = dd_sqdist(A, B), b = dd_sqdist(B, C), c = dd_sqdist(C, A);
    dd N = dd_mul(dd_mul(a, b), c);
    dd ux = dd_from_diff(B.x, A.x), vy = dd_from_diff(C.y, A.y);
    dd vx = dd_from_diff(C.x, A.x), uy = dd_from_diff(B.y, A.y);
    dd P1 = dd_mul(ux, vy), P2 = dd_mul(vx, uy);
    dd ar = dd_sub(P1, P2);
    double mag = fabs(P1.h) + fabs(P2.h);
    *sliver = !(fabs(ar.h) >= ldexp(mag, -48));
    dd D = dd_mul(ar, ar);
    D.h *= 4.0;
    D.l *= 4.0;
    return dd_div_to_double(N, D);
}

// ------------------------------------------------------------------ kernels
struct EdgeCount {
    const int4 *cv, *cn;
    int *cnt;
    __device__ void operator()(long long ii) const
    {
        int t = (int)ii;
        int4 v = cv[t], n = cn[t];
        int k = 0;
        for (int i = 0; i < 3; i++)
            if (geti(v, p1(i)) < geti(v, m1(i)) || geti(n, i) == -1) k++;
        cnt[t] = k;
    }
};

// The exact attached test, called with coordinates by value: the caller then
// keeps its operands in registers (an array argument would have to live in
// local memory on the hot path, for a call that almost never happens).
__device__ __noinline__ int attached_exact_v(double ix, double iy, double jx, double jy, double kx, double ky)
{
    const double i[2] = {ix, iy}, j[2] = {jx, jy}, k[2] = {kx, ky};
    return attached_exact(i, j, k);
}

// Triangle keys + owned edges + attached test.
struct TriKeys {
    const int4 *cv, *cn;
    const int4 *gv;  // the triangles with the ids that index P
    const double2 *P;
    const int *e_off;
    unsigned long long *keys;
    int *vals;
    int4 *edges;    // p1, p2, tIndex, vOpp
    int *unatt;     // 1 if the edge enters the spectrum
    int *edge_ro;
    int *slivers;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int t = (int)ii;
        int4 v = cv[t], n = cn[t];
        const int4 g = gv[t];
        const double2 Q[3] = {P[g.x], P[g.y], P[g.z]};
        const double2 A = Q[0], B = Q[1], C = Q[2];
        bool sl;
        double r = rho_tri(A, B, C, &sl);
        keys[1 + t] = (unsigned long long)__double_as_longlong(r);
        vals[1 + t] = t;
        if (sl) {
            int k = atomicAdd(&ct->nlist2, 1);
            slivers[k] = t;
        }
        int e = e_off[t];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            int a = geti(v, p1(i)), b = geti(v, m1(i));
            int nb = geti(n, i);
            if (!(a < b || nb == -1)) continue;
            edges[e] = make_int4(a, b, t, i);
            const double2 pa = Q[p1(i)], pb = Q[m1(i)], pk = Q[i];
            double qa[2] = {pa.x, pa.y}, qb[2] = {pb.x, pb.y}, qk[2] = {pk.x, pk.y};
            int att = attached_filter(qa, qb, qk);
            if (att == 2) {
                atomicAdd(&ct->exact_attached, 1ull);
                att = attached_exact_v(pa.x, pa.y, pb.x, pb.y, pk.x, pk.y);
            }
            if (att == 0 && nb >= 0) {
                double2 po = P[geti(gv[dtri(nb)], dori(nb))];
                double qo[2] = {po.x, po.y};
                att = attached_filter(qa, qb, qo);
                if (att == 2) {
                    atomicAdd(&ct->exact_attached, 1ull);
                    att = attached_exact_v(pa.x, pa.y, pb.x, pb.y, po.x, po.y);
                }
            }
            if (att == EXACT_OVERFLOW) set_err(ct, GPUDT_ERR_EXACT, 100);
            unatt[e] = att ? 0 : 1;
            if (att) edge_ro[e] = 0;
            e++;
        }
    }
};

struct SliverKeys {
    const int4 *cv;  // the triangles with the ids that index P
    const double2 *P;
    const int *slivers;
    unsigned long long *keys;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int t = slivers[ii];
        int4 v = cv[t];
        double p[6] = {P[v.x].x, P[v.x].y, P[v.y].x, P[v.y].y, P[v.z].x, P[v.z].y};
        double r = rho_rounded_exact(3, p);
        if (r != r) set_err(ct, GPUDT_ERR_EXACT, 101);
        keys[1 + t] = (unsigned long long)__double_as_longlong(r);
    }
};

struct EdgeKeys {
    const int4 *edges;
    const int4 *gv;  // the triangles with the ids that index P
    const double2 *P;
    const int *unatt, *spos;
    unsigned long long *keys;
    int *vals;
    int base, nT;
    __device__ void operator()(long long ii) const
    {
        int e = (int)ii;
        if (!unatt[e]) return;
        int4 E = edges[e];
        int k = base + spos[e];
        const int4 g = gv[E.z];
        keys[k] = (unsigned long long)__double_as_longlong(rho_edge(P[geti(g, p1(E.w))], P[geti(g, m1(E.w))]));
        vals[k] = nT + e;
    }
};

// --------------------------------------------------------- ranks and runs
__device__ __forceinline__ bool near_equal(unsigned long long ka, unsigned long long kb)
{
    // kb >= ka (sorted); keys carry <= 1 ulp of error each
    double a = __longlong_as_double((long long)ka), b = __longlong_as_double((long long)kb);
    double u = __longlong_as_double((long long)kb + 1) - b;  // ulp of the positive key b
    return (b - a) <= 2.0 * u;
}

// nr[i] = 1 when entry i certainly starts a new rank.  Links within 2 ulp are
// listed for one exact comparison each.
struct MarkRuns {
    const unsigned long long *keys;
    int *nr;
    int *unc;
    int n;
    Counters *ct;
    const int *seg;  // set of each entry (batched stage) or nullptr
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        if (i == 0) {
            nr[0] = 0;
            return;
        }
        if (i >= 2 && (!seg || seg[i] == seg[i - 1]) && near_equal(keys[i - 1], keys[i])) {
            nr[i] = 0;
            int k = atomicAdd(&ct->nlist, 1);
            unc[k] = i;
        } else {
            nr[i] = 1;
        }
    }
};

__device__ __forceinline__ void entry_points(int val, int nT, const int4 *cv, const int4 *edges,
                                             const double2 *P, int *kind, double *p)
{
    if (val < nT) {
        int4 v = cv[val];
        double2 a = P[v.x], b = P[v.y], c = P[v.z];
        p[0] = a.x; p[1] = a.y; p[2] = b.x; p[3] = b.y; p[4] = c.x; p[5] = c.y;
        *kind = 3;
    } else {
        int4 E = edges[val - nT];
        const int4 g = cv[E.z];  // cv: the triangles with the ids that index P
        double2 a = P[geti(g, p1(E.w))], b = P[geti(g, m1(E.w))];
        p[0] = a.x; p[1] = a.y; p[2] = b.x; p[3] = b.y;
        *kind = 2;
    }
}

__device__ __forceinline__ int exact_cmp_vals(int va, int vb, int nT, const int4 *cv, const int4 *edges,
                                              const double2 *P)
{
    int ka, kb;
    double pa[6], pb[6];
    entry_points(va, nT, cv, edges, P, &ka, pa);
    entry_points(vb, nT, cv, edges, P, &kb, pb);
    return compare_rho_exact(ka, pa, kb, pb);
}

// One exact comparison per uncertain adjacent pair (parallel over pairs): a
// smaller left value starts a new rank, an exact tie shares the rank, and an
// order violation sends the whole run to k_resolve (rare: it needs two distinct
// values within one ulp whose keys rounded the wrong way).
struct ExactAdjacent {
    const unsigned long long *keys;
    const int *vals;
    int *nr, *slow, *slowflag;
    const int *unc;
    const int4 *cv, *edges;
    const double2 *P;
    int nT;
    Counters *ct;
    const int *seg;
    __device__ void operator()(long long ii) const
    {
        int i = unc[ii];
        int cmp = exact_cmp_vals(vals[i - 1], vals[i], nT, cv, edges, P);
        atomicAdd(&ct->exact_compares, 1ull);
        if (cmp == EXACT_OVERFLOW) {
            set_err(ct, GPUDT_ERR_EXACT, 110);
            return;
        }
        if (cmp < 0) {
            nr[i] = 1;
        } else if (cmp == 0) {
            nr[i] = 0;
            atomicAdd(&ct->nties, 1);
        } else {
            int s = i - 1;
            while (s >= 2 && (!seg || seg[s - 1] == seg[s]) && near_equal(keys[s - 1], keys[s])) s--;
            if (atomicCAS(&slowflag[s], 0, 1) == 0) {
                int k = atomicAdd(&ct->nlist2, 1);
                slow[k] = s;
            }
        }
    }
};

// Rare path: a run with an order violation is re-sorted with the exact
// comparator and its rank-start flags recomputed: one thread per run of at
// most kThreadRun entries (insertion sort), one block per longer run
// (k_resolve_long: merge sort), and a run longer than Ctx::block_run by many
// blocks, one launch per merge level (k_merge_level; a lattice of
// non-dyadic spacing gives runs of millions of near-equal radii).
constexpr int kThreadRun = 512;
struct ResolveRuns {
    unsigned long long *keys;
    int *vals, *nr;
    const int *runs;
    const int4 *cv, *edges;
    const double2 *P;
    int n, nT;
    Counters *ct;
    const int *seg;
    int *longs;  // runs longer than kThreadRun, for k_resolve_long (count in ct->nlong)
    __device__ void operator()(long long ii) const
    {
        int s = runs[ii];
        int e = s;
        while (e + 1 < n && (!seg || seg[e] == seg[e + 1]) && near_equal(keys[e], keys[e + 1])) {
            e++;
            if (e - s >= kThreadRun) {
                longs[atomicAdd(&ct->nlong, 1)] = s;
                return;
            }
        }
        for (int a = s + 1; a <= e; a++) {
            unsigned long long kc = keys[a];
            int vc = vals[a];
            int b = a - 1;
            for (; b >= s; b--) {
                int cmp = exact_cmp_vals(vals[b], vc, nT, cv, edges, P);
                if (cmp == EXACT_OVERFLOW) {
                    set_err(ct, GPUDT_ERR_EXACT, 111);
                    return;
                }
                if (cmp <= 0) break;
                keys[b + 1] = keys[b];
                vals[b + 1] = vals[b];
            }
            keys[b + 1] = kc;
            vals[b + 1] = vc;
        }
        for (int a = s + 1; a <= e; a++) {
            int cmp = exact_cmp_vals(vals[a - 1], vals[a], nT, cv, edges, P);
            if (cmp == EXACT_OVERFLOW) {
                set_err(ct, GPUDT_ERR_EXACT, 112);
                return;
            }
            nr[a] = cmp != 0 ? 1 : 0;
        }
    }
};

// Order of two spectrum entries: by key where the keys are more than 2 ulp
// apart (each carries at most 1 ulp of error), else exactly.
__device__ __forceinline__ int cmp_entries(unsigned long long ka, int va, unsigned long long kb, int vb, int nT,
                                           const int4 *cv, const int4 *edges, const double2 *P)
{
    if (ka < kb && !near_equal(ka, kb)) return -1;
    if (kb < ka && !near_equal(kb, ka)) return 1;
    return exact_cmp_vals(va, vb, nT, cv, edges, P);
}

// One block per long run starting at runs[blockIdx.x]: the run's end by
// block-wide scans, a stable bottom-up merge sort of (keys, vals)[s..e] with
// the exact comparator (each thread merges a share of the outputs from a
// merge-path split found by binary search; ties take the left run first),
// through (tk, tv)[s..e] as the second buffer, then the rank-start flags.
constexpr int kLongThreads = 256;
__global__ void __launch_bounds__(kLongThreads) k_resolve_long(unsigned long long *keys, int *vals, int *nr,
                                                               unsigned long long *tk, int *tv, const int *runs,
                                                               const int4 *cv, const int4 *edges, const double2 *P,
                                                               int n, int nT, Counters *ct, const int *seg,
                                                               int block_run, int2 *huge)
{
    __shared__ int red[kLongThreads / 32];
    __shared__ int s_end;
    const int s = runs[blockIdx.x];
    if (threadIdx.x == 0) s_end = n - 1;
    __syncthreads();
    // the run ends before the first j > s that is not linked to j - 1
    for (long long w0 = s + 1; w0 < n; w0 += kLongThreads) {
        const long long j = w0 + threadIdx.x;
        const bool brk = j < n && (!((!seg || seg[j - 1] == seg[j]) && near_equal(keys[j - 1], keys[j])));
        int m = __reduce_min_sync(0xffffffffu, brk ? (int)j : n);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        m = red[0];
        for (int q = 1; q < kLongThreads / 32; q++) m = min(m, red[q]);
        __syncthreads();
        if (m < n) {
            if (threadIdx.x == 0) s_end = m - 1;
            break;
        }
    }
    __syncthreads();
    const int e = s_end, L = e - s + 1;
    if (L > block_run) {  // left to the multi-block merge
        if (threadIdx.x == 0) huge[atomicAdd(&ct->nhuge, 1)] = make_int2(s, L);
        return;
    }
    bool bad = false;
    unsigned long long *sk = keys + s, *dk = tk + s;
    int *sv = vals + s, *dv = tv + s;
    const int chunk = (L + kLongThreads - 1) / kLongThreads;
    for (int w = 1; w < L; w <<= 1) {
        const int o0 = min(L, (int)threadIdx.x * chunk), o1 = min(L, o0 + chunk);
        for (int pos = o0; pos < o1;) {
            const int lo = pos / (2 * w) * (2 * w), mid = min(L, lo + w), hi = min(L, lo + 2 * w);
            const int na = mid - lo, nb = hi - mid;
            const int k0 = pos - lo, kend = min(o1, hi) - lo;
            // merge-path split of diagonal k0: i elements of A before it
            int a0 = max(0, k0 - nb), a1 = min(k0, na);
            while (a0 < a1) {
                const int m = (a0 + a1) >> 1;
                int c = cmp_entries(sk[lo + m], sv[lo + m], sk[mid + k0 - m - 1], sv[mid + k0 - m - 1], nT, cv, edges, P);
                if (c == EXACT_OVERFLOW) {
                    bad = true;
                    c = 0;
                }
                if (c <= 0) a0 = m + 1;
                else a1 = m;
            }
            int i = a0, j = k0 - a0;
            for (int k = k0; k < kend; k++) {
                bool takeA = i < na;
                if (takeA && j < nb) {
                    int c = cmp_entries(sk[lo + i], sv[lo + i], sk[mid + j], sv[mid + j], nT, cv, edges, P);
                    if (c == EXACT_OVERFLOW) {
                        bad = true;
                        c = 0;
                    }
                    takeA = c <= 0;
                }
                const int src = takeA ? lo + i++ : mid + j++;
                dk[lo + k] = sk[src];
                dv[lo + k] = sv[src];
            }
            pos = lo + kend;
        }
        __syncthreads();  // every output of this level written before the next reads it
        unsigned long long *t1 = sk;
        sk = dk;
        dk = t1;
        int *t2 = sv;
        sv = dv;
        dv = t2;
    }
    if (sk != keys + s)  // the last level wrote the second buffer
        for (int k = threadIdx.x; k < L; k += kLongThreads) {
            keys[s + k] = sk[k];
            vals[s + k] = sv[k];
        }
    __syncthreads();
    for (int a = s + 1 + threadIdx.x; a <= e; a += kLongThreads) {
        int cmp = exact_cmp_vals(vals[a - 1], vals[a], nT, cv, edges, P);
        if (cmp == EXACT_OVERFLOW) {
            bad = true;
            cmp = 1;
        }
        nr[a] = cmp != 0 ? 1 : 0;
    }
    if (bad) set_err(ct, GPUDT_ERR_EXACT, 111);
}

// One merge level of the multi-block exact sort of a run of L entries:
// sorted blocks of w entries are merged pairwise from (sk, sv) into (dk, dv).
// Thread t writes outputs [t*kMergeChunk, (t+1)*kMergeChunk): for each pair
// of blocks its outputs fall in, it finds where its first output's merge path
// crosses the pair by binary search (ties take the left block first, so the
// sort is stable), then merges.
constexpr int kMergeChunk = 16;
__global__ void __launch_bounds__(256) k_merge_level(const unsigned long long *__restrict__ sk,
                                                     const int *__restrict__ sv, unsigned long long *__restrict__ dk,
                                                     int *__restrict__ dv, int L, int w, const int4 *cv,
                                                     const int4 *edges, const double2 *P, int nT, Counters *ct)
{
    const long long o0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kMergeChunk;
    if (o0 >= L) return;
    const long long o1 = min((long long)L, o0 + kMergeChunk);
    bool bad = false;
    // the chunk may span several pairs of blocks while 2w < kMergeChunk
    for (long long pos = o0; pos < o1;) {
        const int lo = (int)(pos / (2ll * w) * (2ll * w));
        const int mid = (int)min((long long)L, (long long)lo + w);
        const int hi = (int)min((long long)L, (long long)lo + 2ll * w);
        const int na = mid - lo, nb = hi - mid;
        const int k0 = (int)pos - lo, kend = (int)min((long long)hi, o1) - lo;
        int a0 = max(0, k0 - nb), a1 = min(k0, na);
        while (a0 < a1) {
            const int m = (a0 + a1) >> 1;
            int c = cmp_entries(sk[lo + m], sv[lo + m], sk[mid + k0 - m - 1], sv[mid + k0 - m - 1], nT, cv, edges,
                                P);
            if (c == EXACT_OVERFLOW) {
                bad = true;
                c = 0;
            }
            if (c <= 0) a0 = m + 1;
            else a1 = m;
        }
        int i = a0, j = k0 - a0;
        for (int k = k0; k < kend; k++) {
            bool takeA = i < na;
            if (takeA && j < nb) {
                int c = cmp_entries(sk[lo + i], sv[lo + i], sk[mid + j], sv[mid + j], nT, cv, edges, P);
                if (c == EXACT_OVERFLOW) {
                    bad = true;
                    c = 0;
                }
                takeA = c <= 0;
            }
            const int src = takeA ? lo + i++ : mid + j++;
            dk[lo + k] = sk[src];
            dv[lo + k] = sv[src];
        }
        pos = lo + kend;
    }
    if (bad) set_err(ct, GPUDT_ERR_EXACT, 114);
}

// Rank-start flags of a sorted run [s, s + L): an entry starts a new rank
// unless it equals its left neighbour exactly.
struct RunFlags {
    const int *vals;
    int *nr;
    const int4 *cv, *edges;
    const double2 *P;
    int s, nT;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int a = s + 1 + (int)ii;
        int cmp = exact_cmp_vals(vals[a - 1], vals[a], nT, cv, edges, P);
        if (cmp == EXACT_OVERFLOW) {
            set_err(ct, GPUDT_ERR_EXACT, 115);
            cmp = 1;
        }
        nr[a] = cmp != 0 ? 1 : 0;
    }
};

// The multi-block exact sort of one long run [s, s + L) of (keys, vals),
// through (tk, tv)[s, s + L) as the second buffer.
static int merge_sort_run(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *tk, int *tv, int *nr,
                          int s, int L, int nT)
{
    unsigned long long *sk = keys + s, *dk = tk + s;
    int *sv = vals + s, *dv = tv + s;
    const long long threads = ((long long)L + kMergeChunk - 1) / kMergeChunk;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    for (long long w = 1; w < L; w <<= 1) {
        k_merge_level<<<blocks, 256, 0, c.stream>>>(sk, sv, dk, dv, L, (int)w, alpha_geom_tris(c), c.edges, c.opos,
                                                     nT, c.ctr);
        count_launch();
        std::swap(sk, dk);
        std::swap(sv, dv);
    }
    GALPHA_CUDA(cudaGetLastError());
    if (sk != keys + s) {
        launch_n(c, CopyElems<unsigned long long>{keys + s, sk}, L);
        launch_n(c, CopyElems<int>{vals + s, sv}, L);
    }
    launch_n(c, RunFlags{vals, nr, alpha_geom_tris(c), c.edges, c.opos, s, nT, c.ctr}, L - 1);
    return GPUDT_OK;
}

struct ScatterRanks {
    const unsigned long long *keys;
    const int *vals, *nr, *excl;
    int *tri_ro, *edge_ro;
    double *spectrum;
    int nT;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        int r = excl[i] + nr[i];
        if (i == 0) {
            spectrum[0] = 0.0;
            return;
        }
        int v = vals[i];
        if (v < nT) tri_ro[v] = r;
        else edge_ro[v - nT] = r;
        if (nr[i]) spectrum[r] = __longlong_as_double((long long)keys[i]);
    }
};

struct EdgeIntervals {
    const int4 *edges, *cn;
    const int *tri_ro, *edge_ro;
    int2 *edge_nu;
    int2 *pt;  // (min, max) accumulators
    __device__ void operator()(long long ii) const
    {
        int e = (int)ii;
        int4 E = edges[e];
        int nb = geti(cn[E.z], E.w);
        int tr = tri_ro[E.z];
        int2 nu;
        if (nb == -1) {
            nu = make_int2(tr, 0);
        } else {
            int o = tri_ro[dtri(nb)];
            nu = tr <= o ? make_int2(tr, o) : make_int2(o, tr);
        }
        edge_nu[e] = nu;
        int ro = edge_ro[e];
        int vmin = ro != 0 ? ro : nu.x;
        atomicMin(&pt[E.x].x, vmin);
        atomicMax(&pt[E.x].y, nu.y);
        atomicMin(&pt[E.y].x, vmin);
        atomicMax(&pt[E.y].y, nu.y);
    }
};

struct InitPt {
    int2 *pt;
    __device__ void operator()(long long i) const { pt[i] = make_int2(0x7fffffff, -1); }
};

struct FixPt {
    int2 *pt;
    __device__ void operator()(long long i) const
    {
        if (pt[i].x == 0x7fffffff) pt[i] = make_int2(-1, -1);
    }
};

// ------------------------------------------------------- batched segments
// Set of each value-sorted entry (triangle, or the triangle that owns the edge).
// Set of every entry id in entry order (triangles, then edges in triangle
// order): coalesced reads, so the sorted entries need one gather each.
// First edge of each set (and [K] = nE): edges are numbered in triangle
// order and triangles are grouped by set.
struct SetEdgeBases {
    const int *e_off, *tbase;
    int nT, nE;
    int *ebase;
    __device__ void operator()(long long s) const
    {
        const int t = tbase[s];
        ebase[s] = t < nT ? e_off[t] : nE;
    }
};

// Set of each value-sorted entry, by binary search of its id in the per-set
// bases (triangles and edges are each grouped by set, bases non-decreasing;
// the last set whose base is at most the id owns it) -- no gather by id.
// A coarse table gives the owner of every kEntryBlock-th id, so the search
// runs only over the sets that start inside the entry's block.
constexpr int kEntryBlockBits = 10;

__device__ __forceinline__ int set_owner(const int *b, int lo, int hi, int x)
{
    // the answer lies in [lo, hi): b[lo] <= x < b[hi]
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if (b[m] <= x) lo = m;
        else hi = m;
    }
    return lo;
}

// coarse[j]: owner of id j << kEntryBlockBits, for the triangle ids (j <
// nbt) and then the edge ids
struct EntryBlocks {
    const int *tbase, *ebase;
    int K, nbt;
    int *coarse;
    __device__ void operator()(long long jj) const
    {
        const int j = (int)jj;
        const bool tri = j < nbt;
        const int x = (tri ? j : j - nbt) << kEntryBlockBits;
        coarse[j] = set_owner(tri ? tbase : ebase, 0, K, x);
    }
};

struct EntrySet {
    const int *vals;
    const int *tbase, *ebase;
    const int *coarse;
    int K, nT, nbt, nbe;
    unsigned *key;
    __device__ void operator()(long long i) const
    {
        const int v = vals[i];
        const bool tri = v < nT;
        const int *b = tri ? tbase : ebase;
        const int x = tri ? v : v - nT;
        const int j = x >> kEntryBlockBits;
        const int *cb = tri ? coarse : coarse + nbt;
        const int nb = tri ? nbt : nbe;
        // the owner of the block's first id, up to the owner of the next block's
        const int lo = cb[j], hi = j + 1 < nb ? min(K, cb[j + 1] + 1) : K;
        key[i] = (unsigned)set_owner(b, lo, hi, x);
    }
};

struct SetOfSorted {
    const unsigned *setkey;
    int *seg;  // indexed like the full entry array (entry 0 = sentinel)
    __device__ void operator()(long long i) const
    {
        seg[1 + i] = (int)setkey[i];
        if (i == 0) seg[0] = -1;
    }
};

// Per set: the global rank count before its first entry, and its number of
// distinct values (entries of a set are contiguous; each set's first entry
// starts a rank).
struct SetRankBounds {
    const int *seg, *nr, *excl;
    int n;
    int *firstexcl, *endrank;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        if (i == 0) return;
        int s = seg[i];
        if (i == 1 || seg[i - 1] != s) firstexcl[s] = excl[i];
        if (i == n - 1 || seg[i + 1] != s) endrank[s] = excl[i] + nr[i];
    }
};

struct SetDistinct {
    const int *firstexcl;
    int *nd;  // in: end rank (0 for a set without entries); out: distinct values
    __device__ void operator()(long long s) const { nd[s] -= firstexcl[s]; }
};

struct ScatterRanksSeg {
    const unsigned long long *keys;
    const int *vals, *nr, *excl, *seg, *firstexcl, *spec_off;
    int *tri_ro, *edge_ro;
    double *spectrum;
    int nT;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        if (i == 0) return;
        int s = seg[i];
        int r = excl[i] + nr[i] - firstexcl[s];
        int v = vals[i];
        if (v < nT) tri_ro[v] = r;
        else edge_ro[v - nT] = r;
        if (nr[i]) spectrum[spec_off[s] + s + r] = __longlong_as_double((long long)keys[i]);
    }
};

struct SetSentinels {
    const int *spec_off;
    double *spectrum;
    __device__ void operator()(long long s) const { spectrum[spec_off[s] + s] = 0.0; }
};

// ------------------------------------------------------------------ stage
int stage_alpha(Ctx &c, AlphaSegs *segs)
{
    int r;
    const int nT = c.nT_out;
    int *cnt = c.aux, *e_off = c.e_off;
    // an alpha call on a resident mesh starts without the error of an earlier
    // failed alpha call (err and errinfo are adjacent words)
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->err, 0, 2 * sizeof(int), c.stream));
    launch_n(c, EdgeCount{c.cv, c.cn, cnt}, nT);
    r = exclusive_scan_int(c, cnt, e_off, nT, &c.ctr->nlist);
    if (r) return r;
    r = read_counters(c);
    if (r) return r;
    const int nE = c.hctr->nlist;
    c.nE = nE;
    int *unatt = c.aux2, *spos = c.rank;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.keys, 0, sizeof(unsigned long long), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.vals, 0, sizeof(int), c.stream));
    launch_occ<4>(c, TriKeys{c.cv, c.cn, alpha_geom_tris(c), c.opos, e_off, c.keys, c.vals, c.edges, unatt, c.edge_ro, c.list, c.ctr}, nT);
    // the sliver list's length stays on the device; TriKeys' errors are read
    // with the spectrum length below
    launch_dev(c, SliverKeys{alpha_geom_tris(c), c.opos, c.list, c.keys, c.ctr}, &c.ctr->nlist2, nT);
    r = exclusive_scan_int(c, unatt, spos, nE, &c.ctr->nlist);
    if (r) return r;
    launch_n(c, EdgeKeys{c.edges, alpha_geom_tris(c), c.opos, unatt, spos, c.keys, c.vals, 1 + nT, nT}, nE);
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
    const int nIn = 1 + nT + c.hctr->nlist;
    c.nSpecIn = nIn;
    c.sort_passes = 0;
    if (c.events) {
        cudaEventRecord(c.kev[8], c.stream);
        c.kev_rec[8] = true;
    }
    bool second = false;
    r = radix_sort(c, c.keys + 1, c.vals + 1, c.keys2 + 1, c.vals2 + 1, nIn - 1, &second);
    if (r) return r;
    if (second) {
        // the sorted entries are in the second buffers: they become keys / vals
        // (sentinel entry 0 included) for the rest of this result's life
        GALPHA_CUDA(cudaMemsetAsync(c.keys2, 0, sizeof(unsigned long long), c.stream));
        GALPHA_CUDA(cudaMemsetAsync(c.vals2, 0, sizeof(int), c.stream));
        std::swap(c.keys, c.keys2);
        std::swap(c.vals, c.vals2);
    }
    if (c.events) {
        cudaEventRecord(c.kev[9], c.stream);
        c.kev_rec[9] = true;
    }
    c.st.sortKeys = nIn - 1;
    c.st.sortPasses = c.sort_passes;
    if (segs) {
        // stable sort by set, carrying each entry's key and value: entries end
        // up ordered by (set, value)
        const int m = nIn - 1;
        unsigned *ka = (unsigned *)c.rank, *kb = (unsigned *)c.aux2;  // both free until the ranks
        launch_n(c, SetEdgeBases{c.e_off, segs->tbase, nT, nE, segs->ebase}, segs->K + 1);
        // c.list is free here (the sliver list has been consumed)
        const int nbt = (nT >> kEntryBlockBits) + 1, nbe = (nE >> kEntryBlockBits) + 1;
        int *coarse = c.list;
        launch_n(c, EntryBlocks{segs->tbase, segs->ebase, segs->K, nbt, coarse}, nbt + nbe);
        launch_n(c, EntrySet{c.vals + 1, segs->tbase, segs->ebase, coarse, segs->K, nT, nbt, nbe, ka}, m);
        int bits = 0;
        while ((1ll << bits) < segs->K) bits++;
        r = radix_sort_set_kv(c, ka, kb, c.keys + 1, c.vals + 1, c.keys2 + 1, c.vals2 + 1, m, bits);
        if (r) return r;
        launch_n(c, SetOfSorted{ka, segs->seg}, m);
    }
    // ranks
    int *nr = c.aux, *unc = c.list, *slow = c.list2, *slowflag = c.stamp;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, 2 * sizeof(int), c.stream));
    launch_n(c, MarkRuns{c.keys, nr, unc, nIn, c.ctr, segs ? segs->seg : nullptr}, nIn);
    r = read_counters(c);
    if (r) return r;
    int nunc = c.hctr->nlist;
    if (nunc > 0) {
        GALPHA_CUDA(cudaMemsetAsync(slowflag, 0, sizeof(int) * (size_t)nIn, c.stream));
        launch_n(c, ExactAdjacent{c.keys, c.vals, nr, slow, slowflag, unc, alpha_geom_tris(c), c.edges, c.opos, nT, c.ctr,
                                  segs ? segs->seg : nullptr},
                 nunc);
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
        if (c.hctr->nlist2 > 0) {
            // runs longer than kThreadRun are listed after the slow runs
            const int nslow = c.hctr->nlist2;
            int *longs = slow + nslow;
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlong, 0, sizeof(int), c.stream));
            launch_n(c, ResolveRuns{c.keys, c.vals, nr, slow, alpha_geom_tris(c), c.edges, c.opos, nIn, nT, c.ctr,
                                    segs ? segs->seg : nullptr, longs},
                     nslow);
            r = read_counters(c);
            if (r) return r;
            if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
            if (c.hctr->nlong > 0) {
                // (keys2, vals2) are free now: the second buffer of each run's merge sort
                const int nlong = c.hctr->nlong;
                // runs for the multi-block merge: (start, length) pairs after the long runs, 8-byte aligned
                uintptr_t hp = reinterpret_cast<uintptr_t>(longs + nlong);
                int2 *huge = reinterpret_cast<int2 *>((hp + 7) & ~(uintptr_t)7);
                GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nhuge, 0, sizeof(int), c.stream));
                k_resolve_long<<<(unsigned)nlong, kLongThreads, 0, c.stream>>>(
                    c.keys, c.vals, nr, c.keys2, c.vals2, longs, alpha_geom_tris(c), c.edges, c.opos, nIn, nT, c.ctr,
                    segs ? segs->seg : nullptr, c.block_run, huge);
                count_launch();
                GALPHA_CUDA(cudaGetLastError());
                r = read_counters(c);
                if (r) return r;
                if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
                const int nhuge = c.hctr->nhuge;
                if (nhuge > 0) {
                    std::vector<int2> hs(nhuge);
                    r = read_small(c, hs.data(), huge, sizeof(int2) * (size_t)nhuge);
                    if (r) return r;
                    for (const int2 &h : hs) {
                        r = merge_sort_run(c, c.keys, c.vals, c.keys2, c.vals2, nr, h.x, h.y, nT);
                        if (r) return r;
                    }
                    r = read_counters(c);
                    if (r) return r;
                    if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
                }
            }
        }
    }
    r = exclusive_scan_int(c, nr, c.rank, nIn, &c.ctr->nlist);
    if (r) return r;
    if (!segs) {
        launch_n(c, ScatterRanks{c.keys, c.vals, nr, c.rank, c.tri_ro, c.edge_ro, c.spectrum, nT}, nIn);
    } else {
        GALPHA_CUDA(cudaMemsetAsync(segs->nd, 0, sizeof(int) * (size_t)segs->K, c.stream));
        GALPHA_CUDA(cudaMemsetAsync(segs->firstexcl, 0, sizeof(int) * (size_t)segs->K, c.stream));
        launch_n(c, SetRankBounds{segs->seg, nr, c.rank, nIn, segs->firstexcl, segs->nd}, nIn);
        launch_n(c, SetDistinct{segs->firstexcl, segs->nd}, segs->K);
        r = exclusive_scan_int(c, segs->nd, segs->spec_off, segs->K, nullptr);
        if (r) return r;
        launch_n(c, ScatterRanksSeg{c.keys, c.vals, nr, c.rank, segs->seg, segs->firstexcl, segs->spec_off,
                                    c.tri_ro, c.edge_ro, c.spectrum, nT},
                 nIn);
        launch_n(c, SetSentinels{segs->spec_off, c.spectrum}, segs->K);
    }
    launch_n(c, InitPt{c.pt_nu}, c.N);
    launch_n(c, EdgeIntervals{c.edges, c.cn, c.tri_ro, c.edge_ro, c.edge_nu, c.pt_nu}, nE);
    launch_n(c, FixPt{c.pt_nu}, c.N);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return stage_fail(c, c.hctr->err, "alpha");
    c.nSpec = c.hctr->nlist + (segs ? segs->K : 1);  // distinct ranks incl. the sentinel(s)
    return GPUDT_OK;
}

// ------------------------------------------------------------ alpha query
// Classification of every simplex of the alpha complex at a value alpha
// (a squared radius, the unit of the spectrum), from the intervals above:
// R = the largest rank with spectrum[R] <= alpha, then
//   triangle:  ro <= R                                    -> interior
//   edge:      nu_max != 0 (finite) && nu_max <= R        -> interior
//              nu_min <= R                                -> regular
//              ro != 0 (unattached) && ro <= R            -> singular
//   point:     (nu_min, nu_max) the same way, with the singular interval
//              starting at rank 0 (every vertex is in the complex at alpha >= 0)
//   otherwise exterior.  Points dropped as duplicates (no incident edge) are
// exterior.  These are the interval semantics of kernel.cu:427-624 that the
// reference's viewer draws from (Visualizer.cu:296-337: an edge is drawn from
// its ro / nu_min entry until its nu_max entry, a triangle from its ro entry).
namespace {

struct QueryRank {
    const double *spectrum;
    int nSpec;
    double alpha, q;
    int by_quantile;
    Counters *ct;
    __device__ void operator()(long long) const
    {
        double a = alpha;
        if (by_quantile) {
            double qq = q < 0.0 ? 0.0 : (q > 1.0 ? 1.0 : q);
            int k = (int)llrint(qq * (double)(nSpec - 1));
            a = spectrum[k];
        }
        int R = -1;
        if (a >= 0.0) {
            int lo = 0, hi = nSpec - 1;  // spectrum[0] = 0 <= a
            while (lo < hi) {
                int mid = lo + (hi - lo + 1) / 2;
                if (spectrum[mid] <= a) lo = mid;
                else hi = mid - 1;
            }
            R = lo;
        }
        ct->qrank = R;
        ct->qalpha = a;
        for (int k = 0; k < 12; k++) ct->qcount[k] = 0;
    }
};

__device__ __forceinline__ int interval_class(int ro, int nu_min, int nu_max, int R)
{
    if (nu_max > 0 && nu_max <= R) return 3;
    if (nu_min <= R) return 2;
    if (ro >= 0 && ro <= R) return 1;
    return 0;
}

struct QueryClassify {
    const int2 *pt;
    const int *edge_ro;
    const int2 *edge_nu;
    const int *tri_ro;
    uint8_t *cls;
    int N, nE, nT;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        const int R = ct->qrank;
        int type, k;
        if (i < N) {
            type = 0;
            int2 v = pt[i];
            k = (v.x < 0 || R < 0) ? 0 : interval_class(0, v.x, v.y, R);
        } else if (i < N + nE) {
            type = 1;
            int e = i - N;
            int ro = edge_ro[e];
            int2 nu = edge_nu[e];
            k = R < 0 ? 0 : interval_class(ro != 0 ? ro : -1, nu.x, nu.y, R);
        } else {
            type = 2;
            k = (R >= 0 && tri_ro[i - N - nE] <= R) ? 3 : 0;
        }
        cls[i] = (uint8_t)k;
        int bin = type * 4 + k;
        unsigned peers = __match_any_sync(__activemask(), bin);
        if ((peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(&ct->qcount[bin], __popc(peers));
    }
};

// Per set of a batch: the set's spectrum is spectrum[spec_off[s] + s ..] of
// length nd[s] + 1 (its own rank-0 sentinel first).
struct QueryRankSets {
    const double *spectrum;
    const int *spec_off, *nd;
    const double *param;
    int by_quantile;
    int *R;
    double *alpha;
    __device__ void operator()(long long ss) const
    {
        int s = (int)ss;
        const double *sp = spectrum + spec_off[s] + s;
        int ns = nd[s] + 1;
        double a = param[s];
        if (by_quantile) {
            double qq = a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a);
            a = sp[(int)llrint(qq * (double)(ns - 1))];
        }
        int r = -1;
        if (a >= 0.0) {
            int lo = 0, hi = ns - 1;
            while (lo < hi) {
                int mid = lo + (hi - lo + 1) / 2;
                if (sp[mid] <= a) lo = mid;
                else hi = mid - 1;
            }
            r = lo;
        }
        R[s] = r;
        alpha[s] = a;
    }
};

struct QueryClassifySets {
    const int2 *pt;
    const int *edge_ro;
    const int2 *edge_nu;
    const int4 *edges;
    const int *tri_ro;
    const int *vset, *tset, *R;
    uint8_t *cls;
    int *counts;  // [K][12]
    int N, nE, nT;
    __device__ void operator()(long long ii) const
    {
        int i = (int)ii;
        int type, k, s;
        if (i < N) {
            type = 0;
            s = vset[i];
            int r = R[s];
            int2 v = pt[i];
            k = (v.x < 0 || r < 0) ? 0 : interval_class(0, v.x, v.y, r);
        } else if (i < N + nE) {
            type = 1;
            int e = i - N;
            s = tset[edges[e].z];
            int r = R[s];
            int ro = edge_ro[e];
            int2 nu = edge_nu[e];
            k = r < 0 ? 0 : interval_class(ro != 0 ? ro : -1, nu.x, nu.y, r);
        } else {
            type = 2;
            int t = i - N - nE;
            s = tset[t];
            int r = R[s];
            k = (r >= 0 && tri_ro[t] <= r) ? 3 : 0;
        }
        cls[i] = (uint8_t)k;
        int bin = s * 12 + type * 4 + k;
        unsigned peers = __match_any_sync(__activemask(), bin);
        if ((peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(&counts[bin], __popc(peers));
    }
};

}  // namespace

int alpha_query_sets(Ctx &c, int K, const int *vset, const int *tset, const int *spec_off, const int *nd,
                     const double *param, int by_quantile, int *R, double *alpha, int *counts)
{
    GALPHA_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * 12 * (size_t)K, c.stream));
    launch_n(c, QueryRankSets{c.spectrum, spec_off, nd, param, by_quantile, R, alpha}, K);
    long long n = (long long)c.N + c.nE + c.nT_out;
    launch_n(c, QueryClassifySets{c.pt_nu, c.edge_ro, c.edge_nu, c.edges, c.tri_ro, vset, tset, R, c.qclass, counts,
                                  c.N, c.nE, c.nT_out},
             n);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int alpha_query(Ctx &c, double alpha, double q, bool by_quantile)
{
    launch_n(c, QueryRank{c.spectrum, c.nSpec, alpha, q, by_quantile ? 1 : 0, c.ctr}, 1);
    long long n = (long long)c.N + c.nE + c.nT_out;
    launch_n(c, QueryClassify{c.pt_nu, c.edge_ro, c.edge_nu, c.tri_ro, c.qclass, c.N, c.nE, c.nT_out, c.ctr}, n);
    GALPHA_CUDA(cudaGetLastError());
    return read_counters(c);
}

}  // namespace galpha
