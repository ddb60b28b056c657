// dt_mesh.cu -- mesh stages of the Delaunay pipeline, all on the device.
//
// Stage map (reference -> here):
//   cpuVertexArray + kernelFindNextTriangles      stage_links: per-vertex incidence lists
//   (cudaReconstruction.cu:348-436; a host pass)   (count / scan / fill) and a matching
//                                                  kernel; validates the mesh (one
//                                                  triangle per directed edge, the hull is
//                                                  exactly the fake ring)
//   kernelDetectShifting / kernelShiftable         stage_shift: a site moves from its grid
//   (cudaReconstruction.cu:241-341,                 position to its true position when its
//    cudaShifting.cu:117-170)                       whole fan stays counterclockwise; rounds
//                                                  of local priority minima (hashed ids)
//   kernelDetectBadCases / DeleteTriangles /       stage_shift (second half): unshiftable
//   FixVertexArray / PatchHoles /                   sites are removed; one thread clips the
//   UpdateTriangleLinks (cudaShifting.cu:175-488)   star hole around the site's kernel point
//   kernelLocateTriangleContainer ... kernel       stage_missing: straight-line walk with
//   UpdateMissingTriangleLinks (cudaMissing.cu:     exact orientation, 1->3 / 2->4 splits,
//   166-527)                                        exact duplicates dropped (lowest id kept)
//   cudaFixBoundary (cudaBoundary.cu:106-608)      stage_boundary: fake ring sites removed
//                                                  in priority rounds, pockets patched with
//                                                  the ccw>0 stack rule, then reflex hull
//                                                  vertices filled so the hull is convex
//   cudaFlipping (cudaFlipping.cu:227-685) +       stage_flip: Lawson flips with exact
//   host gpudtRecursiveFlip (gpudt.cpp:191-304,     in-circle on device, min-id voting, an
//   879-914)                                        active work list; no host fix-up
//   kernelMarkValidTriangles1 ... FixIndices1      stage_compact: scan-compaction of live
//   (cudaMissing.cu:529-617, cudaBoundary.cu)       slots, links remapped, AoS output
//
// Concurrent local operations in one round (hole patches, splits, flips) use a
// two-phase relink: phase 1 writes each operation's own new triangles, records
// where every outer edge went (fwd[] of the consumed slot, epoch[] = round) and
// appends (new location, old outer link) records; phase 2 resolves each record
// against the forwarding of the neighbour if that neighbour was consumed in the
// same round, else writes the neighbour's back-link.  No operation ever writes
// a triangle owned by another operation of the same round.
#include <cstdio>
#include <algorithm>
#include <mutex>
#include "internal.cuh"
#include "exact.cuh"

namespace galpha {

// ------------------------------------------------------------ small helpers
// Orientation tests of one thread, added to the counters once (in a walk, an
// atomic per test costs more than the FP32 test it counts).
struct OrientTally {
    int tests = 0, fp64 = 0;
    __device__ __forceinline__ void flush(Counters *ct) const
    {
        warp_add_spread(ct->ori_spread, tests);
        warp_add_spread(ct->ori64_spread, fp64);
    }
};

// Staged orientation: FP32 filter, FP64 filter, exact.
__device__ __forceinline__ int orient_staged(double2 A, double2 B, double2 C, Counters *ct, OrientTally &n)
{
    n.tests++;
    int s = orient2d_filter32(A.x, A.y, B.x, B.y, C.x, C.y);
    if (s != 2) return s;
    s = orient2d_filter(A.x, A.y, B.x, B.y, C.x, C.y);
    if (s != 2) {
        n.fp64++;
        return s;
    }
    atomicAdd(&ct->exact_orient, 1ull);
    s = orient2d_exact(A.x, A.y, B.x, B.y, C.x, C.y);
    if (s == EXACT_OVERFLOW) {
        set_err(ct, GPUDT_ERR_EXACT, 2);
        return 0;
    }
    return s;
}

// One counted test (call sites outside loops).
__device__ __forceinline__ int orientp(double2 A, double2 B, double2 C, Counters *ct)
{
    OrientTally n;
    const int s = orient_staged(A, B, C, ct, n);
    warp_count_spread(ct->ori_spread);
    if (n.fp64) warp_count_spread(ct->ori64_spread);
    return s;
}

__device__ __forceinline__ int4 ldv(const int4 *tv, int t) { return tv[t]; }

__device__ __forceinline__ void set_link(int4 *tn, int loc, int val)
{
    int *p = (int *)&tn[dtri(loc)];
    p[dori(loc)] = val;
}

__device__ __forceinline__ int get_link(const int4 *tn, int loc)
{
    const int *p = (const int *)&tn[dtri(loc)];
    return p[dori(loc)];
}

__device__ __forceinline__ void push_rec(Relink *rec, Counters *ct, int loc, int old)
{
    int k = atomicAdd(&ct->nrec, 1);
    rec[k] = Relink{loc, old};
}

__device__ __forceinline__ void set_fwd(int4 *fwd, int t, int i, int loc)
{
    int *p = (int *)&fwd[t];
    p[i] = loc;
}

// Pops a free slot, else takes one from the tail; -1 (and GPUDT_ERR_NOMEM)
// when the slot array is full.
__device__ __forceinline__ int alloc_slot(int *freelist, Counters *ct, int cap)
{
    int k = atomicSub(&ct->nfree, 1) - 1;
    if (k >= 0) return freelist[k];
    int s = atomicAdd(&ct->ntris, 1);
    if (s >= cap) {
        set_err(ct, GPUDT_ERR_NOMEM, 5);
        return -1;
    }
    return s;
}

// After a round of allocations: a free-list count driven below zero by pops
// that fell through to the tail is reset, so that a later free_slot appends
// at index 0.
struct ClampFree {
    Counters *ct;
    __device__ void operator()(long long) const
    {
        if (ct->nfree < 0) ct->nfree = 0;
    }
};

__device__ __forceinline__ void free_slot(int4 *tv, int *freelist, Counters *ct, int t)
{
    tv[t] = make_int4(-1, -1, -1, 0);
    int k = atomicAdd(&ct->nfree, 1);
    freelist[k] = t;
}

// ------------------------------------------------------------------- links
struct CountDeg {
    const int4 *tv;
    int *deg;
    __device__ void operator()(long long i) const
    {
        int4 v = tv[i];
        if (v.x < 0) return;  // released slot
        atomicAdd(&deg[v.x], 1);
        atomicAdd(&deg[v.y], 1);
        atomicAdd(&deg[v.z], 1);
    }
};

// Incidence entry of vertex v in triangle t (v = vtx[k]): the oriented slot
// and the next vertex counterclockwise, so matching reads only the list.
struct FillInc {
    const int4 *tv;
    const int *start;
    int *cursor;
    int2 *inc;
    __device__ void operator()(long long i) const
    {
        int t = (int)i;
        int4 v = tv[t];
        if (v.x < 0) return;
        int a[3] = {v.x, v.y, v.z};
        for (int k = 0; k < 3; k++) {
            int s = start[a[k]] + atomicAdd(&cursor[a[k]], 1);
            inc[s] = make_int2(enc(t, k), a[p1(k)]);
        }
    }
};

struct MatchLinks {
    const int4 *tv;
    int4 *tn;
    const int *start;
    const int2 *inc;
    int *vtri;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        int t = (int)i;
        int4 v = tv[t];
        if (v.x < 0) {
            tn[t] = make_int4(-1, -1, -1, 0);
            return;
        }
        // A directed edge held by two triangles shows up as two twins in the
        // twin's scan (cnt > 1) or, on the hull, in the hull edge count, which
        // must equal the fake ring's; so a's own list is not scanned.
        int n[3];
        for (int k = 0; k < 3; k++) {
            int a = geti(v, p1(k)), b = geti(v, m1(k));  // edge a -> b, opposite vtx[k]
            int found = -1, cnt = 0;
            for (int s = start[b], e = start[b + 1]; s < e; s++) {
                int2 x = inc[s];
                if (x.y == a) {  // a triangle with b -> a
                    found = enc(dtri(x.x), m1(dori(x.x)));
                    cnt++;
                }
            }
            if (cnt > 1) set_err(ct, GPUDT_ERR_TOPOLOGY, 20);
            if (found < 0) atomicAdd(&ct->changed, 1);  // hull edge
            n[k] = found;
        }
        tn[t] = make_int4(n[0], n[1], n[2], 0);
    }
};

struct SetVtri {
    const int4 *tv;
    int *vtri;
    __device__ void operator()(long long i) const
    {
        int t = (int)i;
        int4 v = tv[t];
        if (v.x < 0) return;
        vtri[v.x] = enc(t, 0);
        vtri[v.y] = enc(t, 1);
        vtri[v.z] = enc(t, 2);
    }
};

int stage_links(Ctx &c)
{
    int r = read_counters(c);
    if (r) return r;
    int nt = c.hctr->ntris;
    int *deg = c.deg;       // [V+1]
    int *start = c.aux2;    // [V+1]
    GALPHA_CUDA(cudaMemsetAsync(deg, 0, sizeof(int) * (size_t)(c.V + 1), c.stream));
    launch_n(c, CountDeg{c.tv, deg}, nt);
    r = exclusive_scan_int(c, deg, start, c.V + 1, nullptr);
    if (r) return r;
    GALPHA_CUDA(cudaMemsetAsync(deg, 0, sizeof(int) * (size_t)(c.V + 1), c.stream));
    int2 *inc = (int2 *)c.rec;  // relink records are not in use yet: 3*cap int2
    launch_n(c, FillInc{c.tv, start, deg, inc}, nt);
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    launch_n(c, MatchLinks{c.tv, c.tn, start, inc, c.vtri, c.ctr}, nt);
    launch_n(c, SetVtri{c.tv, c.vtri}, nt);
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return c.hctr->err;
    // the only hull edges are the F edges of the fake ring
    if (c.hctr->changed != c.F) {
        c.hctr->errinfo = c.hctr->changed;
        return GPUDT_ERR_TOPOLOGY;
    }
    return GPUDT_OK;
}

// ------------------------------------------------------------------- relink
struct Relinker {
    int4 *tn;
    const int4 *fwd;
    const int *epoch;
    const Relink *rec;
    const int4 *tv;
    int *vtri;
    int round;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        Relink r = rec[i];
        if (r.old < 0) {
            if (r.loc >= 0) set_link(tn, r.loc, -1);
            return;
        }
        int u = dtri(r.old), b = dori(r.old);
        if (epoch[u] == round) {
            const int *f = (const int *)&fwd[u];
            int there = f[b];
            if (r.loc >= 0) set_link(tn, r.loc, there);
            else if (there < 0) set_err(ct, GPUDT_ERR_TOPOLOGY, 30);  // both sides became hull
        } else {
            if (r.loc >= 0) set_link(tn, r.loc, r.old);
            int *p = (int *)&tn[u];
            p[b] = r.loc;  // -1 when the edge became a hull edge
            if (r.loc < 0) {
                int4 w = tv[u];
                vtri[geti(w, p1(b))] = enc(u, p1(b));
                vtri[geti(w, m1(b))] = enc(u, m1(b));
            }
        }
    }
};

// Every operation round gets a fresh id from the handle's counter (the
// round-stamped arrays belong to the handle's arena, so ids must not repeat
// on a handle, whichever thread drives it).
static int next_round(Ctx &c)
{
    return ++c.round_counter;
}
// Marks the k ids after `first` (first + 1 .. first + k) as used by rounds
// that device code numbered itself.
static void skip_rounds(Ctx &c, int first, int k)
{
    if (first + k > c.round_counter) c.round_counter = first + k;
}

// ------------------------------------------------------------------- shift
// A fan walk around interior vertex v: calls f(t, i, a, b) for every
// triangle (v, a, b) counterclockwise; returns false on a fan over kMaxFan*4.
template <class Fn>
__device__ __forceinline__ bool walk_fan(const int4 *tv, const int4 *tn, int start, Fn f)
{
    int e = start;
    for (int guard = 0; guard < 4 * kMaxFan; guard++) {
        int t = dtri(e), i = dori(e);
        int4 w = tv[t];
        if (!f(t, i, geti(w, p1(i)), geti(w, m1(i)))) return true;
        int nx = geti(tn[t], p1(i));  // across (b, v)
        if (nx < 0) return true;
        e = enc(dtri(nx), p1(dori(nx)));
        if (e == start) return true;
    }
    return false;
}

struct ShiftRound {
    const int4 *tv, *tn;
    double2 *pos;
    const double2 *opos;
    int8_t *vstate;
    int *vround;
    const int *vtri;
    int round;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int v = (int)ii;
        if (vstate[v] != VS_UNDECIDED) return;
        uint32_t pv = prio((uint32_t)v);
        bool wait = false, ok = true;
        double2 q = opos[v];
        OrientTally tally;
        bool fine = walk_fan(tv, tn, vtri[v], [&](int t, int i, int a, int b) {
            int ra = vround[a];
            if ((ra == 0 || ra == round) && prio((uint32_t)a) < pv) {
                wait = true;
                return false;
            }
            if (ok && orient_staged(q, pos[a], pos[b], ct, tally) <= 0) ok = false;
            return true;
        });
        tally.flush(ct);
        if (!fine) {
            set_err(ct, GPUDT_ERR_TOPOLOGY, 40);
            return;
        }
        if (wait) {
            atomicAdd(&ct->nlist, 1);
            return;
        }
        vround[v] = round;
        if (ok) {
            pos[v] = q;
            vstate[v] = VS_SHIFTED;
        } else {
            vstate[v] = VS_BAD;
            atomicAdd(&ct->changed, 1);
        }
    }
};

// Optimistic shifting: every undecided site is a candidate for its true
// position; a triangle that would not stay counterclockwise with its candidate
// vertices moved drops those candidates; repeated until no triangle drops
// anything.  At the fixed point every triangle is counterclockwise with all
// remaining candidates moved together, so they are committed at once and only
// the dropped sites go through the priority rounds (ShiftRound).
struct ShiftCandidates {
    const int8_t *vstate;
    int8_t *cand;
    __device__ void operator()(long long i) const { cand[i] = vstate[i] == VS_UNDECIDED ? 1 : 0; }
};

// Drops candidate v (once per iteration) and lists it.
__device__ __forceinline__ void shift_drop(int v, const int8_t *cand, int *drop, int *list, int *n)
{
    if (cand[v] && atomicExch(&drop[v], 1) == 0) list[atomicAdd(n, 1)] = v;
}

// A triangle with candidate vertices that would not stay counterclockwise with
// them moved drops them.
__device__ __forceinline__ void shift_check(int4 v, const double2 *pos, const double2 *opos, const int8_t *cand,
                                            int *drop, int *list, int *n, Counters *ct)
{
    const int8_t c0 = cand[v.x], c1 = cand[v.y], c2 = cand[v.z];
    if (!(c0 | c1 | c2)) return;
    const double2 a = c0 ? opos[v.x] : pos[v.x];
    const double2 b = c1 ? opos[v.y] : pos[v.y];
    const double2 c = c2 ? opos[v.z] : pos[v.z];
    if (orientp(a, b, c, ct) > 0) return;
    if (c0) shift_drop(v.x, cand, drop, list, n);
    if (c1) shift_drop(v.y, cand, drop, list, n);
    if (c2) shift_drop(v.z, cand, drop, list, n);
}

// First iteration: every triangle.
struct ShiftCheckTris {
    const int4 *tv;
    const double2 *pos, *opos;
    const int8_t *cand;
    int *drop, *list, *n;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int4 v = tv[ii];
        if (v.x < 0) return;
        shift_check(v, pos, opos, cand, drop, list, n, ct);
    }
};

// Later iterations: only a triangle with a vertex dropped in the previous
// iteration can change its outcome, so the fans of those vertices are checked.
struct ShiftCheckFans {
    const int4 *tv, *tn;
    const int *vtri;
    const double2 *pos, *opos;
    const int8_t *cand;
    const int *prev;
    int *drop, *list, *n;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int v = prev[ii];
        const bool fine = walk_fan(tv, tn, vtri[v], [&](int t, int, int, int) {
            shift_check(tv[t], pos, opos, cand, drop, list, n, ct);
            return true;
        });
        if (!fine) set_err(ct, GPUDT_ERR_TOPOLOGY, 41);
    }
};

// Takes the listed vertices out of the candidate set and appends them to the
// list of all dropped vertices (its order is immaterial: the priority rounds
// decide by vertex priority, not by list position).
struct ShiftDropList {
    const int *list;
    int8_t *cand;
    int *drop, *all, *total;
    int cap;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        const int v = list[i];
        drop[v] = 0;
        cand[v] = 0;
        const int k = atomicAdd(total, 1);
        if (k < cap) all[k] = v;
        else set_err(ct, GPUDT_ERR_TOPOLOGY, 42);
    }
};

// The undecided sites for the priority rounds: ring position ii of a list.
struct ShiftRoundList {
    ShiftRound r;
    const int *list;
    __device__ void operator()(long long ii) const { r(list[ii]); }
};

struct ShiftCommit {
    const int8_t *cand;
    double2 *pos;
    const double2 *opos;
    int8_t *vstate;
    int *vround;
    __device__ void operator()(long long i) const
    {
        if (!cand[i]) return;
        pos[i] = opos[i];
        vstate[i] = VS_SHIFTED;
        vround[i] = 1;  // decided before the priority rounds start
    }
};

// Select BAD vertices that are the priority minimum among their BAD neighbours.
struct BadSelect {
    const int4 *tv, *tn;
    const int8_t *vstate;
    const int *vtri;
    int *list;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int v = (int)ii;
        if (vstate[v] != VS_BAD) return;
        uint32_t pv = prio((uint32_t)v);
        bool wait = false;
        walk_fan(tv, tn, vtri[v], [&](int t, int i, int a, int b) {
            if (vstate[a] == VS_BAD && prio((uint32_t)a) < pv) {
                wait = true;
                return false;
            }
            return true;
        });
        if (wait) return;
        int k = atomicAdd(&ct->nlist, 1);
        list[k] = v;
    }
};

// BAD sites are among the dropped ones.
struct BadSelectList {
    BadSelect b;
    const int *list;
    __device__ void operator()(long long ii) const { b(list[ii]); }
};

// Remove vertex v (interior) and triangulate its star hole by ear clipping
// with the kernel point K = pos[v] (cudaShifting.cu:350-450 semantics: an ear
// (A,B,C) is cut when ccw(A,B,C) > 0 and K is strictly left of A->C).
struct BadRemove {
    int4 *tv, *tn, *fwd;
    int *epoch, *freelist, *vtri, *anchor;
    const int *list;
    double2 *pos;
    int8_t *vstate;
    Relink *rec;
    int round, nreal;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int v = list[ii];
        int U[kMaxFan], Fs[kMaxFan], Fi[kMaxFan], O[kMaxFan];
        int d = 0;
        bool over = false;
        bool fine = walk_fan(tv, tn, vtri[v], [&](int t, int i, int a, int b) {
            if (d >= kMaxFan) {
                over = true;
                return false;
            }
            U[d] = a;
            Fs[d] = t;
            Fi[d] = i;
            O[d] = geti(tn[t], i);
            d++;
            return true;
        });
        if (!fine || over || d < 3) {
            set_err(ct, GPUDT_ERR_TOPOLOGY, 50);
            return;
        }
        double2 K = pos[v];
        // polygon ring with owners of each current edge (U[k] -> U[next])
        int nxt[kMaxFan], prv[kMaxFan], own[kMaxFan];  // own: -2-k original edge k, else loc
        for (int k = 0; k < d; k++) {
            nxt[k] = (k + 1) % d;
            prv[k] = (k + d - 1) % d;
            own[k] = -2 - k;
        }
        int used = 0, remaining = d, cur = 0, stall = 0;
        auto owner_link = [&](int ownv, int loc) {
            if (ownv <= -2) {
                int k = -2 - ownv;
                set_fwd(fwd, Fs[k], Fi[k], loc);
                push_rec(rec, ct, loc, O[k]);
            } else {
                set_link(tn, loc, ownv);
                set_link(tn, ownv, loc);
            }
        };
        for (int k = 0; k < d; k++) epoch[Fs[k]] = round;
        // strict pass first (K strictly inside what remains); when a full
        // cycle finds no such ear, K lies on a candidate diagonal and the
        // closed test is used (the rest stays star-shaped from K)
        bool strict = true;
        while (remaining > 3) {
            int A = prv[cur], B = cur, C = nxt[cur];
            bool ear = orientp(pos[U[A]], pos[U[B]], pos[U[C]], ct) > 0;
            if (ear && remaining > 4) {
                int k = orientp(pos[U[A]], pos[U[C]], K, ct);
                ear = strict ? k > 0 : k >= 0;
            } else if (ear) {
                // last quad: any diagonal giving two counterclockwise triangles
                int D = nxt[C];
                ear = orientp(pos[U[A]], pos[U[C]], pos[U[D]], ct) > 0;
            }
            if (ear) {
                int s = Fs[used++];
                tv[s] = make_int4(U[A], U[B], U[C], 0);
                tn[s] = make_int4(-1, -1, -1, 0);
                // edges: opp A (0) = B->C owned by own[B]; opp C (2) = A->B owned by own[A];
                // opp B (1) = C->A: the new diagonal, owner of ring edge A->C
                owner_link(own[B], enc(s, 0));
                owner_link(own[A], enc(s, 2));
                own[A] = enc(s, 1);
                vtri[U[A]] = enc(s, 0);
                vtri[U[B]] = enc(s, 1);
                vtri[U[C]] = enc(s, 2);
                nxt[A] = C;
                prv[C] = A;
                remaining--;
                cur = C;
                stall = 0;
                strict = true;
            } else {
                cur = nxt[cur];
                if (++stall > remaining + 1) {
                    if (strict) {
                        strict = false;
                        stall = 0;
                        continue;
                    }
                    set_err(ct, GPUDT_ERR_TOPOLOGY, 51);
                    return;
                }
            }
        }
        {
            int A = cur, B = nxt[cur], C = nxt[nxt[cur]];
            if (orientp(pos[U[A]], pos[U[B]], pos[U[C]], ct) <= 0) {
                set_err(ct, GPUDT_ERR_TOPOLOGY, 52);
                return;
            }
            int s = Fs[used++];
            tv[s] = make_int4(U[A], U[B], U[C], 0);
            tn[s] = make_int4(-1, -1, -1, 0);
            owner_link(own[B], enc(s, 0));
            owner_link(own[C], enc(s, 1));
            owner_link(own[A], enc(s, 2));
            vtri[U[A]] = enc(s, 0);
            vtri[U[B]] = enc(s, 1);
            vtri[U[C]] = enc(s, 2);
        }
        for (int k = used; k < d; k++) free_slot(tv, freelist, ct, Fs[k]);
        int an = U[0];
        for (int k = 0; k < d; k++)
            if (U[k] < nreal) {
                an = U[k];
                break;
            }
        vtri[v] = -1;
        vstate[v] = VS_MISSING;
        anchor[v] = an;
    }
};

struct CountState {
    const int8_t *vstate;
    int8_t s;
    int *list;
    Counters *ct;
    __device__ void operator()(long long i) const
    {
        const bool hit = vstate[i] == s;
        const int k = warp_reserve(&ct->nlist, hit ? 1 : 0);  // one atomic per warp
        if (hit && list) list[k] = (int)i;
    }
};

// Rounds of the shifting loops run in groups of c.shift_group between counter
// reads: list lengths stay on the device (launch_dev), each round's count is
// kept in ct->grp[], and a round after the loop's last one does nothing (an
// empty list, or no site left in the state it acts on), so running past the
// end of a loop changes no result.

int stage_shift(Ctx &c)
{
    const int kShiftGroup = c.shift_group;
    int r;
    int shiftRounds = 0, badCount = 0;
    int *dropped = c.aux2;  // every site the optimistic phase dropped: the only undecided ones after it
    {
        // candidate flags (bytes) and per-iteration drop flags (ints) share list2
        int8_t *cand = (int8_t *)c.list2;
        int *drop = c.list2 + ((c.V + 1023) >> 2) + 256;
        int *lists[2] = {c.list, c.aux};  // vertices dropped in an iteration (ping-pong)
        launch_n(c, ShiftCandidates{c.vstate, cand}, c.V);
        GALPHA_CUDA(cudaMemsetAsync(drop, 0, sizeof(int) * (size_t)c.V, c.stream));
        GALPHA_CUDA(cudaMemsetAsync(c.ctr->sh_n, 0, 3 * sizeof(int), c.stream));  // sh_n[2], sh_total
        bool settled = false;
        for (int it = 0; !settled;) {
            for (int j = 0; j < kShiftGroup; j++, it++) {
                int *cur = lists[it & 1], *prev = lists[(it + 1) & 1];
                int *curn = &c.ctr->sh_n[it & 1], *prevn = &c.ctr->sh_n[(it + 1) & 1];
                GALPHA_CUDA(cudaMemsetAsync(curn, 0, sizeof(int), c.stream));
                if (it == 0)
                    launch_dev(c, ShiftCheckTris{c.tv, c.pos, c.opos, cand, drop, cur, curn, c.ctr}, &c.ctr->ntris,
                               c.cap_tris);
                else
                    launch_dev(c, ShiftCheckFans{c.tv, c.tn, c.vtri, c.pos, c.opos, cand, prev, drop, cur, curn,
                                                 c.ctr},
                               prevn, c.V);
                launch_dev(c, ShiftDropList{cur, cand, drop, dropped, &c.ctr->sh_total, c.N, c.ctr}, curn, c.V);
                launch_n(c, CopyElems<int>{&c.ctr->grp[j], curn}, 1);
            }
            r = read_counters(c);
            if (r) return r;
            if (c.hctr->err) return c.hctr->err;
            for (int j = 0; j < kShiftGroup && !settled; j++) {
                shiftRounds++;
                settled = c.hctr->grp[j] == 0;
            }
            if (!settled && shiftRounds >= c.max_rounds) return GPUDT_ERR_NOCONVERGE;
        }
        launch_n(c, ShiftCommit{cand, c.pos, c.opos, c.vstate, c.vround}, c.V);
    }
    // vertices fixed from the start (fake ring) and the optimistic set count
    // as decided in the first shifting round (id 1); the rest go through
    // priority rounds
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    for (int round = 2, done = 0; !done;) {
        for (int j = 0; j < kShiftGroup; j++, round++) {
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
            launch_dev(c,
                       ShiftRoundList{ShiftRound{c.tv, c.tn, c.pos, c.opos, c.vstate, c.vround, c.vtri, round, c.ctr},
                                      dropped},
                       &c.ctr->sh_total, c.N);
            launch_n(c, CopyElems<int>{&c.ctr->grp[j], &c.ctr->nlist}, 1);
        }
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        for (int j = 0; j < kShiftGroup && !done; j++) {
            shiftRounds++;
            done = c.hctr->grp[j] == 0;
        }
        if (!done && shiftRounds > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
    }
    badCount = c.hctr->changed;
    c.st.shiftRounds = shiftRounds;
    c.st.nBadShift = badCount;
    // remove the unshiftable sites in independent rounds
    int guard = 0;
    const long long recn = 4LL * c.cap_tris;
    while (badCount > 0) {
        for (int j = 0; j < kShiftGroup; j++) {
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
            launch_dev(c, BadSelectList{BadSelect{c.tv, c.tn, c.vstate, c.vtri, c.list, c.ctr}, dropped},
                       &c.ctr->sh_total, c.N);
            launch_n(c, CopyElems<int>{&c.ctr->grp[j], &c.ctr->nlist}, 1);
            const int round = next_round(c);
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nrec, 0, sizeof(int), c.stream));
            // a round selects at most the bad sites left (the grid is sized by them:
            // an empty round of this local-memory-heavy kernel then stays cheap)
            launch_dev(c, BadRemove{c.tv, c.tn, c.fwd, c.epoch, c.freelist, c.vtri, c.anchor, c.list, c.pos,
                                    c.vstate, c.rec, round, c.N, c.ctr},
                       &c.ctr->nlist, badCount);
            launch_dev(c, Relinker{c.tn, c.fwd, c.epoch, c.rec, c.tv, c.vtri, round, c.ctr}, &c.ctr->nrec, recn);
        }
        GALPHA_CUDA(cudaGetLastError());
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        bool stuck = false;
        for (int j = 0; j < kShiftGroup && !stuck; j++) {
            stuck = c.hctr->grp[j] == 0;
            badCount -= c.hctr->grp[j];
        }
        if (stuck) break;
        guard += kShiftGroup;
        if (guard > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
    }
    return GPUDT_OK;
}

// ----------------------------------------------------------------- missing
// Straight-line walk from vertex a to point q.  Returns the triangle and the
// location kind: 0 inside, 1 on the edge opposite vtx[k] (k in *edge),
// 2 on vertex vtx[k] (coincident), -1 failure.
__device__ int locate_walk(const int4 *tv, const int4 *tn, const double2 *P, const int *vtri, int a, double2 q,
                           int *tri, int *edge, Counters *ct, OrientTally &n)
{
    int budget = 1 << 22;  // total walk steps over all restarts
    for (int restart = 0; restart < 4096; restart++) {
        double2 A = P[a];
        if (A.x == q.x && A.y == q.y) {
            int e = vtri[a];
            *tri = dtri(e);
            *edge = dori(e);
            return 2;
        }
        // 1. wedge of a containing q: counterclockwise from vtri[a]; a hull
        //    vertex's fan is open, so the clockwise side is searched after
        int e = vtri[a], t = -1, ia = 0;
        for (int dir = 0; dir < 2 && t < 0; dir++) {
            e = vtri[a];
            for (int guard = 0; guard < 4 * kMaxFan; guard++) {
                int tt = dtri(e), i = dori(e);
                int4 w = tv[tt];
                int b = geti(w, p1(i)), c = geti(w, m1(i));
                if (orient_staged(A, P[b], q, ct, n) >= 0 && orient_staged(A, P[c], q, ct, n) <= 0) {
                    t = tt;
                    ia = i;
                    break;
                }
                int nx = dir == 0 ? geti(tn[tt], p1(i)) : geti(tn[tt], m1(i));
                if (nx < 0) break;
                e = dir == 0 ? enc(dtri(nx), p1(dori(nx))) : enc(dtri(nx), m1(dori(nx)));
                if (e == vtri[a]) break;
            }
        }
        if (t < 0) return -1;
        // 2. walk along a -> q
        int4 w = tv[t];
        int b = geti(w, p1(ia)), c = geti(w, m1(ia));
        int cross = ia;  // index (in t) of the vertex opposite the edge to cross
        if (orient_staged(P[b], P[c], q, ct, n) >= 0) {
            goto classify_t;
        }
        for (; budget > 0; budget--) {
            // cross edge (b, c) of t (opposite vtx[cross]); b right of a->q, c left
            int nx = geti(tn[t], cross);
            if (nx < 0) return -1;
            t = dtri(nx);
            int j = dori(nx);
            w = tv[t];
            int d = geti(w, j);  // new triangle (d, c, b)
            int o1 = orient_staged(P[b], P[d], q, ct, n), o2 = orient_staged(P[d], P[c], q, ct, n);
            if (o1 >= 0 && o2 >= 0) goto classify_t;
            int od = orient_staged(A, q, P[d], ct, n);
            if (od > 0) {
                // exit through (b, d): opposite c = vtx[p1(j)]
                c = d;
                cross = p1(j);
            } else if (od < 0) {
                // exit through (d, c): opposite b = vtx[m1(j)]
                b = d;
                cross = m1(j);
            } else {
                a = d;  // the walk runs through vertex d: restart there
                goto next_restart;
            }
        }
        return -1;
    classify_t: {
        int4 v = tv[t];
        int x[3] = {v.x, v.y, v.z};
        int o[3], zeros = 0, zk = -1, nzk = -1;
        for (int k = 0; k < 3; k++) {
            o[k] = orient_staged(P[x[p1(k)]], P[x[m1(k)]], q, ct, n);
            if (o[k] < 0) return -1;
            if (o[k] == 0) {
                zeros++;
                zk = k;
            } else {
                nzk = k;
            }
        }
        *tri = t;
        if (zeros == 0) {
            *edge = 0;
            return 0;
        }
        if (zeros == 1) {
            *edge = zk;
            return 1;
        }
        *edge = nzk;
        return 2;
    }
    next_restart:;
    }
    return -1;
}

struct MissingLocate {
    const int4 *tv, *tn;
    const double2 *pos, *opos;
    const int *vtri, *anchor;
    int8_t *vstate;
    const int *list;
    int *loc;  // [nlist] encoded (t<<2)|edge, kind in bit 30..31 via separate array
    int *kind;
    int *vote;
    int fallback;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int m = list[ii];
        if (vstate[m] != VS_MISSING) {
            kind[ii] = -1;
            return;
        }
        int a = anchor[m];
        for (int g = 0; g < 64 && a >= 0 && vtri[a] < 0; g++) a = anchor[a];
        if (a < 0 || vtri[a] < 0) a = fallback;
        int t, e;
        OrientTally tally;
        int k = locate_walk(tv, tn, pos, vtri, a, opos[m], &t, &e, ct, tally);
        tally.flush(ct);
        kind[ii] = k;
        if (k < 0) {
            set_err(ct, GPUDT_ERR_TOPOLOGY, 60);
            return;
        }
        loc[ii] = enc(t, e);
        if (k == 2) return;
        atomicMin(&vote[t], m);
        if (k == 1) {
            int nb = geti(tn[t], e);
            if (nb < 0) {
                set_err(ct, GPUDT_ERR_TOPOLOGY, 61);
                return;
            }
            atomicMin(&vote[dtri(nb)], m);
        }
    }
};

struct MissingInsert {
    int4 *tv, *tn, *fwd;
    int *epoch, *freelist, *vtri, *vote;
    double2 *pos;
    const double2 *opos;
    int8_t *vstate;
    const int *list, *loc, *kind;
    Relink *rec;
    int round, cap;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int k = kind[ii];
        if (k < 0) return;
        int p = list[ii];
        int t = dtri(loc[ii]), i = dori(loc[ii]);
        if (k == 2) {
            vstate[p] = VS_DUP;
            atomicAdd(&ct->changed, 1);
            atomicAdd(&ct->ndup, 1);
            return;
        }
        if (vote[t] != p) return;
        int4 v = tv[t], n = tn[t];
        if (k == 0) {
            int v0 = v.x, v1 = v.y, v2 = v.z;
            int s1 = alloc_slot(freelist, ct, cap), s2 = alloc_slot(freelist, ct, cap);
            if (s1 < 0 || s2 < 0) return;
            epoch[t] = round;
            tv[t] = make_int4(p, v1, v2, 0);
            tv[s1] = make_int4(p, v2, v0, 0);
            tv[s2] = make_int4(p, v0, v1, 0);
            tn[t] = make_int4(-1, enc(s1, 2), enc(s2, 1), 0);
            tn[s1] = make_int4(-1, enc(s2, 2), enc(t, 1), 0);
            tn[s2] = make_int4(-1, enc(t, 2), enc(s1, 1), 0);
            fwd[t] = make_int4(enc(t, 0), enc(s1, 0), enc(s2, 0), 0);
            push_rec(rec, ct, enc(t, 0), n.x);
            push_rec(rec, ct, enc(s1, 0), n.y);
            push_rec(rec, ct, enc(s2, 0), n.z);
            vtri[p] = enc(t, 0);
            vtri[v1] = enc(t, 1);
            vtri[v2] = enc(t, 2);
            vtri[v0] = enc(s1, 2);
        } else {
            int o0 = geti(n, i);
            int u = dtri(o0), j = dori(o0);
            if (vote[u] != p) return;
            int v0 = geti(v, i), v1 = geti(v, p1(i)), v2 = geti(v, m1(i));
            int o1 = geti(n, p1(i)), o2 = geti(n, m1(i));
            int4 wv = tv[u], wn = tn[u];
            int w = geti(wv, j);
            int ou1 = geti(wn, p1(j)), ou2 = geti(wn, m1(j));
            int s1 = alloc_slot(freelist, ct, cap), s2 = alloc_slot(freelist, ct, cap);
            if (s1 < 0 || s2 < 0) return;
            epoch[t] = round;
            epoch[u] = round;
            // A = t (p,v2,v0), B = s1 (p,v0,v1), C = u (p,v1,w), D = s2 (p,w,v2)
            tv[t] = make_int4(p, v2, v0, 0);
            tv[s1] = make_int4(p, v0, v1, 0);
            tv[u] = make_int4(p, v1, w, 0);
            tv[s2] = make_int4(p, w, v2, 0);
            tn[t] = make_int4(-1, enc(s1, 2), enc(s2, 1), 0);
            tn[s1] = make_int4(-1, enc(u, 2), enc(t, 1), 0);
            tn[u] = make_int4(-1, enc(s2, 2), enc(s1, 1), 0);
            tn[s2] = make_int4(-1, enc(t, 2), enc(u, 1), 0);
            int4 ft = make_int4(0, 0, 0, 0), fu = make_int4(0, 0, 0, 0);
            seti(ft, i, -1);
            seti(ft, p1(i), enc(t, 0));
            seti(ft, m1(i), enc(s1, 0));
            seti(fu, j, -1);
            seti(fu, p1(j), enc(u, 0));
            seti(fu, m1(j), enc(s2, 0));
            fwd[t] = ft;
            fwd[u] = fu;
            push_rec(rec, ct, enc(t, 0), o1);
            push_rec(rec, ct, enc(s1, 0), o2);
            push_rec(rec, ct, enc(u, 0), ou1);
            push_rec(rec, ct, enc(s2, 0), ou2);
            vtri[p] = enc(t, 0);
            vtri[v2] = enc(t, 1);
            vtri[v0] = enc(t, 2);
            vtri[v1] = enc(u, 1);
            vtri[w] = enc(u, 2);
        }
        pos[p] = opos[p];
        vstate[p] = VS_SHIFTED;
        atomicAdd(&ct->changed, 1);
    }
};

struct ResetVotes {
    int *vote;
    const int4 *tn;
    const int *loc, *kind;
    __device__ void operator()(long long ii) const
    {
        int k = kind[ii];
        if (k < 0 || k == 2) return;
        int t = dtri(loc[ii]);
        vote[t] = 0x7fffffff;
    }
};

struct ResetVotesEdge {
    int *vote;
    const int *list2;  // neighbour slots tagged for edge insertions
    __device__ void operator()(long long ii) const { vote[list2[ii]] = 0x7fffffff; }
};

// Record the neighbour slot of every on-edge insertion (before the mesh changes).
struct EdgeTags {
    const int4 *tn;
    const int *loc, *kind;
    int *list2;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        if (kind[ii] != 1) return;
        int t = dtri(loc[ii]), e = dori(loc[ii]);
        int nb = geti(tn[t], e);
        if (nb < 0) return;
        int k = atomicAdd(&ct->nlist2, 1);
        list2[k] = dtri(nb);
    }
};

int stage_missing(Ctx &c)
{
    int r;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
    launch_n(c, CountState{c.vstate, VS_MISSING, c.list, c.ctr}, c.N);
    r = read_counters(c);
    if (r) return r;
    int nmiss = c.hctr->nlist;
    c.st.nMissing = nmiss;
    if (nmiss == 0) return GPUDT_OK;
    int *loc = c.aux, *kind = c.aux2 + 0;
    // aux2 holds kind at [0, nmiss) ; edge tags in list2.  Rounds run in
    // groups of c.missing_group between counter reads (a round after the last
    // insertion finds no missing site and does nothing); each round's
    // insertions are kept in ct->grp[].
    const int kMissingGroup = c.missing_group;
    const long long recn = 4LL * c.cap_tris;
    int rounds = 0, remaining = nmiss, dups = 0;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->ndup, 0, sizeof(int), c.stream));
    while (remaining > 0) {
        for (int j = 0; j < kMissingGroup; j++) {
            int round = next_round(c);
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nrec, 0, sizeof(int), c.stream));
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
            launch_n(c, MissingLocate{c.tv, c.tn, c.pos, c.opos, c.vtri, c.anchor, c.vstate, c.list, loc, kind,
                                      c.vote, c.N, c.ctr},
                     nmiss);
            launch_n(c, EdgeTags{c.tn, loc, kind, c.list2, c.ctr}, nmiss);
            launch_n(c, MissingInsert{c.tv, c.tn, c.fwd, c.epoch, c.freelist, c.vtri, c.vote, c.pos, c.opos,
                                      c.vstate, c.list, loc, kind, c.rec, round, c.cap_tris, c.ctr},
                     nmiss);
            launch_n(c, ClampFree{c.ctr}, 1);  // a pop past the free list took tail slots
            launch_dev(c, Relinker{c.tn, c.fwd, c.epoch, c.rec, c.tv, c.vtri, round, c.ctr}, &c.ctr->nrec, recn);
            launch_n(c, ResetVotes{c.vote, c.tn, loc, kind}, nmiss);
            launch_dev(c, ResetVotesEdge{c.vote, c.list2}, &c.ctr->nlist2, c.cap_tris);
            launch_n(c, CopyElems<int>{&c.ctr->grp[j], &c.ctr->changed}, 1);
        }
        GALPHA_CUDA(cudaGetLastError());
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        if (c.hctr->ntris > c.cap_tris) return GPUDT_ERR_NOMEM;
        for (int j = 0; j < kMissingGroup && remaining > 0; j++) {
            const int done = c.hctr->grp[j];
            remaining -= done;
            rounds++;
            if (done == 0 || rounds > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
        }
    }
    dups = c.hctr->ndup;
    c.st.nDuplicates = dups;
    c.st.missingRounds = rounds;
    return GPUDT_OK;
}

// ---------------------------------------------------------------- boundary
// Fan of a hull vertex f: from the clockwise-most triangle (whose edge f->u0 is
// a hull edge) counterclockwise to the triangle whose edge ud->f is a hull edge.
// Fake ring sites are removed class by class (ring index mod 4 in the order
// 0, 2, 1, 3): sites of one class are separated along the border by sites of
// other classes that are still present, so they are not adjacent and their
// fans are disjoint; the priority test below only matters in the rare case of
// an edge cutting a texture corner.
constexpr int kMaxChain = 256;

// Selection of fake sites to remove together: a fake whose fan (walked once
// each way from vtri) holds no competing fake of lower priority -- in the
// first pass only fakes of its ring class (ring position modulo 4) compete,
// later every remaining fake does.  The selected fake's fan is stored (slot
// and index of f, packed, and the outer neighbour across the chain edge) so
// that the removal reads it with independent loads instead of walking again;
// fans of selected fakes are disjoint, so they stay valid until the removal.
constexpr int kMaxFanLong = 4096;  // longest fan a fake may have (error beyond)

struct FakeSelect {
    const int4 *tv, *tn;
    const int8_t *vstate;
    const int *vtri;
    int *list, *fanoff, *fanlen;
    int2 *fan;
    int *count, *fan_n;
    int N, cls;  // cls < 0: every remaining fake competes by priority
    Counters *ct;
    __device__ bool conflicts(int g, uint32_t pf) const
    {
        return g >= N && vstate[g] == VS_FAKE && (cls < 0 || ((g - N) & 3) == cls) && prio((uint32_t)g) < pf;
    }
    __device__ void operator()(long long ii) const
    {
        const int f = N + (int)ii;
        constexpr int M = kMaxChain;
        int2 E[2 * M];  // (packed f-corner, outer neighbour) per fan triangle, fans of up to M
        int lo = M, hi = M, nccw = 0, ncw = 0, ecw = -1;
        bool pick = (cls < 0 || ((int)ii & 3) == cls) && vstate[f] == VS_FAKE;
        if (pick) {
            const uint32_t pf = prio((uint32_t)f);
            const int e0 = vtri[f];
            int e = e0;
            ecw = e0;
            for (;;) {  // counterclockwise from e0
                const int t = dtri(e), i = dori(e);
                const int4 w = tv[t], n = tn[t];
                if (conflicts(geti(w, p1(i)), pf) || conflicts(geti(w, m1(i)), pf)) {
                    pick = false;
                    break;
                }
                if (hi < 2 * M) E[hi++] = make_int2(e, geti(n, i));
                nccw++;
                const int nx = geti(n, p1(i));  // across (b, f)
                if (nx < 0) break;
                e = enc(dtri(nx), p1(dori(nx)));
                if (e == e0 || nccw > kMaxFanLong) {
                    set_err(ct, GPUDT_ERR_TOPOLOGY, 70);
                    pick = false;
                    break;
                }
            }
            e = e0;
            while (pick) {  // clockwise from e0
                const int nx = geti(tn[dtri(e)], m1(dori(e)));  // across (f, a)
                if (nx < 0) break;
                e = enc(dtri(nx), m1(dori(nx)));
                const int t = dtri(e), i = dori(e);
                const int4 w = tv[t];
                if (conflicts(geti(w, p1(i)), pf)) {
                    pick = false;
                    break;
                }
                if (nccw + ncw >= kMaxFanLong) {
                    set_err(ct, GPUDT_ERR_TOPOLOGY, 71);
                    pick = false;
                    break;
                }
                if (lo > 0) E[--lo] = make_int2(e, geti(tn[t], i));
                ncw++;
                ecw = e;
            }
        }
        const int d = pick ? nccw + ncw : 0;
        const int k = warp_reserve(count, pick ? 1 : 0);
        const int base = warp_reserve(fan_n, d);
        if (pick) {
            list[k] = f;
            fanoff[k] = base;
            fanlen[k] = d;
            if (d <= M) {
                for (int q = 0; q < d; q++) fan[base + q] = E[lo + q];
            } else {
                // a long fan: walk it again from its clockwise end, into the store
                int e = ecw;
                for (int q = 0; q < d; q++) {
                    const int t = dtri(e), i = dori(e);
                    const int4 n = tn[t];
                    fan[base + q] = make_int2(e, geti(n, i));
                    const int nx = geti(n, p1(i));
                    if (nx < 0) break;
                    e = enc(dtri(nx), p1(dori(nx)));
                }
            }
        }
        warp_reserve(&ct->changed, pick ? 1 : 0);
    }
};

// Runs of fake sites removed as one unit.  Removing one ring class after
// another leaves the last class as a chain: collinear fakes on a side of the
// texture become hull neighbours through the chords their removed neighbours
// leave, so every fake of the last class touches the next one and the
// priority rounds take out only about a third of the chain per round.  A run
// -- selected fakes that follow each other along the hull -- has as outer
// boundary the concatenation of its members' fan chains without the one
// triangle each consecutive pair shares; the stack rule patches that chain
// exactly as it patches one fake's.  Selection by separator levels over the
// class's chain (j = ring position / 4): level l takes the fakes with j a
// multiple of 16^l but not of 16^(l+1), so the kept multiples separate the
// runs of one level (level 0: runs of 15 between every 16th fake).  The
// leader (the member whose clockwise hull neighbour is not selected) stores
// the kept fan entries followed by the shared triangles (outer link -1);
// fanlen holds kept | shared << 16.  A run whose fans touch a selected fake
// of another run, or that closes on itself, is left to the priority rounds.
constexpr int kMaxRunMembers = 64;

// Separator-level selection of the fakes of one ring class (see above).
__device__ __forceinline__ bool run_selected(const int8_t *vstate, int N, int cls, int level, int g)
{
    if (g < N || vstate[g] != VS_FAKE || ((g - N) & 3) != cls) return false;
    const int j = (g - N) >> 2, sh = 4 * level;
    return (j & ((1 << sh) - 1)) == 0 && ((j >> sh) & 15) != 0;
}

// Per selected fake, its own fan: the entries (clockwise end first) in the
// staging array, and a record {offset, length, clockwise end vertex U[0],
// counterclockwise end vertex U[d], valid}.  A fan holding a selected fake
// strictly inside its chain is not valid (it touches another run).  Each
// thread walks one fan, so the latency is that of one fan, not of a run.
struct FakeRunStage {
    const int4 *tv, *tn;
    const int8_t *vstate;
    const int *vtri;
    int N, cls, level;
    int2 *stage;
    int *stage_n;
    int *rec;  // 5 ints per ring position
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int f = N + (int)ii;
        const bool sel = run_selected(vstate, N, cls, level, f);
        int ecw = -1, d = 0, a0 = -1, bend = -1;
        bool ok = sel;
        if (ok) {
            const int e0 = vtri[f];
            int e = e0;
            for (int g = 0;; g++) {  // clockwise to the hull edge (f, U[0])
                const int nx = geti(tn[dtri(e)], m1(dori(e)));
                if (nx < 0) break;
                e = enc(dtri(nx), m1(dori(nx)));
                if (e == e0 || g > kMaxFanLong) {
                    e = -1;
                    break;
                }
            }
            ecw = e;
            ok = ecw >= 0;
        }
        if (ok) {
            int ee = ecw;
            for (;;) {  // counterclockwise: count, ends, foreign selected fakes
                const int t = dtri(ee), i = dori(ee);
                const int4 w = tv[t];
                if (d == 0) a0 = geti(w, p1(i));
                const int bv = geti(w, m1(i));
                bend = bv;
                d++;
                const int nx = geti(tn[t], p1(i));
                if (nx < 0) break;
                if (run_selected(vstate, N, cls, level, bv) || d > kMaxFanLong) {  // U[k] inside the chain
                    ok = false;
                    break;
                }
                ee = enc(dtri(nx), p1(dori(nx)));
            }
        }
        const int off = warp_reserve(stage_n, ok ? d : 0);
        if (ok) {
            int ee = ecw;
            for (int k = 0; k < d; k++) {
                const int t = dtri(ee), i = dori(ee);
                const int4 n = tn[t];
                stage[off + k] = make_int2(ee, geti(n, i));
                const int nx = geti(n, p1(i));
                if (nx < 0) break;
                ee = enc(dtri(nx), p1(dori(nx)));
            }
        }
        if (sel) {
            int *r = rec + 5 * ii;
            r[0] = off;
            r[1] = d;
            r[2] = a0;
            r[3] = bend;
            r[4] = ok ? 1 : 0;
        }
    }
};

// Per run leader (a selected fake whose clockwise hull neighbour is not
// selected): follows the members through their records, checks that each
// next member's clockwise end is the current one, and copies the kept
// entries followed by the shared triangles (outer link -1) into the fan
// store; fanlen = kept | shared << 16.
struct FakeRunJoin {
    const int8_t *vstate;
    int N, cls, level;
    const int2 *stage;
    const int *rec;
    int *list, *fanoff, *fanlen;
    int2 *fan;
    int *count, *fan_n;
    Counters *ct;
    // members and counts of the run led by ring position ii; 0 if invalid
    __device__ int scan(int ii, int *kept, int *nsh) const
    {
        const int f = N + ii;
        int m = ii, nk = 0, ns = 0;
        for (int mi = 0; mi < kMaxRunMembers; mi++) {
            const int *r = rec + 5 * m;
            if (!r[4] || (mi > 0 && r[1] < 2)) return 0;
            const int nxt = r[3];
            const bool next = nxt != f && run_selected(vstate, N, cls, level, nxt);
            if (next && rec[5 * (nxt - N) + 2] != N + m) return 0;  // not hull neighbours
            nk += r[1] - (mi > 0 ? 1 : 0) - (next ? 1 : 0);
            ns += next ? 1 : 0;
            if (!next) {
                *kept = nk;
                *nsh = ns;
                return nk > 0 && nk <= kMaxFanLong ? mi + 1 : 0;
            }
            m = nxt - N;
        }
        return 0;
    }
    __device__ void operator()(long long ii) const
    {
        const int f = N + (int)ii;
        bool pick = run_selected(vstate, N, cls, level, f) && rec[5 * ii + 4] &&
                    !run_selected(vstate, N, cls, level, rec[5 * ii + 2]);
        int kept = 0, nsh = 0, nmem = 0;
        if (pick) {
            nmem = scan((int)ii, &kept, &nsh);
            pick = nmem > 0;
        }
        const int k = warp_reserve(count, pick ? 1 : 0);
        const int base = warp_reserve(fan_n, pick ? kept + nsh : 0);
        if (pick) {
            list[k] = f;
            fanoff[k] = base;
            fanlen[k] = kept | (nsh << 16);
            int m = (int)ii, q = 0;
            for (int mi = 0; mi < nmem; mi++) {
                const int *r = rec + 5 * m;
                const bool next = mi + 1 < nmem;
                const int s0 = mi > 0 ? 1 : 0, s1 = r[1] - (next ? 1 : 0);
                for (int j = s0; j < s1; j++) fan[base + q++] = stage[r[0] + j];
                if (next) {
                    fan[base + kept + mi] = make_int2(stage[r[0] + r[1] - 1].x, -1);
                    m = r[3] - N;
                }
            }
        }
        warp_reserve(&ct->changed, pick ? nmem : 0);
    }
};

struct ZeroInts {
    int *a, *b;
    __device__ void operator()(long long) const
    {
        *a = 0;
        if (b) *b = 0;
    }
};


// Removal of the selected fake sites, one warp per fake: the lanes load the
// stored fan, the chain U[0..d] and its positions into shared memory, then
// patch the pocket with the stack rule (the ccw > 0 rule of
// cudaBoundary.cu:278): for each chain vertex in order, while the last two
// stack vertices and it turn left, they and it become a triangle and the top
// is popped.  The chain is cut into up to 32 pieces that share their end
// vertices; each lane runs the rule on its piece (its pops are pops of the
// whole chain too: a vertex inside the hull of a piece is inside the hull of
// the chain), then lane 0 runs it once more over the pieces' leftover stacks
// in order.  The triangles differ from one sequential pass but fill the same
// pocket (the chain is star-shaped from the removed site), and the flip stage
// makes the mesh Delaunay either way.  The lanes then write the remaining
// hull edges, the boundary candidates and the released slots.
struct FakeRemoveArgs {
    int4 *tv, *tn, *fwd;
    int *epoch, *freelist, *vtri;
    const int *list, *fanoff, *fanlen;
    const int2 *fan;
    const double2 *pos;
    int8_t *vstate;
    Relink *rec;
    int *cand;  // boundary-candidate vertices
    int round;
    Counters *ct;
};

constexpr int kFrPieces = 32;    // one piece per lane
constexpr int kFrMinPiece = 16;  // chain edges per piece at least

// Dynamic shared memory for fans of up to M triangles: Fs, Fi, O (M ints),
// U (M + 1), the stacks S, SO (M + 1 + kFrPieces each: each piece's stack
// starts at its first chain position plus its lane), positions P (M + 1).
__host__ __device__ constexpr size_t fake_remove_ints(int M) { return (size_t)(6 * M + 3 + 2 * kFrPieces); }
__host__ __device__ constexpr size_t fake_remove_smem(int M)
{
    return (fake_remove_ints(M) * sizeof(int) + 15) / 16 * 16 + (size_t)(M + 1) * sizeof(double2);
}

// One step of the stack rule: chain position k arrives through the edge owned
// by wown (-2 - j: original chain edge j; >= 0: an edge of a new triangle;
// -1: none).  Pops (and makes triangles) while the turn is left; returns the
// new stack height.  Slots come from take().
struct FrRule {
    const FakeRemoveArgs &a;
    const int *Fs, *Fi, *O, *U;
    const double2 *P;
    int rbase;
    int *nrec_orig;  // original chain edges linked so far (this lane)
    __device__ void owner_link(int ownv, int loc) const
    {
        if (ownv <= -2) {
            const int q = -2 - ownv;
            set_fwd(a.fwd, Fs[q], Fi[q], loc);
            a.rec[rbase + q] = Relink{loc, O[q]};
            (*nrec_orig)++;
        } else {
            set_link(a.tn, loc, ownv);
            set_link(a.tn, ownv, loc);
        }
    }
    template <class Take>
    __device__ int push(int *S, int *SO, int top, int k, int wown, Take take, OrientTally &tally) const
    {
        const int wv = U[k];
        while (top >= 2 && orient_staged(P[S[top - 2]], P[S[top - 1]], P[k], a.ct, tally) > 0) {
            const int s = take();
            if (s < 0) {  // more triangles than chain edges: not a pocket
                set_err(a.ct, GPUDT_ERR_TOPOLOGY, 75);
                break;
            }
            const int A = U[S[top - 2]], B = U[S[top - 1]];
            a.tv[s] = make_int4(A, B, wv, 0);
            a.tn[s] = make_int4(-1, -1, -1, 0);
            // opp wv (2): A->B owned by SO[top-1]; opp A (0): B->wv owned by wown;
            // opp B (1): wv->A, the new chain edge A->wv
            owner_link(SO[top - 1], enc(s, 2));
            owner_link(wown, enc(s, 0));
            wown = enc(s, 1);
            a.vtri[A] = enc(s, 0);
            a.vtri[B] = enc(s, 1);
            a.vtri[wv] = enc(s, 2);
            top--;
        }
        S[top] = k;
        SO[top] = wown;
        return top + 1;
    }
};

// Items whose fan has dmin..M triangles (the short and the long launch).
__global__ void __launch_bounds__(32) k_fake_remove(FakeRemoveArgs a, const int *n_dev, int M, int dmin)
{
    extern __shared__ __align__(16) unsigned char fr_smem[];
    int *Fs = (int *)fr_smem, *Fi = Fs + M, *O = Fi + M, *U = O + M, *S = U + M + 1, *SO = S + M + 1 + kFrPieces;
    double2 *P = (double2 *)(fr_smem + (fake_remove_ints(M) * sizeof(int) + 15) / 16 * 16);
    __shared__ int s_top[kFrPieces], s_used[kFrPieces];
    __shared__ int s_top2, s_cl, s_co;
    const int lane = threadIdx.x;
    const int n = *n_dev;
    for (int item = blockIdx.x; item < n; item += gridDim.x) {
        const int f = a.list[item], d = a.fanlen[item] & 0xffff, nsh = a.fanlen[item] >> 16,
                  base = a.fanoff[item];
        if (d < dmin || d > M) continue;  // the other launch's item
        for (int k = lane; k < d; k += 32) {
            const int2 q = a.fan[base + k];
            const int t = dtri(q.x), i = dori(q.x);
            Fs[k] = t;
            Fi[k] = i;
            O[k] = q.y;
            const int4 w = a.tv[t];
            U[k] = geti(w, p1(i));
            if (k == d - 1) U[d] = geti(w, m1(i));
            a.epoch[t] = a.round;
            const int fk = geti(w, i);  // the fake of this fan triangle (a run has several)
            if (fk != f) {
                a.vtri[fk] = -1;
                a.vstate[fk] = VS_GONE;
            }
        }
        __syncwarp();
        for (int k = lane; k <= d; k += 32) P[k] = a.pos[U[k]];
        // every one of the d chain edges ends with exactly one relink record,
        // at rbase + its index (linked to a new triangle, or left as a hull edge)
        int rbase = 0;
        if (lane == 0 && d > 0) rbase = atomicAdd(&a.ct->nrec, d);
        rbase = __shfl_sync(0xffffffffu, rbase, 0);
        __syncwarp();
        const int G = max(1, min(kFrPieces, d / kFrMinPiece));
        int nrec_orig = 0;
        OrientTally tally;
        const FrRule rule{a, Fs, Fi, O, U, P, rbase, &nrec_orig};
        // 1. each lane's piece [b0, b1]; its stack at S + b0 + lane
        const int b0 = (int)((long long)lane * d / G), b1 = (int)((long long)(lane + 1) * d / G);
        if (lane < G) {
            int *LS = S + b0 + lane, *LSO = SO + b0 + lane;
            int top = 0, used = 0;
            for (int k = b0; k <= b1; k++)
                top = rule.push(LS, LSO, top, k, k > b0 ? -2 - (k - 1) : -1, [&] { return Fs[b0 + used++]; },
                                tally);
            s_top[lane] = top;
            s_used[lane] = used;
        }
        __syncwarp();
        // 2. lane 0: the leftover stacks in order (a piece's first vertex is the
        // previous piece's last); the stack is rebuilt in place at S[0..)
        // (it never passes the entry being read).  Slots: the pieces' unused
        // ones, in piece order.
        if (lane == 0) {
            int cl = 0, co = 0;  // next free slot: piece cl, offset co past its used ones
            auto take = [&]() {
                for (; cl < G; cl++, co = 0) {
                    const int pb0 = (int)((long long)cl * d / G), pb1 = (int)((long long)(cl + 1) * d / G);
                    if (pb0 + s_used[cl] + co < pb1) return Fs[pb0 + s_used[cl] + co++];
                }
                return -1;
            };
            int top2 = 0;
            for (int L = 0; L < G; L++) {
                const int pb0 = (int)((long long)L * d / G);
                for (int j = L == 0 ? 0 : 1; j < s_top[L]; j++) {
                    const int idx = pb0 + L + j;
                    top2 = rule.push(S, SO, top2, S[idx], SO[idx], take, tally);
                }
            }
            s_top2 = top2;
            s_cl = cl;
            s_co = co;
        }
        __syncwarp();
        tally.flush(a.ct);
        const int top = s_top2, cl = s_cl, co = s_co;
        // 3. the remaining chain edges are hull edges now
        for (int k = 1 + lane; k < top; k += 32) {
            const int ownv = SO[k];
            if (ownv > -2) {
                set_link(a.tn, ownv, -1);
            } else {
                const int q = -2 - ownv;
                set_fwd(a.fwd, Fs[q], Fi[q], -1);
                a.rec[rbase + q] = Relink{-1, O[q]};
                nrec_orig++;
            }
        }
        {
            int tot = nrec_orig;
            for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
            if (lane == 0 && tot != d) set_err(a.ct, GPUDT_ERR_TOPOLOGY, 74);
        }
        {
            // released slots: each piece's unused ones past what step 2 took
            int mine = 0, from = 0;
            if (lane < G && lane >= cl) {
                from = b0 + s_used[lane] + (lane == cl ? co : 0);
                mine = max(0, b1 - from);
            }
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int nrel = __shfl_sync(0xffffffffu, incl, 31);
            int cb = 0, fb = 0;
            if (lane == 0) {
                cb = atomicAdd(&a.ct->nlist2, top);
                fb = nrel || nsh ? atomicAdd(&a.ct->nfree, nrel + nsh) : 0;
            }
            cb = __shfl_sync(0xffffffffu, cb, 0);
            fb = __shfl_sync(0xffffffffu, fb, 0);
            for (int k = lane; k < top; k += 32) a.cand[cb + k] = U[S[k]];
            for (int k = 0; k < mine; k++) {
                const int t = Fs[from + k];
                a.tv[t] = make_int4(-1, -1, -1, 0);
                a.freelist[fb + incl - mine + k] = t;
            }
            // triangles shared by consecutive members of a run: inside the removed
            // region.  Both members are marked here: a middle member whose fan is
            // just its two shared triangles has no kept entry to be marked by.
            for (int k = lane; k < nsh; k += 32) {
                const int e = a.fan[base + d + k].x, t = dtri(e), i = dori(e);
                const int4 w = a.tv[t];
                const int m0 = geti(w, i), m2 = geti(w, m1(i));  // this member, the next one
                a.vtri[m0] = -1;
                a.vstate[m0] = VS_GONE;
                a.vtri[m2] = -1;
                a.vstate[m2] = VS_GONE;
                a.tv[t] = make_int4(-1, -1, -1, 0);
                a.freelist[fb + nrel + k] = t;
            }
        }
        if (lane == 0) {
            a.vtri[f] = -1;
            a.vstate[f] = VS_GONE;
        }
        __syncwarp();
    }
}

static int launch_fake_remove(Ctx &c, const FakeRemoveArgs &a, const int *n_dev, int max_n)
{
    {
        static std::mutex mu;
        static bool attr_set[64];
        const int dv = c.device >= 0 && c.device < 64 ? c.device : 0;
        std::lock_guard<std::mutex> lk(mu);
        if (!attr_set[dv]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_fake_remove, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)fake_remove_smem(kMaxFanLong)));
            attr_set[dv] = true;
        }
    }
    const int blocks = std::max(1, std::min(max_n, c.sm_count * 16));
    k_fake_remove<<<blocks, 32, fake_remove_smem(kMaxChain), c.stream>>>(a, n_dev, kMaxChain, 0);
    count_launch();
    // fans longer than kMaxChain (sparse input: chords across empty regions)
    k_fake_remove<<<std::max(1, std::min(max_n, c.sm_count)), 32, fake_remove_smem(kMaxFanLong), c.stream>>>(
        a, n_dev, kMaxFanLong, kMaxChain + 1);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

// Convexity check of a boundary candidate: finds its hull edges (u->v, v->w)
// and reports reflex vertices (orient(u,v,w) < 0).
__device__ bool hull_neighbours(const int4 *tv, const int4 *tn, int v, int start, int *u, int *w, int *tin,
                                int *tout)
{
    // clockwise to the outgoing hull edge v->w (edge opposite b of (v,a,b) ... )
    int e = start;
    for (int guard = 0; guard < 8 * kMaxFan; guard++) {
        int t = dtri(e), i = dori(e);
        int nx = geti(tn[t], m1(i));  // across (v, a)
        if (nx < 0) {
            *w = geti(tv[t], p1(i));
            *tout = enc(t, m1(i));
            break;
        }
        e = enc(dtri(nx), m1(dori(nx)));
        if (e == start) return false;  // interior vertex
    }
    e = start;
    for (int guard = 0; guard < 8 * kMaxFan; guard++) {
        int t = dtri(e), i = dori(e);
        int nx = geti(tn[t], p1(i));  // across (b, v)
        if (nx < 0) {
            *u = geti(tv[t], m1(i));
            *tin = enc(t, p1(i));
            return true;
        }
        e = enc(dtri(nx), p1(dori(nx)));
    }
    return false;
}

struct ReflexCheck {
    const int4 *tv, *tn;
    const double2 *pos;
    const int *vtri, *cand;
    const int8_t *vstate;
    int *list, *stamp;
    int round;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int v = cand[ii];
        if (vtri[v] < 0) return;
        int u, w, tin, tout;
        if (!hull_neighbours(tv, tn, v, vtri[v], &u, &w, &tin, &tout)) return;
        if (orientp(pos[u], pos[v], pos[w], ct) < 0 && atomicExch(&stamp[v], round) != round) {
            int k = atomicAdd(&ct->nlist, 1);
            list[k] = v;
        }
    }
};

// Parallel fill of reflex hull vertices, in rounds.  A reflex v (orient(u, v,
// w) < 0 for its hull neighbours u, w) gets the triangle (u, w, v); an
// operation claims u, v and w (minimum vertex id wins), so concurrent
// operations touch disjoint hull triangles.  Winners requeue u and w (they may
// have become reflex), losers requeue themselves.
struct ConvexPropose {
    const int4 *tv, *tn;
    const double2 *pos;
    const int *vtri, *list;
    const int *n_in;
    int *vote;
    int4 *prop;  // (u, w, tin, tout) per list entry, u = -1: nothing to do
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        int v = list[ii];
        prop[ii] = make_int4(-1, -1, -1, -1);
        if (vtri[v] < 0) return;
        int u, w, tin, tout;
        if (!hull_neighbours(tv, tn, v, vtri[v], &u, &w, &tin, &tout)) return;
        if (orientp(pos[u], pos[v], pos[w], ct) >= 0) return;
        prop[ii] = make_int4(u, w, tin, tout);
        atomicMin(&vote[u], v);
        atomicMin(&vote[v], v);
        atomicMin(&vote[w], v);
    }
};

struct ConvexApply {
    int4 *tv, *tn;
    int *vtri, *freelist, *stamp;
    const int *list, *vote;
    const int4 *prop;
    int *list_out, *n_out;
    int cap, round;
    Counters *ct;
    __device__ void push(int x) const
    {
        if (atomicExch(&stamp[x], round) != round) list_out[atomicAdd(n_out, 1)] = x;
    }
    __device__ void operator()(long long ii) const
    {
        int4 p = prop[ii];
        if (p.x < 0) return;
        int v = list[ii], u = p.x, w = p.y, tin = p.z, tout = p.w;
        if (vote[u] != v || vote[v] != v || vote[w] != v) {
            push(v);
            return;
        }
        int s = alloc_slot(freelist, ct, cap);
        if (s < 0) return;
        // (u, w, v): opp u (0) = w->v, the reverse of hull edge v->w (tout);
        //            opp w (1) = v->u, the reverse of hull edge u->v (tin); opp v (2) = new hull u->w
        tv[s] = make_int4(u, w, v, 0);
        tn[s] = make_int4(tout, tin, -1, 0);
        set_link(tn, tout, enc(s, 0));
        set_link(tn, tin, enc(s, 1));
        vtri[u] = enc(s, 0);
        vtri[w] = enc(s, 1);
        vtri[v] = enc(s, 2);
        push(u);
        push(w);
    }
};

struct ConvexReset {
    const int4 *prop;
    const int *list;
    int *vote;
    __device__ void operator()(long long ii) const
    {
        int4 p = prop[ii];
        if (p.x < 0) return;
        vote[p.x] = 0x7fffffff;
        vote[p.y] = 0x7fffffff;
        vote[list[ii]] = 0x7fffffff;
    }
};

int stage_boundary(Ctx &c)
{
    int r;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    int *cand = c.aux;  // boundary candidates
    const int order[4] = {0, 2, 1, 3};
    const long long recn = 4LL * c.cap_tris;
    int removed = 0;
    // stored fans of the selected fakes: (offset, length) per list entry and
    // the entries; the incidence array of the links stage is free by now
    int *fanoff = c.anchor, *fanlen = c.vround;  // per list entry (F <= V)
    int2 *fan = (int2 *)c.inc;                    // 3 cap ints: 1.5 cap entries
    int run_levels = 1;  // separator levels covering the last class's chain of F / 4 fakes
    while (run_levels < 6 && (1LL << (4 * run_levels)) < (c.F + 3) / 4) run_levels++;
    // first pass: the four ring classes in turn (independent by construction);
    // then rounds of priority-minimal fakes among all that remain
    for (int pass = 0; removed < c.F; pass++) {
        if (pass > c.max_rounds / 4) return GPUDT_ERR_NOCONVERGE;
        // pass 0: three ring classes one fake at a time, then the last class
        // (a chain by then) as runs, one separator level after another; later
        // passes: priority rounds among the fakes left
        const int nsub = pass == 0 ? 3 + run_levels : 1;
        for (int q = 0; q < nsub; q++) {
            int round = next_round(c);
            launch_n(c, ZeroInts{&c.ctr->nlist, &c.ctr->nrec}, 1);
            GALPHA_CUDA(cudaMemsetAsync(&c.ctr->cand, 0, sizeof(int), c.stream));  // fan entries
            if (pass == 0 && q >= 3) {
                // staging in alpha-stage buffers, idle until the mesh is final
                int2 *stage = (int2 *)c.keys2;
                int *rec5 = (int *)c.spectrum;
                GALPHA_CUDA(cudaMemsetAsync(&c.ctr->runstage, 0, sizeof(int), c.stream));
                launch_n(c, FakeRunStage{c.tv, c.tn, c.vstate, c.vtri, c.N, order[3], q - 3, stage, &c.ctr->runstage,
                                         rec5, c.ctr},
                         c.F);
                launch_n(c, FakeRunJoin{c.vstate, c.N, order[3], q - 3, stage, rec5, c.list, fanoff, fanlen, fan,
                                        &c.ctr->nlist, &c.ctr->cand, c.ctr},
                         c.F);
            } else
                launch_n(c, FakeSelect{c.tv, c.tn, c.vstate, c.vtri, c.list, fanoff, fanlen, fan, &c.ctr->nlist,
                                       &c.ctr->cand, c.N, pass == 0 ? order[q] : -1, c.ctr},
                         c.F);
            r = launch_fake_remove(c,
                               FakeRemoveArgs{c.tv, c.tn, c.fwd, c.epoch, c.freelist, c.vtri, c.list, fanoff, fanlen, fan,
                                              c.pos, c.vstate, c.rec, cand, round, c.ctr},
                               &c.ctr->nlist, c.F);
            if (r) return r;
            launch_dev(c, Relinker{c.tn, c.fwd, c.epoch, c.rec, c.tv, c.vtri, round, c.ctr}, &c.ctr->nrec, recn);
        }
        GALPHA_CUDA(cudaGetLastError());
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        if (c.hctr->changed == removed) return GPUDT_ERR_NOCONVERGE;  // a full pass removed nothing
        removed = c.hctr->changed;
    }
    r = read_counters(c);
    if (r) return r;
    int ncand = c.hctr->nlist2;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist, 0, sizeof(int), c.stream));
    // per-vertex stamps of the convexify rounds: this arena region may hold
    // another stage's data (or a differently planned call's)
    GALPHA_CUDA(cudaMemsetAsync(c.stamp, 0xff, sizeof(int) * (size_t)c.V, c.stream));
    launch_n(c, ReflexCheck{c.tv, c.tn, c.pos, c.vtri, cand, c.vstate, c.list, c.stamp, next_round(c), c.ctr}, ncand);
    r = read_counters(c);
    if (r) return r;
    int n = c.hctr->nlist;
    int *lin = c.list, *lout = c.list2;
    int4 *prop = c.fwd;
    for (int guard = 0; n > 0; guard++) {
        if (guard > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
        int round = next_round(c);
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
        launch_n(c, ConvexPropose{c.tv, c.tn, c.pos, c.vtri, lin, nullptr, c.vote, prop, c.ctr}, n);
        launch_n(c, ConvexApply{c.tv, c.tn, c.vtri, c.freelist, c.stamp, lin, c.vote, prop, lout, &c.ctr->nlist2,
                                c.cap_tris, round, c.ctr},
                 n);
        launch_n(c, ConvexReset{prop, lin, c.vote}, n);
        GALPHA_CUDA(cudaGetLastError());
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        n = c.hctr->nlist2;
        std::swap(lin, lout);
    }
    if (c.hctr->nfree < 0) GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nfree, 0, sizeof(int), c.stream));
    return GPUDT_OK;
}

// -------------------------------------------------------------------- flip
// Rounds run back to back on device-side counts (ping-pong active lists);
// the host looks at the counters only every c.flip_sync rounds.

// The first round tests every edge once, from the triangle with the lower
// slot.  A flip replaces edge (b, c) of the quad (a, b, d, c) by (a, d); only
// the quad's four outer edges can then have stopped being locally Delaunay,
// so the two new triangles are listed with their outer edges marked
// (eflag), and later rounds test marked edges only.  A candidate that loses
// its vote keeps its marks (all three after the one-sided first round).
// Set of constrained edges: open addressing over keys (min id << 32 | max id),
// empty slots ~0 (constraints, section below).
__device__ __forceinline__ unsigned long long cons_key(int a, int b)
{
    const unsigned lo = (unsigned)min(a, b), hi = (unsigned)max(a, b);
    return ((unsigned long long)lo << 32) | hi;
}

__device__ __forceinline__ unsigned cons_slot(unsigned long long k, unsigned mask)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return (unsigned)k & mask;
}

__device__ __forceinline__ bool cons_has(const unsigned long long *h, unsigned mask, int a, int b)
{
    const unsigned long long k = cons_key(a, b);
    for (unsigned s = cons_slot(k, mask), n = 0; n <= mask; s = (s + 1) & mask, n++) {
        const unsigned long long x = h[s];
        if (x == k) return true;
        if (x == ~0ull) return false;
    }
    return false;
}

struct FlipCheck {
    const int4 *tv, *tn;
    const double2 *pos;
    const int *act;
    int *vote, *prop, *target, *cands;
    int *cand_n;
    Counters *ct;
    int8_t *eflag;
    const unsigned long long *chash;  // constrained edges, never flipped (null: none)
    unsigned cmask;
    __device__ void operator()(long long ii) const
    {
        const int t = act ? act[ii] : (int)ii;  // no list: every slot (the first round)
        // a list entry of -1 is a hole left by a fixed-slot FlipApply: nothing to test
        const int4 v = t >= 0 ? tv[t] : make_int4(-1, -1, -1, 0);
        int ci = -1, cu = -1, ntest = 0, nfilt = 0;
        bool err = false;
        // the first round tests every edge once (from the lower slot); later
        // rounds test the edges a flip or a lost vote left marked
        const int fl = t < 0 ? 0 : (act ? eflag[t] : 7);
        if (v.x >= 0 && fl) {
            const int4 n = tn[t];
            const int nb[3] = {n.x, n.y, n.z};
            const double2 P[3] = {pos[v.x], pos[v.y], pos[v.z]};  // once per triangle, not per edge
            // the neighbours and their apexes of every edge to be tested are
            // gathered up front, each level of loads in flight together (the
            // kernel is bound by the latency of these dependent gathers)
            bool want[3];
            int4 tu[3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const int e = nb[i];
                want[i] = e >= 0 && ((fl >> i) & 1) && (act || dtri(e) >= t);  // first round: the lower slot tests
                if (want[i] && chash && cons_has(chash, cmask, geti(v, p1(i)), geti(v, m1(i)))) want[i] = false;
                tu[i] = want[i] ? tv[dtri(e)] : make_int4(0, 0, 0, 0);
            }
            double2 D[3];
#pragma unroll
            for (int i = 0; i < 3; i++) D[i] = want[i] ? pos[geti(tu[i], dori(nb[i]))] : make_double2(0.0, 0.0);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                if (ci >= 0 || err) break;
                if (!want[i]) continue;
                const double2 A = P[p1(i)], B = P[m1(i)], C = P[i];
                double pa[2] = {A.x, A.y}, pb[2] = {B.x, B.y}, pc[2] = {C.x, C.y}, pd[2] = {D[i].x, D[i].y};
                ntest++;
                int s = incircle_filter32(pa, pb, pc, pd);
                if (s == 2) {
                    s = incircle_filter(pa, pb, pc, pd);
                    if (s == 2) {
                        atomicAdd(&ct->exact_incircle, 1ull);
                        s = incircle_exact(pa, pb, pc, pd);
                        if (s == EXACT_OVERFLOW) err = true;
                    } else {
                        nfilt++;
                    }
                }
                if (!err && s > 0) {
                    ci = i;
                    cu = dtri(nb[i]);
                }
            }
        }
        if (err) set_err(ct, GPUDT_ERR_EXACT, 90);
        warp_add_spread(ct->icc_spread, ntest);
        warp_add_spread(ct->filt_spread, nfilt);
        const bool has = ci >= 0;
        if (act && !has && fl) eflag[t] = 0;  // every marked edge is locally Delaunay
        if (has) {
            prop[t] = ci;
            target[t] = cu;
            // votes carry a hashed priority (prio is a bijection on 32 bits):
            // chains of competing flips then resolve in about log rounds
            // instead of one step per round along increasing slot ids
            const unsigned pt = prio((uint32_t)t);
            atomicMin((unsigned *)&vote[t], pt);
            atomicMin((unsigned *)&vote[cu], pt);
        }
        const int slot = warp_reserve(cand_n, has ? 1 : 0);
        if (has) cands[slot] = t;
    }
};

// Outputs of candidate ii go to fixed slots when the record array has room
// for four per candidate: relink records rec[4ii, 4ii+4) and next-round
// entries next[2ii, 2ii+2), unused ones written as no-ops ({-1, -1} records,
// -1 entries, which the relinker and FlipCheck skip).  That replaces three
// returning atomics per candidate (record, flip and list reservations) --
// the tail of the kernel's latency chain -- by plain stores.
struct FlipApply {
    int4 *tv, *tn, *fwd;
    int *epoch, *vtri, *vote, *stamp, *next;
    int *next_n;
    const int *prop, *target, *cands;
    Relink *rec;
    int round;
    Counters *ct;
    int8_t *eflag;
    bool first;  // first round: a losing candidate was tested one-sided, so all its edges stay marked
    const int *cand_n;  // candidates of the round (the launch count)
    long long rec_cap;  // relink records the array holds
    __device__ bool fresh(int x) const { return x >= 0 && atomicExch(&stamp[x], round) != round; }
    __device__ void operator()(long long ii) const
    {
        const int t = cands[ii];
        const int u = target[t];
        const unsigned pt = prio((uint32_t)t);
        // the vote words and both triangles are loaded together (a winner
        // needs all of them; the kernel is bound by these gathers' latency)
        const unsigned vt = (unsigned)vote[t], vu = (unsigned)vote[u];
        const int i = prop[t];
        const int4 tvv = tv[t], tnn = tn[t], uvv = tv[u], unn = tn[u];
        const bool win = vt == pt && vu == pt;
        int nx[6], nn = 0;
        Relink r4[4];
        if (!win) {
            if (first) eflag[t] = 7;
            if (fresh(t)) nx[nn++] = t;
        } else {
            const int e = geti(tnn, i);
            const int j = dori(e);
            const int a = geti(tvv, i), b = geti(tvv, p1(i)), cc = geti(tvv, m1(i)), d = geti(uvv, j);
            const int ot1 = geti(tnn, p1(i)), ot2 = geti(tnn, m1(i));
            const int ou1 = geti(unn, p1(j)), ou2 = geti(unn, m1(j));
            epoch[t] = round;
            epoch[u] = round;
            tv[t] = make_int4(a, b, d, 0);
            tv[u] = make_int4(d, cc, a, 0);
            tn[t] = make_int4(-1, enc(u, 1), -1, 0);
            tn[u] = make_int4(-1, enc(t, 1), -1, 0);
            int4 ft = make_int4(0, 0, 0, 0), fu = make_int4(0, 0, 0, 0);
            seti(ft, i, -1);
            seti(ft, p1(i), enc(u, 0));
            seti(ft, m1(i), enc(t, 2));
            seti(fu, j, -1);
            seti(fu, p1(j), enc(t, 0));
            seti(fu, m1(j), enc(u, 2));
            fwd[t] = ft;
            fwd[u] = fu;
            r4[0] = Relink{enc(t, 0), ou1};
            r4[1] = Relink{enc(t, 2), ot2};
            r4[2] = Relink{enc(u, 0), ot1};
            r4[3] = Relink{enc(u, 2), ou2};
            vtri[a] = enc(t, 0);
            vtri[b] = enc(t, 1);
            vtri[d] = enc(t, 2);
            vtri[cc] = enc(u, 1);
            // only the four outer edges of the new pair can have stopped being
            // locally Delaunay: edges 0 and 2 of t and of u
            eflag[t] = 5;
            eflag[u] = 5;
            if (fresh(t)) nx[nn++] = t;
            if (fresh(u)) nx[nn++] = u;
        }
        const int nc = *cand_n;  // the same for every thread of the launch
        if (4ll * nc <= rec_cap) {
            if (ii == 0) {
                ct->nrec = 4 * nc;
                *next_n = 2 * nc;
            }
            Relink *rr = rec + 4 * ii;
            for (int k = 0; k < 4; k++) rr[k] = win ? r4[k] : Relink{-1, -1};
            next[2 * ii] = nn > 0 ? nx[0] : -1;
            next[2 * ii + 1] = nn > 1 ? nx[1] : -1;
            const unsigned m = __activemask();
            const int wins = __popc(__ballot_sync(m, win));
            if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && wins) atomicAdd(&ct->nflips, wins);
            return;
        }
        // one atomic per warp for each of the records, the flip count and the next list
        const int rb = warp_reserve(&ct->nrec, win ? 4 : 0);
        if (win)
            for (int k = 0; k < 4; k++) rec[rb + k] = r4[k];
        warp_reserve(&ct->nflips, win ? 1 : 0);
        const int nb = warp_reserve(next_n, nn);
        for (int k = 0; k < nn; k++) next[nb + k] = nx[k];
    }
};

struct FlipReset {
    int *vote;
    const int *target, *cands;
    __device__ void operator()(long long ii) const
    {
        int t = cands[ii];
        vote[t] = -1;  // 0xffffffff: no unsigned vote yet
        vote[target[t]] = -1;
    }
};

// Start of a flip round: the next list becomes current (counts stay in the
// counter block; the host alternates the list buffers).
struct FlipRoundStart {
    int p;  // parity of the round: act[p] is current
    Counters *ct;
    __device__ void operator()(long long) const
    {
        ct->act[1 - p] = 0;
        ct->flips_total += ct->nflips;
        ct->nflips = 0;
        ct->cand = 0;
        ct->nrec = 0;
    }
};

// The tail of the stage: once the active list is short, whole rounds run
// inside ONE block, with __syncthreads between their phases instead of a launch
// per phase (long flip chains -- a retriangulated hull pocket, a dense cluster
// -- otherwise cost five launches per round for a handful of flips).  The same
// functors run in the same phase order with consecutive round ids, so the mesh
// is the one the launched rounds produce.  The block stops when the list
// empties, when a round's list exceeds `leave` (the host goes back to launched
// rounds) or after max_rounds; no thread ever waits on another block.
constexpr int kTailThreads = 1024;
// c.tail_enter: the host hands over at or below this many active triangles;
// c.tail_leave: the block hands back above this many.

__global__ void __launch_bounds__(kTailThreads) k_flip_tail(FlipCheck ck, FlipApply ap, Relinker rl, FlipReset rs,
                                                             int *l0, int *l1, int p0, int round0,
                                                             int max_rounds, int leave)
{
    Counters *ct = ck.ct;
    int k = 0;
    for (; k < max_rounds; k++) {
        const int p = (p0 + k) & 1;
        const int n = *(volatile int *)&ct->act[p];
        if (n == 0 || n > leave) break;
        if (threadIdx.x == 0) FlipRoundStart{p, ct}(0);
        __syncthreads();
        const int round = round0 + k;
        ck.act = p ? l1 : l0;
        for (int i = threadIdx.x; i < n; i += kTailThreads) ck(i);
        __syncthreads();
        const int nc = *(volatile int *)&ct->cand;
        ap.next = p ? l0 : l1;
        ap.next_n = &ct->act[1 - p];
        ap.round = round;
        for (int i = threadIdx.x; i < nc; i += kTailThreads) ap(i);
        __syncthreads();
        const int nr = *(volatile int *)&ct->nrec;
        rl.round = round;
        for (int i = threadIdx.x; i < nr; i += kTailThreads) rl(i);
        for (int i = threadIdx.x; i < nc; i += kTailThreads) rs(i);  // independent of the relinks
        __syncthreads();
    }
    if (threadIdx.x == 0) ct->tail_rounds = k;
}

struct AllAlive {
    const int4 *tv;
    int *list;
    int *count;
    __device__ void operator()(long long i) const
    {
        if (tv[i].x >= 0) {
            int k = atomicAdd(count, 1);
            list[k] = (int)i;
        }
    }
};

int stage_flip(Ctx &c)
{
    int r = read_counters(c);
    if (r) return r;
    int nt = c.hctr->ntris;
    int *lists[2] = {c.list, c.list2};
    int *prop = c.aux, *target = c.aux2, *cands = c.inc, *stamp = c.stamp;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->act[0], 0, 2 * sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->flips_total, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nflips, 0, sizeof(int), c.stream));
    // the first launched round tests every slot directly; the in-block tail
    // (small meshes) starts from a list of the live slots
    if (nt <= c.tail_enter) launch_n(c, AllAlive{c.tv, lists[0], &c.ctr->act[0]}, nt);
    // marked edges: none before the first launched round (it tests all), all
    // when the in-block rounds start from the list of live slots
    GALPHA_CUDA(cudaMemsetAsync(c.eflag, nt <= c.tail_enter ? 7 : 0, (size_t)c.cap_tris, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.vote, 0xff, sizeof(int) * (size_t)nt, c.stream));  // unsigned votes start at max
    GALPHA_CUDA(cudaMemsetAsync(stamp, 0xff, sizeof(int) * (size_t)c.cap_tris, c.stream));
    const long long capn = c.cap_tris, recn = 4LL * c.cap_tris;
    int rounds = 0;
    long long known = nt;  // active-list length at `rounds`, as last read (nt bounds the first)
    while (known > 0) {
        if (known <= c.tail_enter) {
            const int p = rounds & 1;
            const int round0 = next_round(c);
            k_flip_tail<<<1, kTailThreads, 0, c.stream>>>(
                FlipCheck{c.tv, c.tn, c.pos, nullptr, c.vote, prop, target, cands, &c.ctr->cand, c.ctr, c.eflag,
                          c.chash, c.cmask},
                FlipApply{c.tv, c.tn, c.fwd, c.epoch, c.vtri, c.vote, stamp, nullptr, nullptr, prop, target, cands,
                          c.rec, 0, c.ctr, c.eflag, false, &c.ctr->cand, 3ll * c.cap_tris},
                Relinker{c.tn, c.fwd, c.epoch, c.rec, c.tv, c.vtri, 0, c.ctr}, FlipReset{c.vote, target, cands},
                lists[0], lists[1], p, round0, c.max_rounds + 1 - rounds, c.tail_leave);
            count_launch();
            GALPHA_CUDA(cudaGetLastError());
            r = read_counters(c);
            if (r) return r;
            if (c.hctr->err) return c.hctr->err;
            const int k = c.hctr->tail_rounds;
            skip_rounds(c, round0, k - 1);
            rounds += k;
            known = c.hctr->act[rounds & 1];
            if (known == 0) break;
            if (rounds > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
            if (known <= c.tail_leave) return set_last_error("flip: in-block rounds stopped early"), GPUDT_ERR_TOPOLOGY;
        }
        for (int k = 0; k < c.flip_sync; k++) {
            int p = rounds & 1;
            int round = next_round(c);
            launch_n(c, FlipRoundStart{p, c.ctr}, 1);
            if (rounds == 0)
                launch_n(c, FlipCheck{c.tv, c.tn, c.pos, nullptr, c.vote, prop, target, cands, &c.ctr->cand, c.ctr,
                                      c.eflag, c.chash, c.cmask},
                         nt);
            else
                launch_dev(c, FlipCheck{c.tv, c.tn, c.pos, lists[p], c.vote, prop, target, cands, &c.ctr->cand,
                                        c.ctr, c.eflag, c.chash, c.cmask},
                           &c.ctr->act[p], capn);
            launch_dev(c, FlipApply{c.tv, c.tn, c.fwd, c.epoch, c.vtri, c.vote, stamp, lists[1 - p],
                                    &c.ctr->act[1 - p], prop, target, cands, c.rec, round, c.ctr, c.eflag,
                                    rounds == 0, &c.ctr->cand, 3ll * c.cap_tris},
                       &c.ctr->cand, capn);
            launch_dev(c, Relinker{c.tn, c.fwd, c.epoch, c.rec, c.tv, c.vtri, round, c.ctr}, &c.ctr->nrec, recn);
            launch_dev(c, FlipReset{c.vote, target, cands}, &c.ctr->cand, capn);
            rounds++;
        }
        GALPHA_CUDA(cudaGetLastError());
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        known = c.hctr->act[rounds & 1];
        if (rounds > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
    }
    c.st.nFlips = c.hctr->flips_total + c.hctr->nflips;
    c.st.flipRounds = rounds;
    return GPUDT_OK;
}

// ------------------------------------------------------------ constraints
// Constrained edges (GPUDTPARAMS.nConstraints > 0; the reference inserts them
// in cudaConstraint, gpudt/Cuda/cudaConstraint.cu:828-939, and its flipping
// never flips a marked edge, cudaFlipping.cu:111-220, gpudt.cpp:88-155).
// Here they are inserted after the fake ring is gone and before the flip
// stage, in rounds:
//   1. each constraint (a, b) that is not yet an edge walks from a along the
//      segment, counting the triangles it crosses, and claims them and their
//      neighbours (atomicMin of its index on the vote words);
//   2. a constraint that holds every claim records its walk: the crossed
//      triangles (their slots are reused), the chains of vertices right and
//      left of the segment, and the outer link of every chain edge;
//   3. each winner re-triangulates the two cavities on either side of the
//      segment (every chain vertex lies strictly on its side), each by the
//      Delaunay choice of apex over the base (for the base (u, w), the chain
//      vertex whose circle through u and w holds no other one) applied
//      recursively; the segment becomes the edge shared by the two roots.
//      A vertex whose whole star was crossed lies inside a cavity (the walk
//      records it as a spike u, x, u): it is left out of the chain and put
//      back afterwards by a split of the new triangle that holds it.
// Winners own their crossed triangles and the neighbours around them, so their
// writes never meet, and the constraint with the lowest index among those
// left always wins: every round inserts at least one.  The flip stage then
// leaves the constrained edges in place (FlipCheck looks them up in a hash
// set), which yields the constrained Delaunay triangulation.  A segment that
// passes through another vertex, or a vertex that is not in the mesh, is an
// argument error (GPUDT_ERR_ARG); crossing constraints exhaust the round cap.
constexpr int kConsWalkMax = 1 << 22;  // crossed edges of one constraint

struct ConsWalker {
    const int4 *tv, *tn;
    const double2 *pos;
    const int *vtri;
    Counters *ct;
    // The first crossed edge of (a, b): the triangle (a, p, q) whose corner at
    // a holds the direction of b.  Returns 1 and (t, ja), 0 when (a, b) is an
    // edge already, -1 on an error (recorded in the counters).
    __device__ int start(int a, int b, int &t, int &ja, OrientTally &n) const
    {
        const int s0 = vtri[a];
        if (s0 < 0) {
            set_err(ct, GPUDT_ERR_ARG, 123);
            return -1;
        }
        const double2 A = pos[a], B = pos[b];
        int tt = dtri(s0), j = dori(s0), dir = 0;
        for (int steps = 0; steps < kConsWalkMax; steps++) {
            const int4 v = tv[tt];
            const int p = geti(v, p1(j)), q = geti(v, m1(j));
            if (p == b || q == b) return 0;
            const int o1 = orient_staged(A, pos[p], B, ct, n), o2 = orient_staged(A, pos[q], B, ct, n);
            if (o1 > 0 && o2 < 0) {
                t = tt;
                ja = j;
                return 1;
            }
            if (o1 == 0) {
                const double2 P = pos[p];
                if ((P.x - A.x) * (B.x - A.x) + (P.y - A.y) * (B.y - A.y) > 0) {
                    set_err(ct, GPUDT_ERR_ARG, 120);  // p lies on the segment
                    return -1;
                }
            }
            const int4 nb = tn[tt];
            const int e = dir == 0 ? geti(nb, p1(j)) : geti(nb, m1(j));
            if (e < 0) {
                if (dir == 1) break;
                dir = 1;
                tt = dtri(s0);
                j = dori(s0);
                continue;
            }
            tt = dtri(e);
            j = dir == 0 ? p1(dori(e)) : m1(dori(e));
            if (enc(tt, j) == s0) break;
        }
        set_err(ct, GPUDT_ERR_TOPOLOGY, 122);
        return -1;
    }
};

__device__ __forceinline__ int index_of(const int4 &v, int x) { return v.x == x ? 0 : (v.y == x ? 1 : 2); }

// Round step 1: walk, count the crossed triangles, claim them and their
// neighbours.  size[k] = the record size of the constraint (0 when inserted).
struct ConsClaim {
    ConsWalker w;
    const int2 *cons;
    const unsigned long long *hash;
    unsigned mask;
    int *done, *size, *vote;
    int m;
    __device__ void operator()(long long kk) const
    {
        const int k = (int)kk;
        size[k] = 0;
        if (done[k]) return;
        const int a = cons[k].x, b = cons[k].y;
        OrientTally n;
        int t, ja;
        const int st = w.start(a, b, t, ja, n);
        if (st <= 0) {
            if (st == 0) done[k] = 1;
            n.flush(w.ct);
            return;
        }
        int p = geti(w.tv[t], p1(ja)), q = geti(w.tv[t], m1(ja)), jt = ja, cnt = 1;
        const double2 A = w.pos[a], B = w.pos[b];
        for (;;) {
            atomicMin(&vote[t], k);
            const int4 nb = w.tn[t];
            if (nb.x >= 0) atomicMin(&vote[dtri(nb.x)], k);
            if (nb.y >= 0) atomicMin(&vote[dtri(nb.y)], k);
            if (nb.z >= 0) atomicMin(&vote[dtri(nb.z)], k);
            const int e = geti(nb, jt);
            if (e < 0 || cnt > kConsWalkMax) {
                set_err(w.ct, GPUDT_ERR_TOPOLOGY, 124);
                break;
            }
            if (cons_has(hash, mask, p, q)) {
                set_err(w.ct, GPUDT_ERR_ARG, 130);  // crosses another constraint
                break;
            }
            const int u = dtri(e);
            const int4 uv = w.tv[u];
            const int r = geti(uv, dori(e));
            cnt++;
            if (r == b) {
                atomicMin(&vote[u], k);
                const int4 un = w.tn[u];
                if (un.x >= 0) atomicMin(&vote[dtri(un.x)], k);
                if (un.y >= 0) atomicMin(&vote[dtri(un.y)], k);
                if (un.z >= 0) atomicMin(&vote[dtri(un.z)], k);
                break;
            }
            const int o = orient_staged(A, B, w.pos[r], w.ct, n);
            if (o == 0) {
                set_err(w.ct, GPUDT_ERR_ARG, 121);  // r lies on the segment
                break;
            }
            if (o > 0) {
                jt = index_of(uv, q);
                q = r;
            } else {
                jt = index_of(uv, p);
                p = r;
            }
            t = u;
        }
        n.flush(w.ct);
        // slots (cnt), two chains (cnt + 2 each) with their edge links, the
        // vertices inside the region (fewer than cnt) and the
        // re-triangulation stack (4 ints per level)
        size[k] = 12 * (cnt + 4);
        atomicAdd(&w.ct->changed, 1);
    }
};

// Round step 2: a constraint that holds all its claims records its walk at
// rec = pool + off[k]: [0] crossed triangles n, [1] right chain length nr,
// [2] left chain length nl, [3] unused, then slots[n], right chain[nr],
// right links[nr - 1], left chain[nl], left links[nl - 1] (chain i: vertices
// in order from a to b; link i: the neighbour across chain edge i), room for
// the inner vertices and the stack of step 3.
struct ConsRecord {
    ConsWalker w;
    const int2 *cons;
    const int *done, *size, *off, *vote;
    int *win, *pool;
    long long pool_ints;
    __device__ bool mine(int t, int k) const
    {
        if (vote[t] != k) return false;
        const int4 nb = w.tn[t];
        return (nb.x < 0 || vote[dtri(nb.x)] == k) && (nb.y < 0 || vote[dtri(nb.y)] == k) &&
               (nb.z < 0 || vote[dtri(nb.z)] == k);
    }
    __device__ void operator()(long long kk) const
    {
        const int k = (int)kk;
        win[k] = 0;
        if (done[k] || size[k] == 0) return;
        if (off[k] < 0 || (long long)off[k] + size[k] > pool_ints) {  // (a wrapped offset scan included)
            set_err(w.ct, GPUDT_ERR_NOMEM, 125);
            return;
        }
        const int a = cons[k].x, b = cons[k].y;
        OrientTally n;
        int t, ja;
        if (w.start(a, b, t, ja, n) <= 0) {
            n.flush(w.ct);
            return;
        }
        const int cap = size[k] / 12 - 4;  // crossed triangles the record holds
        int *rec = pool + off[k];
        int *slots = rec + 4;
        int *R = slots + cap, *RL = R + cap + 2, *L = RL + cap + 1, *LL = L + cap + 2;
        const double2 A = w.pos[a], B = w.pos[b];
        bool ok = mine(t, k);
        int4 tv0 = w.tv[t];
        int p = geti(tv0, p1(ja)), q = geti(tv0, m1(ja)), jt = ja, cnt = 0, nr = 0, nl = 0;
        const int4 tn0 = w.tn[t];
        slots[cnt++] = t;
        R[nr] = a;
        RL[nr++] = geti(tn0, m1(ja));  // edge (a, p), opposite q
        R[nr] = p;
        L[nl] = a;
        LL[nl++] = geti(tn0, p1(ja));  // edge (q, a), opposite p
        L[nl] = q;
        for (;;) {
            const int e = geti(w.tn[t], jt);
            const int u = dtri(e);
            if (e < 0 || cnt >= cap) {
                set_err(w.ct, GPUDT_ERR_TOPOLOGY, 126);
                ok = false;
                break;
            }
            const int4 uv = w.tv[u], un = w.tn[u];
            const int r = geti(uv, dori(e));
            ok = ok && mine(u, k);
            slots[cnt++] = u;
            if (r == b) {
                RL[nr++] = geti(un, index_of(uv, q));  // edge (p, b), opposite q
                R[nr] = b;
                LL[nl++] = geti(un, index_of(uv, p));  // edge (q, b), opposite p
                L[nl] = b;
                break;
            }
            const int o = orient_staged(A, B, w.pos[r], w.ct, n);
            if (o > 0) {  // r left: the boundary edge (q, r) is opposite p
                LL[nl++] = geti(un, index_of(uv, p));
                L[nl] = r;
                jt = index_of(uv, q);
                q = r;
            } else {  // r right: the boundary edge (p, r) is opposite q
                RL[nr++] = geti(un, index_of(uv, q));
                R[nr] = r;
                jt = index_of(uv, p);
                p = r;
            }
            t = u;
        }
        n.flush(w.ct);
        rec[0] = cnt;
        rec[1] = nr + 1;
        rec[2] = nl + 1;
        win[k] = ok ? 1 : 0;
    }
};

// Links edge ei of triangle t to the encoded neighbour o and o back to it.
__device__ __forceinline__ void cons_link(int4 *tn, int t, int ei, int o)
{
    set_link(tn, enc(t, ei), o);
    if (o >= 0) set_link(tn, o, enc(t, ei));
}

// Removes the dangling trees from a chain in place: a vertex whose whole star
// is crossed lies inside the region of the crossed triangles, and the walk
// passes round the edges to it in both directions (u, x, u).  Those vertices
// go to orph[]; the remaining chain is the simple boundary of the region on
// its side, and its links all lead to triangles outside it.  Returns the new
// chain length.
__device__ __forceinline__ int cons_reduce(int *c, int *cl, int len, int *orph, int &no)
{
    int top = 0;  // c[0..top] kept, cl[0..top) their links
    for (int i = 1; i < len; i++) {
        if (top >= 1 && c[top - 1] == c[i]) {
            orph[no++] = c[top];  // (c[top-1], c[top]) and back: a spike
            top--;
        } else {
            cl[top] = cl[i - 1];
            c[++top] = c[i];
        }
    }
    return top + 1;
}

// Round step 3: re-triangulate a winner's cavities.  Chain c[0..len) with
// links cl[0..len-1) forms a counterclockwise polygon closed by the base edge
// (c[len-1], c[0]); each sub-polygon (i, j) becomes the triangle
// (c[i], c[x], c[j]) whose circle holds no other c[i+1..j-1], plus its two
// sub-polygons.  Triangle edges: 0 = (c[x], c[j]), 1 = the base (c[j], c[i]),
// 2 = (c[i], c[x]).  The vertices taken off the chains as dangling trees are
// then put back, each by splitting the new triangle that holds it (or the two
// on either side of the new edge through it); the slots of the crossed
// triangles hold exactly the result.  The flip stage restores the Delaunay
// property around them.
struct ConsApply {
    int4 *tv, *tn;
    const double2 *pos;
    int *vtri, *done;
    const int *win, *off, *size;
    int *pool;
    Counters *ct;
    __device__ int cavity(const int *c, const int *cl, int len, const int *slots, int &next, int *stack,
                          int nstack) const
    {
        int sp = 0, root = -1;
        stack[0] = 0;
        stack[1] = len - 1;
        stack[2] = -1;
        stack[3] = -1;
        sp = 1;
        while (sp > 0) {
            sp--;
            const int i = stack[4 * sp], j = stack[4 * sp + 1], pt = stack[4 * sp + 2], pe = stack[4 * sp + 3];
            int x = i + 1;
            const double2 I = pos[c[i]], J = pos[c[j]];
            for (int l = i + 2; l < j; l++) {
                const double2 X = pos[c[x]], Lp = pos[c[l]];
                double pa[2] = {I.x, I.y}, pb[2] = {X.x, X.y}, pc[2] = {J.x, J.y}, pd[2] = {Lp.x, Lp.y};
                int s = incircle_filter32(pa, pb, pc, pd);
                if (s == 2) s = incircle_filter(pa, pb, pc, pd);
                if (s == 2) {
                    atomicAdd(&ct->exact_incircle, 1ull);
                    s = incircle_exact(pa, pb, pc, pd);
                    if (s == EXACT_OVERFLOW) {
                        set_err(ct, GPUDT_ERR_EXACT, 127);
                        return -1;
                    }
                }
                if (s > 0) x = l;
            }
            const int T = slots[next++];
            tv[T] = make_int4(c[i], c[x], c[j], 0);
            vtri[c[i]] = enc(T, 0);
            vtri[c[x]] = enc(T, 1);
            vtri[c[j]] = enc(T, 2);
            if (pt >= 0) cons_link(tn, T, 1, enc(pt, pe));
            else root = T;
            if (x == i + 1) cons_link(tn, T, 2, cl[i]);
            else if (sp < nstack) {
                stack[4 * sp] = i;
                stack[4 * sp + 1] = x;
                stack[4 * sp + 2] = T;
                stack[4 * sp + 3] = 2;
                sp++;
            } else {
                set_err(ct, GPUDT_ERR_TOPOLOGY, 128);
                return -1;
            }
            if (j == x + 1) cons_link(tn, T, 0, cl[x]);
            else if (sp < nstack) {
                stack[4 * sp] = x;
                stack[4 * sp + 1] = j;
                stack[4 * sp + 2] = T;
                stack[4 * sp + 3] = 0;
                sp++;
            } else {
                set_err(ct, GPUDT_ERR_TOPOLOGY, 128);
                return -1;
            }
        }
        return root;
    }
    // Writes triangle T = (a, b, c) with the links (na, nb, nc) of its edges
    // opposite a, b, c; `ext` bit i: link i leads outside the triangles being
    // written, so its far side is pointed back at T.
    __device__ void put(int T, int a, int b, int c, int na, int nb, int nc, int ext) const
    {
        tv[T] = make_int4(a, b, c, 0);
        tn[T] = make_int4(na, nb, nc, 0);
        if ((ext & 1) && na >= 0) set_link(tn, na, enc(T, 0));
        if ((ext & 2) && nb >= 0) set_link(tn, nb, enc(T, 1));
        if ((ext & 4) && nc >= 0) set_link(tn, nc, enc(T, 2));
        vtri[a] = enc(T, 0);
        vtri[b] = enc(T, 1);
        vtri[c] = enc(T, 2);
    }
    // Puts vertex v back into the triangles slots[0..next): a 1-3 split of the
    // one that holds it, or a 2-4 split of the two beside the edge through it.
    __device__ bool orphan(int v, const int *slots, int &next, OrientTally &n) const
    {
        const double2 V = pos[v];
        for (int k = 0; k < next; k++) {
            const int T = slots[k];
            const int4 t = tv[T];
            const double2 P0 = pos[t.x], P1 = pos[t.y], P2 = pos[t.z];
            const int s0 = orient_staged(P1, P2, V, ct, n);
            if (s0 < 0) continue;
            const int s1 = orient_staged(P2, P0, V, ct, n);
            if (s1 < 0) continue;
            const int s2 = orient_staged(P0, P1, V, ct, n);
            if (s2 < 0) continue;
            const int4 nb = tn[T];
            if (s0 > 0 && s1 > 0 && s2 > 0) {
                const int B = slots[next++], C = slots[next++];
                put(T, v, t.y, t.z, nb.x, enc(B, 2), enc(C, 1), 0);
                put(B, v, t.z, t.x, nb.y, enc(C, 2), enc(T, 1), 1);
                put(C, v, t.x, t.y, nb.z, enc(T, 2), enc(B, 1), 1);
                return true;
            }
            if ((s0 == 0) + (s1 == 0) + (s2 == 0) != 1) break;
            // v on the edge opposite corner i of T = (a, b, c): U = (u, c, b)
            const int i = s0 == 0 ? 0 : (s1 == 0 ? 1 : 2);
            const int a = geti(t, i), b = geti(t, p1(i)), c = geti(t, m1(i));
            const int na = geti(nb, i), nbb = geti(nb, p1(i)), nc = geti(nb, m1(i));
            if (na < 0) break;
            const int U = dtri(na), j = dori(na);
            bool ours = false;  // the edge through v is one of the new ones
            for (int q = 0; q < next && !ours; q++) ours = slots[q] == U;
            if (!ours) break;
            const int4 uv = tv[U], un = tn[U];
            const int u = geti(uv, j), ub = geti(un, p1(j)), uc = geti(un, m1(j));
            const int T2 = slots[next++], U2 = slots[next++];
            put(T, a, b, v, enc(U2, 0), enc(T2, 2), nc, 4);
            put(T2, a, v, c, enc(U, 0), nbb, enc(T, 1), 2);
            put(U, u, c, v, enc(T2, 0), enc(U2, 2), uc, 4);
            put(U2, u, v, b, enc(T, 0), ub, enc(U, 1), 2);
            return true;
        }
        set_err(ct, GPUDT_ERR_TOPOLOGY, 131);
        return false;
    }
    __device__ void operator()(long long kk) const
    {
        const int k = (int)kk;
        if (!win[k]) return;
        int *rec = pool + off[k];
        const int cnt = rec[0];
        int nr = rec[1], nl = rec[2];
        const int cap = size[k] / 12 - 4;
        const int *slots = rec + 4;
        int *R = (int *)slots + cap, *RL = R + cap + 2;
        int *L = RL + cap + 1, *LL = L + cap + 2;
        int *orph = LL + cap + 1;
        int *stack = orph + cap;
        const int nstack = (size[k] - (int)(stack - rec)) / 4;
        if (nr + nl - 4 != cnt || nr > cap + 2 || nl > cap + 2) {
            set_err(ct, GPUDT_ERR_TOPOLOGY, 129);
            return;
        }
        int no = 0;
        nr = cons_reduce(R, RL, nr, orph, no);
        nl = cons_reduce(L, LL, nl, orph, no);
        if (nr < 3 || nl < 3 || nr + nl - 4 + 2 * no != cnt) {
            set_err(ct, GPUDT_ERR_TOPOLOGY, 132);
            return;
        }
        // the left chain, reversed (b ... a), is counterclockwise like the right one
        for (int i = 0, j = nl - 1; i < j; i++, j--) {
            const int x = L[i];
            L[i] = L[j];
            L[j] = x;
        }
        for (int i = 0, j = nl - 2; i < j; i++, j--) {
            const int x = LL[i];
            LL[i] = LL[j];
            LL[j] = x;
        }
        int next = 0;
        const int rr = cavity(R, RL, nr, slots, next, stack, nstack);
        if (rr < 0) return;
        const int rl = cavity(L, LL, nl, slots, next, stack, nstack);
        if (rl < 0) return;
        cons_link(tn, rr, 1, enc(rl, 1));  // the constraint: base of both roots
        OrientTally n;
        for (int o = 0; o < no; o++)
            if (!orphan(orph[o], slots, next, n)) break;
        n.flush(ct);
        done[k] = 1;
    }
};

struct ConsMap {
    const int2 *in;
    const int *iperm;  // input -> internal id (null: identity)
    int2 *cons;
    int *done;
    __device__ void operator()(long long k) const
    {
        int2 c = in[k];
        if (iperm) c = make_int2(iperm[c.x], iperm[c.y]);
        cons[k] = c;
        done[k] = 0;
    }
};

struct InvPerm {
    const int *perm;
    int *iperm;
    __device__ void operator()(long long i) const { iperm[perm[i]] = (int)i; }
};

struct VtriOfTris {
    const int4 *tv;
    int *vtri;
    __device__ void operator()(long long t) const
    {
        const int4 v = tv[t];
        if (v.x < 0) return;
        vtri[v.x] = enc((int)t, 0);
        vtri[v.y] = enc((int)t, 1);
        vtri[v.z] = enc((int)t, 2);
    }
};

struct ConsHashInsert {
    const int2 *cons;
    unsigned long long *h;
    unsigned mask;
    __device__ void operator()(long long k) const
    {
        const unsigned long long key = cons_key(cons[k].x, cons[k].y);
        for (unsigned s = cons_slot(key, mask), n = 0; n <= mask; s = (s + 1) & mask, n++) {
            const unsigned long long old = atomicCAS(&h[s], ~0ull, key);
            if (old == ~0ull || old == key) return;
        }
    }
};

int stage_constraints(Ctx &c)
{
    const int m = c.n_cons;
    c.chash = nullptr;
    c.cons_rounds = 0;
    if (m <= 0) return GPUDT_OK;
    unsigned S = 64;
    while (S < 2u * (unsigned)m + 2u) S <<= 1;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t need = al(sizeof(int2) * (size_t)m) * 2 + al(4 * (size_t)(m + 1)) * 4 + al(8 * (size_t)S) +
                        al(4 * (size_t)c.N + 4);
    if (need > c.cons_bytes) {
        if (c.cons_buf) cudaFree(c.cons_buf);
        c.cons_buf = nullptr;
        c.cons_bytes = 0;
        GALPHA_CUDA(cudaMalloc(&c.cons_buf, need));
        c.cons_bytes = need;
    }
    char *p = c.cons_buf;
    auto take = [&](size_t b) {
        char *q = p;
        p += al(b);
        return q;
    };
    int2 *in = (int2 *)take(sizeof(int2) * (size_t)m);
    int2 *cons = (int2 *)take(sizeof(int2) * (size_t)m);
    int *done = (int *)take(4 * (size_t)(m + 1));
    int *size = (int *)take(4 * (size_t)(m + 1));
    int *off = (int *)take(4 * (size_t)(m + 1));
    int *win = (int *)take(4 * (size_t)(m + 1));
    unsigned long long *hash = (unsigned long long *)take(8 * (size_t)S);
    int *iperm = (int *)take(4 * (size_t)c.N + 4);
    GALPHA_CUDA(cudaMemcpyAsync(in, c.h_cons, sizeof(int2) * (size_t)m, cudaMemcpyHostToDevice, c.stream));
    if (c.renumbered) launch_n(c, InvPerm{c.perm, iperm}, c.N);
    launch_n(c, ConsMap{in, c.renumbered ? iperm : nullptr, cons, done}, m);
    GALPHA_CUDA(cudaMemsetAsync(hash, 0xff, 8 * (size_t)S, c.stream));
    launch_n(c, ConsHashInsert{cons, hash, S - 1}, m);
    // one incident triangle per vertex of the mesh (vertices not in it: -1)
    int r = read_counters(c);
    if (r) return r;
    const int nt = c.hctr->ntris;
    GALPHA_CUDA(cudaMemsetAsync(c.vtri, 0xff, sizeof(int) * (size_t)c.V, c.stream));
    launch_n(c, VtriOfTris{c.tv, c.vtri}, nt);
    const ConsWalker w{c.tv, c.tn, c.pos, c.vtri, c.ctr};
    int round = 0;
    for (;; round++) {
        if (round > c.max_rounds) return GPUDT_ERR_NOCONVERGE;
        GALPHA_CUDA(cudaMemsetAsync(c.vote, 0x7f, sizeof(int) * (size_t)c.cap_tris, c.stream));
        GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
        launch_n(c, ConsClaim{w, cons, hash, S - 1, done, size, c.vote, m}, m);
        r = exclusive_scan_int(c, size, off, m, &c.ctr->nlist);
        if (r) return r;
        r = read_counters(c);
        if (r) return r;
        if (c.hctr->err) return c.hctr->err;
        if (c.hctr->changed == 0) break;
        const long long total = (long long)(unsigned)c.hctr->nlist;
        if (total > c.cons_pool_ints) {
            if (c.cons_pool) cudaFree(c.cons_pool);
            c.cons_pool = nullptr;
            c.cons_pool_ints = 0;
            const long long ints = std::max(total + total / 2, 1ll << 16);
            GALPHA_CUDA(cudaMalloc(&c.cons_pool, sizeof(int) * (size_t)ints));
            c.cons_pool_ints = ints;
        }
        launch_n(c, ConsRecord{w, cons, done, size, off, c.vote, win, c.cons_pool, c.cons_pool_ints}, m);
        launch_n(c, ConsApply{c.tv, c.tn, c.pos, c.vtri, done, win, off, size, c.cons_pool, c.ctr}, m);
        GALPHA_CUDA(cudaGetLastError());
    }
    c.chash = hash;
    c.cmask = S - 1;
    c.cons_rounds = round;
    c.st.constraintRounds = round;
    return GPUDT_OK;
}

// ----------------------------------------------------------------- compact
struct MarkAlive {
    const int4 *tv;
    int *flag;
    __device__ void operator()(long long i) const { flag[i] = tv[i].x >= 0 ? 1 : 0; }
};

struct CompactWrite {
    const int4 *tv, *tn;
    const int *newidx;
    int4 *cv, *cn;
    gpudtTriangle *out;
    const int *perm;  // internal -> input vertex index (nullptr: identity)
    int4 *cvi;        // with perm: the triangles with internal ids (alpha-stage geometry)
    __device__ void operator()(long long ii) const
    {
        int t = (int)ii;
        int4 v = tv[t];
        if (v.x < 0) return;
        if (perm) {
            cvi[newidx[t]] = make_int4(v.x, v.y, v.z, 0);
            v = make_int4(perm[v.x], perm[v.y], perm[v.z], 0);
        }
        int4 n = tn[t];
        int k = newidx[t];
        int nn[3] = {n.x, n.y, n.z};
        for (int q = 0; q < 3; q++)
            if (nn[q] >= 0) nn[q] = enc(newidx[dtri(nn[q])], dori(nn[q]));
        cv[k] = make_int4(v.x, v.y, v.z, 0);
        cn[k] = make_int4(nn[0], nn[1], nn[2], 0);
        if (!out) return;
        gpudtTriangle g;
        g.tri[0] = nn[0];
        g.tri[1] = nn[1];
        g.tri[2] = nn[2];
        g.vtx[0] = v.x;
        g.vtx[1] = v.y;
        g.vtx[2] = v.z;
        g.tmp[0] = g.tmp[1] = g.tmp[2] = 0;
        out[k] = g;
    }
};

// The same compaction driven by the new order: new triangle j is slot
// order[j] (alive slots sorted by set, slot order kept within a set), so the
// writes are consecutive and only the reads follow the slots.
struct CompactGather {
    const int4 *tv, *tn;
    const int *order, *newidx;
    int4 *cv, *cn;
    const int *perm;  // internal -> input vertex index (nullptr: identity)
    int4 *cvi;        // with perm: the triangles with internal ids (alpha-stage geometry)
    __device__ void operator()(long long jj) const
    {
        const int j = (int)jj, t = order[j];
        int4 v = tv[t];
        const int4 n = tn[t];
        if (perm) {
            cvi[j] = make_int4(v.x, v.y, v.z, 0);
            v = make_int4(perm[v.x], perm[v.y], perm[v.z], 0);
        }
        int nn[3] = {n.x, n.y, n.z};
        for (int q = 0; q < 3; q++)
            if (nn[q] >= 0) nn[q] = enc(newidx[dtri(nn[q])], dori(nn[q]));
        cv[j] = make_int4(v.x, v.y, v.z, 0);
        cn[j] = make_int4(nn[0], nn[1], nn[2], 0);
    }
};

void launch_compact_gather(Ctx &c, const int *order, const int *newidx, int nalive)
{
    launch_n(c, CompactGather{c.tv, c.tn, order, newidx, c.cv, c.cn, c.renumbered ? c.perm : nullptr, c.fwd},
             nalive);
    c.outtri_ready = false;
}

// gpudtTriangle records of the compacted mesh (tmp[] zero).
struct SoaToAos {
    const int4 *cv, *cn;
    gpudtTriangle *out;
    __device__ void operator()(long long k) const
    {
        const int4 v = cv[k], n = cn[k];
        gpudtTriangle g;
        g.tri[0] = n.x;
        g.tri[1] = n.y;
        g.tri[2] = n.z;
        g.vtx[0] = v.x;
        g.vtx[1] = v.y;
        g.vtx[2] = v.z;
        g.tmp[0] = g.tmp[1] = g.tmp[2] = 0;
        out[k] = g;
    }
};

int ensure_outtri(Ctx &c)
{
    if (c.outtri_ready) return GPUDT_OK;
    if (c.nT_out > 0) launch_n(c, SoaToAos{c.cv, c.cn, c.outtri}, c.nT_out);
    GALPHA_CUDA(cudaGetLastError());
    c.outtri_ready = true;
    return GPUDT_OK;
}

int stage_compact(Ctx &c)
{
    int r = read_counters(c);
    if (r) return r;
    int nt = c.hctr->ntris;
    launch_n(c, MarkAlive{c.tv, c.aux}, nt);
    r = exclusive_scan_int(c, c.aux, c.aux2, nt, &c.ctr->nlist);
    if (r) return r;
    // cv / cn, and the gpudtTriangle records when the call will return them
    // (otherwise they are built when a download asks for them)
    launch_n(c, CompactWrite{c.tv, c.tn, c.aux2, c.cv, c.cn, c.want_outtri ? c.outtri : nullptr,
                             c.renumbered ? c.perm : nullptr, c.fwd},
             nt);
    c.outtri_ready = c.want_outtri;
    GALPHA_CUDA(cudaGetLastError());
    r = read_counters(c);
    if (r) return r;
    c.nT_out = c.hctr->nlist;
    return GPUDT_OK;
}

}  // namespace galpha
