// api.cu -- C ABI of libgalpha: handles, device arena, stage orchestration.
//
// Entry points and the reference interfaces they replace are listed in
// include/gpudt.h and include/galpha.h.  The reference keeps global host and
// device state and exits on any CUDA error (gpudt.cpp:64-77, cudaMain.cu:69-92,
// common.h:55-93); here each handle owns its stream and buffers, every entry
// point returns a GPUDT_* status, and device-side errors (topology, iteration
// caps, exact-arithmetic scratch) are reported through the counter block.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <mutex>
#include <new>
#include "internal.cuh"

namespace galpha {

static thread_local std::string g_err;
unsigned long long g_launches = 0;

int cuda_fail(cudaError_t e, const char *what)
{
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? GPUDT_ERR_NOMEM : GPUDT_ERR_CUDA;
}

const char *last_error_text() { return g_err.c_str(); }
void set_last_error(const char *text) { g_err = text; }

// Device words to mapped host memory.  The stores travel as PCIe writes of
// the SMs, not through a copy engine, so a pipeline's counter reads do not
// wait for result downloads queued by this or another handle.
__global__ void k_read_words(const unsigned *__restrict__ src, unsigned *dst, int nwords)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += gridDim.x * blockDim.x) dst[i] = src[i];
    __threadfence_system();
}

int read_counters(Ctx &c)
{
    static_assert(sizeof(Counters) % 4 == 0, "counter block is read as 32-bit words");
    const int nw = (int)(sizeof(Counters) / 4);
    k_read_words<<<1, 256, 0, c.stream>>>((const unsigned *)c.ctr, (unsigned *)c.hctr_dev, nw);
    count_launch();
    c.host_reads++;
    GALPHA_CUDA(cudaGetLastError());
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    return GPUDT_OK;
}

// Predicate stage counts of the last run (counter block already read).
static void fill_predicate_stats(Ctx &c)
{
    const Counters &h = *c.hctr;
    c.st.exactOrient = (long long)h.exact_orient;
    c.st.exactIncircle = (long long)h.exact_incircle;
    c.st.filteredIncircle = c.st.incircleTests = c.st.orientTests = c.st.filteredOrient = 0;
    for (int k = 0; k < 64; k++) {
        c.st.filteredIncircle += (long long)h.filt_spread[k];
        c.st.incircleTests += (long long)h.icc_spread[k];
        c.st.orientTests += (long long)h.ori_spread[k];
        c.st.filteredOrient += (long long)h.ori64_spread[k];
    }
}

int read_small(Ctx &c, void *host_dst, const void *dev_src, size_t bytes)
{
    if (bytes == 0) return GPUDT_OK;
    c.host_reads++;
    if (bytes > kMailBytes || (bytes & 3) || ((uintptr_t)dev_src & 3)) {
        GALPHA_CUDA(cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, c.stream));
        GALPHA_CUDA(cudaStreamSynchronize(c.stream));
        return GPUDT_OK;
    }
    const int nw = (int)(bytes / 4);
    k_read_words<<<(nw + 255) / 256, 256, 0, c.stream>>>((const unsigned *)dev_src, (unsigned *)c.hmail_dev, nw);
    count_launch();
    GALPHA_CUDA(cudaGetLastError());
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    memcpy(host_dst, c.hmail, bytes);
    return GPUDT_OK;
}

// One arena per handle; carve() hands out 256-byte aligned pieces.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
    void *carve(size_t bytes)
    {
        size_t off = (used + 255) & ~(size_t)255;
        if (off + bytes > cap) return nullptr;
        used = off + bytes;
        return base + off;
    }
};

struct Sizes {
    size_t V, T2, cap, lists, ntiles;
    size_t occw = 0, bandw = 0;  // occupancy words (0: a single T x T texture)
};

static size_t plan(const Sizes &z, Ctx *c, Arena *A)
{
    size_t total = 0;
    auto take = [&](size_t bytes) -> void * {
        size_t off = (total + 255) & ~(size_t)255;
        total = off + bytes;
        return A ? A->carve(bytes) : nullptr;
    };
    size_t V = z.V, cap = z.cap, T2 = z.T2, L = z.lists;
    size_t T = (size_t)std::llround(std::sqrt((double)T2));
    size_t W2 = ((T >> 6) + 31) / 32;
    const size_t occw = z.occw ? z.occw : T * (T / 32), bandw = z.bandw ? z.bandw : T * W2;
#define TAKE(field, type, count) \
    {                            \
        void *p_ = take(sizeof(type) * (size_t)(count)); \
        if (c) c->field = (type *)p_; \
    }
    TAKE(opos, double2, V);
    TAKE(pos, double2, V);
    TAKE(gpix, short2, V);
    TAKE(idmap, int, T2);
    TAKE(occ, uint32_t, occw);
    TAKE(bandocc, uint32_t, bandw);
    TAKE(ycol, int16_t, T2);
    TAKE(colour, int, T2);
    TAKE(list, int, L);
    TAKE(list2, int, L);
    TAKE(aux, int, L);
    TAKE(aux2, int, L);
    TAKE(tv, int4, cap);
    TAKE(tn, int4, cap);
    TAKE(fwd, int4, cap);
    TAKE(cv, int4, cap);
    TAKE(cn, int4, cap);
    TAKE(epoch, int, cap);
    TAKE(vote, int, cap);
    TAKE(eflag, int8_t, cap);
    TAKE(stamp, int, L);
    TAKE(freelist, int, cap);
    TAKE(rec, Relink, 3 * cap);
    TAKE(vtri, int, V);
    TAKE(vstate, int8_t, V);
    TAKE(vround, int, V);
    TAKE(anchor, int, V);
    TAKE(perm, int, V);
    TAKE(deg, int, V + 1);
    TAKE(inc, int, 3 * cap);
    TAKE(tilecount, int, z.ntiles + 1);
    TAKE(hist, int, 65536);
    TAKE(rhist, int, radix_sort_scratch_ints((long long)(3 * cap)) + 16);
    if (c) c->rhist_ints = radix_sort_scratch_ints((long long)(3 * cap)) + 16;
    TAKE(e_off, int, cap + 1);
    TAKE(edges, int4, 2 * cap);
    TAKE(edge_ro, int, 2 * cap);
    TAKE(edge_nu, int2, 2 * cap);
    TAKE(tri_ro, int, cap);
    TAKE(pt_nu, int2, V);
    TAKE(keys, unsigned long long, 3 * cap);
    TAKE(keys2, unsigned long long, 3 * cap);
    TAKE(vals, int, 3 * cap);
    TAKE(vals2, int, 3 * cap);
    TAKE(rank, int, 3 * cap);
    TAKE(spectrum, double, 3 * cap);
    TAKE(outtri, gpudtTriangle, cap);
    TAKE(edge_aos, galphaEdgeInterval, 2 * cap);
    TAKE(qclass, uint8_t, V + 3 * cap);
    TAKE(ctr, Counters, 1);
#undef TAKE
    return total + 4096;
}

struct HandleState {
    Ctx c;
    Arena arena;
    BatchHost bh;
    BatchDev bd;
    double *d_xy = nullptr;
    size_t d_xy_cap = 0;
    cudaStream_t side = nullptr;  // downloads that overlap later stages (galphaComputeAll)
    cudaEvent_t side_ev = nullptr;
};

static int ensure_sizes(HandleState &H, const Sizes &z);

static int ensure(HandleState &H, int V, int T, long long nExtraTris)
{
    Sizes z;
    z.V = (size_t)V;
    z.T2 = (size_t)T * T;
    z.cap = (size_t)2 * V + 64 + (size_t)(nExtraTris > 0 ? nExtraTris : 0);
    z.lists = std::max(z.cap * 3, z.V + 1);
    z.ntiles = ((size_t)(T - 1) * (T - 1) + 255) / 256 + 1;
    return ensure_sizes(H, z);
}

static int ensure_sizes(HandleState &H, const Sizes &z)
{
    Ctx &c = H.c;
    size_t need = plan(z, nullptr, nullptr);
    if (c.budget > 0 && (long long)need > c.budget) {
        g_err = "device memory budget exceeded";
        return GPUDT_ERR_NOMEM;
    }
    if (need > H.arena.cap) {
        if (H.arena.base) cudaFree(H.arena.base);
        H.arena.base = nullptr;
        H.arena.cap = 0;
        void *p = nullptr;
        GALPHA_CUDA(cudaMalloc(&p, need));
        H.arena.base = (char *)p;
        H.arena.cap = need;
        c.reserved = (long long)need;
        GALPHA_CUDA(cudaMemsetAsync(p, 0, need, c.stream));
    }
    H.arena.used = 0;
    plan(z, &c, &H.arena);
    c.cap_tris = (int)z.cap;
    // per-call initialisation of the slot state
    // round ids restart well before the int range ends; every stage that
    // compares stamps with round ids initialises its stamps first
    if (c.round_counter > (1 << 30)) c.round_counter = 1;
    GALPHA_CUDA(cudaMemsetAsync(c.epoch, 0, sizeof(int) * z.cap, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.vote, 0x7f, sizeof(int) * z.cap, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(c.ctr, 0, sizeof(Counters), c.stream));
    return GPUDT_OK;
}

static void ev_record(Ctx &c, int k)
{
    c.reads_at[k] = c.host_reads;
    if (c.events) cudaEventRecord(c.ev[k], c.stream);
}

static int fbo_ok(int T) { return T >= 256 && T <= 16384 && (T & (T - 1)) == 0; }

// Records which stage failed and the device-side detail code.
int stage_fail(Ctx &c, int r, const char *stage)
{
    if (r == GPUDT_ERR_CUDA || r == GPUDT_ERR_NOMEM) {
        if (g_err.find(stage) == std::string::npos) g_err = std::string(stage) + ": " + g_err;
        return r;
    }
    read_counters(c);
    char buf[160];
    snprintf(buf, sizeof(buf), "stage %s: device error %d, detail %d", stage, c.hctr->err, c.hctr->errinfo);
    g_err = buf;
    return r;
}

// DT of n device points (interleaved xy).  Leaves the compacted mesh in c.cv/c.cn.
static int run_dt(HandleState &H, const double *d_xy, int n, double minX, double minY, double maxX, double maxY,
                  int T)
{
    Ctx &c = H.c;
    int r;
    int nside = (T - 1 + kFakeSpacing - 1) / kFakeSpacing;
    int V = n + 4 * nside;
    r = ensure(H, V, T, 0);
    if (r) return r;
    memset(&c.st, 0, sizeof(c.st));
    c.host_reads = 0;
    c.chash = nullptr;  // no constrained edges unless this call's constraint stage sets them
    for (int k = 0; k < 10; k++) c.kev_rec[k] = false;
    c.have_mesh = c.have_alpha = c.have_master = false;
    ev_record(c, 1);
    int nonempty = has_triangles(c, d_xy, n);
    if (nonempty < 0) return stage_fail(c, nonempty, "precheck");
    if (nonempty == 0) {
        // fewer than three distinct points, or all collinear: no triangle
        // (the reference has no defined output here; this returns an empty mesh)
        c.N = n;
        c.nT_out = 0;
        c.have_mesh = true;
        for (int k = 2; k <= 8; k++) ev_record(c, k);
        return GPUDT_OK;
    }
    const char *stage = "setup";
#define STAGE(name, call)        \
    stage = name;                \
    r = (call);                  \
    if (r) return stage_fail(c, r, stage)
    STAGE("setup", stage_setup(c, d_xy, n, minX, minY, maxX, maxY, T));
    STAGE("voronoi", stage_voronoi(c));
    ev_record(c, 2);
    STAGE("triangles", stage_triangles(c));
    STAGE("links", stage_links(c));
    ev_record(c, 3);
    STAGE("shift", stage_shift(c));
    ev_record(c, 4);
    STAGE("missing", stage_missing(c));
    ev_record(c, 5);
    STAGE("boundary", stage_boundary(c));
    STAGE("constraints", stage_constraints(c));
    ev_record(c, 6);
    STAGE("flip", stage_flip(c));
    ev_record(c, 7);
    STAGE("compact", stage_compact(c));
#undef STAGE
    ev_record(c, 8);
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return stage_fail(c, c.hctr->err, "final");
    c.st.nVerts = c.V;
    c.st.nFake = c.F;
    fill_predicate_stats(c);
    c.have_mesh = true;
    return GPUDT_OK;
}

// ------------------------------------------------------------------ batches
struct EdgeBases {
    const int *e_off, *tbase;
    int nT, nE;
    int *out;
    __device__ void operator()(long long s) const
    {
        int t = tbase[s];
        out[s] = t < nT ? e_off[t] : nE;
    }
};

static int run_batch(HandleState &H, int K, const int *sizes, const double *d_xy, const double *bounds, int withAlpha)
{
    Ctx &c = H.c;
    BatchHost &bh = H.bh;
    bh.valid = false;
    int r = batch_plan(bh, K, sizes, bounds);
    if (r) {
        g_err = "galphaRunBatch: invalid set sizes or bounds";
        return r;
    }
    Sizes z;
    z.V = (size_t)bh.N + bh.Fmax;
    z.T2 = (size_t)bh.T2;
    z.occw = (size_t)bh.occw;
    z.bandw = (size_t)bh.band;
    z.cap = 2 * z.V + 64;
    z.lists = std::max(z.cap * 3, z.V + 1);
    int Tmax = 128;
    for (auto &C : bh.classes) Tmax = std::max(Tmax, C.T);
    z.ntiles = std::max<size_t>(((size_t)(Tmax - 1) * (Tmax - 1) + 255) / 256 + 1,
                                (size_t)bh.T2 / 256 + bh.K + 1);  // envelope emission tiles of all cells
    r = ensure_sizes(H, z);
    if (r) return r;
    r = batch_buffers(c, H.bd, K, bh.N, (int)z.V, c.cap_tris, 3 * c.cap_tris + 8, bh.ntiles);
    if (r) return r;
    memset(&c.st, 0, sizeof(c.st));
    c.host_reads = 0;
    c.chash = nullptr;  // no constrained edges unless this call's constraint stage sets them
    for (int k = 0; k < 10; k++) c.kev_rec[k] = false;
    c.have_mesh = c.have_alpha = c.have_master = false;
    ev_record(c, 1);
    const char *stage = "setup";
#define STAGE(name, call)        \
    stage = name;                \
    r = (call);                  \
    if (r) return stage_fail(c, r, stage)
    STAGE("setup", batch_setup(c, H.bd, bh, d_xy));
    STAGE("voronoi", batch_voronoi(c, H.bd, bh));
    ev_record(c, 2);
    STAGE("links", stage_links(c));
    ev_record(c, 3);
    STAGE("shift", stage_shift(c));
    ev_record(c, 4);
    STAGE("missing", stage_missing(c));
    ev_record(c, 5);
    STAGE("boundary", stage_boundary(c));
    STAGE("constraints", stage_constraints(c));
    ev_record(c, 6);
    STAGE("flip", stage_flip(c));
    ev_record(c, 7);
    STAGE("compact", batch_compact(c, H.bd, bh));
    ev_record(c, 8);
    c.have_mesh = true;
    bh.alpha = false;
    if (withAlpha) {
        AlphaSegs segs{H.bd.tset, K, H.bd.seg, H.bd.firstexcl, H.bd.nd, H.bd.spec_off, H.bd.tbase, H.bd.ebase};
        STAGE("alpha", stage_alpha(c, &segs));
        c.have_alpha = true;
        bh.alpha = true;
        launch_n(c, EdgeBases{c.e_off, H.bd.tbase, c.nT_out, c.nE, H.bd.firstexcl}, K);
        bh.ebase.resize(K);
        bh.nd.resize(K);
        bh.specoff.resize(K);
        GALPHA_CUDA(cudaMemcpyAsync(bh.ebase.data(), H.bd.firstexcl, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost,
                                    c.stream));
        GALPHA_CUDA(cudaMemcpyAsync(bh.nd.data(), H.bd.nd, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost, c.stream));
        GALPHA_CUDA(cudaMemcpyAsync(bh.specoff.data(), H.bd.spec_off, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost,
                                    c.stream));
        GALPHA_CUDA(cudaStreamSynchronize(c.stream));
        for (int s2 = 0; s2 < K; s2++) bh.specoff[s2] += s2;  // one rank-0 sentinel per set
    }
    ev_record(c, 9);
#undef STAGE
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return stage_fail(c, c.hctr->err, "final");
    c.st.nVerts = c.V;
    c.st.nFake = c.F;
    fill_predicate_stats(c);
    bh.valid = true;
    return GPUDT_OK;
}

static void fill_times(Ctx &c, int last)
{
    if (!c.events) return;
    cudaEventSynchronize(c.ev[last]);
    for (int k = 1; k < last; k++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c.ev[k], c.ev[k + 1]) == cudaSuccess && k < 12) c.st.ms[k] = ms;
        if (k < 12) c.st.hostReadsStage[k] = c.reads_at[k + 1] - c.reads_at[k];
    }
    float tot = 0.f;
    if (cudaEventElapsedTime(&tot, c.ev[0], c.ev[last]) == cudaSuccess) c.st.ms[GALPHA_STAGE_TOTAL] = tot;
    auto kms = [&](int k) -> float {
        float v = 0.f;
        if (c.kev_rec[2 * k] && c.kev_rec[2 * k + 1]) {
            if (cudaEventElapsedTime(&v, c.kev[2 * k], c.kev[2 * k + 1]) != cudaSuccess) v = 0.f;
        }
        return v;
    };
    c.st.kernelMs[0] = kms(0);
    c.st.kernelMs[1] = kms(1);
    c.st.kernelMs[2] = kms(2) + kms(3);
    c.st.kernelMs[3] = kms(4);
    cudaGetLastError();  // a timing query never leaves an error behind
}

static int upload_points(HandleState &H, const gpudtVertex *pts, int n)
{
    Ctx &c = H.c;
    size_t bytes = sizeof(double) * 2 * (size_t)(n > 0 ? n : 1);
    if (bytes > H.d_xy_cap) {
        if (H.d_xy) cudaFree(H.d_xy);
        H.d_xy = nullptr;
        H.d_xy_cap = 0;
        GALPHA_CUDA(cudaMalloc(&H.d_xy, bytes));
        H.d_xy_cap = bytes;
    }
    if (n > 0)
        GALPHA_CUDA(cudaMemcpyAsync(H.d_xy, pts, sizeof(double) * 2 * (size_t)n, cudaMemcpyHostToDevice, c.stream));
    return GPUDT_OK;
}

static int check_params(const GPUDTPARAMS *p)
{
    if (!p) return GPUDT_ERR_ARG;
    if (p->nPoints < 0 || (p->nPoints > 0 && !p->points)) return GPUDT_ERR_ARG;
    if (p->nConstraints < 0 || (p->nConstraints > 0 && !p->constraints)) return GPUDT_ERR_ARG;
    for (int k = 0; k < p->nConstraints; k++) {
        const int a = p->constraints[2 * k], b = p->constraints[2 * k + 1];
        if (a < 0 || b < 0 || a >= p->nPoints || b >= p->nPoints || a == b) {
            set_last_error("constraint with an endpoint out of range, or with equal endpoints");
            return GPUDT_ERR_ARG;
        }
    }
    if (!fbo_ok(p->fboSize)) return GPUDT_ERR_ARG;
    if (p->nPoints >= (1 << 28)) return GPUDT_ERR_ARG;
    if (!(std::isfinite(p->minX) && std::isfinite(p->minY) && std::isfinite(p->maxX) && std::isfinite(p->maxY)))
        return GPUDT_ERR_ARG;
    if (p->minX > p->maxX || p->minY > p->maxY) return GPUDT_ERR_ARG;
    return GPUDT_OK;
}

}  // namespace galpha

using namespace galpha;

struct galpha_ctx {
    HandleState H;
    std::mutex mu;
};

static int handle_init(galpha_ctx *h, int device, long long budget)
{
    Ctx &c = h->H.c;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_err = "no CUDA device";
        return GPUDT_ERR_NODEVICE;
    }
    if (device < 0) GALPHA_CUDA(cudaGetDevice(&device));
    GALPHA_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    GALPHA_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        g_err = "libgalpha is built for sm_100a";
        return GPUDT_ERR_NODEVICE;
    }
    c.device = device;
    c.sm_count = prop.multiProcessorCount;
    c.budget = budget;
    GALPHA_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.own_stream = true;
    {
        // counter mirror + mailbox: pinned, mapped into the device's address space
        const size_t ctr_bytes = (sizeof(Counters) + 255) & ~(size_t)255;
        void *hp = nullptr, *dp = nullptr;
        GALPHA_CUDA(cudaHostAlloc(&hp, ctr_bytes + kMailBytes, cudaHostAllocMapped));
        memset(hp, 0, ctr_bytes + kMailBytes);
        GALPHA_CUDA(cudaHostGetDevicePointer(&dp, hp, 0));
        c.hctr = (Counters *)hp;
        c.hctr_dev = (Counters *)dp;
        c.hmail = (char *)hp + ctr_bytes;
        c.hmail_dev = (char *)dp + ctr_bytes;
    }
    for (int k = 0; k < GALPHA_STAGE_TOTAL + 2; k++) GALPHA_CUDA(cudaEventCreate(&c.ev[k]));
    for (int k = 0; k < 10; k++) GALPHA_CUDA(cudaEventCreate(&c.kev[k]));
    c.events = true;
    // exact fall-back paths keep expansion arrays on the per-thread stack
    GALPHA_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, 18432));  // largest kernel frame is ~16 KB
    return GPUDT_OK;
}

extern "C" {

const char *galphaVersion(void) { return "galpha-b200 0.1 (sm_100a)"; }

unsigned long long galphaLaunchCount(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

const char *galphaLastError(void) { return last_error_text(); }

int galphaCreate(int device, long long budgetBytes, galphaHandle *out)
{
    if (!out) return GPUDT_ERR_ARG;
    galpha_ctx *h = new (std::nothrow) galpha_ctx;
    if (!h) return GPUDT_ERR_NOMEM;
    int r = handle_init(h, device, budgetBytes);
    if (r) {
        delete h;
        *out = nullptr;
        return r;
    }
    *out = h;
    return GPUDT_OK;
}

int galphaDestroy(galphaHandle h)
{
    if (!h) return GPUDT_OK;
    Ctx &c = h->H.c;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    if (h->H.arena.base) cudaFree(h->H.arena.base);
    if (h->H.d_xy) cudaFree(h->H.d_xy);
    if (c.ml_buf) cudaFree(c.ml_buf);
    if (c.cons_buf) cudaFree(c.cons_buf);
    if (c.cons_pool) cudaFree(c.cons_pool);
    if (h->H.bd.buf) cudaFree(h->H.bd.buf);
    if (c.hctr) cudaFreeHost(c.hctr);
    for (int k = 0; k < GALPHA_STAGE_TOTAL + 2 && c.events; k++) cudaEventDestroy(c.ev[k]);
    for (int k = 0; k < 10 && c.events; k++) cudaEventDestroy(c.kev[k]);
    if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
    if (h->H.side) {
        cudaStreamSynchronize(h->H.side);
        cudaStreamDestroy(h->H.side);
    }
    if (h->H.side_ev) cudaEventDestroy(h->H.side_ev);
    delete h;
    return GPUDT_OK;
}

int galphaSetStream(galphaHandle h, void *stream)
{
    if (!h) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (stream) {
        if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
        c.stream = (cudaStream_t)stream;
        c.own_stream = false;
    }
    return GPUDT_OK;
}

int galphaSetLimits(galphaHandle h, int maxRounds, int spinLimit, int holdFirstTile)
{
    if (!h) {
        noalloc_set_limits(spinLimit, holdFirstTile);
        return GPUDT_OK;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    c.max_rounds = maxRounds > 0 ? maxRounds : kMaxRounds;
    c.spin_limit = spinLimit > 0 ? spinLimit : kSpinLimit;
    c.hold_first = holdFirstTile > 0 ? 1 : 0;
    return GPUDT_OK;
}

int galphaSetSchedule(galphaHandle h, int shiftGroup, int missingGroup, int flipSync, int flipTailEnter,
                      int flipTailLeave)
{
    if (!h) return GPUDT_ERR_ARG;
    const int sg = shiftGroup > 0 ? shiftGroup : kShiftGroupDefault;
    const int mg = missingGroup > 0 ? missingGroup : kMissingGroupDefault;
    const int fs = flipSync > 0 ? flipSync : kFlipSyncDefault;
    const int te = flipTailEnter >= 0 ? flipTailEnter : kTailEnterDefault;
    const int tl = flipTailLeave > 0 ? flipTailLeave : kTailLeaveDefault;
    if (sg > kMaxGroup || mg > kMaxGroup || fs > 64 || te > (1 << 20) || tl > (1 << 22) || tl < te)
        return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    c.shift_group = sg;
    c.missing_group = mg;
    c.flip_sync = fs;
    c.tail_enter = te;
    c.tail_leave = tl;
    return GPUDT_OK;
}

int galphaGetSchedule(galphaHandle h, int *out5)
{
    if (!h || !out5) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    const Ctx &c = h->H.c;
    out5[0] = c.shift_group;
    out5[1] = c.missing_group;
    out5[2] = c.flip_sync;
    out5[3] = c.tail_enter;
    out5[4] = c.tail_leave;
    return GPUDT_OK;
}

int galphaSetBlockRun(galphaHandle h, int entries)
{
    if (!h) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    h->H.c.block_run = entries > 0 ? entries : kBlockRun;
    return GPUDT_OK;
}

int galphaRunDevice(galphaHandle h, const double *d_xy, int n, double minX, double minY, double maxX, double maxY,
                    int fboSize, int withAlpha, gpudtStatus *st)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || n < 0 || !fbo_ok(fboSize)) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    const int level = withAlpha & 3;
    ev_record(c, 0);
    c.want_outtri = (withAlpha & GALPHA_RUN_TRIANGLES) != 0;  // written by the compaction
    int r = run_dt(h->H, d_xy, n, minX, minY, maxX, maxY, fboSize);
    c.want_outtri = false;
    if (!r && level) {
        ev_record(c, 8);
        r = stage_alpha(c);
        if (!r) c.have_alpha = true;
        ev_record(c, 9);
        if (!r && level >= 2) {
            r = master_list(c);
            ev_record(c, 10);
        }
        if (!r) fill_times(c, 9);
        if (!r && level >= 2 && c.events) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c.ev[9], c.ev[10]) == cudaSuccess) c.st.ms[GALPHA_STAGE_MASTER] = ms;
            if (cudaEventElapsedTime(&ms, c.ev[0], c.ev[10]) == cudaSuccess) c.st.ms[GALPHA_STAGE_TOTAL] = ms;
            cudaGetLastError();
        }
    } else if (!r) {
        fill_times(c, 8);
    }
    c.st.status = r;
    c.st.hostReads = c.host_reads;
    if (st) *st = c.st;
    return r;
}

int galphaTriangulate(galphaHandle h, const GPUDTPARAMS *params, GPUDTOUTPUT *out, gpudtStatus *st)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h) return GPUDT_ERR_ARG;
    int r = check_params(params);
    if (r) return r;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    ev_record(c, 0);
    r = upload_points(h->H, params->points, params->nPoints);
    c.n_cons = params->nConstraints;
    c.h_cons = params->constraints;
    c.want_outtri = out != nullptr;
    if (!r)
        r = run_dt(h->H, h->H.d_xy, params->nPoints, params->minX, params->minY, params->maxX, params->maxY,
                   params->fboSize);
    c.want_outtri = false;
    c.n_cons = 0;
    c.h_cons = nullptr;
    if (!r && out) {
        int n = params->nPoints;
        gpudtTriangle *tris = nullptr;
        if (out->triangles) {
            // caller buffer: out->nTris is its capacity
            if (out->nTris < c.nT_out) {
                g_err = "galphaTriangulate: output buffer too small";
                r = GPUDT_ERR_NOMEM;
            } else {
                tris = out->triangles;
            }
        } else {
            int nv = n + std::max(4, (int)(std::sqrt((double)n) / 10));
            int capacity = std::max(2 * nv, c.nT_out);
            tris = new (std::nothrow) gpudtTriangle[capacity > 0 ? capacity : 1];
            if (!tris) r = GPUDT_ERR_NOMEM;
        }
        if (!r) r = ensure_outtri(c);
        if (!r) {
            if (c.nT_out > 0) {
                cudaError_t e = cudaMemcpyAsync(tris, c.outtri, sizeof(gpudtTriangle) * (size_t)c.nT_out,
                                                cudaMemcpyDeviceToHost, c.stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
                if (e != cudaSuccess) r = cuda_fail(e, "download triangles");
            }
            out->triangles = tris;
            out->nTris = c.nT_out;
        }
    }
    if (!r) fill_times(c, 8);
    c.st.status = r;
    c.st.hostReads = c.host_reads;
    if (st) *st = c.st;
    return r;
}

int galphaGetCounts(galphaHandle h, int *nTris, int *nEdges, int *nSpectrum)
{
    if (!h) return GPUDT_ERR_ARG;
    Ctx &c = h->H.c;
    if (nTris) *nTris = c.have_mesh ? c.nT_out : 0;
    if (nEdges) *nEdges = c.have_alpha ? c.nE : 0;
    if (nSpectrum) *nSpectrum = c.have_alpha ? c.nSpec : 0;
    return GPUDT_OK;
}

static int run_query(galphaHandle h, double alpha, double q, bool by_quantile, galphaQueryResult *res)
{
    if (!h || !res) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (!c.have_alpha) {
        g_err = "galphaQuery: no alpha result on this handle";
        return GPUDT_ERR_ARG;
    }
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    int r = alpha_query(c, alpha, q, by_quantile);
    if (r) return r;
    if (c.hctr->err) return c.hctr->err;
    res->alpha = c.hctr->qalpha;
    res->rank = c.hctr->qrank;
    for (int k = 0; k < 4; k++) {
        res->nPoints[k] = c.hctr->qcount[k];
        res->nEdges[k] = c.hctr->qcount[4 + k];
        res->nTris[k] = c.hctr->qcount[8 + k];
    }
    return GPUDT_OK;
}

int galphaQuery(galphaHandle h, double alpha, galphaQueryResult *res)
{
    return run_query(h, alpha, 0.0, false, res);
}

int galphaQueryQuantile(galphaHandle h, double q, galphaQueryResult *res)
{
    return run_query(h, 0.0, q, true, res);
}

int galphaCopyClasses(galphaHandle h, unsigned char *pointClass, unsigned char *edgeClass, unsigned char *triClass)
{
    if (!h) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (!c.have_alpha) return GPUDT_ERR_ARG;
    cudaStream_t s = c.stream;
    if (pointClass && c.N > 0)
        GALPHA_CUDA(cudaMemcpyAsync(pointClass, c.qclass, (size_t)c.N, cudaMemcpyDeviceToHost, s));
    if (edgeClass && c.nE > 0)
        GALPHA_CUDA(cudaMemcpyAsync(edgeClass, c.qclass + c.N, (size_t)c.nE, cudaMemcpyDeviceToHost, s));
    if (triClass && c.nT_out > 0)
        GALPHA_CUDA(cudaMemcpyAsync(triClass, c.qclass + c.N + c.nE, (size_t)c.nT_out, cudaMemcpyDeviceToHost, s));
    GALPHA_CUDA(cudaStreamSynchronize(s));
    return GPUDT_OK;
}

int galphaCopyTriangles(galphaHandle h, gpudtTriangle *dst, int cap)
{
    if (!h || !dst) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (!c.have_mesh) return GPUDT_ERR_ARG;
    int n = std::min(cap, c.nT_out);
    int r = ensure_outtri(c);
    if (r) return r;
    if (n > 0) {
        GALPHA_CUDA(cudaMemcpyAsync(dst, c.outtri, sizeof(gpudtTriangle) * (size_t)n, cudaMemcpyDeviceToHost, c.stream));
        GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    }
    return GPUDT_OK;
}

// Edge records in the reference's edge_interval layout, built on the device.
struct EdgeAos {
    const int4 *edges;
    const int *ero;
    const int2 *enu;
    galphaEdgeInterval *out;
    __device__ void operator()(long long e) const
    {
        galphaEdgeInterval E;
        int4 q = edges[e];
        E.ro_rank = ero[e];
        E.nu_min_rank = enu[e].x;
        E.nu_max_rank = enu[e].y;
        E.sc = E.ro_rank == 0 ? 0 : 1;
        E.tIndex = q.z;
        E.vOpp = q.w;
        out[e] = E;
    }
};

// Copies the alpha result to host memory.  When the caller passes buffers
// (non-NULL pointers, capacities in the count fields) they are filled in place
// -- pinned buffers make these single DMA copies; otherwise the arrays are
// allocated with malloc and released by galphaReleaseOutput.
static int download_alpha(Ctx &c, GAlphaOutput *out)
{
    bool caller = out->spectrum && out->point_list && out->edge_list && out->tri_list;
    if (caller) {
        if (out->nSpectrum < c.nSpec || out->nPoints < c.N || out->nEdges < c.nE || out->nTris < c.nT_out) {
            g_err = "galphaComputeResident: output buffers too small (see galphaGetCounts)";
            return GPUDT_ERR_NOMEM;
        }
    } else {
        memset(out, 0, sizeof(*out));
        out->spectrum = (double *)malloc(sizeof(double) * (size_t)std::max(1, c.nSpec));
        out->point_list = (galphaPointInterval *)malloc(sizeof(galphaPointInterval) * (size_t)std::max(1, c.N));
        out->edge_list = (galphaEdgeInterval *)malloc(sizeof(galphaEdgeInterval) * (size_t)std::max(1, c.nE));
        out->tri_list = (galphaTriangleInterval *)malloc(sizeof(galphaTriangleInterval) * (size_t)std::max(1, c.nT_out));
        if (!out->spectrum || !out->point_list || !out->edge_list || !out->tri_list) {
            galphaReleaseOutput(out);
            return GPUDT_ERR_NOMEM;
        }
    }
    out->nSpectrum = c.nSpec;
    out->nPoints = c.N;
    out->nEdges = c.nE;
    out->nTris = c.nT_out;
    cudaStream_t s = c.stream;
    galphaEdgeInterval *d_edges = (galphaEdgeInterval *)c.edge_aos;
    launch_n(c, EdgeAos{c.edges, c.edge_ro, c.edge_nu, d_edges}, c.nE);
    GALPHA_CUDA(cudaMemcpyAsync(out->spectrum, c.spectrum, sizeof(double) * (size_t)c.nSpec, cudaMemcpyDeviceToHost, s));
    if (c.N > 0)
        GALPHA_CUDA(cudaMemcpyAsync(out->point_list, c.pt_nu, sizeof(int2) * (size_t)c.N, cudaMemcpyDeviceToHost, s));
    if (c.nT_out > 0)
        GALPHA_CUDA(cudaMemcpyAsync(out->tri_list, c.tri_ro, sizeof(int) * (size_t)c.nT_out, cudaMemcpyDeviceToHost, s));
    if (c.nE > 0)
        GALPHA_CUDA(cudaMemcpyAsync(out->edge_list, d_edges, sizeof(galphaEdgeInterval) * (size_t)c.nE,
                                    cudaMemcpyDeviceToHost, s));
    GALPHA_CUDA(cudaStreamSynchronize(s));
    out->exactCompares = (long long)c.hctr->exact_compares;
    out->exactTies = c.hctr->nties;
    out->exactAttached = (long long)c.hctr->exact_attached;
    return GPUDT_OK;
}

int galphaComputeResident(galphaHandle h, GAlphaOutput *out)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || !out) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (!c.have_mesh) return GPUDT_ERR_ARG;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    int r = GPUDT_OK;
    if (!c.have_alpha) {
        r = stage_alpha(c);
        if (r) return r;
        c.have_alpha = true;
    }
    return download_alpha(c, out);
}

// Alpha of a host triangulation: the points and triangles are uploaded into
// the handle's mesh arrays, then the same device stage runs.
struct AosToSoa {
    const gpudtTriangle *in;
    int4 *cv, *cn;
    __device__ void operator()(long long i) const
    {
        gpudtTriangle g = in[i];
        cv[i] = make_int4(g.vtx[0], g.vtx[1], g.vtx[2], 0);
        cn[i] = make_int4(g.tri[0], g.tri[1], g.tri[2], 0);
    }
};

int galphaCompute(galphaHandle h, const GPUDTPARAMS *params, const GPUDTOUTPUT *dt, GAlphaOutput *out)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || !params || !dt || !out || params->nPoints < 0 || dt->nTris < 0) return GPUDT_ERR_ARG;
    if (dt->nTris > 0 && !dt->triangles) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    int n = params->nPoints;
    int r = ensure(h->H, n + 4, 256, (long long)dt->nTris);
    if (r) return r;
    r = upload_points(h->H, params->points, n);
    if (r) return r;
    c.N = n;
    c.V = n;
    c.renumbered = false;  // a host mesh: input ids throughout
    GALPHA_CUDA(cudaMemcpyAsync(c.opos, h->H.d_xy, sizeof(double2) * (size_t)n, cudaMemcpyDeviceToDevice, c.stream));
    GALPHA_CUDA(cudaMemcpyAsync(c.outtri, dt->triangles, sizeof(gpudtTriangle) * (size_t)dt->nTris,
                                cudaMemcpyHostToDevice, c.stream));
    launch_n(c, AosToSoa{c.outtri, c.cv, c.cn}, dt->nTris);
    c.outtri_ready = true;
    c.nT_out = dt->nTris;
    c.have_mesh = true;
    c.have_alpha = c.have_master = false;
    r = stage_alpha(c);
    if (r) return r;
    c.have_alpha = true;
    return download_alpha(c, out);
}

// gpudtComputeDT + Alpha_Shapes_2D in one call with host outputs: the
// triangles are copied back on a second stream while the alpha stage runs on
// the handle's stream, so their transfer overlaps the alpha computation.
int galphaComputeAll(galphaHandle h, const GPUDTPARAMS *params, GPUDTOUTPUT *dt, GAlphaOutput *out, gpudtStatus *st)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || !dt || !out) return GPUDT_ERR_ARG;
    int r = check_params(params);
    if (r) return r;
    std::lock_guard<std::mutex> lk(h->mu);
    HandleState &H = h->H;
    Ctx &c = H.c;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    if (!H.side) {
        GALPHA_CUDA(cudaStreamCreateWithFlags(&H.side, cudaStreamNonBlocking));
        GALPHA_CUDA(cudaEventCreateWithFlags(&H.side_ev, cudaEventDisableTiming));
    }
    ev_record(c, 0);
    r = upload_points(H, params->points, params->nPoints);
    c.n_cons = params->nConstraints;
    c.h_cons = params->constraints;
    c.want_outtri = true;
    if (!r)
        r = run_dt(H, H.d_xy, params->nPoints, params->minX, params->minY, params->maxX, params->maxY,
                   params->fboSize);
    c.want_outtri = false;
    c.n_cons = 0;
    c.h_cons = nullptr;
    gpudtTriangle *tris = nullptr;
    bool owned = false, copying = false;
    if (!r) {
        const int n = params->nPoints;
        if (dt->triangles) {
            if (dt->nTris < c.nT_out) {
                g_err = "galphaComputeAll: triangle buffer too small";
                r = GPUDT_ERR_NOMEM;
            } else {
                tris = dt->triangles;
            }
        } else {
            int nv = n + std::max(4, (int)(std::sqrt((double)n) / 10));
            int capacity = std::max(2 * nv, c.nT_out);
            tris = new (std::nothrow) gpudtTriangle[capacity > 0 ? capacity : 1];
            owned = true;
            if (!tris) r = GPUDT_ERR_NOMEM;
        }
    }
    if (!r) r = ensure_outtri(c);
    if (!r && c.nT_out > 0) {
        cudaError_t e = cudaEventRecord(H.side_ev, c.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(H.side, H.side_ev, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(tris, c.outtri, sizeof(gpudtTriangle) * (size_t)c.nT_out, cudaMemcpyDeviceToHost,
                                H.side);
        if (e != cudaSuccess) r = cuda_fail(e, "galphaComputeAll: download triangles");
        else copying = true;
    }
    if (!r) {
        ev_record(c, 8);
        r = stage_alpha(c);
        if (!r) c.have_alpha = true;
        ev_record(c, 9);
    }
    if (!r) r = download_alpha(c, out);
    if (copying) {
        // the side copy reads c.outtri: wait for it whatever happened above
        cudaError_t e = cudaStreamSynchronize(H.side);
        if (!r && e != cudaSuccess) r = cuda_fail(e, "galphaComputeAll: download triangles");
    }
    if (!r) {
        dt->triangles = tris;
        dt->nTris = c.nT_out;
        fill_times(c, 9);
    } else if (owned) {
        delete[] tris;
    }
    c.st.status = r;
    c.st.hostReads = c.host_reads;
    if (st) *st = c.st;
    return r;
}

int galphaRunBatch(galphaHandle h, int nSets, const int *setSizes, const double *d_xy, const double *bounds,
                   int withAlpha, gpudtStatus *st)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || nSets <= 0 || !setSizes || !bounds) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    ev_record(c, 0);
    int r = run_batch(h->H, nSets, setSizes, d_xy, bounds, withAlpha);
    if (!r) fill_times(c, withAlpha ? 9 : 8);
    c.st.status = r;
    c.st.hostReads = c.host_reads;
    if (st) *st = c.st;
    return r;
}

int galphaRunBatchHost(galphaHandle h, int nSets, const int *setSizes, const double *xy, const double *bounds,
                       int withAlpha, gpudtStatus *st)
{
    g_err.clear();  // a compute call starts without a stale message
    if (!h || nSets <= 0 || !setSizes || !bounds) return GPUDT_ERR_ARG;
    long long n = 0;
    for (int s = 0; s < nSets; s++) n += setSizes[s] > 0 ? setSizes[s] : 0;
    if (n > 0x3fffffffLL || (n > 0 && !xy)) return GPUDT_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        cudaSetDevice(h->H.c.device);
        cudaGetLastError();
        ev_record(h->H.c, 0);
        int r = upload_points(h->H, (const gpudtVertex *)xy, (int)n);
        if (r) return r;
    }
    return galphaRunBatch(h, nSets, setSizes, h->H.d_xy, bounds, withAlpha, st);
}

int galphaSetBatchDensity(galphaHandle h, double pixelsPerPoint)
{
    if (!h || !(pixelsPerPoint >= 1.0 && pixelsPerPoint <= 64.0)) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    h->H.bh.density = pixelsPerPoint;
    return GPUDT_OK;
}

int galphaBatchSets(galphaHandle h, galphaBatchSet *sets)
{
    if (!h || !sets) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    BatchHost &bh = h->H.bh;
    Ctx &c = h->H.c;
    if (!bh.valid) return GPUDT_ERR_ARG;
    for (int s = 0; s < bh.K; s++) {
        galphaBatchSet &o = sets[s];
        o.nPoints = bh.sets[s].n;
        o.pointBase = bh.sets[s].vbase;
        o.triBase = bh.tbase[s];
        o.nTris = bh.tbase[s + 1] - bh.tbase[s];
        if (bh.alpha) {
            o.edgeBase = bh.ebase[s];
            o.nEdges = (s + 1 < bh.K ? bh.ebase[s + 1] : c.nE) - bh.ebase[s];
            o.specBase = bh.specoff[s];
            o.nSpectrum = bh.nd[s] + 1;
        } else {
            o.edgeBase = o.nEdges = o.specBase = o.nSpectrum = 0;
        }
    }
    return GPUDT_OK;
}

int galphaBatchCopy(galphaHandle h, gpudtTriangle *tris, galphaPointInterval *points, galphaEdgeInterval *edges,
                    int *triRanks, double *spectrum)
{
    if (!h) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    BatchHost &bh = h->H.bh;
    Ctx &c = h->H.c;
    if (!bh.valid) return GPUDT_ERR_ARG;
    if (!bh.alpha && (points || edges || triRanks || spectrum)) return GPUDT_ERR_ARG;
    cudaSetDevice(c.device);
    cudaStream_t s = c.stream;
    gpudtTriangle *dtri = h->H.bd.otri;
    galphaEdgeInterval *dedge = c.edge_aos;
    int r = batch_local_outputs(c, h->H.bd, tris ? dtri : nullptr, edges ? dedge : nullptr);
    if (r) return r;
    if (tris && c.nT_out > 0)
        GALPHA_CUDA(cudaMemcpyAsync(tris, dtri, sizeof(gpudtTriangle) * (size_t)c.nT_out, cudaMemcpyDeviceToHost, s));
    if (edges && c.nE > 0)
        GALPHA_CUDA(cudaMemcpyAsync(edges, dedge, sizeof(galphaEdgeInterval) * (size_t)c.nE, cudaMemcpyDeviceToHost, s));
    if (points && c.N > 0)
        GALPHA_CUDA(cudaMemcpyAsync(points, c.pt_nu, sizeof(int2) * (size_t)c.N, cudaMemcpyDeviceToHost, s));
    if (triRanks && c.nT_out > 0)
        GALPHA_CUDA(cudaMemcpyAsync(triRanks, c.tri_ro, sizeof(int) * (size_t)c.nT_out, cudaMemcpyDeviceToHost, s));
    if (spectrum && c.nSpec > 0)
        GALPHA_CUDA(cudaMemcpyAsync(spectrum, c.spectrum, sizeof(double) * (size_t)c.nSpec, cudaMemcpyDeviceToHost, s));
    GALPHA_CUDA(cudaStreamSynchronize(s));
    return GPUDT_OK;
}

int galphaBatchQuery(galphaHandle h, const double *values, int byQuantile, galphaQueryResult *res)
{
    if (!h || !values || !res) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    BatchHost &bh = h->H.bh;
    BatchDev &B = h->H.bd;
    Ctx &c = h->H.c;
    if (!bh.valid || !bh.alpha) {
        g_err = "galphaBatchQuery: no batched alpha result on this handle";
        return GPUDT_ERR_ARG;
    }
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    const int K = bh.K;
    GALPHA_CUDA(cudaMemcpyAsync(B.qparam, values, sizeof(double) * (size_t)K, cudaMemcpyHostToDevice, c.stream));
    int r = alpha_query_sets(c, K, B.vsetall, B.tset, B.spec_off, B.nd, B.qparam, byQuantile ? 1 : 0, B.qR, B.qalpha,
                             B.qcounts);
    if (r) return r;
    std::vector<int> R(K), cnt(12 * (size_t)K);
    std::vector<double> a(K);
    GALPHA_CUDA(cudaMemcpyAsync(R.data(), B.qR, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaMemcpyAsync(a.data(), B.qalpha, sizeof(double) * (size_t)K, cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaMemcpyAsync(cnt.data(), B.qcounts, sizeof(int) * 12 * (size_t)K, cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    for (int s2 = 0; s2 < K; s2++) {
        res[s2].alpha = a[s2];
        res[s2].rank = R[s2];
        for (int k = 0; k < 4; k++) {
            res[s2].nPoints[k] = cnt[12 * (size_t)s2 + k];
            res[s2].nEdges[k] = cnt[12 * (size_t)s2 + 4 + k];
            res[s2].nTris[k] = cnt[12 * (size_t)s2 + 8 + k];
        }
    }
    return GPUDT_OK;
}

static const int kMinusOneHost = -1;

int galphaMasterList(galphaHandle h, GAlphaMasterList *out)
{
    if (!h || !out) return GPUDT_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    Ctx &c = h->H.c;
    if (!c.have_alpha) {
        g_err = "galphaMasterList: no alpha result on this handle";
        return GPUDT_ERR_ARG;
    }
    cudaSetDevice(c.device);
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    if (!c.have_master) {
        int r = master_list(c);
        if (r) return r;
    }
    bool caller = out->master_list && out->spec_pointers;
    if (caller) {
        if (out->nMaster < c.nMaster || out->nSpecPointers < c.nSpecPtr) {
            g_err = "galphaMasterList: output buffers too small";
            return GPUDT_ERR_ARG;
        }
    } else {
        out->master_list = (galphaAlpha *)malloc(sizeof(galphaAlpha) * (size_t)(c.nMaster > 0 ? c.nMaster : 1));
        out->spec_pointers = (int *)malloc(sizeof(int) * (size_t)(c.nSpecPtr > 0 ? c.nSpecPtr : 1));
        if (!out->master_list || !out->spec_pointers) {
            free(out->master_list);
            free(out->spec_pointers);
            out->master_list = nullptr;
            out->spec_pointers = nullptr;
            return GPUDT_ERR_NOMEM;
        }
    }
    if (c.nMaster > 0)
        GALPHA_CUDA(cudaMemcpyAsync(out->master_list, c.ml_out, sizeof(galphaAlpha) * (size_t)c.nMaster,
                                    cudaMemcpyDeviceToHost, c.stream));
    if (c.nMaster > 0)
        GALPHA_CUDA(cudaMemcpyAsync(out->spec_pointers, c.ml_sp, sizeof(int) * (size_t)c.nSpecPtr,
                                    cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    if (c.nMaster == 0) out->spec_pointers[0] = kMinusOneHost;
    out->nMaster = c.nMaster;
    out->nSpecPointers = c.nSpecPtr;
    return GPUDT_OK;
}

void galphaReleaseMasterList(GAlphaMasterList *out)
{
    if (!out) return;
    free(out->master_list);
    free(out->spec_pointers);
    out->master_list = nullptr;
    out->spec_pointers = nullptr;
    out->nMaster = out->nSpecPointers = 0;
}

void galphaReleaseOutput(GAlphaOutput *out)
{
    if (!out) return;
    free(out->spectrum);
    free(out->point_list);
    free(out->edge_list);
    free(out->tri_list);
    memset(out, 0, sizeof(*out));
}

// ------------------------------------------------------ reference entry points
static galpha_ctx *g_default = nullptr;
static std::mutex g_default_mu;

static galpha_ctx *default_handle(int *status)
{
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default) {
        galphaHandle h = nullptr;
        int r = galphaCreate(-1, 0, &h);
        if (r) {
            if (status) *status = r;
            return nullptr;
        }
        g_default = h;
    }
    return g_default;
}

int gpudtComputeDTEx(const GPUDTPARAMS *pParam, GPUDTOUTPUT *pOutput, gpudtStatus *status)
{
    g_err.clear();  // a compute call starts without a stale message
    int r = GPUDT_OK;
    galpha_ctx *h = default_handle(&r);
    if (!h) {
        if (status) {
            memset(status, 0, sizeof(*status));
            status->status = r;
        }
        return r;
    }
    if (!pOutput) return GPUDT_ERR_ARG;
    pOutput->triangles = nullptr;
    pOutput->nTris = 0;
    return galphaTriangulate(h, pParam, pOutput, status);
}

PGPUDTOUTPUT gpudt_compute_dt(PGPUDTPARAMS pParam)
{
    PGPUDTOUTPUT out = new (std::nothrow) GPUDTOUTPUT;
    if (!out) return nullptr;
    out->triangles = nullptr;
    out->nTris = 0;
    gpudtStatus st;
    int r = gpudtComputeDTEx(pParam, out, &st);
    if (r) {
        fprintf(stderr, "gpudtComputeDT failed: status %d (%s)\n", r, last_error_text());
        delete[] out->triangles;
        out->triangles = nullptr;
        out->nTris = 0;
    }
    return out;
}

// As gpudt.cpp:926-929: frees the triangle array only.
void gpudt_release_dt_output(PGPUDTOUTPUT pGpudtOutput)
{
    if (!pGpudtOutput) return;
    delete[] pGpudtOutput->triangles;
    pGpudtOutput->triangles = nullptr;
}

}  // extern "C"

// C++-linkage symbols of the reference header (gpudt.h:131-132).
PGPUDTOUTPUT gpudtComputeDT(PGPUDTPARAMS pParam) { return gpudt_compute_dt(pParam); }
void gpudtReleaseDTOutput(PGPUDTOUTPUT pGpudtOutput) { gpudt_release_dt_output(pGpudtOutput); }
