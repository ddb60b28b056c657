// noalloc.cu -- galphaEdgeListNoAlloc: the alpha stage's edge numbering of a
// device-resident triangle-neighbour mesh, computed without allocating.
//
// The handle path numbers edges in three launches over arena scratch
// (EdgeCount -> exclusive_scan_int -> the edge writes of TriKeys, which
// restate computeTriEdgeCount + thrust::exclusive_scan + the edge fill of
// Alpha_Shapes_2D.cu:170-199).  This variant does the same in ONE kernel: each
// block takes the next tile of triangles from a ticket, counts the edges its
// triangles own, finds the tile's global offset by a single-pass decoupled
// look-back over the per-tile descriptors of earlier tiles, and writes the
// (tIndex, vOpp) pairs.  The descriptors, the ticket and a done counter live in
// one file-scope device array (g_el_scratch, 512 KB), so a call allocates
// nothing: not device memory, not pinned host memory, not events.
//
// Shared-state rules:
//  * every call on a device uses the same array, so calls on one device must
//    be ordered (same stream, or synchronised): two calls in flight at once
//    race on the ticket and descriptors and give wrong results;
//  * the ticket, the done counter, the error word and every descriptor must
//    be zero when a call starts; the first call on a device (and the first
//    after a cudaDeviceReset, which reloads the module) zeroes the array,
//    stream-ordered on the caller's stream, and the last block of every call
//    zeroes what the call used before it exits.
#include <cstdint>
#include <cstdio>
#include <mutex>
#include "internal.cuh"

namespace galpha {
namespace {

constexpr int kElThreads = 256;
constexpr int kElItems = 4;
constexpr int kElTile = kElThreads * kElItems;  // 1024 triangles per tile
constexpr int kElMaxTiles = 65536;
constexpr long long kElMaxTris = (long long)kElTile * kElMaxTiles;  // 67,108,864
constexpr int kElHeader = 32;  // [0] ticket, [1] blocks done, [2] error word
constexpr unsigned long long kStAgg = 1ull << 62;   // descriptor holds the tile's own count
constexpr unsigned long long kStPre = 2ull << 62;   // descriptor holds the inclusive prefix
constexpr unsigned long long kValMask = (1ull << 62) - 1;
constexpr int kMaxDevices = 64;

// 512 KB: the header words and one descriptor per tile
static __device__ __align__(256) unsigned long long g_el_scratch[kElHeader + kElMaxTiles];

__device__ __forceinline__ void st_release(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Owned edges of one triangle record staged in shared memory (9 ints: tri[3],
// vtx[3], tmp[3]): edge i = (vtx[i+1], vtx[i+2]) belongs to the triangle when
// its first vertex has the smaller index or it lies on the hull (kernel.cu's
// computeTriEdgeCount rule, the same test as EdgeCount in alpha.cu).
__device__ __forceinline__ int owned_mask(const int *r)
{
    int m = 0;
    for (int i = 0; i < 3; i++) {
        int a = r[3 + p1(i)], b = r[3 + m1(i)];
        if (a < b || r[i] == -1) m |= 1 << i;
    }
    return m;
}

// spin_limit bounds every look-back wait; hold_first (a failure-detection
// test switch, 0 in normal use) makes tile 0 withhold its descriptor so that
// tile 1's wait runs out and the call reports GPUDT_ERR_NOCONVERGE.
__global__ void __launch_bounds__(kElThreads) k_edge_list(const int *__restrict__ tris, int nTris,
                                                          int2 *__restrict__ edges, int cap,
                                                          int *__restrict__ nEdges,
                                                          unsigned long long *__restrict__ scratch,
                                                          int spin_limit, int hold_first)
{
    __shared__ int s_rec[kElTile * 9];  // the tile's triangle records, 36 KB
    __shared__ unsigned char s_mask[kElTile];
    __shared__ int s_tile, s_last;
    __shared__ int s_warp[kElThreads / 32];
    __shared__ unsigned long long s_excl;
    unsigned long long *hdr = scratch;
    unsigned long long *desc = scratch + kElHeader;
    const int ntiles = gridDim.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    if (threadIdx.x == 0) s_tile = (int)atomicAdd(&hdr[0], 1ull);
    __syncthreads();
    const int tile = s_tile;
    const long long tbase = (long long)tile * kElTile;
    const int ntile = (int)min((long long)kElTile, (long long)nTris - tbase);

    // stage the records with consecutive 4-byte loads (a warp reads 128
    // contiguous bytes), then find each triangle's owned edges from shared
    // memory (stride 9 words between threads: no bank conflicts)
    const int *src = tris + tbase * 9;
    for (int j = threadIdx.x; j < ntile * 9; j += kElThreads) s_rec[j] = src[j];
    __syncthreads();
    for (int t = threadIdx.x; t < kElTile; t += kElThreads)
        s_mask[t] = t < ntile ? (unsigned char)owned_mask(s_rec + 9 * t) : 0;
    __syncthreads();

    // this thread's kElItems consecutive triangles
    unsigned masks = 0;  // 3 bits per item
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < kElItems; k++) {
        int m = s_mask[threadIdx.x * kElItems + k];
        masks |= (unsigned)m << (3 * k);
        cnt += __popc(m);
    }
    // block-wide exclusive scan of the counts
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    int wbase = 0, agg = 0;
    for (int q = 0; q < kElThreads / 32; q++) {
        int v = s_warp[q];
        if (q < w) wbase += v;
        agg += v;
    }
    const int texcl = wbase + incl - cnt;

    // decoupled look-back for the tile's global offset
    if (threadIdx.x == 0) {
        unsigned long long excl = 0;
        if (tile == 0) {
            if (!hold_first) st_release(&desc[0], kStPre | (unsigned long long)agg);
        } else {
            st_release(&desc[tile], kStAgg | (unsigned long long)agg);
            bool bad = false;
            for (int j = tile - 1; j >= 0; j--) {
                unsigned long long d = 0;
                int spins = 0;
                // tile j took its ticket before this one, so its block is running
                // and publishes; the bound only guards against a broken invariant
                while (((d = ld_acquire(&desc[j])) >> 62) == 0) {
                    if (++spins > spin_limit) {
                        bad = true;
                        break;
                    }
                    __nanosleep(32);
                }
                if (bad) break;
                excl += d & kValMask;
                if ((d >> 62) == 2) break;
            }
            if (bad) atomicOr(&hdr[2], 1ull);
            st_release(&desc[tile], kStPre | (excl + (unsigned long long)agg));
        }
        s_excl = excl;
    }
    __syncthreads();

    long long e = (long long)s_excl + texcl;
#pragma unroll
    for (int k = 0; k < kElItems; k++) {
        long long t = tbase + threadIdx.x * kElItems + k;
        if (t >= nTris) break;
        for (int i = 0; i < 3; i++) {
            if ((masks >> (3 * k + i)) & 1u) {
                if (e < cap) edges[e] = make_int2((int)t, i);
                e++;
            }
        }
    }

    // the last block to finish reports the count and zeroes the scratch it used
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&hdr[1], 1ull) == (unsigned long long)(ntiles - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned long long total = ld_acquire(&desc[ntiles - 1]) & kValMask;
        bool err = ld_acquire(&hdr[2]) != 0ull;
        *nEdges = err ? GPUDT_ERR_NOCONVERGE : (total > 0x7fffffffull ? GPUDT_ERR_NOMEM : (int)total);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < ntiles; j += kElThreads) desc[j] = 0ull;
    if (threadIdx.x < 3) hdr[threadIdx.x] = 0ull;
}

std::mutex g_el_mu;
unsigned long long *g_el_ptr[kMaxDevices];  // the address the array was last zeroed at
int g_el_spin_limit = kSpinLimit;
int g_el_hold_first = 0;

// The array's device address, looked up on every call with the caller's
// device current (a cudaDeviceReset reloads the module, so an address kept
// from before would be stale), and a zero fill ordered on the caller's stream
// whenever the address is new: the first call on a device, the first after a
// reset.
int el_scratch(cudaStream_t stream, unsigned long long **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "galphaEdgeListNoAlloc: cudaGetDevice"), GPUDT_ERR_NODEVICE;
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("galphaEdgeListNoAlloc: device index out of range");
        return GPUDT_ERR_NODEVICE;
    }
    unsigned long long *p = nullptr;
    e = cudaGetSymbolAddress((void **)&p, g_el_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "galphaEdgeListNoAlloc: cudaGetSymbolAddress"), GPUDT_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_el_mu);
    if (g_el_ptr[dev] != p) {
        e = cudaMemsetAsync(p, 0, sizeof(g_el_scratch), stream);
        if (e != cudaSuccess) return cuda_fail(e, "galphaEdgeListNoAlloc: zeroing scratch"), GPUDT_ERR_CUDA;
        g_el_ptr[dev] = p;
    }
    *out = p;
    return GPUDT_OK;
}

}  // namespace

// Failure-detection limits of galphaEdgeListNoAlloc (galphaSetLimits with a
// NULL handle); values <= 0 restore the defaults.
void noalloc_set_limits(int spin_limit, int hold_first)
{
    std::lock_guard<std::mutex> lk(g_el_mu);
    g_el_spin_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
    g_el_hold_first = hold_first > 0 ? 1 : 0;
}

}  // namespace galpha

using namespace galpha;

extern "C" int galphaEdgeListNoAlloc(const gpudtTriangle *d_tris, int nTris, int *d_edges, int edgeCapacity,
                                     int *d_nEdges, void *stream_)
{
    if (nTris < 0 || edgeCapacity < 0 || !d_nEdges || (nTris > 0 && !d_tris) || (edgeCapacity > 0 && !d_edges)) {
        set_last_error("galphaEdgeListNoAlloc: invalid argument");
        return GPUDT_ERR_ARG;
    }
    if (((uintptr_t)d_edges & 7u) != 0 || ((uintptr_t)d_tris & 3u) != 0 || ((uintptr_t)d_nEdges & 3u) != 0) {
        set_last_error("galphaEdgeListNoAlloc: misaligned buffer (d_edges needs 8 bytes, the others 4)");
        return GPUDT_ERR_ARG;
    }
    if ((long long)nTris > kElMaxTris) {
        char buf[160];
        snprintf(buf, sizeof(buf), "galphaEdgeListNoAlloc: %d triangles exceed the fixed scratch limit of %lld",
                 nTris, kElMaxTris);
        set_last_error(buf);
        return GPUDT_ERR_ARG;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    cudaGetLastError();  // clear an error left by unrelated runtime calls
    unsigned long long *scratch = nullptr;
    int r = el_scratch(stream, &scratch);
    if (r) return r;
    if (nTris == 0) {
        cudaError_t e = cudaMemsetAsync(d_nEdges, 0, sizeof(int), stream);
        if (e != cudaSuccess) return cuda_fail(e, "galphaEdgeListNoAlloc"), GPUDT_ERR_CUDA;
        return GPUDT_OK;
    }
    int ntiles = (int)(((long long)nTris + kElTile - 1) / kElTile);
    int spin_limit, hold_first;
    {
        std::lock_guard<std::mutex> lk(g_el_mu);
        spin_limit = g_el_spin_limit;
        hold_first = g_el_hold_first;
    }
    k_edge_list<<<ntiles, kElThreads, 0, stream>>>((const int *)d_tris, nTris, (int2 *)d_edges, edgeCapacity,
                                                   d_nEdges, scratch, spin_limit, hold_first);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "galphaEdgeListNoAlloc: launch"), GPUDT_ERR_CUDA;
    return GPUDT_OK;
}
