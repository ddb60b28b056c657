// scan.cu -- exclusive prefix sum of int32 arrays (reduce-then-scan).
//
// Replaces the reference's recursive Blelloch scan (cudaScanLargeArray.cu:
// 222-477, prescanArray) and its host-side row prefix sum
// (cudaReconstruction.cu:470-478).  Each block scans a 4096-element tile held
// in registers (16 per thread) with warp shuffles.  Up to 32736 tiles, one
// launch scans the whole array (tile offsets by decoupled look-back, int4
// accesses); above that, tile sums are scanned recursively and a final pass
// adds the tile offsets.  Scratch comes from a per-handle buffer, so a scan
// allocates nothing.
#include "internal.cuh"

namespace galpha {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl(int v)
{
    int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ int block_scan(int v, int &excl)
{
    __shared__ int ws[kScanThreads / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = warp_incl(v);
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        int s = lane < kScanThreads / 32 ? ws[lane] : 0;
        int si = warp_incl(s);
        if (lane < kScanThreads / 32) ws[lane] = si - s;
    }
    __syncthreads();
    excl = incl - v + ws[w];
    __shared__ int total;
    if (threadIdx.x == kScanThreads - 1) total = excl + v;
    __syncthreads();
    int t = total;
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int *__restrict__ in, int *__restrict__ out,
                                                             int *__restrict__ tilesum, long long n)
{
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    int excl;
    int tot = block_scan(s, excl);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        long long i = base + k;
        if (i < n) out[i] = excl;
        excl += v[k];
    }
    if (threadIdx.x == 0) tilesum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_add(int *__restrict__ out, const int *__restrict__ tileoff,
                                                           long long n)
{
    long long base = (long long)blockIdx.x * kScanTile;
    int add = tileoff[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += kScanThreads) {
        long long i = base + k;
        if (i < n) out[i] += add;
    }
}

__global__ void k_scan_total(const int *in_last, const int *out_last, int *total)
{
    *total = *in_last + *out_last;
}

size_t scan_scratch_bytes(int n)
{
    size_t total = 0;
    long long m = n;
    while (m > 1) {
        m = (m + kScanTile - 1) / kScanTile;
        total += sizeof(int) * (size_t)(m + 1);
    }
    return total + 64;
}

static int scan_rec(Ctx &c, const int *in, int *out, long long n, int *scratch)
{
    long long tiles = (n + kScanTile - 1) / kScanTile;
    int *tilesum = scratch;
    k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, c.stream>>>(in, out, tilesum, n);
    count_launch();
    if (tiles > 1) {
        int r = scan_rec(c, tilesum, tilesum, tiles, scratch + tiles + 1);
        if (r) return r;
        k_scan_add<<<(unsigned)tiles, kScanThreads, 0, c.stream>>>(out, tilesum, n);
        count_launch();
    }
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

// ---------------------------------------------------------- single pass
// One launch: tiles are taken in ticket order; each tile publishes its sum,
// then warp 0 looks back over the published sums of up to 32 earlier tiles at
// a time until it meets a tile that has published its inclusive prefix
// (decoupled look-back), and publishes its own.  A tile only waits on tiles
// with earlier tickets, whose blocks are running; the bounded wait guards a
// broken invariant and reports it in the counter block.
constexpr unsigned long long kScAgg = 1ull << 62;  // status: the tile's own sum
constexpr unsigned long long kScPre = 2ull << 62;  // status: the sum of this and all earlier tiles
constexpr unsigned long long kScVal = (1ull << 62) - 1;
constexpr int kScanSpinLimit = 1 << 22;
constexpr int kScanStatusOff = 64;  // ints before the status words in the scratch (ticket at [2])
constexpr long long kScanMaxTiles = (65536 - kScanStatusOff) / 2;

__device__ __forceinline__ void sc_st_release(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long sc_ld_acquire(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// A tile is kScanSlices slices of 4 * kScanThreads elements; thread t holds
// elements [4t, 4t + 4) of each slice as one int4, so every load and store
// of a warp covers 512 contiguous bytes.  The warp sums of all slices, in
// slice-major order, are the tile's 32 partial sums in element order: one
// warp scan gives every warp's offset and the tile total.
constexpr int kScanSlices = kScanItems / 4;
static_assert(kScanSlices * (kScanThreads / 32) == 32, "one warp scans the partial sums of a tile");

__global__ void __launch_bounds__(kScanThreads) k_scan_1p(const int *__restrict__ in, int *__restrict__ out,
                                                          long long n, unsigned long long *status, int *ticket,
                                                          int *total, Counters *ct, bool vec)
{
    __shared__ int s_tile;
    __shared__ long long s_excl;
    __shared__ int s_part[32];
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1);
    __syncthreads();
    const int tile = s_tile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long base = (long long)tile * kScanTile + 4ll * threadIdx.x;
    int4 a[kScanSlices];
    int incl[kScanSlices], sum[kScanSlices];
#pragma unroll
    for (int k = 0; k < kScanSlices; k++) {
        const long long i = base + (long long)k * 4 * kScanThreads;
        if (vec && i + 3 < n) {
            a[k] = *reinterpret_cast<const int4 *>(in + i);
        } else {
            a[k].x = i < n ? in[i] : 0;
            a[k].y = i + 1 < n ? in[i + 1] : 0;
            a[k].z = i + 2 < n ? in[i + 2] : 0;
            a[k].w = i + 3 < n ? in[i + 3] : 0;
        }
        sum[k] = a[k].x + a[k].y + a[k].z + a[k].w;
        incl[k] = warp_incl(sum[k]);
        if (lane == 31) s_part[k * (kScanThreads / 32) + w] = incl[k];
    }
    __syncthreads();
    if (w == 0) {
        const int v = s_part[lane];
        const int x = warp_incl(v);
        s_part[lane] = x - v;  // exclusive offset of (slice, warp) in the tile
        if (lane == 31) s_tile = x;  // the tile total (the ticket is no longer needed)
    }
    __syncthreads();
    const int tot = s_tile;
    if (threadIdx.x < 32) {
        long long acc = 0;
        if (tile > 0) {
            if (lane == 0) sc_st_release(&status[tile], kScAgg | (unsigned long long)(unsigned)tot);
            bool bad = false;
            for (int j = tile - 1;; j -= 32) {
                const int idx = j - lane;
                unsigned long long wd = kScPre;  // before tile 0: nothing to add
                if (idx >= 0) {
                    int spins = 0;
                    while (((wd = sc_ld_acquire(&status[idx])) >> 62) == 0) {
                        if (++spins > kScanSpinLimit) {
                            bad = true;
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                if (__any_sync(0xffffffffu, bad)) {
                    bad = true;
                    break;
                }
                const unsigned pre = __ballot_sync(0xffffffffu, (wd >> 62) == 2);
                const int first = pre ? __ffs(pre) - 1 : 31;  // lanes up to the nearest prefix count
                long long mine = (lane <= first && idx >= 0) ? (long long)(wd & kScVal) : 0;
                for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
                acc += mine;
                if (pre) break;
            }
            if (bad && lane == 0) set_err(ct, GPUDT_ERR_NOCONVERGE, 97);
        }
        if (lane == 0) {
            sc_st_release(&status[tile], kScPre | (unsigned long long)(acc + tot));
            s_excl = acc;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanSlices; k++) {
        const long long i = base + (long long)k * 4 * kScanThreads;
        int4 o;
        o.x = (int)s_excl + s_part[k * (kScanThreads / 32) + w] + incl[k] - sum[k];
        o.y = o.x + a[k].x;
        o.z = o.y + a[k].y;
        o.w = o.z + a[k].z;
        if (vec && i + 3 < n) {
            *reinterpret_cast<int4 *>(out + i) = o;
        } else {
            if (i < n) out[i] = o.x;
            if (i + 1 < n) out[i + 1] = o.y;
            if (i + 2 < n) out[i + 2] = o.z;
            if (i + 3 < n) out[i + 3] = o.w;
        }
    }
    if (total && threadIdx.x == 0 && (long long)(tile + 1) * kScanTile >= n) *total = (int)(s_excl + tot);
}

// out may alias in.  total_dev (optional) receives sum(in).
int exclusive_scan_int(Ctx &c, const int *in, int *out, int n, int *total_dev)
{
    if (n <= 0) {
        if (total_dev) GALPHA_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(int), c.stream));
        return GPUDT_OK;
    }
    const long long tiles = ((long long)n + kScanTile - 1) / kScanTile;
    if (tiles > 1 && tiles <= kScanMaxTiles) {
        int *ticket = c.hist + 2;
        unsigned long long *status = reinterpret_cast<unsigned long long *>(c.hist + kScanStatusOff);
        GALPHA_CUDA(cudaMemsetAsync(ticket, 0, sizeof(int), c.stream));
        GALPHA_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned long long) * (size_t)tiles, c.stream));
        const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
        k_scan_1p<<<(unsigned)tiles, kScanThreads, 0, c.stream>>>(in, out, n, status, ticket, total_dev, c.ctr, vec);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        return GPUDT_OK;
    }
    int *scratch = c.hist;  // scan scratch lives at the start of the histogram buffer
    if (total_dev) {
        // keep the last input before an in-place scan overwrites it
        launch_n(c, CopyElems<int>{scratch, in + n - 1}, 1);
    }
    int r = scan_rec(c, in, out, n, scratch + 16);
    if (r) return r;
    if (total_dev) {
        k_scan_total<<<1, 1, 0, c.stream>>>(scratch, out + n - 1, total_dev);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
    }
    return GPUDT_OK;
}

}  // namespace galpha
