// scan.cu -- exclusive prefix sum of int32 arrays (reduce-then-scan).
//
// Replaces the reference's recursive Blelloch scan (cudaScanLargeArray.cu:
// 222-477, prescanArray) and its host-side row prefix sum
// (cudaReconstruction.cu:470-478).  Each block scans a 4096-element tile held
// in registers (16 per thread) with warp shuffles; tile sums are scanned
// recursively; a final pass adds the tile offsets.  Scratch comes from a
// per-handle buffer, so a scan allocates nothing.
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

// out may alias in.  total_dev (optional) receives sum(in).
int exclusive_scan_int(Ctx &c, const int *in, int *out, int n, int *total_dev)
{
    if (n <= 0) {
        if (total_dev) GALPHA_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(int), c.stream));
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
