// sort.cu -- LSD radix sort of 64-bit keys with an int payload.
//
// Replaces thrust::sort_by_key on the FP64 spectrum (Alpha_Shapes_2D.cu:317):
// the keys are the IEEE bit patterns of positive doubles, so their unsigned
// order is the numeric order.  8-bit digits; digits on which all keys agree are
// skipped (an OR of key XOR first-key finds them).  Each pass: a per-block
// shared-memory histogram, a scan of the digit-major histogram table, and a
// stable scatter in which every warp ranks its 32 keys per round with
// __match_any_sync.
#include <algorithm>
#include "internal.cuh"

namespace galpha {

// ------------------------------------------------------------- radix sort
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 keys per block

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned long long *__restrict__ keys, int n,
                                                        int shift, int *__restrict__ hist, int nblocks)
{
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kRsTile;
    for (int k = threadIdx.x; k < kRsTile; k += kRsThreads) {
        long long i = base + k;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: warp w owns tile elements [w*512, (w+1)*512) in 16 rounds of
// 32; ranks within a round come from __match_any_sync on the digit.
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned long long *__restrict__ kin,
                                                           const int *__restrict__ vin,
                                                           unsigned long long *__restrict__ kout,
                                                           int *__restrict__ vout, int n, int shift,
                                                           const int *__restrict__ hoff, int nblocks)
{
    __shared__ int wcnt[kRsThreads / 32][256];
    __shared__ int boff[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = lane; d < 256; d += 32) wcnt[w][d] = 0;
    boff[threadIdx.x] = hoff[threadIdx.x * nblocks + blockIdx.x];
    __syncwarp();
    long long base = (long long)blockIdx.x * kRsTile + (long long)w * (kRsItems * 32);
    unsigned long long key[kRsItems];
    int dig[kRsItems];
    unsigned lanemask_lt = (1u << lane) - 1u;
    // sweep 1: per-warp digit counts
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        long long i = base + r * 32 + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : 0ull;
        dig[r] = ok ? (int)((key[r] >> shift) & 255) : 256 + lane;  // unique dummy digits
        unsigned peers = __match_any_sync(0xffffffffu, dig[r]);
        if (ok && (peers & lanemask_lt) == 0) wcnt[w][dig[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive scan over warps
    {
        int d = threadIdx.x;
        int s = 0;
        for (int q = 0; q < kRsThreads / 32; q++) {
            int c = wcnt[q][d];
            wcnt[q][d] = s;
            s += c;
        }
    }
    __syncthreads();
    // sweep 2: scatter
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        long long i = base + r * 32 + lane;
        bool ok = i < n;
        unsigned peers = __match_any_sync(0xffffffffu, dig[r]);
        int rank = __popc(peers & lanemask_lt);
        int d = ok ? dig[r] : 0;
        int pos = 0;
        if (ok) pos = boff[d] + wcnt[w][d] + rank;
        __syncwarp();
        if (ok && (peers & lanemask_lt) == 0) wcnt[w][d] += __popc(peers);
        __syncwarp();
        if (ok) {
            kout[pos] = key[r];
            vout[pos] = vin[i];
        }
    }
}

// OR over all keys of (key XOR first key): the bits on which keys differ.
// Reduced per warp and per block; one 64-bit atomic per block.
__global__ void __launch_bounds__(256) k_or_xor(const unsigned long long *__restrict__ keys, long long n,
                                                unsigned long long *acc)
{
    __shared__ unsigned long long ws[8];
    unsigned long long k0 = acc[0], x = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x |= keys[i] ^ k0;
    for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) x |= ws[w];
        if (x) atomicOr(&acc[1], x);
    }
}

// Sorts (keys, vals)[0..n) ascending; result in keys/vals.  Uses keys2/vals2.
int radix_sort(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *keys2, int *vals2, int n)
{
    if (n <= 1) return GPUDT_OK;
    unsigned long long *acc = (unsigned long long *)c.rhist;
    GALPHA_CUDA(cudaMemcpyAsync(acc, keys, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(acc + 1, 0, sizeof(unsigned long long), c.stream));
    {
        long long blocks = std::min<long long>((n + 255) / 256, (long long)c.sm_count * 4);
        k_or_xor<<<(unsigned)blocks, 256, 0, c.stream>>>(keys, n, acc);
        count_launch();
    }
    unsigned long long hv[2];
    GALPHA_CUDA(cudaMemcpyAsync(hv, acc, sizeof(hv), cudaMemcpyDeviceToHost, c.stream));
    GALPHA_CUDA(cudaStreamSynchronize(c.stream));
    unsigned long long varying = hv[1];
    int nblocks = (n + kRsTile - 1) / kRsTile;
    int *hist = c.rhist + 8;
    unsigned long long *ki = keys, *ko = keys2;
    int *vi = vals, *vo = vals2;
    for (int shift = 0; shift < 64; shift += 8) {
        if (((varying >> shift) & 255ull) == 0) continue;
        k_rs_hist<<<nblocks, kRsThreads, 0, c.stream>>>(ki, n, shift, hist, nblocks);
        count_launch();
        int r = exclusive_scan_int(c, hist, hist, 256 * nblocks, nullptr);
        if (r) return r;
        k_rs_scatter<<<nblocks, kRsThreads, 0, c.stream>>>(ki, vi, ko, vo, n, shift, hist, nblocks);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    if (ki != keys) {
        GALPHA_CUDA(cudaMemcpyAsync(keys, ki, sizeof(unsigned long long) * (size_t)n, cudaMemcpyDeviceToDevice,
                                    c.stream));
        GALPHA_CUDA(cudaMemcpyAsync(vals, vi, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, c.stream));
    }
    return GPUDT_OK;
}

}  // namespace galpha
