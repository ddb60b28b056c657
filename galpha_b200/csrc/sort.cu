// sort.cu -- stable LSD radix sort of 64- or 32-bit keys with an int payload.
//
// Replaces thrust::sort_by_key on the FP64 spectrum (Alpha_Shapes_2D.cu:317,
// keys = the IEEE bit patterns of positive doubles, whose unsigned order is
// the numeric order) and on the master-list ranks (Alpha_Shapes_2D.cu:658).
// 8-bit digits; digits on which all keys agree are skipped (an OR of
// key XOR first-key finds them).  Each pass: a per-block shared-memory
// histogram, a scan of the digit-major histogram table, and a scatter that
// first sorts the block's 2048-key tile by digit in shared memory (warp ranks
// from 8 ballots per round, stable) and then writes each digit's run to its
// global offset, so consecutive threads store consecutive addresses.
#include <algorithm>
#include <mutex>
#include "internal.cuh"

namespace galpha {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;  // 2048 keys per block (several blocks per SM)
constexpr int kRsWarps = kRsThreads / 32;

template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const K *__restrict__ keys, int n, int shift,
                                                        int *__restrict__ hist, int nblocks)
{
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kRsTile;
    for (int k = threadIdx.x; k < kRsTile; k += kRsThreads) {
        long long i = base + k;
        if (i < n) atomicAdd(&h[(int)((keys[i] >> shift) & 255)], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

template <typename K>
struct RsSmem {
    K key[kRsTile];
    int val[kRsTile];
    int wcnt[kRsWarps][256];  // per-warp digit counts, then tile-local offsets
    int lstart[256];          // tile-local start of each digit's run
    int gbase[256];           // global start of this tile's run of each digit
};

// Stable scatter of one tile: warp w owns tile elements [w*256, (w+1)*256) in
// 8 rounds of 32; an element's tile-local rank is (digit run start) + (keys
// of the same digit in earlier warps) + (earlier rounds of its warp) + (lower
// lanes of its round).
template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const K *__restrict__ kin, const int *__restrict__ vin,
                                                           K *__restrict__ kout, int *__restrict__ vout, int n,
                                                           int shift, const int *__restrict__ hoff, int nblocks)
{
    extern __shared__ __align__(16) unsigned char rs_smem[];
    RsSmem<K> &S = *reinterpret_cast<RsSmem<K> *>(rs_smem);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = lane; d < 256; d += 32) S.wcnt[w][d] = 0;
    S.gbase[threadIdx.x] = hoff[threadIdx.x * nblocks + blockIdx.x];
    __syncwarp();
    const long long tile0 = (long long)blockIdx.x * kRsTile;
    const long long base = tile0 + (long long)w * (kRsItems * 32);
    K key[kRsItems];
    int val[kRsItems];
    int rk[kRsItems];  // rank within the warp's keys of the same digit
    const unsigned lanemask_lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        long long i = base + r * 32 + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : (K)0;
        val[r] = ok ? vin[i] : 0;
    }
    // lanes with the same digit: 8 ballots; the lowest such lane adds the
    // group to the warp's digit count and hands the old count to the group
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        const bool ok = base + r * 32 + lane < n;
        const int dg = (int)((key[r] >> shift) & 255);
        unsigned peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const unsigned bb = __ballot_sync(0xffffffffu, (dg >> b) & 1);
            peers &= ((dg >> b) & 1) ? bb : ~bb;
        }
        const int leader = ok ? __ffs(peers) - 1 : lane;
        int before = 0;
        if (ok && lane == leader) before = atomicAdd(&S.wcnt[w][dg], __popc(peers));
        before = __shfl_sync(0xffffffffu, before, leader);
        rk[r] = before + __popc(peers & lanemask_lt);
    }
    __syncthreads();
    // per digit: totals over warps, then the digit-major exclusive scan
    {
        const int d = threadIdx.x;
        int s = 0;
        for (int q = 0; q < kRsWarps; q++) {
            int c = S.wcnt[q][d];
            S.wcnt[q][d] = s;
            s += c;
        }
        S.lstart[d] = s;  // digit total for now
    }
    __syncthreads();
    if (w == 0) {
        int carry = 0;
        for (int d0 = 0; d0 < 256; d0 += 32) {
            int v = S.lstart[d0 + lane];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            S.lstart[d0 + lane] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        long long i = base + r * 32 + lane;
        if (i < n) {
            const int dg = (int)((key[r] >> shift) & 255);
            int p = S.lstart[dg] + S.wcnt[w][dg] + rk[r];
            S.key[p] = key[r];
            S.val[p] = val[r];
        }
    }
    __syncthreads();
    const int cnt = (int)min((long long)kRsTile, (long long)n - tile0);
    for (int p = threadIdx.x; p < cnt; p += kRsThreads) {
        K k = S.key[p];
        int d = (int)((k >> shift) & 255);
        long long g = (long long)S.gbase[d] + (p - S.lstart[d]);
        kout[g] = k;
        vout[g] = S.val[p];
    }
}

// OR over all keys of (key XOR first key): the bits on which keys differ.
// Reduced per warp and per block; one atomic per block.
template <typename K>
__global__ void __launch_bounds__(256) k_or_xor(const K *__restrict__ keys, long long n, K *acc)
{
    __shared__ K ws[8];
    K k0 = acc[0], x = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x |= keys[i] ^ k0;
    for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < 8; q++) x |= ws[q];
        if (x) atomicOr(&acc[1], x);
    }
}

// Scratch ints needed by radix_sort_keys for n keys.
long long radix_scratch_ints(long long n)
{
    return 8 + 256 * ((n + kRsTile - 1) / kRsTile + 1);
}

// Sorts (keys, vals)[0..n) ascending (stable) on the key bits from min_shift
// up; result in keys/vals.  Uses keys2/vals2 and `scratch`
// (radix_scratch_ints(n) ints).
template <typename K>
static int radix_sort_keys(Ctx &c, K *keys, int *vals, K *keys2, int *vals2, int n, int *scratch, int min_shift = 0,
                           bool *in_second = nullptr)
{
    if (in_second) *in_second = false;
    if (n <= 1) return GPUDT_OK;
    static_assert(sizeof(K) == 4 || sizeof(K) == 8, "32- or 64-bit keys");
    const int smem = (int)sizeof(RsSmem<K>);
    {
        static std::mutex mu;
        static bool attr_set[64];  // per key type and device: the opt-in above 48 KB, once
        std::lock_guard<std::mutex> lk(mu);
        if (c.device < 0 || c.device >= 64 || !attr_set[c.device]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_scatter<K>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             cudaSharedmemCarveoutMaxShared));
            if (c.device >= 0 && c.device < 64) attr_set[c.device] = true;
        }
    }
    K *acc = reinterpret_cast<K *>(scratch);
    launch_n(c, CopyElems<K>{acc, keys}, 1);
    GALPHA_CUDA(cudaMemsetAsync(acc + 1, 0, sizeof(K), c.stream));
    {
        long long blocks = std::min<long long>((n + 255) / 256, (long long)c.sm_count * 4);
        k_or_xor<K><<<(unsigned)blocks, 256, 0, c.stream>>>(keys, n, acc);
        count_launch();
    }
    K hv[2];
    int rr = read_small(c, hv, acc, sizeof(hv));
    if (rr) return rr;
    const unsigned long long varying = (unsigned long long)hv[1];
    const int nblocks = (n + kRsTile - 1) / kRsTile;
    int *hist = scratch + 8;
    K *ki = keys, *ko = keys2;
    int *vi = vals, *vo = vals2;
    for (int shift = min_shift; shift < (int)(8 * sizeof(K)); shift += 8) {
        if (((varying >> shift) & 255ull) == 0) continue;
        c.sort_passes++;
        k_rs_hist<K><<<nblocks, kRsThreads, 0, c.stream>>>(ki, n, shift, hist, nblocks);
        count_launch();
        int r = exclusive_scan_int(c, hist, hist, 256 * nblocks, nullptr);
        if (r) return r;
        k_rs_scatter<K><<<nblocks, kRsThreads, smem, c.stream>>>(ki, vi, ko, vo, n, shift, hist, nblocks);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    if (ki != keys) {
        if (in_second) {  // the caller takes the result where the last pass left it
            *in_second = true;
            return GPUDT_OK;
        }
        launch_n(c, CopyElems<K>{keys, ki}, n);
        launch_n(c, CopyElems<int>{vals, vi}, n);
    }
    return GPUDT_OK;
}

// ---------------------------------------------------------- 64-bit keys
// The radix passes run on the top 40 bits only (5 digits instead of 8).
// Entries whose top 40 bits agree are then put in full-key order: each such
// group that is out of order is insertion-sorted (stable) by one thread.  A
// group longer than kMaxFixGroup sends the whole array through the 3 low
// digits as well (an LSD sort of the partly sorted array keeps equal keys in
// their current, i.e. input, order), so the result is always the stable
// sort of the full keys.
constexpr int kLowBits = 24;
constexpr int kMaxFixGroup = 64;

struct FixFind {
    const unsigned long long *keys;
    int *starts, *flag;
    int n;
    Counters *ct;
    __device__ void operator()(long long ii) const
    {
        const int i = (int)ii;
        const unsigned long long k = keys[i], kp = keys[i - 1];
        if ((k >> kLowBits) != (kp >> kLowBits) || k >= kp) return;
        int s = i - 1, len = 2;
        while (s > 0 && (keys[s - 1] >> kLowBits) == (k >> kLowBits)) {
            s--;
            if (++len > kMaxFixGroup) {
                ct->changed = 1;  // too long: full sort
                return;
            }
        }
        for (int e = i + 1; e < n && (keys[e] >> kLowBits) == (k >> kLowBits); e++)
            if (++len > kMaxFixGroup) {
                ct->changed = 1;
                return;
            }
        if (atomicExch(&flag[s], 1) == 0) starts[atomicAdd(&ct->nlist2, 1)] = s;
    }
};

struct FixFindOffset {
    const unsigned long long *keys;
    int *starts, *flag;
    int n;
    Counters *ct;
    __device__ void operator()(long long i) const { FixFind{keys, starts, flag, n, ct}(i + 1); }
};

struct FixGroups {
    unsigned long long *keys;
    int *vals;
    const int *starts;
    int *flag;
    int n;
    __device__ void operator()(long long ii) const
    {
        const int s = starts[ii];
        flag[s] = 0;
        const unsigned long long hi = keys[s] >> kLowBits;
        int e = s + 1;
        while (e < n && (keys[e] >> kLowBits) == hi) e++;
        for (int a = s + 1; a < e; a++) {
            unsigned long long kc = keys[a];
            int vc = vals[a];
            int b = a - 1;
            for (; b >= s && keys[b] > kc; b--) {
                keys[b + 1] = keys[b];
                vals[b + 1] = vals[b];
            }
            keys[b + 1] = kc;
            vals[b + 1] = vc;
        }
    }
};

// The result is left in (keys, vals) or, when *in_second comes back true, in
// (keys2, vals2): an odd number of passes ends there, and a copy back would
// cost a full read and write of both arrays.
int radix_sort(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *keys2, int *vals2, int n,
               bool *in_second)
{
    bool sec = false;
    int r = radix_sort_keys<unsigned long long>(c, keys, vals, keys2, vals2, n, c.rhist, kLowBits, &sec);
    *in_second = sec;
    if (r || n <= 1) return r;
    unsigned long long *rk = sec ? keys2 : keys, *fk = sec ? keys : keys2;
    int *rv = sec ? vals2 : vals, *fv = sec ? vals : vals2;
    // group fix-up (starts / flags in the other key buffer, free now)
    int *starts = (int *)fk, *flag = starts + ((n + 63) & ~63);
    GALPHA_CUDA(cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)n, c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    launch_n(c, FixFindOffset{rk, starts, flag, n, c.ctr}, n - 1);
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->changed) {
        bool sec2 = false;
        r = radix_sort_keys<unsigned long long>(c, rk, rv, fk, fv, n, c.rhist, 0, &sec2);
        if (sec2) *in_second = !sec;
        return r;
    }
    if (c.hctr->nlist2 > 0) launch_n(c, FixGroups{rk, rv, starts, flag, n}, c.hctr->nlist2);
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int radix_sort32(Ctx &c, unsigned int *keys, int *vals, unsigned int *keys2, int *vals2, int n, int *scratch)
{
    return radix_sort_keys<unsigned int>(c, keys, vals, keys2, vals2, n, scratch);
}

}  // namespace galpha
