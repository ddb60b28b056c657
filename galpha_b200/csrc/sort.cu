// sort.cu -- stable LSD radix sort of 64- or 32-bit keys with an int payload.
//
// Replaces thrust::sort_by_key on the FP64 spectrum (Alpha_Shapes_2D.cu:317,
// keys = the IEEE bit patterns of positive doubles, whose unsigned order is
// the numeric order) and on the master-list ranks (Alpha_Shapes_2D.cu:658).
// 8-bit digits.  Every pass sorts the block's 2048-key tile by digit in
// shared memory (warp ranks from 8 ballots per round, stable) and then writes
// each digit's run to its global offset, so consecutive threads store
// consecutive addresses.  The spectrum's 5 passes over the top 40 key bits
// are one kernel each (digit counts of all passes from one read of the keys,
// tile offsets by decoupled look-back); the other sorts take a per-block
// histogram and a scan of the digit-major histogram table per pass, and skip
// the digits on which all keys agree (an OR of key XOR first-key finds them).
#include <algorithm>
#include <mutex>
#include <vector>
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
// key_bits > 0: the keys are known to fit in key_bits bits, and every digit
// below that is sorted without first reading which bits vary.
template <typename K>
static int radix_sort_keys(Ctx &c, K *keys, int *vals, K *keys2, int *vals2, int n, int *scratch, int min_shift = 0,
                           bool *in_second = nullptr, int key_bits = 0)
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
    unsigned long long varying;
    if (key_bits > 0) {
        varying = key_bits >= 64 ? ~0ull : (1ull << key_bits) - 1ull;
    } else {
        K *acc = reinterpret_cast<K *>(scratch);
        launch_n(c, CopyElems<K>{acc, keys}, 1);
        GALPHA_CUDA(cudaMemsetAsync(acc + 1, 0, sizeof(K), c.stream));
        long long blocks = std::min<long long>((n + 255) / 256, (long long)c.sm_count * 4);
        k_or_xor<K><<<(unsigned)blocks, 256, 0, c.stream>>>(keys, n, acc);
        count_launch();
        K hv[2];
        int rr = read_small(c, hv, acc, sizeof(hv));
        if (rr) return rr;
        varying = (unsigned long long)hv[1];
    }
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
// group that is out of order is insertion-sorted (stable) by one thread if it
// has at most kMaxFixGroup entries; a longer group is sorted as a sub-array
// by the radix passes (its top digits are constant and skipped).  With more
// than kMaxLongGroups long groups (or more than kMaxLongPairs recorded pairs)
// the whole array goes through all 8 digits instead (an LSD sort of the
// partly sorted array keeps equal keys in their current, i.e. input, order).
// Either way the result is the stable sort of the full keys.
constexpr int kLowBits = 24;
constexpr int kMaxFixGroup = 64;
constexpr int kMaxLongPairs = 4096;  // extents read back through the mailbox (8 B each)
constexpr int kMaxLongGroups = 64;

// Thread i checks the pair (i-1, i) of the sorted array.  Of the out-of-order
// pairs of one top-40-bit group only the first reports the group's start, so
// every group that needs fixing is listed once.
// A pair of a group longer than kMaxFixGroup is recorded in `longs` instead
// (several pairs of one long group may be; their extents are merged later).
struct FixFind {
    const unsigned long long *keys;
    int *starts, *longs;
    int n, lcap;  // lcap: room of longs
    Counters *ct;
    __device__ void long_pair(int i) const
    {
        const int k = atomicAdd(&ct->nlong, 1);
        if (k < lcap) longs[k] = i;
        else ct->changed = 1;  // too many: full sort
    }
    __device__ void operator()(long long ii) const
    {
        const int i = (int)ii;
        const unsigned long long k = keys[i], kp = keys[i - 1], hi = k >> kLowBits;
        if ((kp >> kLowBits) != hi || k >= kp) return;
        int s = i - 1, len = 2;
        unsigned long long right = kp;  // keys[s]
        while (s > 0) {
            const unsigned long long left = keys[s - 1];
            if ((left >> kLowBits) != hi) break;
            if (left > right) return;  // an earlier pair of the group is out of order: it reports
            right = left;
            s--;
            if (++len > kMaxFixGroup) {
                long_pair(i);
                return;
            }
        }
        for (int e = i + 1; e < n && (keys[e] >> kLowBits) == hi; e++)
            if (++len > kMaxFixGroup) {
                long_pair(i);
                return;
            }
        // one counter atomic per converged group of lanes
        const unsigned m = __activemask();
        const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&ct->nlist2, __popc(m));
        base = __shfl_sync(m, base, leader);
        starts[base + __popc(m & ((1u << lane) - 1u))] = s;
    }
};

// Extent [start, end) of the top-40-bit group around the recorded pair of
// block b, by block-wide scans of 256 keys per step (the group is contiguous).
__device__ __forceinline__ int block_max_int(int v, int *red)
{
    v = __reduce_max_sync(0xffffffffu, v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    int m = red[0];
    for (int q = 1; q < 8; q++) m = max(m, red[q]);
    return m;
}

__global__ void __launch_bounds__(256) k_group_extent(const unsigned long long *__restrict__ keys, int n,
                                                      const int *__restrict__ pairs, int2 *ext)
{
    __shared__ int red[8];
    const int i = pairs[blockIdx.x];
    const unsigned long long hi = keys[i] >> kLowBits;
    int start = 0, end = n;
    for (long long w0 = i; w0 > 0; w0 -= 256) {  // keys [w0 - 256, w0) before i
        const long long j = w0 - 1 - threadIdx.x;
        const bool diff = j >= 0 && (keys[j] >> kLowBits) != hi;
        const int m = block_max_int(diff ? (int)j + 1 : -1, red);
        if (m >= 0) {
            start = m;
            break;
        }
    }
    for (long long w0 = i + 1; w0 < n; w0 += 256) {  // keys [w0, w0 + 256) after i
        const long long j = w0 + threadIdx.x;
        const bool diff = j < n && (keys[j] >> kLowBits) != hi;
        const int m = block_max_int(diff ? -(int)j : -n - 1, red);  // the smallest such j
        if (m > -n - 1) {
            end = -m;
            break;
        }
    }
    if (threadIdx.x == 0) ext[blockIdx.x] = make_int2(start, end);
}

// FixFind over every pair (i - 1, i), 0 < i < n, each examined once: thread t
// reads 8 keys with 16-byte loads (plus the key before them) and hands the
// rare out-of-order pair to FixFind.  `keys` is 8-byte aligned: the chunks
// start at the first 16-byte boundary (key 0 or 1; key 0 has no pair), and
// the keys after the last whole chunk are checked one by one.
__global__ void __launch_bounds__(256) k_fix_find(const unsigned long long *__restrict__ keys, int *starts,
                                                  int *longs, int n, int lcap, Counters *ct)
{
    const FixFind f{keys, starts, longs, n, lcap, ct};
    const int lead = (int)((reinterpret_cast<uintptr_t>(keys) >> 3) & 1);  // keys before the 16-byte boundary
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nchunk = ((long long)n - lead) / 8;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = tid; t < nchunk; t += stride) {
        const long long i0 = lead + 8 * t;
        const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(keys + i0);
        const ulonglong2 a = p[0], b = p[1], c = p[2], d = p[3];
        const unsigned long long k[8] = {a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y};
        unsigned long long prev = i0 > 0 ? keys[i0 - 1] : 0ull;
#pragma unroll
        for (int u = 0; u < 8; u++) {
            // a pair in order never needs fixing; most pairs are
            if (i0 + u > 0 && k[u] < prev && (k[u] >> kLowBits) == (prev >> kLowBits)) f(i0 + u);
            prev = k[u];
        }
    }
    // the keys after the last whole chunk
    const long long rest0 = lead + 8 * nchunk;
    for (long long i = rest0 + tid; i < n; i += stride)
        if (i > 0) f(i);
}

struct FixGroups {
    unsigned long long *keys;
    int *vals;
    const int *starts;
    int n;
    __device__ void operator()(long long ii) const
    {
        const int s = starts[ii];
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

// ------------------------------------------- single-pass digit passes (64-bit)
// The spectrum sort's 5 passes over the top 40 key bits: one kernel first
// counts every pass's digits in one read of the keys (the global digit
// counts do not depend on the order); then each pass is one kernel.  A block
// takes the next tile by ticket, ranks it in shared memory as k_rs_scatter
// does, publishes its per-digit counts, and finds, per digit, the keys of
// that digit in earlier tiles by decoupled look-back: thread d reads the
// status word of digit d of the previous tiles until one holds an inclusive
// count (a tile's own count alone means: keep going back), then publishes
// its own inclusive count.  A tile waits only on tiles with earlier tickets,
// whose blocks are running; the bounded wait guards a broken invariant and
// reports it in the counter block.  Status words: bits 63-62 kind (1 the
// tile's count, 2 inclusive), bits 61-32 the pass (so the passes share
// the words, zeroed once per sort), bits 31-0 the count.
constexpr int kOsPasses = (64 - kLowBits) / 8;
constexpr int kOsTicketOff = kOsPasses * 256;  // after the digit counts [kOsPasses][256]
constexpr int kOsHeadInts = 2048;              // then the status words (256 per tile)
constexpr unsigned long long kOsAgg = 1ull << 62, kOsInc = 2ull << 62;
constexpr unsigned long long kOsPassMask = ((1ull << 30) - 1) << 32;
constexpr int kOsWindow = 8;  // earlier tiles read at once by the look-back

// A status word carries its own payload (nothing else is read after it), so
// relaxed accesses at GPU scope suffice, and the loads of a look-back window
// can be in flight together.
__device__ __forceinline__ void os_st(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long os_ld(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}

// Digit counts of all kOsPasses passes.  The top digits (sign and exponent)
// take few values, so their shared-memory increments are aggregated per warp
// over lanes with the same digit.
__global__ void __launch_bounds__(256) k_rs_hist_top(const unsigned long long *__restrict__ keys, int n,
                                                     int *__restrict__ ghist)
{
    constexpr int kU = 4;  // keys loaded before their digits are counted
    __shared__ int h[kOsPasses * 256];
    for (int i = threadIdx.x; i < kOsPasses * 256; i += 256) h[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * 256 * kU;
    // whole warps iterate together (the aggregated increments need them)
    const long long nw = ((long long)n + 31) & ~31ll;
    for (long long i0 = (long long)blockIdx.x * 256 * kU + threadIdx.x; i0 < nw; i0 += stride) {
        unsigned long long k[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const long long i = i0 + u * 256;
            k[u] = i < n ? keys[i] : 0ull;
        }
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const long long i = i0 + u * 256;
            if (i >= nw) break;  // uniform over the warp
            const bool ok = i < n;
#pragma unroll
            for (int p = 0; p < kOsPasses - 2; p++)
                if (ok) atomicAdd(&h[p * 256 + (int)((k[u] >> (kLowBits + 8 * p)) & 255)], 1);
#pragma unroll
            for (int p = kOsPasses - 2; p < kOsPasses; p++) {
                const int dg = ok ? (int)((k[u] >> (kLowBits + 8 * p)) & 255) : 256 + lane;
                const unsigned peers = __match_any_sync(0xffffffffu, dg);
                if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[p * 256 + dg], __popc(peers));
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kOsPasses * 256; i += 256)
        if (h[i]) atomicAdd(&ghist[i], h[i]);
}

__global__ void __launch_bounds__(kRsThreads, 5) k_rs_onesweep(const unsigned long long *__restrict__ kin,
                                                            const int *__restrict__ vin,
                                                            unsigned long long *__restrict__ kout,
                                                            int *__restrict__ vout, int n, int shift,
                                                            const int *__restrict__ dcount,
                                                            unsigned long long *status, int *ticket,
                                                            unsigned long long pass_tag, Counters *ct,
                                                            int spin_limit, int hold_first)
{
    typedef unsigned long long K;
    extern __shared__ __align__(16) unsigned char rs_smem[];
    RsSmem<K> &S = *reinterpret_cast<RsSmem<K> *>(rs_smem);
    __shared__ int s_tile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1);
    for (int d = lane; d < 256; d += 32) S.wcnt[w][d] = 0;
    __syncthreads();
    const int tile = s_tile;
    const long long tile0 = (long long)tile * kRsTile;
    const long long base = tile0 + (long long)w * (kRsItems * 32);
    K key[kRsItems];
    int val[kRsItems];
    int rk[kRsItems];
    const unsigned lanemask_lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        long long i = base + r * 32 + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : (K)0;
        val[r] = ok ? vin[i] : 0;
    }
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
    // per digit: totals over warps, published at once for the later tiles
    const int d = threadIdx.x;
    int tot = 0;
    for (int q = 0; q < kRsWarps; q++) {
        int c = S.wcnt[q][d];
        S.wcnt[q][d] = tot;
        tot += c;
    }
    S.lstart[d] = tot;
    unsigned long long *mine = status + (long long)tile * 256 + d;
    // (hold_first: a failure-detection test switch under which tile 0 withholds
    // its counts, so that tile 1's bounded wait runs out; 0 in normal use)
    if (tile != 0 || !hold_first) os_st(mine, (tile == 0 ? kOsInc : kOsAgg) | pass_tag | (unsigned)tot);
    __syncthreads();
    if (w == 0) {  // tile-local digit starts
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
    } else if (w == 1) {  // global digit starts of the pass
        int carry = 0;
        for (int d0 = 0; d0 < 256; d0 += 32) {
            int v = dcount[d0 + lane];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            S.gbase[d0 + lane] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    // the tile sorted by digit in shared memory (the key registers are free
    // for the look-back after this)
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
    // look-back for digit d over the earlier tiles, kOsWindow at a time: the
    // window's words are loaded together, then summed from the nearest tile
    // back to the first inclusive count (a word not yet published is re-read)
    long long acc = 0;
    if (tile > 0) {
        bool bad = false, done = false;
        for (long long j = tile - 1; j >= 0 && !done && !bad; j -= kOsWindow) {
            unsigned long long v[kOsWindow];
#pragma unroll
            for (int k = 0; k < kOsWindow; k++)
                v[k] = j - k >= 0 ? os_ld(status + (j - k) * 256 + d) : (kOsInc | pass_tag);
#pragma unroll
            for (int k = 0; k < kOsWindow; k++) {
                if (!done && !bad) {
                    unsigned long long x = v[k];
                    int spins = 0;
                    while (((x >> 62) == 0 || (x & kOsPassMask) != pass_tag) && spins <= spin_limit) {
                        spins++;
                        __nanosleep(32);
                        x = os_ld(status + (j - k) * 256 + d);
                    }
                    if (spins > spin_limit) {
                        bad = true;
                    } else {
                        acc += (unsigned)x;
                        if ((x >> 62) == 2) done = true;
                    }
                }
            }
        }
        if (bad) set_err(ct, GPUDT_ERR_NOCONVERGE, 98);
        os_st(mine, kOsInc | pass_tag | (unsigned)(acc + tot));
    }
    S.gbase[d] += (int)acc;
    __syncthreads();
    const int cnt = (int)min((long long)kRsTile, (long long)n - tile0);
    for (int p = threadIdx.x; p < cnt; p += kRsThreads) {
        K k = S.key[p];
        int dd = (int)((k >> shift) & 255);
        long long g = (long long)S.gbase[dd] + (p - S.lstart[dd]);
        if (g < n) {  // always, unless a look-back gave up (error 98 is set then)
            kout[g] = k;
            vout[g] = S.val[p];
        }
    }
}

// Scratch ints of the single-pass sort of n keys.
static long long onesweep_scratch_ints(long long n)
{
    return kOsHeadInts + 512 * ((n + kRsTile - 1) / kRsTile);
}

long long radix_sort_scratch_ints(long long n)
{
    return std::max(radix_scratch_ints(n), onesweep_scratch_ints(n));
}

// The kOsPasses passes; the result ends in (keys, vals) after an even number
// of passes, in (keys2, vals2) after an odd one.
static int onesweep_top(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *keys2, int *vals2, int n)
{
    typedef unsigned long long K;
    const int smem = (int)sizeof(RsSmem<K>);
    {
        static std::mutex mu;
        static bool attr_set[64];
        std::lock_guard<std::mutex> lk(mu);
        if (c.device < 0 || c.device >= 64 || !attr_set[c.device]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_onesweep, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             cudaSharedmemCarveoutMaxShared));
            if (c.device >= 0 && c.device < 64) attr_set[c.device] = true;
        }
    }
    const long long tiles = ((long long)n + kRsTile - 1) / kRsTile;
    int *ghist = c.rhist, *tickets = c.rhist + kOsTicketOff;
    unsigned long long *status = reinterpret_cast<unsigned long long *>(c.rhist + kOsHeadInts);
    GALPHA_CUDA(cudaMemsetAsync(ghist, 0, sizeof(int) * (kOsTicketOff + 8), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned long long) * 256 * (size_t)tiles, c.stream));
    {
        const long long blocks = std::max(1ll, std::min<long long>((n + 1023) / 1024, (long long)c.sm_count * 8));
        k_rs_hist_top<<<(unsigned)blocks, 256, 0, c.stream>>>(keys, n, ghist);
        count_launch();
    }
    K *ki = keys, *ko = keys2;
    int *vi = vals, *vo = vals2;
    for (int p = 0; p < kOsPasses; p++) {
        c.sort_passes++;
        k_rs_onesweep<<<(unsigned)tiles, kRsThreads, smem, c.stream>>>(ki, vi, ko, vo, n, kLowBits + 8 * p,
                                                                      ghist + 256 * p, status, tickets + p,
                                                                      (unsigned long long)(p + 1) << 32, c.ctr,
                                                                      c.spin_limit, c.hold_first);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    return GPUDT_OK;
}

// The result is left in (keys, vals) or, when *in_second comes back true, in
// (keys2, vals2): where the last digit pass left it, since a copy back would
// cost a full read and write of both arrays.
int radix_sort(Ctx &c, unsigned long long *keys, int *vals, unsigned long long *keys2, int *vals2, int n,
               bool *in_second)
{
    bool sec = false;
    int r;
    if (n > 1 && n < (1 << 30) && onesweep_scratch_ints(n) <= c.rhist_ints) {
        r = onesweep_top(c, keys, vals, keys2, vals2, n);
        sec = (kOsPasses & 1) != 0;  // the passes alternate between the two buffer pairs
    } else {
        r = radix_sort_keys<unsigned long long>(c, keys, vals, keys2, vals2, n, c.rhist, kLowBits, &sec);
    }
    *in_second = sec;
    if (r || n <= 1) return r;
    unsigned long long *rk = sec ? keys2 : keys, *fk = sec ? keys : keys2;
    int *rv = sec ? vals2 : vals, *fv = sec ? vals : vals2;
    // group fix-up in the other key buffer (2n ints, free now): group starts
    // (at most n / 2), then the long pairs and their extents (3 ints each)
    int *starts = (int *)fk;
    const long long soff = ((long long)n / 2 + 2) & ~1ll;
    const int lcap = (int)(std::min<long long>(kMaxLongPairs, (2ll * n - soff) / 3) & ~1ll);
    int *longs = starts + soff;
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlist2, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->nlong, 0, sizeof(int), c.stream));
    GALPHA_CUDA(cudaMemsetAsync(&c.ctr->changed, 0, sizeof(int), c.stream));
    {
        const long long blocks = std::max(1ll, std::min<long long>(((long long)n / 8 + 255) / 256, (long long)c.sm_count * 8));
        k_fix_find<<<(unsigned)blocks, 256, 0, c.stream>>>(rk, starts, longs, n, std::max(lcap, 0), c.ctr);
        count_launch();
    }
    r = read_counters(c);
    if (r) return r;
    if (c.hctr->err) return stage_fail(c, c.hctr->err, "spectrum sort");
    const int nlong = std::min(c.hctr->nlong, std::max(lcap, 0));
    std::vector<int2> groups;
    if (!c.hctr->changed && nlong > 0) {
        // extents of the long groups, merged on the host
        int2 *ext = reinterpret_cast<int2 *>(longs + lcap);
        k_group_extent<<<(unsigned)nlong, 256, 0, c.stream>>>(rk, n, longs, ext);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        std::vector<int2> h(nlong);
        r = read_small(c, h.data(), ext, sizeof(int2) * (size_t)nlong);
        if (r) return r;
        std::sort(h.begin(), h.end(), [](int2 a, int2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
        for (const int2 &g : h)
            if (groups.empty() || g.x != groups.back().x) groups.push_back(g);
    }
    if (c.hctr->changed || groups.size() > (size_t)kMaxLongGroups) {
        bool sec2 = false;
        r = radix_sort_keys<unsigned long long>(c, rk, rv, fk, fv, n, c.rhist, 0, &sec2);
        if (sec2) *in_second = !sec;
        return r;
    }
    if (c.hctr->nlist2 > 0) launch_n(c, FixGroups{rk, rv, starts, n}, c.hctr->nlist2);
    GALPHA_CUDA(cudaGetLastError());
    // each long group as a sub-array (the other buffers are free now)
    for (const int2 &g : groups) {
        const int len = g.y - g.x;
        bool sec2 = false;
        r = radix_sort_keys<unsigned long long>(c, rk + g.x, rv + g.x, fk, fv, len, c.rhist, 0, &sec2);
        if (r) return r;
        if (sec2) {
            launch_n(c, CopyElems<unsigned long long>{rk + g.x, fk}, len);
            launch_n(c, CopyElems<int>{rv + g.x, fv}, len);
        }
    }
    GALPHA_CUDA(cudaGetLastError());
    return GPUDT_OK;
}

int radix_sort32(Ctx &c, unsigned int *keys, int *vals, unsigned int *keys2, int *vals2, int n, int *scratch,
                 int key_bits)
{
    return radix_sort_keys<unsigned int>(c, keys, vals, keys2, vals2, n, scratch, 0, nullptr, key_bits);
}

}  // namespace galpha

namespace galpha {

// ------------------------------------- set-key sort with a (key, value) payload
// Stable LSD sort of 32-bit set ids that moves each entry's 64-bit key and int
// value with it: the batched alpha stage turns its value-sorted entries into
// (set, value) order in ceil(bits / 8) passes of coalesced reads and run-wise
// writes, instead of sorting positions and gathering the entries afterwards.
struct RsKvSmem {
    unsigned key[kRsTile];
    unsigned long long pk[kRsTile];
    int pv[kRsTile];
    int wcnt[kRsWarps][256];
    int lstart[256];
    int gbase[256];
};

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter_kv(const unsigned *__restrict__ kin,
                                                              const unsigned long long *__restrict__ pkin,
                                                              const int *__restrict__ pvin, unsigned *__restrict__ kout,
                                                              unsigned long long *__restrict__ pkout,
                                                              int *__restrict__ pvout, int n, int shift,
                                                              const int *__restrict__ hoff, int nblocks)
{
    extern __shared__ __align__(16) unsigned char rs_smem_kv[];
    RsKvSmem &S = *reinterpret_cast<RsKvSmem *>(rs_smem_kv);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = lane; d < 256; d += 32) S.wcnt[w][d] = 0;
    S.gbase[threadIdx.x] = hoff[threadIdx.x * nblocks + blockIdx.x];
    __syncwarp();
    const long long tile0 = (long long)blockIdx.x * kRsTile;
    const long long base = tile0 + (long long)w * (kRsItems * 32);
    unsigned key[kRsItems];
    unsigned long long pk[kRsItems];
    int pv[kRsItems], rk[kRsItems];
    const unsigned lanemask_lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        const long long i = base + r * 32 + lane;
        const bool ok = i < n;
        key[r] = ok ? kin[i] : 0u;
        pk[r] = ok ? pkin[i] : 0ull;
        pv[r] = ok ? pvin[i] : 0;
    }
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
    {
        const int d = threadIdx.x;
        int s = 0;
        for (int q = 0; q < kRsWarps; q++) {
            const int c = S.wcnt[q][d];
            S.wcnt[q][d] = s;
            s += c;
        }
        S.lstart[d] = s;
    }
    __syncthreads();
    if (w == 0) {
        int carry = 0;
        for (int d0 = 0; d0 < 256; d0 += 32) {
            const int v = S.lstart[d0 + lane];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            S.lstart[d0 + lane] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsItems; r++) {
        const long long i = base + r * 32 + lane;
        if (i < n) {
            const int dg = (int)((key[r] >> shift) & 255);
            const int p = S.lstart[dg] + S.wcnt[w][dg] + rk[r];
            S.key[p] = key[r];
            S.pk[p] = pk[r];
            S.pv[p] = pv[r];
        }
    }
    __syncthreads();
    const int cnt = (int)min((long long)kRsTile, (long long)n - tile0);
    for (int p = threadIdx.x; p < cnt; p += kRsThreads) {
        const unsigned k = S.key[p];
        const int d = (int)((k >> shift) & 255);
        const long long g = (long long)S.gbase[d] + (p - S.lstart[d]);
        kout[g] = k;
        pkout[g] = S.pk[p];
        pvout[g] = S.pv[p];
    }
}

int radix_sort_set_kv(Ctx &c, unsigned *skey, unsigned *skey2, unsigned long long *keys, int *vals,
                      unsigned long long *keys2, int *vals2, int n, int nbits)
{
    if (n <= 1 || nbits <= 0) return GPUDT_OK;
    const int smem = (int)sizeof(RsKvSmem);
    {
        static std::mutex mu;
        static bool attr_set[64];
        std::lock_guard<std::mutex> lk(mu);
        if (c.device < 0 || c.device >= 64 || !attr_set[c.device]) {
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_scatter_kv, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            GALPHA_CUDA(cudaFuncSetAttribute(k_rs_scatter_kv, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             cudaSharedmemCarveoutMaxShared));
            if (c.device >= 0 && c.device < 64) attr_set[c.device] = true;
        }
    }
    const int nblocks = (n + kRsTile - 1) / kRsTile;
    int *hist = c.rhist + 8;
    unsigned *ki = skey, *ko = skey2;
    unsigned long long *pki = keys, *pko = keys2;
    int *pvi = vals, *pvo = vals2;
    for (int shift = 0; shift < nbits; shift += 8) {
        c.sort_passes++;
        k_rs_hist<unsigned><<<nblocks, kRsThreads, 0, c.stream>>>(ki, n, shift, hist, nblocks);
        count_launch();
        int r = exclusive_scan_int(c, hist, hist, 256 * nblocks, nullptr);
        if (r) return r;
        k_rs_scatter_kv<<<nblocks, kRsThreads, smem, c.stream>>>(ki, pki, pvi, ko, pko, pvo, n, shift, hist, nblocks);
        count_launch();
        GALPHA_CUDA(cudaGetLastError());
        std::swap(ki, ko);
        std::swap(pki, pko);
        std::swap(pvi, pvo);
    }
    if (pki != keys) {  // an odd number of passes: the result is in the second buffers
        launch_n(c, CopyElems<unsigned long long>{keys, pki}, n);
        launch_n(c, CopyElems<int>{vals, pvi}, n);
        launch_n(c, CopyElems<unsigned>{skey, ki}, n);
    }
    return GPUDT_OK;
}

}  // namespace galpha
