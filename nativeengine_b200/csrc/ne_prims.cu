// ne_prims.cu -- device-wide exclusive scan and stable LSD radix sort.
//
// Both are HBM-streaming primitives written for deterministic output: the scan
// is a three-phase tile scan, and the sort ranks elements inside each 256-item
// warp sub-tile with __match_any_sync in element order, so equal keys keep
// their input order (stability is what keeps bodies in a cell, and contacts in
// an island, in the reference's index order).
//
// Both take a host-side capacity n (launch size) and an optional device-side
// count n_dev: only the first min(n, *n_dev) elements are scanned or sorted,
// so a buffer sized for the worst case costs only what the step filled.
#include "ne_internal.cuh"

namespace neb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;   // 2048
constexpr int kTopThreads = 1024;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t& excl, uint32_t* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) sm[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < NT / 32) ? sm[lane] : 0u;
        uint32_t wi = warp_incl_scan(w);
        if (lane < NT / 32) sm[lane] = wi - w;
        if (lane == NT / 32 - 1) sm[32] = wi;
    }
    __syncthreads();
    excl = inc - v + sm[warp];
    uint32_t total = sm[32];
    __syncthreads();
    return total;
}

__device__ __forceinline__ uint32_t live_count(uint32_t n, const uint64_t* n_dev) {
    if (!n_dev) return n;
    const uint64_t v = *n_dev;
    return v < (uint64_t)n ? (uint32_t)v : n;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in,
                                                             uint32_t* __restrict__ out, uint32_t ncap,
                                                             uint32_t* __restrict__ tsum,
                                                             const Ctl* __restrict__ ctl,
                                                             const uint64_t* __restrict__ n_dev) {
    if (ctl->abort) return;
    __shared__ uint32_t sm[33];
    const uint32_t n = live_count(ncap, n_dev);
    if ((uint64_t)blockIdx.x * kScanTile >= n) {
        if (threadIdx.x == 0) tsum[blockIdx.x] = 0u;
        return;
    }
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t x[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        x[k] = (base + k < n) ? in[base + k] : 0u;
        s += x[k];
    }
    uint32_t excl;
    uint32_t total = block_excl_scan<kScanThreads>(s, excl, sm);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = excl;
        excl += x[k];
    }
    if (threadIdx.x == 0) tsum[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile sums, u64 grand total.
__global__ void __launch_bounds__(kTopThreads) k_scan_top(uint32_t* __restrict__ tsum, uint32_t ntiles,
                                                          uint64_t* __restrict__ total,
                                                          const Ctl* __restrict__ ctl) {
    if (ctl->abort) return;
    __shared__ uint32_t sm[33];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0ull;
    __syncthreads();
    for (uint32_t base = 0; base < ntiles; base += kTopThreads) {
        const uint32_t idx = base + threadIdx.x;
        uint32_t v = (idx < ntiles) ? tsum[idx] : 0u;
        uint32_t excl;
        uint32_t t = block_excl_scan<kTopThreads>(v, excl, sm);
        if (idx < ntiles) tsum[idx] = (uint32_t)(carry + excl);
        __syncthreads();
        if (threadIdx.x == 0) carry += t;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t ncap, const uint32_t* __restrict__ tsum,
                           const Ctl* __restrict__ ctl, const uint64_t* __restrict__ n_dev) {
    if (ctl->abort) return;
    const uint32_t n = live_count(ncap, n_dev);
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tsum[i / kScanTile];
}

// ---- radix sort ---------------------------------------------------------

constexpr int kSortWarps = 8;
constexpr int kSub = 256;      // elements per warp sub-tile (8 chunks of 32)

template <typename K>
__device__ __forceinline__ int digit_of(K k, int shift) {
    return (int)((k >> shift) & (K)0xFF);
}

// Digit histogram per 256-element sub-tile, laid out [digit][sub-tile] over
// the live sub-tiles; block 0 publishes that layout's length for the scan.
template <typename K>
__global__ void __launch_bounds__(kSortWarps * 32) k_radix_hist(const K* __restrict__ keys, uint32_t ncap,
                                                                int shift, uint32_t* __restrict__ hist,
                                                                const Ctl* __restrict__ ctl,
                                                                const uint64_t* __restrict__ n_dev,
                                                                uint64_t* __restrict__ hist_len) {
    if (ctl->abort) return;
    __shared__ uint32_t cnt[kSortWarps][256];
    const uint32_t n = live_count(ncap, n_dev);
    const uint32_t nsub = (n + kSub - 1) / kSub;
    if (blockIdx.x == 0 && threadIdx.x == 0) *hist_len = 256ull * nsub;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t g = blockIdx.x * kSortWarps + w;
    if (blockIdx.x * kSortWarps >= nsub) return;
    for (int d = lane; d < 256; d += 32) cnt[w][d] = 0u;
    __syncwarp();
    if (g < nsub) {
        for (int ch = 0; ch < kSub / 32; ++ch) {
            const uint64_t e = (uint64_t)g * kSub + ch * 32 + lane;
            const int d = (e < n) ? digit_of(keys[e], shift) : 256 + lane;
            const uint32_t m = __match_any_sync(0xffffffffu, d);
            if (d < 256 && lane == __ffs(m) - 1) cnt[w][d] += __popc(m);
            __syncwarp();
        }
        for (int d = lane; d < 256; d += 32) hist[(uint64_t)d * nsub + g] = cnt[w][d];
    }
}

template <typename K>
__global__ void __launch_bounds__(kSortWarps * 32) k_radix_scatter(const K* __restrict__ kin,
                                                                   const uint32_t* __restrict__ vin,
                                                                   K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                                   uint32_t ncap, int shift,
                                                                   const uint32_t* __restrict__ hist,
                                                                   const Ctl* __restrict__ ctl,
                                                                   const uint64_t* __restrict__ n_dev) {
    if (ctl->abort) return;
    __shared__ uint32_t cnt[kSortWarps][256];
    const uint32_t n = live_count(ncap, n_dev);
    const uint32_t nsub = (n + kSub - 1) / kSub;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t g = blockIdx.x * kSortWarps + w;
    if (g >= nsub) return;
    for (int d = lane; d < 256; d += 32) cnt[w][d] = hist[(uint64_t)d * nsub + g];
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    for (int ch = 0; ch < kSub / 32; ++ch) {
        const uint64_t e = (uint64_t)g * kSub + ch * 32 + lane;
        K k = 0;
        uint32_t v = 0;
        int d = 256 + lane;
        if (e < n) { k = kin[e]; v = vin[e]; d = digit_of(k, shift); }
        const uint32_t m = __match_any_sync(0xffffffffu, d);
        if (d < 256) {
            const uint32_t pos = cnt[w][d] + __popc(m & lt);
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncwarp();
        if (d < 256 && lane == __ffs(m) - 1) cnt[w][d] += __popc(m);
        __syncwarp();
    }
}

inline uint32_t ceil_div(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

template <typename K>
int radix_sort_impl(K* key[2], uint32_t* val[2], uint32_t n, int bits, uint32_t* hist, uint32_t* tsum,
                    const Ctl* ctl, cudaStream_t st, uint64_t* launches, const uint64_t* n_dev) {
    int cur = 0;
    if (n <= 1 || bits <= 0) return cur;
    const uint32_t nsub = ceil_div(n, kSub);
    const uint32_t nblk = ceil_div(nsub, kSortWarps);
    const uint32_t hn = 256u * nsub;
    uint64_t* total = const_cast<uint64_t*>(&ctl->scan_total);
    uint64_t* hlen = const_cast<uint64_t*>(&ctl->sort_hist_len);
    for (int shift = 0; shift < bits; shift += 8) {
        k_radix_hist<K><<<nblk, kSortWarps * 32, 0, st>>>(key[cur], n, shift, hist, ctl, n_dev, hlen);
        ++*launches;
        scan_u32(hist, hist, hn, tsum, total, ctl, st, launches, hlen);
        k_radix_scatter<K><<<nblk, kSortWarps * 32, 0, st>>>(key[cur], val[cur], key[cur ^ 1], val[cur ^ 1], n,
                                                              shift, hist, ctl, n_dev);
        ++*launches;
        cur ^= 1;
    }
    return cur;
}

}  // namespace

size_t scan_tsum_words(uint32_t n) { return (size_t)ceil_div(n, kScanTile) + 1; }
size_t radix_hist_words(uint32_t n) { return (size_t)256 * ceil_div(n, kSub) + 1; }

void scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tsum, uint64_t* total, const Ctl* ctl,
              cudaStream_t st, uint64_t* launches, const uint64_t* n_dev) {
    if (n == 0) return;
    const uint32_t ntiles = ceil_div(n, kScanTile);
    k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(in, out, n, tsum, ctl, n_dev);
    k_scan_top<<<1, kTopThreads, 0, st>>>(tsum, ntiles, total, ctl);
    *launches += 2;
    if (ntiles > 1) {
        k_scan_add<<<ceil_div(n, 256), 256, 0, st>>>(out, n, tsum, ctl, n_dev);
        ++*launches;
    }
}

int radix_sort_u64(unsigned long long* key[2], uint32_t* val[2], uint32_t n, int bits, uint32_t* hist,
                   uint32_t* tsum, const Ctl* ctl, cudaStream_t st, uint64_t* launches, const uint64_t* n_dev) {
    return radix_sort_impl<unsigned long long>(key, val, n, bits, hist, tsum, ctl, st, launches, n_dev);
}

int radix_sort_u32(uint32_t* key[2], uint32_t* val[2], uint32_t n, int bits, uint32_t* hist, uint32_t* tsum,
                   const Ctl* ctl, cudaStream_t st, uint64_t* launches, const uint64_t* n_dev) {
    return radix_sort_impl<uint32_t>(key, val, n, bits, hist, tsum, ctl, st, launches, n_dev);
}

}  // namespace neb
