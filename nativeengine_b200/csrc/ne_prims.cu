// ne_prims.cu -- device-wide exclusive scan and stable LSD radix sort.
//
// Both are HBM-streaming primitives written for deterministic output: the scan
// is a single-pass tile scan with chained tile prefixes, and the sort ranks elements inside each 256-item
// warp sub-tile with __match_any_sync in element order, so equal keys keep
// their input order (stability is what keeps bodies in a cell, and contacts in
// an island, in the reference's index order).
//
// Both take a host-side capacity n (launch size) and an optional device-side
// count n_dev: only the first min(n, *n_dev) elements are scanned or sorted,
// so a buffer sized for the worst case costs only what the step filled.
#include <cuda/atomic>

#include "ne_internal.cuh"

namespace neb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;   // 2048

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

// Single-pass exclusive scan: tiles take numbers from a ticket in the order
// they start, publish their sum, then walk back over earlier tiles' published
// sums to the first one that carries its inclusive prefix (chained tile
// prefixes).  A tile only waits on tiles that started before it, so every wait
// ends; it is still bounded in time, and reports through ctl->solve_timeout.
// The last tile to finish clears the tile states and counters for the next
// scan (scans on one stream never overlap).
//   tstat[0, ntiles): (flag << 62) | value, flag 1 = tile sum, 2 = inclusive
//   prefix; the two u32 words after them: ticket and finished count.
constexpr unsigned long long kTileSum = 1ull << 62, kTilePrefix = 2ull << 62, kTileVal = (1ull << 62) - 1;
constexpr unsigned long long kLookbackNs = 2000000000ull;

__device__ __forceinline__ unsigned long long scan_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_1pass(const uint32_t* in, uint32_t* out, uint32_t ncap,
                                                             unsigned long long* __restrict__ tstat,
                                                             uint32_t ntiles_cap, uint64_t* __restrict__ total,
                                                             const Ctl* __restrict__ ctl,
                                                             const uint64_t* __restrict__ n_dev) {
    if (ctl->abort) return;
    __shared__ uint32_t sm[33];
    __shared__ uint32_t s_tile, s_last;
    __shared__ unsigned long long s_prefix;
    uint32_t* ctr = reinterpret_cast<uint32_t*>(tstat + ntiles_cap);
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr[0], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t n = live_count(ncap, n_dev);
    const uint32_t live = (uint32_t)(((uint64_t)n + kScanTile - 1) / kScanTile);
    using Word = cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>;
    if (tile < live) {
        const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
        uint32_t x[kScanItems];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            x[k] = (base + k < n) ? in[base + k] : 0u;
            sum += x[k];
        }
        uint32_t excl;
        const uint32_t tot = block_excl_scan<kScanThreads>(sum, excl, sm);
        if (threadIdx.x == 0) {
            unsigned long long prefix = 0;
            if (tile == 0) {
                Word(tstat[0]).store(kTilePrefix | tot, cuda::memory_order_relaxed);
            } else {
                Word(tstat[tile]).store(kTileSum | tot, cuda::memory_order_relaxed);
                const unsigned long long t0 = scan_ns();
                uint32_t spins = 0;
                for (int64_t q = (int64_t)tile - 1; q >= 0;) {
                    const unsigned long long v = Word(tstat[q]).load(cuda::memory_order_relaxed);
                    const unsigned long long f = v & ~kTileVal;
                    if (f == 0ull) {
                        if ((++spins & 255u) == 0u && scan_ns() - t0 > kLookbackNs) {
                            atomicExch(const_cast<uint32_t*>(&ctl->solve_timeout), 1u);
                            break;
                        }
                        continue;
                    }
                    prefix += v & kTileVal;
                    if (f == kTilePrefix) break;
                    --q;
                }
                Word(tstat[tile]).store(kTilePrefix | (prefix + tot), cuda::memory_order_relaxed);
            }
            s_prefix = prefix;
            if (tile == live - 1) *total = prefix + tot;
        }
        __syncthreads();
        excl += (uint32_t)s_prefix;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < n) out[base + k] = excl;
            excl += x[k];
        }
    } else if (n == 0 && tile == 0 && threadIdx.x == 0) {
        *total = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&ctr[1], 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last) {
        for (uint32_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) tstat[k] = 0ull;
        if (threadIdx.x == 0) { ctr[0] = 0u; ctr[1] = 0u; }
        __threadfence();
    }
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

// u32 words of scan state: one u64 per tile, then the two counters.
size_t scan_tsum_words(uint32_t n) { return 2 * ((size_t)ceil_div(n ? n : 1, kScanTile) + 2); }
size_t radix_hist_words(uint32_t n) { return (size_t)256 * ceil_div(n, kSub) + 1; }

void scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tsum, uint64_t* total, const Ctl* ctl,
              cudaStream_t st, uint64_t* launches, const uint64_t* n_dev) {
    if (n == 0) return;
    const uint32_t ntiles = ceil_div(n, kScanTile);
    k_scan_1pass<<<ntiles, kScanThreads, 0, st>>>(in, out, n, reinterpret_cast<unsigned long long*>(tsum), ntiles,
                                                  total, ctl, n_dev);
    ++*launches;
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
