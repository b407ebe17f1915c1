// ne_noalloc.cu -- a broadphase entry point that allocates no memory.
//
// ne_broadphase_pairs_noalloc computes the same sorted, unique candidate pair
// list as the world step's broadphase (ne_world_pairs), for one body set, but
// without cudaMalloc: its working memory is one file-scope device array that
// the library reserves when it is loaded.  It exists for callers that cannot
// allocate device memory at the point of the call -- code running under a
// fixed memory budget handed out by an embedding engine's own allocator, code
// in a real-time loop where an allocation (and the implicit synchronisation it
// can bring) is not allowed, or tools that probe the pair list of a scene
// without owning a world.
//
// Limits: at most NE_NOALLOC_MAX_BODIES bodies and NE_NOALLOC_MAX_PAIRS
// pairs.  The scratch array is shared by every call in the process on a given
// GPU and keeps the previous call's contents; every value a call reads is
// written by that same call first.  Calls that overlap on the GPU (from
// several host threads at once) race on the array and must be serialised by
// the caller.  The first call on each device looks up the array's device
// address with that device current; make that first call before any stream
// capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ne_cuda.h"
#include "ne_geom.cuh"

namespace neb {
void set_last_error(const std::string& msg);   // defined in ne_capi.cu
}

namespace {

constexpr uint32_t kMaxBodies = NE_NOALLOC_MAX_BODIES;
constexpr uint32_t kMaxPairs = NE_NOALLOC_MAX_PAIRS;
constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;

// Byte layout of the scratch array.
constexpr size_t kOffPos = 0;                                       // double[3*kMaxBodies]
constexpr size_t kOffExcl = kOffPos + sizeof(double) * 3 * kMaxBodies;   // uint32_t[kMaxBodies]
constexpr size_t kOffTotal = kOffExcl + sizeof(uint32_t) * kMaxBodies;   // uint32_t total
constexpr size_t kOffPairI = 65536;                                 // uint32_t[kMaxPairs]
constexpr size_t kOffPairJ = kOffPairI + sizeof(uint32_t) * kMaxPairs;
constexpr size_t kScratchBytes = kOffPairJ + sizeof(uint32_t) * kMaxPairs;
static_assert(kOffTotal + 256 <= kOffPairI, "scratch layout overlaps");

// The whole working set of the entry point (about 2.06 MiB per GPU).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct GridParams {
    uint32_t n;
    int brute, periodic;
    double half, cell;
    long long nc[3];
};

__device__ __forceinline__ long long na_cell(const GridParams& g, double c, int axis) {
    if (g.periodic) {
        long long k = (long long)floor((c + g.half) / g.cell);
        long long m = g.nc[axis];
        return ((k % m) + m) % m;
    }
    return (long long)floor(c / g.cell);
}

__device__ __forceinline__ unsigned long long na_key(long long x, long long y, long long z) {
    return (unsigned long long)(x & 0x1FFFFF) | ((unsigned long long)(y & 0x1FFFFF) << 21) |
           ((unsigned long long)(z & 0x1FFFFF) << 42);
}

__device__ __forceinline__ long long na_wrap(const GridParams& g, long long c, int axis) {
    if (!g.periodic) return c;
    const long long m = g.nc[axis];
    return ((c % m) + m) % m;
}

// One CTA.  Body j > i is a partner of i when either body is grid-excluded
// (planes pair with everyone), when the grid is bypassed (brute force), or
// when j's cell key is one of the 27 neighbour keys of i's cell -- the pair
// set World::broadphasePairs() builds from both sides and de-duplicates.
// Rows are scanned in j order, so each row comes out sorted.
__global__ void __launch_bounds__(kThreads) k_pairs_noalloc(unsigned char* scratch, GridParams g) {
    const double* pos = reinterpret_cast<const double*>(scratch + kOffPos);
    const uint32_t* excl = reinterpret_cast<const uint32_t*>(scratch + kOffExcl);
    uint32_t* total_out = reinterpret_cast<uint32_t*>(scratch + kOffTotal);
    uint32_t* pi = reinterpret_cast<uint32_t*>(scratch + kOffPairI);
    uint32_t* pj = reinterpret_cast<uint32_t*>(scratch + kOffPairJ);

    __shared__ unsigned long long s_key[kMaxBodies];
    __shared__ unsigned char s_excl[kMaxBodies];
    __shared__ uint32_t s_off[kMaxBodies + 1];
    __shared__ unsigned long long s_nk[kWarps][27];
    __shared__ uint32_t s_wsum[kWarps];

    const uint32_t n = g.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t t = threadIdx.x; t < n; t += kThreads) {
        s_excl[t] = excl[t] ? 1 : 0;
        s_key[t] = (g.brute || excl[t])
                       ? ~0ull
                       : na_key(na_cell(g, pos[3 * t], 0), na_cell(g, pos[3 * t + 1], 1), na_cell(g, pos[3 * t + 2], 2));
    }
    __syncthreads();

    // Pass 0 counts each row's partners into s_off; pass 1 writes them.
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = warp; i < n; i += kWarps) {
            const bool all = g.brute || s_excl[i];
            if (!all && lane < 27) {
                const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
                const double* p = pos + 3 * i;
                s_nk[warp][lane] = na_key(na_wrap(g, na_cell(g, p[0], 0) + dx, 0),
                                          na_wrap(g, na_cell(g, p[1], 1) + dy, 1),
                                          na_wrap(g, na_cell(g, p[2], 2) + dz, 2));
            }
            __syncwarp();
            uint32_t cnt = 0;
            const uint32_t base = pass ? s_off[i] : 0u;
            for (uint32_t j0 = i + 1; j0 < n; j0 += 32) {
                const uint32_t j = j0 + lane;
                bool hit = false;
                if (j < n) {
                    if (all || s_excl[j]) {
                        hit = true;
                    } else {
                        const unsigned long long kj = s_key[j];
                        for (int q = 0; q < 27; ++q) hit |= (s_nk[warp][q] == kj);
                    }
                }
                const uint32_t b = __ballot_sync(0xffffffffu, hit);
                if (pass && hit) {
                    const uint32_t slot = base + cnt + __popc(b & ((1u << lane) - 1u));
                    if (slot < kMaxPairs) {
                        pi[slot] = i;
                        pj[slot] = j;
                    }
                }
                cnt += __popc(b);
            }
            if (!pass && lane == 0) s_off[i] = cnt;
            __syncwarp();
        }
        __syncthreads();
        if (!pass) {
            // Exclusive scan of the row counts (n <= 2048, two per thread).
            const uint32_t a0 = 2 * threadIdx.x, a1 = a0 + 1;
            const uint32_t v0 = a0 < n ? s_off[a0] : 0u, v1 = a1 < n ? s_off[a1] : 0u;
            uint32_t incl = v0 + v1;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane == 31) s_wsum[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                uint32_t w = s_wsum[lane];
                uint32_t wi = w;
                for (int o = 1; o < 32; o <<= 1) {
                    uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                    if (lane >= o) wi += t;
                }
                s_wsum[lane] = wi - w;
                if (lane == 31) s_off[kMaxBodies] = wi;
            }
            __syncthreads();
            const uint32_t ex = incl - (v0 + v1) + s_wsum[warp];
            if (a0 < n) s_off[a0] = ex;
            if (a1 < n) s_off[a1] = ex + v0;
            __syncthreads();
            if (threadIdx.x == 0) *total_out = s_off[kMaxBodies];
            if (s_off[kMaxBodies] > kMaxPairs) return;   // uniform: the host reports the overflow
        }
    }
}

std::mutex g_setup_mutex;
void* g_scratch_ptr[64] = {};

int na_err(int code, const std::string& msg) {
    neb::set_last_error(msg);   // readable through ne_last_error()
    return code;
}

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
int scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_err(NE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return na_err(NE_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return na_err(NE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return NE_OK;
}

}  // namespace

extern "C" {

int ne_broadphase_pairs_noalloc(const NeWorldParams* params, const NeBodyArrays* b, uint32_t* pair_i,
                                uint32_t* pair_j, uint64_t cap, uint64_t* count) {
    if (!params || !b || !count) return na_err(NE_ERR_ARG, "NULL argument");
    *count = 0;
    const uint32_t n = b->n;
    if (n > kMaxBodies)
        return na_err(NE_ERR_CAPACITY, "ne_broadphase_pairs_noalloc: more than NE_NOALLOC_MAX_BODIES (" +
                                           std::to_string(kMaxBodies) + ") bodies");
    if (n == 0) return NE_OK;
    if (!b->x || !b->shape || !b->radius || !b->half_height || !b->half_extents)
        return na_err(NE_ERR_ARG, "a required body array is NULL");
    if (cap && (!pair_i || !pair_j)) return na_err(NE_ERR_ARG, "output arrays are NULL");

    // Grid constants of World::broadphasePairs() (src/world.cpp:427-457),
    // from the bodies' bounding radii (src/body.hpp:137-158).
    double maxR = 0.0;
    std::vector<double> xs(3 * (size_t)n);
    std::vector<uint32_t> excl(n);
    for (uint32_t i = 0; i < n; ++i) {
        const int s = b->shape[i];
        if (s < 0 || s > NE_SHAPE_COMPOUND) return na_err(NE_ERR_ARG, "shape tag out of range");
        if (s == NE_SHAPE_COMPOUND) return na_err(NE_ERR_UNSUPPORTED, "compound bodies are not supported");
        for (int k = 0; k < 3; ++k) xs[3 * i + k] = b->x[3 * i + k];
        excl[i] = (s == NE_SHAPE_PLANE || s == NE_SHAPE_MESH) ? 1u : 0u;
        if (excl[i]) continue;
        std::vector<neb::D4> vv;
        if (s == NE_SHAPE_CONVEX) {
            if (!b->verts || !b->vert_offset || !b->vert_count) return na_err(NE_ERR_ARG, "convex body without vertices");
            for (uint32_t k = 0; k < b->vert_count[i]; ++k) {
                const double* v = b->verts + 3 * ((size_t)b->vert_offset[i] + k);
                vv.push_back(neb::D4{v[0], v[1], v[2], 0.0});
            }
        }
        const neb::V3 he = neb::mk(b->half_extents[3 * i], b->half_extents[3 * i + 1], b->half_extents[3 * i + 2]);
        const double r = neb::bounding_radius(s, b->radius[i], b->half_height[i], he, vv.data(), (int)vv.size());
        maxR = (maxR < r) ? r : maxR;
    }
    GridParams g;
    g.n = n;
    g.half = params->half;
    g.periodic = params->periodic ? 1 : 0;
    g.cell = 2.0 * maxR;
    g.brute = (params->force_brute_force || n < 64 || g.cell < 1e-9) ? 1 : 0;
    g.nc[0] = g.nc[1] = g.nc[2] = 1;
    if (g.periodic && !g.brute) {
        const double L = 2.0 * params->half;
        for (int a = 0; a < 3; ++a) {
            long long m = (long long)(int)std::floor(L / g.cell);
            g.nc[a] = m < 1 ? 1 : m;
        }
    }

    unsigned char* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    const cudaStream_t st = cudaStreamPerThread;
    cudaError_t e = cudaMemcpyAsync(scratch + kOffPos, xs.data(), xs.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scratch + kOffExcl, excl.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return na_err(NE_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    k_pairs_noalloc<<<1, kThreads, 0, st>>>(scratch, g);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_err(NE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    uint32_t total = 0;
    e = cudaMemcpyAsync(&total, scratch + kOffTotal, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_err(NE_ERR_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
    *count = total;
    if (total > kMaxPairs)
        return na_err(NE_ERR_CAPACITY, "ne_broadphase_pairs_noalloc: more than NE_NOALLOC_MAX_PAIRS (" +
                                           std::to_string(kMaxPairs) + ") pairs");
    const uint64_t m = total < cap ? total : cap;
    if (m) {
        e = cudaMemcpyAsync(pair_i, scratch + kOffPairI, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(pair_j, scratch + kOffPairJ, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return na_err(NE_ERR_CUDA, std::string("download: ") + cudaGetErrorString(e));
    }
    return NE_OK;
}

}  // extern "C"
