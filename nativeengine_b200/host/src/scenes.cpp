// scenes.cpp -- exact-overlap random sequential placement (see ne/scenes.h).
#include "ne/scenes.h"

#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "ne_geom.cuh"

namespace {

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

uint64_t cell_hash(long x, long y, long z) {
    return ((uint64_t)(x & 0x1FFFFF)) | ((uint64_t)(y & 0x1FFFFF) << 21) | ((uint64_t)(z & 0x1FFFFF) << 42);
}

}  // namespace

extern "C" uint32_t ne_scene_place_periodic(uint32_t n, const int32_t* shape, const double* radius,
                                            const double* half_height, const double* half_extents, const double* q,
                                            const uint32_t* vert_offset, const uint32_t* vert_count,
                                            const double* verts, double L, uint64_t seed, uint32_t max_attempts,
                                            double* x_out) {
    using namespace neb;
    std::vector<D4> vpool;
    uint32_t nv_total = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (shape[i] == SH_CONVEX) nv_total = std::max(nv_total, vert_offset[i] + vert_count[i]);
    vpool.resize(nv_total ? nv_total : 1);
    for (uint32_t k = 0; k < nv_total; ++k) vpool[k] = D4{verts[3 * k], verts[3 * k + 1], verts[3 * k + 2], 0.0};
    std::vector<BodyG> g(n);
    std::vector<double> bound(n);
    double maxb = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        BodyG& b = g[i];
        b.x = mk(0, 0, 0);
        b.q = mkq(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
        b.he = mk(half_extents[3 * i], half_extents[3 * i + 1], half_extents[3 * i + 2]);
        b.radius = radius[i];
        b.half_height = half_height[i];
        b.shape = shape[i];
        b.verts = vpool.data() + (shape[i] == SH_CONVEX ? vert_offset[i] : 0);
        b.nverts = shape[i] == SH_CONVEX ? (int)vert_count[i] : 0;
        bound[i] = bounding_radius(b.shape, b.radius, b.half_height, b.he, b.verts, b.nverts);
        maxb = std::max(maxb, bound[i]);
    }
    const double cell = std::max(2.0 * maxb, 1e-9);
    const long nc = std::max(1L, (long)std::floor(L / cell));
    const double cs = L / (double)nc;
    Domain dom;
    dom.half = 0.5 * L;
    dom.periodic = 1;
    std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
    grid.reserve(2 * (size_t)n);
    SplitMix rng{seed};
    for (uint32_t i = 0; i < n; ++i) {
        bool placed = false;
        for (uint32_t att = 0; att < max_attempts && !placed; ++att) {
            V3 c = mk(L * rng.uniform() - 0.5 * L, L * rng.uniform() - 0.5 * L, L * rng.uniform() - 0.5 * L);
            g[i].x = c;
            const long gx = ((long)std::floor((c.x + 0.5 * L) / cs) % nc + nc) % nc;
            const long gy = ((long)std::floor((c.y + 0.5 * L) / cs) % nc + nc) % nc;
            const long gz = ((long)std::floor((c.z + 0.5 * L) / cs) % nc + nc) % nc;
            bool clash = false;
            for (int dx = -1; dx <= 1 && !clash; ++dx)
                for (int dy = -1; dy <= 1 && !clash; ++dy)
                    for (int dz = -1; dz <= 1 && !clash; ++dz) {
                        auto it = grid.find(cell_hash(((gx + dx) % nc + nc) % nc, ((gy + dy) % nc + nc) % nc,
                                                      ((gz + dz) % nc + nc) % nc));
                        if (it == grid.end()) continue;
                        for (uint32_t j : it->second) {
                            const V3 d = min_image(dom, g[j].x - c);
                            const double rr = bound[i] + bound[j];
                            if (norm2(d) >= rr * rr) continue;
                            SupV tet[4];
                            if (gjk_tetra(g[i], g[j], min_image_shift(g[i], g[j], dom), tet)) { clash = true; break; }
                        }
                    }
            if (!clash) {
                placed = true;
                grid[cell_hash(gx, gy, gz)].push_back(i);
                x_out[3 * i] = c.x;
                x_out[3 * i + 1] = c.y;
                x_out[3 * i + 2] = c.z;
            }
        }
        if (!placed) return i;
    }
    return n;
}
