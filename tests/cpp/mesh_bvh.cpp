// Builds a height-field mesh with the facade's ne::MeshData::build() and prints
// the BVH (order, then one line per node) for comparison with the reference's
// own build.  Usage: mesh_bvh rows cols
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "ne/world.hpp"

int main(int argc, char** argv) {
    const int rows = argc > 1 ? std::atoi(argv[1]) : 6, cols = argc > 2 ? std::atoi(argv[2]) : 6;
    ne::MeshData m;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c)
            m.verts.push_back(ne::V3{1.5 * c, 0.4 * std::sin(0.8 * c) * std::cos(0.6 * r), 1.5 * r});
    for (int r = 0; r + 1 < rows; ++r)
        for (int c = 0; c + 1 < cols; ++c) {
            const int a = r * cols + c, b = a + 1, d = a + cols, e = d + 1;
            m.tris.push_back({a, d, b});
            m.tris.push_back({b, d, e});
        }
    m.build();
    std::printf("order");
    for (int k : m.order) std::printf(" %d", k);
    std::printf("\n");
    for (const ne::MeshData::Node& nd : m.nodes)
        std::printf("node %.17g %.17g %.17g %.17g %.17g %.17g %d %d %d %d\n", nd.lo.x, nd.lo.y, nd.lo.z, nd.hi.x,
                    nd.hi.y, nd.hi.z, nd.left, nd.right, nd.start, nd.count);
    return 0;
}
