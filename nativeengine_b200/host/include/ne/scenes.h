/* ne/scenes.h -- benchmark scene placement helper (host only, C ABI).
 *
 * Random sequential placement of n convex bodies with EXACT overlap rejection
 * (GJK on the bodies' support mappings, the same geometry the step uses) in a
 * periodic cube of edge L.  Orientations and shapes are given; centres are
 * drawn uniformly from a SplitMix64 stream seeded by `seed`.  Bodies are
 * placed in index order; each gets at most max_attempts candidate centres.
 * Returns the number of bodies placed (n when all fit); x_out[3*i..] receives
 * the centre of body i.  Not part of the step path. */
#ifndef NE_SCENES_H
#define NE_SCENES_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
uint32_t ne_scene_place_periodic(uint32_t n, const int32_t* shape, const double* radius, const double* half_height,
                                 const double* half_extents, const double* q, const uint32_t* vert_offset,
                                 const uint32_t* vert_count, const double* verts, double L, uint64_t seed,
                                 uint32_t max_attempts, double* x_out);
#ifdef __cplusplus
}
#endif
#endif
