// ne_internal.cuh -- device-side world layout and the host orchestration API
// shared by the CUDA translation units of libne_cuda.so.
//
// HBM layout (one world):
//   bodies   : structure of 32-byte records, one array per record kind, so a
//              per-body kernel streams each array fully coalesced and a pair
//              kernel gathers one 32-byte sector per record:
//                pos  = (x, y, z, invMass)      quat = (w, x, y, z)
//                vel  = (vx, vy, vz, -)         omg  = (wx, wy, wz, -)
//                frc  = force accumulator       trq  = torque accumulator
//                inert= (invIx, invIy, invIz, boundingRadius)
//                geom = (radius, halfHeight, gravityScale, -)
//                ext  = (halfExtents | plane normal, -)
//                mat  = (friction, restitution, linearDamping, angularDamping)
//                meta = (shape, flags, layer, mask)
//   pairs    : surviving pairs si/sj, CSR by first body, in sorted (i, j) order
//              (rec_i/rec_j: the reference-rule list, when recording).
//   contacts : 4 slots per surviving pair (normal+depth, point).
//   constraints, warm cache, island order: flat arrays in solver order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ne_geom.cuh"
#include "ne_cuda.h"

namespace neb {

// Internal body flag: the solver can change this body's velocity
// (invMass > 0 or a nonzero inverse inertia).  Immovable bodies separate islands.
constexpr uint32_t kFlagMutable = 1u << 16;
// Internal body flag: bounding radius far above its world's typical size (a
// ground box, a wall).  The internal grid pairs such bodies with every body of
// the world, like planes, so they do not set the cell size.
constexpr uint32_t kFlagLarge = 1u << 17;

// Device control block: capacity checks, counters, warm-cache selector.
struct Ctl {
    uint32_t abort;          // a capacity or bit budget was exceeded this step
    uint32_t flags;          // bit0: EPA/clip budget overrun
    uint32_t need_bits;      // sort-key bits the cell keys needed
    uint32_t local_bits;     // widest per-world cell-key layout this step
    uint32_t wsel;           // warm cache buffer holding the previous step
    uint64_t P, S, C;        // grid candidates examined, surviving pairs, contacts (totals, even if over capacity)
    uint64_t P_ref;          // pairs of the reference's broadphase rule (recorded steps)
    uint64_t islands, max_island, epa_cap_hits;
    uint32_t nbig;           // islands solved by the dataflow kernel this step
    uint32_t solve_timeout;  // a bounded dependency wait ran out (error)
    uint32_t wcount[2];      // warm cache entries per buffer
    uint64_t scan_total;     // scratch total of the last scan
    uint64_t sort_hist_len;  // live length of the radix sort's digit histogram
    uint64_t C2;             // 2 * C: rank entries of the dataflow solver
    uint64_t ncells;         // runs of equal cell keys after the sort (internal grid)
    uint64_t S_stage;        // surviving pairs staged so far this step
    // Replayed batches of steps (CUDA graph): a step that aborts sets halt,
    // and with StepArgs::sticky every later step of the batch is a no-op.
    // The rest accumulates over the steps of a batch that completed.
    uint32_t halt;
    uint32_t steps_done;     // completed steps since the batch began
    uint32_t acc_flags;      // OR of flags
    uint32_t acc_timeout;    // OR of solve_timeout
    uint32_t need_max;       // max of need_bits
    uint32_t pad_;
    uint64_t acc_epa;        // sum of epa_cap_hits
    // Big islands in claim order for the shared-memory solver: counts per
    // size class (floor(log2 contacts)), fill cursors, and the claim counter.
    uint32_t big_class[32];
    uint32_t big_fill[32];
    uint32_t big_next;
    uint32_t nlong;          // long partner lists split over many warps this step
};

// Islands with at least kBigIsland contacts go to the team (dataflow)
// solver; smaller ones are solved one thread per island.
constexpr uint32_t kBigIsland = 48;

// Partner lists of at least kLongRow candidates are culled by many warps
// (k_long_mask, k_long_place); up to kLongRows of them per step, the rest on
// one warp each like every other list.
constexpr uint32_t kLongRow = 512;
constexpr uint32_t kLongRows = 64;

// Big-island solver control block: ready-queue head (claims) and tail
// (pushes), updates done, failure flag.
struct BigCtl {
    uint32_t head, tail, done, fail;
};

struct DevWorld {
    // bodies
    D4 *pos, *quat, *vel, *omg, *frc, *trq;
    D4 *inert, *geom, *ext, *mat;
    uint4* meta;
    uint2* vrng;
    D4* verts;
    uint2* ncrng;
    uint32_t* nc;
    uint32_t* planes;        // indices of grid-excluded bodies (planes), ascending
    uint32_t* xlist;         // planes and large bodies, ascending (internal grid)
    // pre-step snapshot (restored when a step is re-run)
    D4 *s_pos, *s_quat, *s_vel, *s_omg, *s_frc, *s_trq;
    // broadphase
    unsigned long long *key[2];
    uint32_t* val[2];
    uint32_t *bcnt, *boff;
    // cell table of the internal grid: run r of equal sorted keys occupies
    // sorted positions [cstart[r], cstart[r+1]); an open-addressing hash maps
    // a cell key to its run
    uint32_t *cflag, *crun, *cstart;   // [n], [n], [n + 1]
    unsigned long long* hkey;          // [hsize] (~0 = empty)
    uint32_t* hval;                    // [hsize]
    uint32_t hsize;                    // power of two >= 2n
    uint32_t *stage_j, *bstage;        // [Scap] staged partner lists, [n] staging offset per body
    // long partner lists (every later body of the world: brute-force worlds
    // and grid-excluded bodies): the body of each slot and one keep bit per
    // candidate, lwords words per slot
    uint32_t *lrow, *lmask;            // [kLongRows], [kLongRows * lwords]
    uint32_t lwords;                   // ceil(n / 32) + 1
    D4* srec;                          // [n] (x, y, z, boundR) in sorted cell order
    uint32_t *rec_i, *rec_j;       // reference-rule pair list (recorded steps only)
    // narrowphase: the pairs that pass the filters and the cull, sorted by (i, j)
    uint32_t *si, *sj;
    uint32_t* sperm;         // [S] survivors in narrowphase order: analytic pairs first, then GJK/EPA
    uint32_t *ccnt, *coff;
    D4 *cn, *cp;             // 4 slots per survivor: (normal, depth), (point, -)
    // constraints
    uint32_t *ci, *cj, *cslot;
    D4 *con_n;               // n, overlap
    D4 *con_ra;              // rA, restBias
    D4 *con_rb;              // rB, mu
    D4 *con_p;               // contact point
    double2* con_imp;        // nImp, tImp
    // warm cache (double buffered)
    unsigned long long* wkey[2];
    double* wimp[2];
    // islands
    uint32_t* parent;
    uint32_t *ilab[2], *iord[2];
    uint32_t *iflag, *ioff, *istart;
    uint32_t* big;           // islands handed to the dataflow solver
    double* con_kn;          // effective mass along n (constant during the solve)
    // per-body update ranks for the dataflow solver
    uint32_t *rkey[2], *rval[2];   // (body, 2*position+side) entries, 2 per contact
    uint32_t* crank;         // [2C] rank of each contact among its body's contacts
    uint32_t* bdeg;          // [n] contacts per body in its island
    uint32_t* bstart;        // [n] first rank entry of each body in the sorted entries
    uint32_t* bcnt10;        // [10C] unfinished-predecessor counts of the solver updates
    uint32_t* bq10;          // [10C] ready queues of the solver updates
    BigCtl* bctl;            // [C/48 + 1] per big island
    uint32_t* bteam;         // [C/48 + 2] first virtual CTA of each big island's team
    uint32_t* bigs;          // [C/48 + 1] big islands, larger size classes first
    uint4* brec;             // [2C] per island position: {c, i, j, flags}, {next on i, next on j} (big islands)
    // compound children and triangle meshes (vrng: child range; mesh index in .x)
    D4* child;               // [4 per child] (localPos, shape), localRot, (r, hh, he.x, he.y), (he.z, -, -, -)
    uint4* mesh_tab;         // [meshes] node, order, triangle and vertex offsets (node offset ~0u: empty)
    D4 *mnode_lo, *mnode_hi; // [nodes] BVH node bounds
    int4* mnode;             // [nodes] (left, right, start, count), mesh-local
    int* morder;             // [tris] BVH-sorted triangle indices, mesh-local
    int4* mtri;              // [tris] vertex indices, mesh-local
    D4* mvert;               // [verts] mesh-frame vertices
    D4 *ext_cn, *ext_cp;     // [C] contacts of mesh and compound pairs, at their constraint index
    // batched FP32 form (null in FP64 mode): FP32 copies of the body state the
    // narrowphase and the solver read, refreshed every step after integration,
    // and the FP32 constraint records.  Poses, the warm-start impulses and the
    // body state between steps stay in the FP64 arrays above.
    F4 *f_v, *f_w;           // [n] (v, invMass), (omega, -): solver working state
    F4 *f_q;                 // [n] orientation (w, x, y, z)
    F4 *f_I;                 // [n] (invI, halfHeight)
    F4 *f_e;                 // [n] (half extents or plane normal, radius)
    F4* f_verts;             // convex vertices (body frame)
    F4 *f_n, *f_ra, *f_rb;   // [C] (n, overlap), (rA, restBias), (rB, mu)
    float* f_kn;             // [C] effective mass along n
    // host-layout state block for per-step transfers (19n doubles, lazily allocated)
    double* io;
    // scratch
    uint32_t *hist, *tsum;
    Ctl* ctl;
};

// Scan / sort primitives (ne_prims.cu).  All are asynchronous on `st`, all skip
// when ctl->abort is set, and all count their launches into *launches.
// Exclusive scan of n u32 values; the u64 total lands in *total (device).
// n is the capacity; with n_dev only the first min(n, *n_dev) elements count.
void scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tsum, uint64_t* total,
              const Ctl* ctl, cudaStream_t st, uint64_t* launches, const uint64_t* n_dev = nullptr);
size_t scan_tsum_words(uint32_t n);
// Stable LSD radix sort of (key, val) pairs on the low `bits` bits.
// Ping-pongs between buffers 0 and 1; returns the buffer index holding the result.
int radix_sort_u64(unsigned long long* key[2], uint32_t* val[2], uint32_t n, int bits, uint32_t* hist,
                   uint32_t* tsum, const Ctl* ctl, cudaStream_t st, uint64_t* launches,
                   const uint64_t* n_dev = nullptr);
int radix_sort_u32(uint32_t* key[2], uint32_t* val[2], uint32_t n, int bits, uint32_t* hist,
                   uint32_t* tsum, const Ctl* ctl, cudaStream_t st, uint64_t* launches,
                   const uint64_t* n_dev = nullptr);
size_t radix_hist_words(uint32_t n);

}  // namespace neb
