// ne_step.cuh -- launch arguments of the step kernels.
//
// One device world holds one or more independent simulation worlds (a
// batch).  Bodies of world w occupy the index range [begin, end); no pair,
// contact or island ever spans two worlds.  A single ne::World is a batch of
// one, so it runs exactly the same kernels.
#pragma once

#include "ne_internal.cuh"

namespace neb {

// Per-world configuration: ne::World's fields (src/world.hpp:75-126) plus the
// broadphase constants World::broadphasePairs() derives (src/world.cpp:427-457).
struct WorldP {
    Domain dom;              // Box (half, periodic)
    double dt, restitution, friction, beta;
    V3 g;                    // gravity
    int rcomb, fcomb;        // material combine modes
    int open_boundary;
    int brute;               // forceBruteForce || n < 64 || cell < 1e-9
    double cell;             // 2 * max bounding radius
    long long nc[3];         // periodic cell counts
    // internal grid: large bodies excluded like planes; the cell bounds every
    // pair the cull can keep (see derive_worlds in ne_capi.cu)
    int fbrute;
    double fcell;
    long long fnc[3];
    uint32_t begin, end;     // body range
    uint32_t plane_begin, plane_end;   // range of this world's planes in DevWorld::planes
    uint32_t xl_begin, xl_end;         // range of this world's planes + large bodies in DevWorld::xlist
};

struct StepArgs {
    DevWorld d;
    uint32_t n;              // bodies, all worlds
    uint32_t nworlds;
    int world_bits;          // bits of a world index in a cell key
    const WorldP* wp;        // [nworlds], device
    const uint32_t* bw;      // [n] world of each body, device
    long long* cext;         // [6 * nworlds] cell extents (min xyz, max xyz) per world
    int key_bits;            // bits the cell-key sort covers this step
    int any_grid;            // some world uses the grid (else every world is brute force)
    int warm;                // warm starting (one setting for the whole batch)
    int record;              // also build the reference-rule pair list
    int f32;                 // batched FP32 form: FP32 narrowphase, constraints and solve
    uint64_t Scap, Ccap, Rcap;
    int num_sms;
    int big_threads;         // threads per CTA of the big-island solver (tuned)
    int big_ctas_per_sm;     // CTAs per SM of the big-island solver (tuned)
    int big_team_max;        // CTAs per big island: 1 = block-local solver, > 1 = team solver (tuned)
    int sticky;              // replayed batch: an aborted step halts the rest of the batch
    uint32_t local_cap;      // big islands up to this many contacts: shared-memory dataflow solver
    int any_ext;             // some body is a triangle mesh or a compound (second narrowphase pass)
    int class_sort;          // some world mixes shapes: narrowphase in class order (d.sperm)
};

// Contacts per island the shared-memory dataflow solver takes (one counter
// byte each: 64 KiB of dynamic shared memory per CTA).
constexpr uint32_t kLocalCap = 65536;
// Opt-in shared-memory sizes of the solver kernels (once per device).
void init_kernel_attrs();
void init_kernel_attrs_f32();

// A second stream and two events: the small-island solve runs on st2 beside
// the big-island solvers on the main stream (fork after the island list, join
// before the boundary).  st2 == nullptr runs everything on the main stream.
struct SideStream {
    cudaStream_t st2;
    cudaEvent_t fork, join;
};

// ev: NE_NUM_STAGES + 1 events recorded at the stage boundaries, or nullptr.
// Grid shapes depend on the capacities in a only (live counts are read on the
// device), so the enqueued step can be captured once and replayed.
void launch_step(const StepArgs& a, cudaStream_t st, uint64_t* launches, cudaEvent_t* ev,
                 const SideStream* side = nullptr);
// Clears the batch fields of ctl (halt, steps_done, accumulators) before a
// replayed batch of steps.
void launch_batch_begin(Ctl* ctl, cudaStream_t st);

// FP32 stages (ne_step_f32.cu), enqueued by launch_step when a.f32 is set;
// the FP64 constraint build writes the FP32 solver records itself.
void launch_narrowphase_f32(const StepArgs& a, cudaStream_t st, uint64_t* launches);
// Small islands (one thread each) and big islands (dataflow solvers).
void launch_solve_small_f32(const StepArgs& a, int ib, cudaStream_t st, uint64_t* launches);
void launch_solve_big_f32(const StepArgs& a, int ib, int rb, cudaStream_t st, uint64_t* launches);
// FP32 velocities back into the FP64 state, after both solves.
void launch_writeback_f32(const StepArgs& a, cudaStream_t st, uint64_t* launches);
// Teams and dataflow state of the big islands (ne_step.cu; both precisions).
void launch_big_prep(const StepArgs& a, int ib, cudaStream_t st, uint64_t* launches);
// Per-position records of the big islands for the shared-memory solver.
void launch_big_rec(const StepArgs& a, int ib, int rb, cudaStream_t st, uint64_t* launches);
// State transfer in the C-ABI's host layout: x[3n] | q[4n] | v[3n] | w[3n] |
// force[3n] | torque[3n] (mask bit k = array k) to and from the records.
void launch_unpack_state(const DevWorld& d, uint32_t n, const double* io, uint32_t mask, cudaStream_t st);
void launch_pack_state(const DevWorld& d, uint32_t n, double* io, uint32_t mask, cudaStream_t st);
// Convex vertex pool D4 -> F4 (upload time).
void convert_verts_f32(const D4* src, F4* dst, uint32_t count, cudaStream_t st);

}  // namespace neb
