/*
 * ne_cuda.h -- C-ABI of the B200 step() path of NativeEngine.
 *
 * The reference engine is a C++17 class API: ne::World::step()
 * (src/world.hpp:138, src/world.cpp:133-146) called from ne::PhysicsWorld::step()
 * (src/physics_world.hpp:217-246).  It has no C ABI and no device.  This header
 * is the one boundary the B200 build adds underneath that API: the host facade
 * (nativeengine_b200/host/include/ne/world.hpp) owns the bodies and calls these
 * functions; bodies, contacts, islands and the warm-start cache live on the GPU.
 *
 * Conventions
 *  - Plain C: POD structs, host pointers and sizes, no torch or CUDA types.
 *  - Every function returns an int status (NE_OK == 0).  The reference has no
 *    error channel (invalid handles are silent no-ops); device faults, capacity
 *    exhaustion and unsupported features are reported here instead.
 *  - One opaque NeWorld per world.  Each world owns one CUDA stream.  A world is
 *    not thread-safe; distinct worlds may be used from distinct threads.
 *  - Vectors are interleaved: x[3*i+0..2]; quaternions are (w,x,y,z) like ne::Q
 *    (src/vmath.hpp:47-48).
 *  - Features that the reference supports but this device path does not yet run
 *    (joints, sleeping, CCD) make ne_world_upload / ne_world_step return
 *    NE_ERR_UNSUPPORTED.  There is no CPU fallback.
 */
#ifndef NE_CUDA_H
#define NE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
    NE_OK = 0,
    NE_ERR_ARG = 1,          /* bad pointer / size / enum value                  */
    NE_ERR_CUDA = 2,         /* a CUDA runtime call failed                        */
    NE_ERR_CAPACITY = 3,     /* a device capacity limit was hit and could not grow */
    NE_ERR_UNSUPPORTED = 4,  /* feature not on the device path (see above)        */
    NE_ERR_TIMEOUT = 5,      /* a bounded device wait ran out                     */
    NE_ERR_NUMERIC = 6,      /* an iteration cap was hit (EPA face budget)        */
    NE_ERR_NO_DEVICE = 7     /* no CUDA device visible                            */
};

/* ---- shapes: same tags and order as ne::Shape (src/body.hpp:24) ----------- */
enum {
    NE_SHAPE_SPHERE = 0,
    NE_SHAPE_CYLINDER = 1,
    NE_SHAPE_BOX = 2,
    NE_SHAPE_CAPSULE = 3,
    NE_SHAPE_CONVEX = 4,
    NE_SHAPE_PLANE = 5,
    NE_SHAPE_MESH = 6,
    NE_SHAPE_COMPOUND = 7
};

/* ---- material combine modes: ne::World::Combine (src/world.hpp:85) ------- */
enum {
    NE_COMBINE_AVERAGE = 0,
    NE_COMBINE_MIN = 1,
    NE_COMBINE_MAX = 2,
    NE_COMBINE_MULTIPLY = 3,
    NE_COMBINE_GEOMETRIC_MEAN = 4
};

/* ---- per-body flag bits (ne::Body booleans, src/body.hpp:106-127) -------- */
#define NE_BODY_DYNAMIC   1u
#define NE_BODY_SLEEPING  2u
#define NE_BODY_KINEMATIC 4u
#define NE_BODY_SENSOR    8u
#define NE_BODY_CCD      16u

/* World configuration: the public fields of ne::World (src/world.hpp:75-136)
 * that step() reads.  Joint counts are carried so that a world with joints
 * is refused (NE_ERR_UNSUPPORTED) rather than silently stepped without them. */
typedef struct NeWorldParams {
    double half;                 /* Box::half (src/box.hpp:17)                  */
    int32_t periodic;            /* Box::periodic                               */
    int32_t open_boundary;       /* World::openBoundary                         */
    double dt;                   /* World::dt                                   */
    double restitution;          /* World::restitution                          */
    double friction;             /* World::friction                             */
    double contact_beta;         /* World::contactBeta                          */
    double gravity[3];           /* World::gravity                              */
    int32_t restitution_combine; /* World::restitutionCombine (NE_COMBINE_*)    */
    int32_t friction_combine;    /* World::frictionCombine                      */
    int32_t warm_start;          /* World::warmStart                            */
    int32_t force_brute_force;   /* World::forceBruteForce                      */
    int32_t capture_contacts;    /* World::captureContacts                      */
    int32_t sleep_enabled;       /* World::sleepEnabled (must be 0 here)        */
    double sleep_lin_vel, sleep_ang_vel, sleep_time, wake_vel;
    uint32_t n_distance_joints;  /* World::distanceJoints.size() (must be 0)    */
    uint32_t n_joints;           /* World::joints.size() (must be 0)            */
} NeWorldParams;

/* Fills p with ne::World's defaults (src/world.hpp:75-126, src/box.hpp:17-18). */
void ne_world_params_default(NeWorldParams* p);

/* A static triangle mesh with its AABB BVH, exactly as ne::MeshData holds it
 * after MeshData::build() (src/mesh.hpp:14-26): the device walks the given
 * nodes in the reference's order (src/mesh.hpp:44-57), so pass the arrays of
 * the reference's own build for contacts in the reference's order. */
typedef struct NeMeshData {
    uint32_t n_verts;
    const double* verts;        /* [3*n_verts] mesh-frame vertices               */
    uint32_t n_tris;
    const int32_t* tris;        /* [3*n_tris] vertex indices a, b, c             */
    const int32_t* order;       /* [n_tris] BVH-sorted triangle indices          */
    uint32_t n_nodes;
    const double* node_lo;      /* [3*n_nodes] node AABB                         */
    const double* node_hi;      /* [3*n_nodes]                                   */
    const int32_t* node_left;   /* [n_nodes] child node indices (-1: leaf)       */
    const int32_t* node_right;  /* [n_nodes]                                     */
    const int32_t* node_start;  /* [n_nodes] leaf range [start, start+count) of order */
    const int32_t* node_count;  /* [n_nodes]                                     */
} NeMeshData;

/* Host-side body arrays (structure of arrays, n bodies).  Mirrors the fields of
 * ne::Body (src/body.hpp:41-130) that step() reads or writes.  For upload every
 * pointer except verts/nocollide (when unused) must be non-NULL; for download
 * only the non-NULL state pointers are filled. */
typedef struct NeBodyArrays {
    uint32_t n;
    /* dynamic state */
    double* x;              /* [3n] centre of mass                           */
    double* q;              /* [4n] orientation w,x,y,z (body -> world)      */
    double* v;              /* [3n] linear velocity                          */
    double* w;              /* [3n] angular velocity (world frame)           */
    double* force;          /* [3n] force accumulator (cleared by step)      */
    double* torque;         /* [3n] torque accumulator (cleared by step)     */
    /* mass */
    double* inv_mass;       /* [n]                                           */
    double* inv_inertia;    /* [3n] diagonal of the body-frame inverse inertia */
    /* shape */
    int32_t* shape;         /* [n] NE_SHAPE_*                                */
    double* radius;         /* [n]                                           */
    double* half_height;    /* [n]                                           */
    double* half_extents;   /* [3n] box half extents, or plane normal        */
    uint32_t* vert_offset;  /* [n] first convex vertex in verts              */
    uint32_t* vert_count;   /* [n] number of convex vertices                 */
    double* verts;          /* [3*n_verts] body-frame convex vertices        */
    uint32_t n_verts;
    /* material, damping, gravity */
    double* friction;       /* [n] (<0: inherit World::friction)             */
    double* restitution;    /* [n] (<0: inherit World::restitution)          */
    double* linear_damping; /* [n]                                           */
    double* angular_damping;/* [n]                                           */
    double* gravity_scale;  /* [n]                                           */
    /* filtering */
    uint32_t* layer;        /* [n]                                           */
    uint32_t* mask;         /* [n]                                           */
    uint32_t* flags;        /* [n] NE_BODY_* bits                            */
    uint32_t* nocollide_offset; /* [n] into nocollide                        */
    uint32_t* nocollide_count;  /* [n]                                       */
    uint32_t* nocollide;    /* [n_nocollide] excluded partner indices         */
    uint32_t n_nocollide;
    /* compound bodies (NE_SHAPE_COMPOUND): children as ne::ChildShape
     * (src/body.hpp:28-39), primitives only (sphere, box, cylinder, capsule);
     * NULL when no body is a compound */
    uint32_t* child_offset; /* [n] first child of each compound body          */
    uint32_t* child_count;  /* [n]                                           */
    uint32_t n_children;
    int32_t* child_shape;   /* [n_children] NE_SHAPE_*                       */
    double* child_pos;      /* [3*n_children] localPos                       */
    double* child_rot;      /* [4*n_children] localRot (w,x,y,z)             */
    double* child_radius;   /* [n_children]                                  */
    double* child_half_height; /* [n_children]                               */
    double* child_half_extents; /* [3*n_children]                            */
    /* triangle-mesh bodies (NE_SHAPE_MESH): mesh_index[i] into meshes; NULL
     * when no body is a mesh */
    uint32_t* mesh_index;   /* [n]                                           */
    uint32_t n_meshes;
    const NeMeshData* meshes; /* [n_meshes]                                  */
} NeBodyArrays;

/* One resolved contact constraint of the last step, in solver order
 * (sorted body pair, then slot) -- the device image of World::debugContacts
 * (src/world.hpp:135-136, src/world.cpp:552) plus the converged impulses. */
typedef struct NeContactArrays {
    uint32_t* i;            /* [c] body index a (i < j)                      */
    uint32_t* j;            /* [c] body index b                              */
    uint32_t* slot;         /* [c] contact slot within the pair              */
    double* point;          /* [3c] world contact point                      */
    double* normal;         /* [3c] unit normal, b -> a                      */
    double* depth;          /* [c] penetration                               */
    double* n_imp;          /* [c] converged accumulated normal impulse      */
    double* t_imp;          /* [c] accumulated friction impulse (scalar)     */
} NeContactArrays;

/* Per-step counters of the last successful step. */
typedef struct NeStepStats {
    uint64_t pairs;          /* reference-rule broadphase pairs when recording,
                                else the internal candidate pairs             */
    uint64_t survivors;      /* pairs passing filters + bounding-sphere cull  */
    uint64_t contacts;       /* contact constraints                           */
    uint64_t islands;        /* solver islands (connected components)         */
    uint64_t max_island;     /* constraints in the largest island             */
    uint64_t epa_cap_hits;   /* EPA runs that stopped at the 64-iteration cap */
    uint64_t steps;          /* steps taken since upload                      */
    uint64_t retries;        /* steps re-run after growing a device buffer    */
    uint64_t candidates;     /* pairs the internal grid handed to the cull    */
    uint64_t graph_steps;    /* steps run by replaying the captured step graph */
    uint64_t graph_captures; /* times the step graph was (re)captured         */
} NeStepStats;

typedef struct NeWorld NeWorld;

/* Lifecycle.  Replaces constructing ne::World (src/world.hpp:73). */
int ne_world_create(const NeWorldParams* params, NeWorld** out);
int ne_world_destroy(NeWorld* world);
/* Replaces assigning World's public config fields (src/world.hpp:75-136). */
int ne_world_set_params(NeWorld* world, const NeWorldParams* params);

/* Full (re)load of all bodies.  Replaces editing World::bodies
 * (src/world.hpp:128) -- add/remove/setters in PhysicsWorld
 * (src/physics_world.hpp:58-165,262-270) end here.  Does not clear the warm
 * cache, matching the reference, whose cache survives body edits. */
int ne_world_upload(NeWorld* world, const NeBodyArrays* bodies);
/* Batch of independent worlds stepped together (no counterpart in the
 * reference, which steps one World at a time).  World k owns bodies
 * [world_begin[k], world_begin[k+1]) of `bodies` (world_begin has nworlds + 1
 * entries, from 0 to bodies->n) and is configured by params[k]; no pair,
 * contact or island spans two worlds, so each world evolves exactly as an
 * ne::World of its own would.  All worlds share one warm_start setting.
 * Pairs, contacts and island labels of a batch use global body indices. */
int ne_world_upload_batch(NeWorld* world, const NeWorldParams* params, uint32_t nworlds,
                          const uint32_t* world_begin, const NeBodyArrays* bodies);
/* Overwrite only x/q/v/w (each may be NULL to keep the device copy).  Same
 * count as the last full upload. */
int ne_world_upload_state(NeWorld* world, const double* x, const double* q,
                          const double* v, const double* w);
/* Copy the non-NULL state fields (x, q, v, w, force, torque) back to the host. */
int ne_world_download(NeWorld* world, NeBodyArrays* out);

/* Advance nsteps steps.  Replaces World::step() (src/world.cpp:133-146):
 * integrate -> broadphase -> narrowphase -> constraint build + warm start ->
 * 8 sequential-impulse iterations -> position correction -> warm-cache store ->
 * wrap (periodic) or walls (reflective).  Synchronous: returns after the last
 * step has finished on the device. */
int ne_world_step(NeWorld* world, uint32_t nsteps);

/* Replaces World::resetWarmCache() (src/world.hpp:140). */
int ne_world_reset_warm_cache(NeWorld* world);

/* Introspection of the last step (parity probes). */
int ne_world_stats(const NeWorld* world, NeStepStats* out);
/* Recording of step intermediates.  With NE_RECORD_PAIRS set, each step also
 * builds the pair list exactly as World::broadphasePairs() does
 * (src/world.cpp:424-501) for ne_world_pairs.  Off by default: internally the
 * step pairs bodies whose bounding radius is far above their world's typical
 * size (a ground box) with everyone, like planes, and grids the rest with a
 * cell sized for them; every pair that can pass the bounding-volume cull is
 * still examined, so contacts and results do not depend on this setting. */
#define NE_RECORD_PAIRS 1u
int ne_world_set_record(NeWorld* world, uint32_t flags);
/* Broadphase pairs of the last step, as World::broadphasePairs() returned them
 * (src/world.cpp:424-501): sorted by (i, j), unique, i < j.  *count receives
 * the total; at most cap pairs are written.  Needs NE_RECORD_PAIRS. */
int ne_world_pairs(NeWorld* world, uint32_t* i, uint32_t* j, uint64_t cap,
                   uint64_t* count);
/* Contacts of the last step in solver order; *count receives the total. */
int ne_world_contacts(NeWorld* world, NeContactArrays* out, uint64_t cap,
                      uint64_t* count);
/* Island partition of the last step: label[b] = smallest body index of the
 * connected component of b over contacts whose two bodies both have
 * invMass > 0 (the union-find of src/world.cpp:332-343 over islandPairs_);
 * bodies in no such contact are their own label. */
int ne_world_islands(NeWorld* world, uint32_t* label, uint32_t n);

/* Arithmetic precision of the narrowphase and the contact solve.  No
 * counterpart in the reference (which is FP64 throughout).
 *   NE_PRECISION_F64  the default: bit-exact with the reference.
 *   NE_PRECISION_F32  the batched FP32 form: support mappings, analytic
 *     pairs, box-box clipping and the sequential-impulse solve in FP32 with
 *     FP32 accumulation, in the reference's contact order; FP64 stays for
 *     pose integration, the minimum-image offsets and the wrap, the
 *     accumulated normal impulses (the warm-start cache), GJK's simplex and
 *     EPA's polytope arithmetic with their near-degenerate containment and
 *     termination tests, and the body state between steps.
 * Takes effect from the next step; may be changed at any time. */
#define NE_PRECISION_F64 0
#define NE_PRECISION_F32 1
int ne_world_set_precision(NeWorld* world, int precision);

/* Launch shape of the big-island solver (islands of >= 48 contacts).  No
 * counterpart in the reference.  Results do not depend on it.
 * threads: a multiple of 32 in 64..512 per CTA; ctas_per_sm: 1..4;
 * team_max: 1 = each big island is solved by one CTA (ready queue in shared
 * memory); 2..64 = an island may be solved by a team of up to team_max CTAs
 * on different SMs (queue and counters in global memory), sized in proportion
 * to its share of the work.  Until set or tuned, the shape follows the last
 * upload: 384 threads x 1 CTA per SM for a single world, 128 x 3 for a
 * batch of several worlds.
 * ne_world_autotune times each candidate shape for `steps` steps from the
 * current state, keeps the fastest and restores the state and warm cache, so
 * the world continues as if it had not been called; *chosen (may be NULL)
 * receives the shape kept. */
typedef struct NeSolverShape {
    uint32_t threads;
    uint32_t ctas_per_sm;
    uint32_t team_max;
} NeSolverShape;
int ne_world_set_solver_shape(NeWorld* world, const NeSolverShape* shape);
int ne_world_get_solver_shape(const NeWorld* world, NeSolverShape* shape);
int ne_world_autotune(NeWorld* world, uint32_t steps, NeSolverShape* chosen);

/* Device checkpoint of everything a step changes: positions, orientations,
 * velocities, angular velocities, pending forces and torques, and the warm
 * cache (last step's accumulated normal impulses).  The device analogue of
 * PhysicsWorld::saveState()/loadState() (src/physics_world.cpp:22-64) kept in
 * HBM; restoring makes the next steps bit-identical to the steps taken after
 * the checkpoint was made.  A checkpoint belongs to the world that made it
 * and must be destroyed before that world. */
typedef struct NeCheckpoint NeCheckpoint;
int ne_world_checkpoint(NeWorld* world, NeCheckpoint** out);
int ne_world_restore(NeWorld* world, const NeCheckpoint* checkpoint);
int ne_checkpoint_destroy(NeCheckpoint* checkpoint);

/* Adjoint of step() (stepBackward).  No counterpart in the reference.
 * Differentiates the trajectory of `nsteps` steps starting from the world's
 * current state and warm cache: given dL/d(x, v after the last step) in
 * `final_grad` (either pointer may be NULL for zero), returns dL/d(initial
 * x, q, v, w), dL/d per-body mass (inverse inertia scaled with the mass, shape
 * fixed), dL/d per-body inverse mass and inverse inertia, and dL/d per-world
 * friction and restitution (through the bodies that inherit the world's
 * values).  Every step is recomputed on the device, one CTA per world,
 * from states checkpointed every `checkpoint_every` steps (0 = one segment);
 * the contact set, clamps and branches are those of the trajectory, so the
 * result is the derivative of the piecewise-smooth map on the piece the
 * trajectory is on.  The world's own state is not changed.  Supported: open
 * or periodic worlds of planes, boxes and convex hulls (spheres only with
 * spheres and planes), at most 1024 bodies per world; otherwise
 * NE_ERR_UNSUPPORTED.  Output pointers may be NULL. */
typedef struct NeStateGrad {
    const double* x;        /* [3n] dL/dx after the last step */
    const double* v;        /* [3n] dL/dv after the last step */
} NeStateGrad;
typedef struct NeParamGrad {
    double* x;              /* [3n] dL/d initial x */
    double* q;              /* [4n] dL/d initial q (w, x, y, z components) */
    double* v;              /* [3n] dL/d initial v */
    double* w;              /* [3n] dL/d initial angular velocity */
    double* mass;           /* [n] dL/d mass (bodies with invMass > 0; else 0) */
    double* inv_mass;       /* [n] */
    double* inv_inertia;    /* [3n] */
    double* friction;       /* [nworlds] dL/d World::friction */
    double* restitution;    /* [nworlds] dL/d World::restitution */
} NeParamGrad;
int ne_world_step_backward(NeWorld* world, uint32_t nsteps, uint32_t checkpoint_every,
                           const NeStateGrad* final_grad, NeParamGrad* out);

/* The CUDA stream the world launches on (as a void*; cast to cudaStream_t). */
int ne_world_stream(const NeWorld* world, void** stream);
/* Number of kernel launches made by the last ne_world_step call (kernels
 * inside replayed graphs included). */
int ne_world_launch_count(const NeWorld* world, uint64_t* launches);

/* CUDA-graph stepping (on by default; no counterpart in the reference).  The
 * kernels of one step are captured once into a CUDA graph and replayed in
 * batches of up to 64 steps, with one read of the control block per batch
 * instead of one per step.  A step that overflows a device buffer halts the
 * rest of its batch on the device; the host restores that step's pre-step
 * state, grows the buffer and takes the step again outside the graph, so
 * results are the same bit for bit with the graph on or off.  Changing
 * capacities, precision, solver shape or parameters re-captures the graph.
 * Steps with stage timing or pair recording enabled run outside the graph. */
int ne_world_set_graph(NeWorld* world, int enable);

/* Per-stage device timing (CUDA events on the world's stream).  Stages:
 * 0 integrate, 1 broadphase, 2 pair filter + cull, 3 narrowphase,
 * 4 constraint build, 5 islands, 6 solve, 7 boundary.  While enabled, each
 * step records NE_NUM_STAGES + 1 events; ne_world_stage_times returns the
 * accumulated milliseconds per stage and the number of steps timed since the
 * last enable.  No counterpart in the reference (it has no timers). */
#define NE_NUM_STAGES 8
int ne_world_profile(NeWorld* world, int enable);
int ne_world_stage_times(NeWorld* world, double* ms, uint64_t* steps);
const char* ne_stage_name(int stage);

/* Broadphase pair list without any device allocation.  No counterpart in the
 * reference: it is for callers that may not allocate GPU memory where they
 * call -- an embedding engine that hands out device memory only from its own
 * fixed pool, or a frame loop in which an allocation (and the synchronisation
 * cudaMalloc/cudaFree can bring) is not allowed.  Returns, for the bodies as
 * given, the sorted unique candidate pairs World::broadphasePairs() would
 * return (the same list ne_world_pairs reports for a step); at most cap pairs
 * are written to the host arrays and *count receives the total.  All device
 * working memory is one file-scope array (about 2.1 MiB) that every GPU the
 * library is loaded on holds until the process exits; more than
 * NE_NOALLOC_MAX_BODIES bodies or NE_NOALLOC_MAX_PAIRS pairs is refused with
 * NE_ERR_CAPACITY.  Every call shares that array, so calls that overlap on the
 * GPU (several host threads at once) race and must be serialised by the
 * caller.  The first call on a device looks up the array's device address;
 * make it before any stream capture.  Synchronous, on the per-thread default
 * stream. */
#define NE_NOALLOC_MAX_BODIES 2048u
#define NE_NOALLOC_MAX_PAIRS 262144u
int ne_broadphase_pairs_noalloc(const NeWorldParams* params, const NeBodyArrays* bodies, uint32_t* pair_i,
                                uint32_t* pair_j, uint64_t cap, uint64_t* count);

/* Human-readable status / last CUDA error text. */
const char* ne_status_string(int status);
const char* ne_last_error(void);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* NE_CUDA_H */
