// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into the
// product.  Drives the reference NativeEngine, compiled unmodified from its own
// sources (src/world.cpp, src/physics_world.cpp) by oracle/Makefile, through a
// C-ABI that uses the same POD structs as include/ne_cuda.h, so the parity
// tests can feed identical inputs to the reference and to the device path.
//
// The reference exposes no hook for its step-internal intermediates, so the
// shim re-sequences World::step() (src/world.cpp:133-146) from World's own
// private members (made reachable with an access-specifier macro around the
// header only; no reference source is edited) and records:
//   * the broadphase pair list of the step (World::broadphasePairs(), called
//     between integrate() and collide() -- it is const and deterministic);
//   * the resolved contacts (World::captureContacts / debugContacts);
//   * the converged normal impulses (World::warmCache_ after collide());
//   * the island partition (union-find over World::islandPairs_, the structure
//     World::updateSleep() builds at src/world.cpp:332-343).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <utility>
#include <vector>

#define private public
#include "world.hpp"
#undef private
#include "detect.hpp"
#include "manifold.hpp"
#include "physics_world.hpp"

#include "ne_cuda.h"

namespace {

struct RefWorld {
    ne::World w;
    std::vector<std::pair<std::size_t, std::size_t>> lastPairs;
    std::vector<uint32_t> islandLabel;
};

ne::V3 v3(const double* p, std::size_t i) { return ne::V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

void applyParams(ne::World& w, const NeWorldParams* p) {
    w.box.half = p->half;
    w.box.periodic = p->periodic != 0;
    w.openBoundary = p->open_boundary != 0;
    w.dt = p->dt;
    w.restitution = p->restitution;
    w.friction = p->friction;
    w.contactBeta = p->contact_beta;
    w.gravity = ne::V3{p->gravity[0], p->gravity[1], p->gravity[2]};
    w.restitutionCombine = static_cast<ne::World::Combine>(p->restitution_combine);
    w.frictionCombine = static_cast<ne::World::Combine>(p->friction_combine);
    w.warmStart = p->warm_start != 0;
    w.forceBruteForce = p->force_brute_force != 0;
    w.captureContacts = true;   // always record; costs nothing on the oracle side
    w.sleepEnabled = p->sleep_enabled != 0;
    w.sleepLinVel = p->sleep_lin_vel;
    w.sleepAngVel = p->sleep_ang_vel;
    w.sleepTime = p->sleep_time;
    w.wakeVel = p->wake_vel;
}

void loadBodies(ne::World& w, const NeBodyArrays* b) {
    w.bodies.clear();
    w.bodies.resize(b->n);
    for (uint32_t i = 0; i < b->n; ++i) {
        ne::Body& o = w.bodies[i];
        o.x = v3(b->x, i);
        o.q = ne::Q{b->q[4 * i], b->q[4 * i + 1], b->q[4 * i + 2], b->q[4 * i + 3]};
        o.v = v3(b->v, i);
        o.w = v3(b->w, i);
        o.force = b->force ? v3(b->force, i) : ne::V3{};
        o.torque = b->torque ? v3(b->torque, i) : ne::V3{};
        o.invMass = b->inv_mass[i];
        o.invInertiaBody = v3(b->inv_inertia, i);
        o.shape = static_cast<ne::Shape>(b->shape[i]);
        o.radius = b->radius[i];
        o.halfHeight = b->half_height[i];
        o.halfExtents = v3(b->half_extents, i);
        if (o.shape == ne::Shape::Convex && b->verts) {
            for (uint32_t k = 0; k < b->vert_count[i]; ++k)
                o.vertices.push_back(v3(b->verts, b->vert_offset[i] + k));
        }
        if (o.shape == ne::Shape::Compound && b->child_shape) {
            for (uint32_t k = b->child_offset[i]; k < b->child_offset[i] + b->child_count[i]; ++k) {
                ne::ChildShape c;
                c.shape = static_cast<ne::Shape>(b->child_shape[k]);
                c.localPos = v3(b->child_pos, k);
                c.localRot = ne::Q{b->child_rot[4 * k], b->child_rot[4 * k + 1], b->child_rot[4 * k + 2],
                                   b->child_rot[4 * k + 3]};
                c.radius = b->child_radius[k];
                c.halfHeight = b->child_half_height[k];
                c.halfExtents = v3(b->child_half_extents, k);
                o.children.push_back(c);
            }
        }
        if (o.shape == ne::Shape::Mesh && b->meshes) {
            // The given BVH as ne::MeshData holds it (not rebuilt).
            const NeMeshData& m = b->meshes[b->mesh_index[i]];
            auto md = std::make_shared<ne::MeshData>();
            for (uint32_t k = 0; k < m.n_verts; ++k) md->verts.push_back(v3(m.verts, k));
            for (uint32_t k = 0; k < m.n_tris; ++k) md->tris.push_back({m.tris[3 * k], m.tris[3 * k + 1], m.tris[3 * k + 2]});
            md->order.assign(m.order, m.order + m.n_tris);
            for (uint32_t k = 0; k < m.n_nodes; ++k) {
                ne::MeshData::Node nd;
                nd.lo = v3(m.node_lo, k);
                nd.hi = v3(m.node_hi, k);
                nd.left = m.node_left[k];
                nd.right = m.node_right[k];
                nd.start = m.node_start[k];
                nd.count = m.node_count[k];
                md->nodes.push_back(nd);
            }
            o.mesh = md;
        }
        o.friction = b->friction[i];
        o.restitution = b->restitution[i];
        o.linearDamping = b->linear_damping[i];
        o.angularDamping = b->angular_damping[i];
        o.gravityScale = b->gravity_scale[i];
        o.layer = b->layer[i];
        o.mask = b->mask[i];
        const uint32_t f = b->flags[i];
        o.dynamic = (f & NE_BODY_DYNAMIC) != 0;
        o.sleeping = (f & NE_BODY_SLEEPING) != 0;
        o.kinematic = (f & NE_BODY_KINEMATIC) != 0;
        o.sensor = (f & NE_BODY_SENSOR) != 0;
        o.ccd = (f & NE_BODY_CCD) != 0;
        if (b->nocollide && b->nocollide_count) {
            for (uint32_t k = 0; k < b->nocollide_count[i]; ++k)
                o.noCollide.push_back(b->nocollide[b->nocollide_offset[i] + k]);
        }
    }
}

void computeIslands(RefWorld& r) {
    const std::size_t n = r.w.bodies.size();
    std::vector<std::size_t> parent(n);
    for (std::size_t i = 0; i < n; ++i) parent[i] = i;
    auto find = [&](std::size_t x) {
        while (parent[x] != x) x = parent[x];
        return x;
    };
    for (const auto& pr : r.w.islandPairs_) {
        std::size_t a = find(pr.first), b = find(pr.second);
        if (a == b) continue;
        if (a < b) parent[b] = a; else parent[a] = b;   // root = smallest index
    }
    r.islandLabel.resize(n);
    for (std::size_t i = 0; i < n; ++i) r.islandLabel[i] = (uint32_t)find(i);
}

// World::step() (src/world.cpp:133-146) with the pair list recorded in between.
void stepOnce(RefWorld& r) {
    ne::World& w = r.w;
    w.applyJointForces();
    for (ne::Body& b : w.bodies) { b.prevX = b.x; b.prevQ = b.q; }
    w.integrate();
    w.ccdPass();
    r.lastPairs = w.broadphasePairs();
    w.collide();
    w.solveRigidJoints(8);
    w.solveJoints(8);
    if (w.box.periodic)
        w.wrapPositions();
    else if (!w.openBoundary)
        w.applyWalls();
    if (w.sleepEnabled) w.updateSleep();
    computeIslands(r);
}

}  // namespace

extern "C" {

void* neref_create(const NeWorldParams* p, const NeBodyArrays* b) {
    auto* r = new RefWorld();
    applyParams(r->w, p);
    loadBodies(r->w, b);
    return r;
}

void neref_destroy(void* h) { delete static_cast<RefWorld*>(h); }

// The reference's own BVH of a triangle mesh (MeshData::build(),
// src/mesh.hpp:38-42), for giving the device the same mesh.  Returns the node
// count, or -1 when node_cap is too small.
int neref_mesh_build(const double* verts, uint32_t nv, const int32_t* tris, uint32_t nt, int32_t* order,
                     uint32_t node_cap, double* lo, double* hi, int32_t* left, int32_t* right, int32_t* start,
                     int32_t* count) {
    ne::MeshData md;
    for (uint32_t k = 0; k < nv; ++k) md.verts.push_back(v3(verts, k));
    for (uint32_t k = 0; k < nt; ++k) md.tris.push_back({tris[3 * k], tris[3 * k + 1], tris[3 * k + 2]});
    md.build();
    if (md.nodes.size() > node_cap) return -1;
    std::copy(md.order.begin(), md.order.end(), order);
    for (std::size_t k = 0; k < md.nodes.size(); ++k) {
        const ne::MeshData::Node& nd = md.nodes[k];
        lo[3 * k] = nd.lo.x; lo[3 * k + 1] = nd.lo.y; lo[3 * k + 2] = nd.lo.z;
        hi[3 * k] = nd.hi.x; hi[3 * k + 1] = nd.hi.y; hi[3 * k + 2] = nd.hi.z;
        left[k] = nd.left; right[k] = nd.right; start[k] = nd.start; count[k] = nd.count;
    }
    return (int)md.nodes.size();
}

void neref_set_params(void* h, const NeWorldParams* p) { applyParams(static_cast<RefWorld*>(h)->w, p); }

void neref_reset_warm_cache(void* h) { static_cast<RefWorld*>(h)->w.resetWarmCache(); }

// Plain World::step(), for timing the reference as it ships.
void neref_step_plain(void* h, uint32_t nsteps) {
    auto* r = static_cast<RefWorld*>(h);
    for (uint32_t s = 0; s < nsteps; ++s) r->w.step();
}

void neref_step(void* h, uint32_t nsteps) {
    auto* r = static_cast<RefWorld*>(h);
    for (uint32_t s = 0; s < nsteps; ++s) stepOnce(*r);
}

void neref_get_state(void* h, NeBodyArrays* out) {
    const ne::World& w = static_cast<RefWorld*>(h)->w;
    for (std::size_t i = 0; i < w.bodies.size() && i < out->n; ++i) {
        const ne::Body& b = w.bodies[i];
        if (out->x) { out->x[3 * i] = b.x.x; out->x[3 * i + 1] = b.x.y; out->x[3 * i + 2] = b.x.z; }
        if (out->q) { out->q[4 * i] = b.q.w; out->q[4 * i + 1] = b.q.x; out->q[4 * i + 2] = b.q.y; out->q[4 * i + 3] = b.q.z; }
        if (out->v) { out->v[3 * i] = b.v.x; out->v[3 * i + 1] = b.v.y; out->v[3 * i + 2] = b.v.z; }
        if (out->w) { out->w[3 * i] = b.w.x; out->w[3 * i + 1] = b.w.y; out->w[3 * i + 2] = b.w.z; }
    }
}

uint64_t neref_pairs(void* h, uint32_t* pi, uint32_t* pj, uint64_t cap) {
    const auto& P = static_cast<RefWorld*>(h)->lastPairs;
    for (uint64_t k = 0; k < P.size() && k < cap; ++k) { pi[k] = (uint32_t)P[k].first; pj[k] = (uint32_t)P[k].second; }
    return P.size();
}

// Broadphase of the current state, without stepping.
uint64_t neref_pairs_now(void* h, uint32_t* pi, uint32_t* pj, uint64_t cap) {
    auto P = static_cast<RefWorld*>(h)->w.broadphasePairs();
    for (uint64_t k = 0; k < P.size() && k < cap; ++k) { pi[k] = (uint32_t)P[k].first; pj[k] = (uint32_t)P[k].second; }
    return P.size();
}

// Contacts of the last step with their converged normal impulses (taken from
// the warm cache the step stored; 0 when warm starting is off).
uint64_t neref_contacts(void* h, NeContactArrays* out, uint64_t cap) {
    const ne::World& w = static_cast<RefWorld*>(h)->w;
    const auto& C = w.debugContacts;
    std::unordered_map<uint64_t, int> slotOf;
    for (uint64_t k = 0; k < C.size() && k < cap; ++k) {
        const ne::ContactViz& c = C[k];
        const uint64_t key = ((uint64_t)c.i << 32) | (uint32_t)c.j;
        int slot = slotOf[key]++;
        out->i[k] = (uint32_t)c.i;
        out->j[k] = (uint32_t)c.j;
        if (out->slot) out->slot[k] = (uint32_t)slot;
        out->point[3 * k] = c.point.x; out->point[3 * k + 1] = c.point.y; out->point[3 * k + 2] = c.point.z;
        out->normal[3 * k] = c.normal.x; out->normal[3 * k + 1] = c.normal.y; out->normal[3 * k + 2] = c.normal.z;
        out->depth[k] = c.depth;
        if (out->n_imp) {
            double imp = 0.0;
            auto it = w.warmCache_.find(key);
            if (it != w.warmCache_.end() && slot < (int)it->second.size()) imp = it->second[slot];
            out->n_imp[k] = imp;
        }
        if (out->t_imp) out->t_imp[k] = 0.0;   // not retained by the reference
    }
    return C.size();
}

void neref_islands(void* h, uint32_t* label, uint32_t n) {
    const auto& L = static_cast<RefWorld*>(h)->islandLabel;
    for (uint32_t i = 0; i < n && i < L.size(); ++i) label[i] = L[i];
}

// Narrowphase of one body pair (a = index ia, b = index ib) on the current
// state: the non-mesh, non-compound branch of gatherContacts
// (src/world.cpp:122-129).  Returns the number of contacts written (<= 4).
int neref_pair_contacts(void* h, uint32_t ia, uint32_t ib, double* point, double* normal, double* depth) {
    const ne::World& w = static_cast<RefWorld*>(h)->w;
    const ne::Body& a = w.bodies[ia];
    const ne::Body& b = w.bodies[ib];
    ne::Contact c = ne::detectContact(a, b, w.box);
    if (!c.hit) return 0;
    int n = 0;
    if (a.shape == ne::Shape::Box && b.shape == ne::Shape::Box) {
        ne::Manifold m = ne::boxBoxManifold(a, b, c.normal, w.box);
        for (int p = 0; p < m.count; ++p) {
            point[3 * p] = m.point[p].x; point[3 * p + 1] = m.point[p].y; point[3 * p + 2] = m.point[p].z;
            normal[3 * p] = c.normal.x; normal[3 * p + 1] = c.normal.y; normal[3 * p + 2] = c.normal.z;
            depth[p] = m.depth[p];
        }
        n = m.count;
    }
    if (n == 0) {
        point[0] = c.point.x; point[1] = c.point.y; point[2] = c.point.z;
        normal[0] = c.normal.x; normal[1] = c.normal.y; normal[2] = c.normal.z;
        depth[0] = c.overlap;
        n = 1;
    }
    return n;
}

// Aggregate diagnostics (src/world.cpp:704-729).
void neref_diagnostics(void* h, double* p3, double* l3, double* ke) {
    const ne::World& w = static_cast<RefWorld*>(h)->w;
    ne::V3 p = w.totalLinearMomentum(), l = w.totalAngularMomentum();
    p3[0] = p.x; p3[1] = p.y; p3[2] = p.z;
    l3[0] = l.x; l3[1] = l.y; l3[2] = l.z;
    *ke = w.totalKinetic();
}

// Mass properties from the reference's own factories (src/body.hpp:206-315),
// so that scene builders can be checked against them.  kind = NE_SHAPE_*;
// p = shape parameters (sphere r; cylinder r,height; box hx,hy,hz; capsule
// r,halfHeight; convex: verts[3*nv]).  Writes invMass and invInertia[3].
void neref_mass_props(int kind, const double* p, const double* verts, uint32_t nv, double density,
                      double* inv_mass, double* inv_inertia) {
    ne::Body b;
    switch (kind) {
        case NE_SHAPE_SPHERE: b = ne::makeSphere(0, ne::V3{}, p[0], density); break;
        case NE_SHAPE_CYLINDER: b = ne::makeCylinder(0, ne::V3{}, ne::Q{}, p[0], p[1], density); break;
        case NE_SHAPE_BOX: b = ne::makeBox(0, ne::V3{}, ne::Q{}, ne::V3{p[0], p[1], p[2]}, density); break;
        case NE_SHAPE_CAPSULE: b = ne::makeCapsule(0, ne::V3{}, ne::Q{}, p[0], p[1], density); break;
        case NE_SHAPE_CONVEX: {
            std::vector<ne::V3> vs;
            for (uint32_t k = 0; k < nv; ++k) vs.push_back(v3(verts, k));
            b = ne::makeConvex(0, ne::V3{}, ne::Q{}, vs, density);
            break;
        }
        default: b.invMass = 0.0; b.invInertiaBody = ne::V3{}; break;
    }
    *inv_mass = b.invMass;
    inv_inertia[0] = b.invInertiaBody.x; inv_inertia[1] = b.invInertiaBody.y; inv_inertia[2] = b.invInertiaBody.z;
}

// The README example (README.md:61-72) through the reference's own facade:
// returns the ball's y after 600 steps.
double neref_readme_example(void) {
    ne::PhysicsWorld w;
    w.setGravity({0.0, -9.81, 0.0});
    w.setTimestep(1.0 / 60.0);
    w.setOpenBoundary(true);
    w.setRestitution(0.2);
    w.setFriction(0.5);
    w.makeStatic(w.addBox({0.0, -1.0, 0.0}, {}, {50.0, 1.0, 50.0}, 1.0));
    ne::BodyId ball = w.addSphere({0.0, 10.0, 0.0}, 0.5, 1.0);
    for (int i = 0; i < 600; ++i) w.step();
    return w.position(ball).y;
}

}  // extern "C"
