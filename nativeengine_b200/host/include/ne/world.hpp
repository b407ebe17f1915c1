// ne/world.hpp -- the host C++17 facade of the B200 step path.
//
// ne::Body, ne::Box, ne::World and ne::PhysicsWorld keep the reference's
// public interface (src/body.hpp:24-130, 206-345; src/box.hpp:16-42;
// src/world.hpp:73-145; src/physics_world.hpp:45-246): the same fields, the
// same factories with the same mass formulas, the same defaults.  The one
// difference is where World::step() runs: the bodies are mirrored into a
// device world (include/ne_cuda.h) and stepped on the GPU, then the state is
// copied back into World::bodies.  Features the device path does not run
// (joints, sleeping, CCD) make step() throw ne::DeviceError instead of
// silently skipping them; there is no CPU path.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "ne/vmath.hpp"

struct NeWorld;

namespace ne {

enum class Shape { Sphere, Cylinder, Box, Capsule, Convex, Plane, Mesh, Compound };

// A child primitive of a compound body in the parent's frame (src/body.hpp:28-39).
struct ChildShape {
    Shape shape = Shape::Sphere;
    V3 localPos;
    Q localRot{1, 0, 0, 0};
    double radius = 1.0;
    double halfHeight = 0.0;
    V3 halfExtents;
    static ChildShape sphere(const V3& p, double r);
    static ChildShape box(const V3& p, const Q& q, const V3& he);
    static ChildShape cylinder(const V3& p, const Q& q, double r, double hh);
    static ChildShape capsule(const V3& p, const Q& q, double r, double hh);
};

// A static triangle mesh with an AABB BVH (src/mesh.hpp:14-26).  build()
// makes the reference's tree (median split of the triangle centroids along
// the longest axis, leaves of at most 4), so contacts come in its order.
struct MeshData {
    struct Tri { int a, b, c; };
    struct Node {
        V3 lo, hi;
        int left = -1, right = -1;
        int start = 0, count = 0;
    };
    std::vector<V3> verts;
    std::vector<Tri> tris;
    std::vector<int> order;
    std::vector<Node> nodes;
    void build();
};

struct Body {
    V3 x, v;
    Q q{1, 0, 0, 0};
    V3 w;
    V3 force, torque;
    double invMass = 0.0;
    V3 invInertiaBody;
    Shape shape = Shape::Sphere;
    double radius = 1.0;
    double halfHeight = 0.0;
    V3 halfExtents;
    std::vector<V3> vertices;
    std::shared_ptr<const MeshData> mesh;     // Mesh only
    std::vector<ChildShape> children;         // Compound only
    int id = -1;
    double friction = -1.0, restitution = -1.0;
    double linearDamping = 0.0, angularDamping = 0.0;
    double gravityScale = 1.0;
    std::uint32_t layer = 0, mask = 0xFFFFFFFFu;
    std::vector<std::uint32_t> noCollide;
    std::uint64_t userData = 0;
    bool dynamic = true, sleeping = false;
    double sleepTimer = 0.0;
    bool kinematic = false, sensor = false, ccd = false;
    V3 prevX;
    Q prevQ{1, 0, 0, 0};
};

// Factories: the reference's mass / inertia formulas, operation for operation.
Body makeSphere(int id, const V3& x, double radius, double density);
Body makeCylinder(int id, const V3& x, const Q& q, double radius, double height, double density);
Body makeBox(int id, const V3& x, const Q& q, const V3& halfExtents, double density);
Body makeCapsule(int id, const V3& x, const Q& q, double radius, double halfHeight, double density);
Body makeConvex(int id, const V3& x, const Q& q, std::vector<V3> verts, double density);
Body makePlane(int id, const V3& point, const V3& normal);
Body makeMesh(int id, const V3& point, const Q& q, std::shared_ptr<const MeshData> data);
Body makeCompound(int id, const V3& x, const Q& q, std::vector<ChildShape> children, double density);

struct Box {
    double half = 12.0;
    bool periodic = false;
    double edge() const { return 2.0 * half; }
    V3 minImage(V3 d) const {
        if (!periodic) return d;
        const double L = edge();
        d.x -= L * std::floor(d.x / L + 0.5);
        d.y -= L * std::floor(d.y / L + 0.5);
        d.z -= L * std::floor(d.z / L + 0.5);
        return d;
    }
    V3 wrap(V3 p) const {
        if (!periodic) return p;
        const double L = edge();
        p.x -= L * std::floor((p.x + half) / L);
        p.y -= L * std::floor((p.y + half) / L);
        p.z -= L * std::floor((p.z + half) / L);
        return p;
    }
};

struct ContactViz {
    V3 point, normal;
    double depth = 0.0;
    std::size_t i = 0, j = 0;
};

class DeviceError : public std::runtime_error {
public:
    DeviceError(int code, const std::string& what) : std::runtime_error(what), code(code) {}
    int code;
};

class World {
public:
    World();
    ~World();
    World(const World&) = delete;
    World& operator=(const World&) = delete;

    Box box;
    double dt = 1.0 / 120.0;
    double restitution = 1.0;
    double friction = 0.0;
    double contactBeta = 0.2;
    V3 gravity;
    enum class Combine { Average, Min, Max, Multiply, GeometricMean };
    Combine restitutionCombine = Combine::Max;
    Combine frictionCombine = Combine::GeometricMean;
    bool sleepEnabled = false;
    double sleepLinVel = 0.05, sleepAngVel = 0.05, sleepTime = 0.5, wakeVel = 0.5;
    bool openBoundary = false;
    bool warmStart = true;
    bool forceBruteForce = false;
    std::vector<Body> bodies;
    std::size_t distanceJointCount = 0;   // joints are not on the device path (must stay 0)
    bool captureContacts = false;
    std::vector<ContactViz> debugContacts;

    // One World::step() on the device: mirrors `bodies` in, steps, copies
    // x/q/v/w (and the cleared force/torque accumulators) back.
    void step();
    // Advance n steps on the device without copying state back in between;
    // call syncFromDevice() to refresh `bodies`.  `bodies` must not be edited
    // in between.
    void stepDevice(std::uint32_t n);
    void syncFromDevice();
    void resetWarmCache();

    V3 totalLinearMomentum() const;
    double totalKinetic() const;

private:
    void upload();
    NeWorld* dev_ = nullptr;
};

using BodyId = std::uint32_t;
constexpr BodyId kInvalidBody = 0;

// Handle-based facade (src/physics_world.hpp:45-246), the part that drives
// step(): configuration, body creation, static/kinematic, removal with
// swap-and-pop, accessors and setters.
class PhysicsWorld {
public:
    void setBox(double half, bool periodic) { w_.box.half = half; w_.box.periodic = periodic; }
    void setOpenBoundary(bool on) { w_.openBoundary = on; }
    void setTimestep(double dt) { w_.dt = dt; }
    void setRestitution(double e) { w_.restitution = e; }
    void setFriction(double mu) { w_.friction = mu; }
    void setGravity(const V3& g) { w_.gravity = g; }
    double timestep() const { return w_.dt; }

    BodyId addSphere(const V3& pos, double radius, double density) { return add(makeSphere(0, pos, radius, density)); }
    BodyId addBox(const V3& pos, const Q& rot, const V3& he, double density) { return add(makeBox(0, pos, rot, he, density)); }
    BodyId addCylinder(const V3& pos, const Q& rot, double r, double h, double density) {
        return add(makeCylinder(0, pos, rot, r, h, density));
    }
    BodyId addCapsule(const V3& pos, const Q& rot, double r, double hh, double density) {
        return add(makeCapsule(0, pos, rot, r, hh, density));
    }
    BodyId addConvex(const V3& pos, const Q& rot, const std::vector<V3>& verts, double density) {
        return add(makeConvex(0, pos, rot, verts, density));
    }
    BodyId addPlane(const V3& point, const V3& normal) { return add(makePlane(0, point, normal)); }
    BodyId addCompound(const V3& pos, const Q& rot, const std::vector<ChildShape>& children, double density) {
        return add(makeCompound(0, pos, rot, children, density));
    }
    // A static triangle mesh: verts + flat indices (triples); the BVH is built here.
    BodyId addMesh(const V3& pos, const Q& rot, const std::vector<V3>& verts, const std::vector<int>& indices);
    // A rows x cols height grid (row-major, spacing in x/z) as a static mesh.
    BodyId addHeightfield(const V3& origin, double spacing, int rows, int cols, const std::vector<double>& heights);

    BodyId makeStatic(BodyId h);
    BodyId makeKinematic(BodyId h);
    void remove(BodyId h);
    void step() { w_.step(); }

    bool valid(BodyId h) const { return slot_.count(h) != 0; }
    V3 position(BodyId h) const { const Body* b = body(h); return b ? b->x : V3{}; }
    Q orientation(BodyId h) const { const Body* b = body(h); return b ? b->q : Q{}; }
    V3 velocity(BodyId h) const { const Body* b = body(h); return b ? b->v : V3{}; }
    V3 angularVelocity(BodyId h) const { const Body* b = body(h); return b ? b->w : V3{}; }
    void setPosition(BodyId h, const V3& p) { if (Body* b = body(h)) b->x = p; }
    void setVelocity(BodyId h, const V3& v) { if (Body* b = body(h)) b->v = v; }
    void setAngularVelocity(BodyId h, const V3& w) { if (Body* b = body(h)) b->w = w; }
    void applyImpulse(BodyId h, const V3& J) { if (Body* b = body(h)) b->v += J * b->invMass; }

    World& world() { return w_; }
    const World& world() const { return w_; }
    std::size_t bodyCount() const { return w_.bodies.size(); }

private:
    BodyId add(Body b);
    Body* body(BodyId h) {
        auto it = slot_.find(h);
        return it == slot_.end() ? nullptr : &w_.bodies[it->second];
    }
    const Body* body(BodyId h) const {
        auto it = slot_.find(h);
        return it == slot_.end() ? nullptr : &w_.bodies[it->second];
    }
    World w_;
    std::unordered_map<BodyId, std::size_t> slot_;
    std::vector<BodyId> handle_;
    BodyId next_ = 1;
};

}  // namespace ne
