// world.cpp -- host facade implementation: factories, body mirroring, and
// World::step() through the C-ABI of libne_cuda.so.
#include "ne/world.hpp"

#include <algorithm>
#include <cstring>

#include "ne_cuda.h"

namespace ne {

namespace {

double inv(double v) { return v > 0 ? 1.0 / v : 0.0; }

void check(int rc, const char* where) {
    if (rc != NE_OK && rc != NE_ERR_NUMERIC)
        throw DeviceError(rc, std::string(where) + ": " + ne_status_string(rc) + ": " + ne_last_error());
}

}  // namespace

// ---- factories (src/body.hpp:206-345) -------------------------------------

Body makeSphere(int id, const V3& x, double radius, double density) {
    Body b;
    b.shape = Shape::Sphere;
    b.id = id;
    b.x = x;
    b.radius = radius;
    const double m = density * (4.0 / 3.0) * PI * radius * radius * radius;
    b.invMass = inv(m);
    const double I = (2.0 / 5.0) * m * radius * radius;
    b.invInertiaBody = {inv(I), inv(I), inv(I)};
    return b;
}

Body makeCylinder(int id, const V3& x, const Q& q, double radius, double height, double density) {
    Body b;
    b.shape = Shape::Cylinder;
    b.id = id;
    b.x = x;
    b.q = q;
    b.radius = radius;
    b.halfHeight = 0.5 * height;
    const double m = density * PI * radius * radius * height;
    b.invMass = inv(m);
    const double Iyy = 0.5 * m * radius * radius;
    const double Ixx = (1.0 / 12.0) * m * (3.0 * radius * radius + height * height);
    b.invInertiaBody = {inv(Ixx), inv(Iyy), inv(Ixx)};
    return b;
}

Body makeBox(int id, const V3& x, const Q& q, const V3& he, double density) {
    Body b;
    b.shape = Shape::Box;
    b.id = id;
    b.x = x;
    b.q = q;
    b.halfExtents = he;
    const double hx = he.x, hy = he.y, hz = he.z;
    const double m = density * 8.0 * hx * hy * hz;
    b.invMass = inv(m);
    b.invInertiaBody = {inv((1.0 / 3.0) * m * (hy * hy + hz * hz)), inv((1.0 / 3.0) * m * (hx * hx + hz * hz)),
                        inv((1.0 / 3.0) * m * (hx * hx + hy * hy))};
    return b;
}

Body makeCapsule(int id, const V3& x, const Q& q, double radius, double halfHeight, double density) {
    Body b;
    b.shape = Shape::Capsule;
    b.id = id;
    b.x = x;
    b.q = q;
    b.radius = radius;
    b.halfHeight = halfHeight;
    const double r = radius, L = 2.0 * halfHeight;
    const double mc = density * PI * r * r * L;
    const double mh = density * (4.0 / 3.0) * PI * r * r * r;
    const double m = mc + mh;
    b.invMass = inv(m);
    const double Iyy = 0.5 * mc * r * r + 0.4 * mh * r * r;
    const double Ixx = mc * (0.25 * r * r + L * L / 12.0) + mh * (0.4 * r * r + 0.25 * L * L);
    b.invInertiaBody = {inv(Ixx), inv(Iyy), inv(Ixx)};
    return b;
}

Body makeConvex(int id, const V3& x, const Q& q, std::vector<V3> verts, double density) {
    Body b;
    b.shape = Shape::Convex;
    b.id = id;
    b.x = x;
    b.q = q;
    b.vertices = std::move(verts);
    V3 lo{1e30, 1e30, 1e30}, hi{-1e30, -1e30, -1e30};
    for (const V3& v : b.vertices) {
        lo = V3{std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z)};
        hi = V3{std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z)};
    }
    const V3 he = (hi - lo) * 0.5;
    const double hx = std::max(he.x, 1e-4), hy = std::max(he.y, 1e-4), hz = std::max(he.z, 1e-4);
    const double m = density * 8.0 * hx * hy * hz;
    b.invMass = inv(m);
    b.invInertiaBody = {inv((1.0 / 3.0) * m * (hy * hy + hz * hz)), inv((1.0 / 3.0) * m * (hx * hx + hz * hz)),
                        inv((1.0 / 3.0) * m * (hx * hx + hy * hy))};
    return b;
}

Body makePlane(int id, const V3& point, const V3& normal) {
    Body b;
    b.shape = Shape::Plane;
    b.id = id;
    b.x = point;
    b.halfExtents = normal.normalized();
    b.invMass = 0.0;
    b.invInertiaBody = {0, 0, 0};
    b.dynamic = false;
    return b;
}

ChildShape ChildShape::sphere(const V3& p, double r) {
    ChildShape c;
    c.shape = Shape::Sphere; c.localPos = p; c.radius = r;
    return c;
}
ChildShape ChildShape::box(const V3& p, const Q& q, const V3& he) {
    ChildShape c;
    c.shape = Shape::Box; c.localPos = p; c.localRot = q; c.halfExtents = he;
    return c;
}
ChildShape ChildShape::cylinder(const V3& p, const Q& q, double r, double hh) {
    ChildShape c;
    c.shape = Shape::Cylinder; c.localPos = p; c.localRot = q; c.radius = r; c.halfHeight = hh;
    return c;
}
ChildShape ChildShape::capsule(const V3& p, const Q& q, double r, double hh) {
    ChildShape c;
    c.shape = Shape::Capsule; c.localPos = p; c.localRot = q; c.radius = r; c.halfHeight = hh;
    return c;
}

namespace {

void tri_bounds(const MeshData& m, int t, V3& lo, V3& hi) {
    const V3 a = m.verts[m.tris[t].a], b = m.verts[m.tris[t].b], c = m.verts[m.tris[t].c];
    lo = {std::min({a.x, b.x, c.x}), std::min({a.y, b.y, c.y}), std::min({a.z, b.z, c.z})};
    hi = {std::max({a.x, b.x, c.x}), std::max({a.y, b.y, c.y}), std::max({a.z, b.z, c.z})};
}

// Node over order[start, start + count): its bounds; a leaf at <= 4
// triangles, else split at the median centroid (lo + hi) of the longest axis.
int build_node(MeshData& m, int start, int count) {
    const int idx = static_cast<int>(m.nodes.size());
    m.nodes.emplace_back();
    V3 lo{1e30, 1e30, 1e30}, hi{-1e30, -1e30, -1e30};
    for (int k = 0; k < count; ++k) {
        V3 tl, th;
        tri_bounds(m, m.order[start + k], tl, th);
        lo = {std::min(lo.x, tl.x), std::min(lo.y, tl.y), std::min(lo.z, tl.z)};
        hi = {std::max(hi.x, th.x), std::max(hi.y, th.y), std::max(hi.z, th.z)};
    }
    MeshData::Node nd;
    nd.lo = lo;
    nd.hi = hi;
    if (count <= 4) {
        nd.start = start;
        nd.count = count;
        m.nodes[idx] = nd;
        return idx;
    }
    const V3 ext = hi - lo;
    const int axis = (ext.x > ext.y && ext.x > ext.z) ? 0 : (ext.y > ext.z ? 1 : 2);
    auto centre = [&](int t) {
        V3 tl, th;
        tri_bounds(m, t, tl, th);
        return axis == 0 ? tl.x + th.x : (axis == 1 ? tl.y + th.y : tl.z + th.z);
    };
    const int mid = start + count / 2;
    std::nth_element(m.order.begin() + start, m.order.begin() + mid, m.order.begin() + start + count,
                     [&](int p, int q) { return centre(p) < centre(q); });
    const int l = build_node(m, start, mid - start);
    const int r = build_node(m, mid, start + count - mid);
    nd.left = l;
    nd.right = r;
    m.nodes[idx] = nd;
    return idx;
}

}  // namespace

void MeshData::build() {
    order.resize(tris.size());
    for (size_t k = 0; k < tris.size(); ++k) order[k] = static_cast<int>(k);
    nodes.clear();
    if (!tris.empty()) build_node(*this, 0, static_cast<int>(tris.size()));
}

Body makeMesh(int id, const V3& point, const Q& q, std::shared_ptr<const MeshData> data) {
    Body b;
    b.shape = Shape::Mesh;
    b.id = id;
    b.x = point;
    b.q = q;
    b.mesh = std::move(data);
    b.invMass = 0.0;
    b.invInertiaBody = {0, 0, 0};
    b.dynamic = false;
    return b;
}

// Mass sums the children; the inertia is the diagonal of the summed tensor by
// the parallel-axis theorem (src/body.hpp:368-400).
Body makeCompound(int id, const V3& x, const Q& q, std::vector<ChildShape> children, double density) {
    Body b;
    b.shape = Shape::Compound;
    b.id = id;
    b.x = x;
    b.q = q;
    b.children = std::move(children);
    double M = 0.0;
    V3 I;
    for (const ChildShape& ch : b.children) {
        Body t;
        switch (ch.shape) {
            case Shape::Box: t = makeBox(0, V3{}, Q{1, 0, 0, 0}, ch.halfExtents, density); break;
            case Shape::Cylinder: t = makeCylinder(0, V3{}, Q{1, 0, 0, 0}, ch.radius, 2.0 * ch.halfHeight, density); break;
            case Shape::Capsule: t = makeCapsule(0, V3{}, Q{1, 0, 0, 0}, ch.radius, ch.halfHeight, density); break;
            default: t = makeSphere(0, V3{}, ch.radius, density); break;
        }
        const double mc = (t.invMass > 0) ? 1.0 / t.invMass : 0.0;
        const V3 Ic{t.invInertiaBody.x > 0 ? 1.0 / t.invInertiaBody.x : 0.0,
                    t.invInertiaBody.y > 0 ? 1.0 / t.invInertiaBody.y : 0.0,
                    t.invInertiaBody.z > 0 ? 1.0 / t.invInertiaBody.z : 0.0};
        const V3 o = ch.localPos;
        M += mc;
        I.x += Ic.x + mc * (o.y * o.y + o.z * o.z);
        I.y += Ic.y + mc * (o.x * o.x + o.z * o.z);
        I.z += Ic.z + mc * (o.x * o.x + o.y * o.y);
    }
    b.invMass = (M > 0) ? 1.0 / M : 0.0;
    b.invInertiaBody = {I.x > 0 ? 1.0 / I.x : 0.0, I.y > 0 ? 1.0 / I.y : 0.0, I.z > 0 ? 1.0 / I.z : 0.0};
    return b;
}

BodyId PhysicsWorld::addMesh(const V3& pos, const Q& rot, const std::vector<V3>& verts,
                             const std::vector<int>& indices) {
    auto md = std::make_shared<MeshData>();
    md->verts = verts;
    for (size_t k = 0; k + 2 < indices.size(); k += 3) md->tris.push_back({indices[k], indices[k + 1], indices[k + 2]});
    md->build();
    return add(makeMesh(0, pos, rot, md));
}

BodyId PhysicsWorld::addHeightfield(const V3& origin, double spacing, int rows, int cols,
                                    const std::vector<double>& heights) {
    std::vector<V3> verts;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c)
            verts.push_back(V3{origin.x + c * spacing, origin.y + heights[(size_t)r * cols + c], origin.z + r * spacing});
    std::vector<int> idx;
    for (int r = 0; r + 1 < rows; ++r)
        for (int c = 0; c + 1 < cols; ++c) {
            const int a = r * cols + c, b = a + 1, d = a + cols, e = d + 1;
            idx.insert(idx.end(), {a, d, b, b, d, e});
        }
    return addMesh(V3{0, 0, 0}, Q{1, 0, 0, 0}, verts, idx);
}

// ---- World ----------------------------------------------------------------

namespace {

NeWorldParams params_of(const World& w) {
    NeWorldParams p;
    ne_world_params_default(&p);
    p.half = w.box.half;
    p.periodic = w.box.periodic ? 1 : 0;
    p.open_boundary = w.openBoundary ? 1 : 0;
    p.dt = w.dt;
    p.restitution = w.restitution;
    p.friction = w.friction;
    p.contact_beta = w.contactBeta;
    p.gravity[0] = w.gravity.x;
    p.gravity[1] = w.gravity.y;
    p.gravity[2] = w.gravity.z;
    p.restitution_combine = static_cast<int32_t>(w.restitutionCombine);
    p.friction_combine = static_cast<int32_t>(w.frictionCombine);
    p.warm_start = w.warmStart ? 1 : 0;
    p.force_brute_force = w.forceBruteForce ? 1 : 0;
    p.capture_contacts = w.captureContacts ? 1 : 0;
    p.sleep_enabled = w.sleepEnabled ? 1 : 0;
    p.sleep_lin_vel = w.sleepLinVel;
    p.sleep_ang_vel = w.sleepAngVel;
    p.sleep_time = w.sleepTime;
    p.wake_vel = w.wakeVel;
    p.n_distance_joints = static_cast<uint32_t>(w.distanceJointCount);
    return p;
}

// Structure-of-arrays image of World::bodies for the C-ABI.
struct Packed {
    std::vector<double> x, q, v, w, f, t, im, ii, r, hh, he, verts, fr, re, ld, ad, gs;
    std::vector<int32_t> shape;
    std::vector<uint32_t> vo, vc, layer, mask, flags, no, nc, nl;
    // compound children and meshes
    std::vector<uint32_t> co, cc, mi;
    std::vector<int32_t> cs;
    std::vector<double> cp, cr, crad, chh, che;
    struct MeshArrays {
        const MeshData* src = nullptr;
        std::vector<double> verts, lo, hi;
        std::vector<int32_t> tris, order, left, right, start, count;
    };
    std::vector<MeshArrays> marr;
    std::vector<NeMeshData> meshes;
    NeBodyArrays view{};

    explicit Packed(const std::vector<Body>& B) {
        const size_t n = B.size();
        for (const Body& b : B) {
            const double s3[][3] = {{b.x.x, b.x.y, b.x.z}, {b.v.x, b.v.y, b.v.z}, {b.w.x, b.w.y, b.w.z},
                                    {b.force.x, b.force.y, b.force.z}, {b.torque.x, b.torque.y, b.torque.z},
                                    {b.invInertiaBody.x, b.invInertiaBody.y, b.invInertiaBody.z},
                                    {b.halfExtents.x, b.halfExtents.y, b.halfExtents.z}};
            std::vector<double>* d3[] = {&x, &v, &w, &f, &t, &ii, &he};
            for (int k = 0; k < 7; ++k) d3[k]->insert(d3[k]->end(), s3[k], s3[k] + 3);
            q.insert(q.end(), {b.q.w, b.q.x, b.q.y, b.q.z});
            im.push_back(b.invMass);
            shape.push_back(static_cast<int32_t>(b.shape));
            r.push_back(b.radius);
            hh.push_back(b.halfHeight);
            vo.push_back(static_cast<uint32_t>(verts.size() / 3));
            vc.push_back(static_cast<uint32_t>(b.vertices.size()));
            for (const V3& p : b.vertices) verts.insert(verts.end(), {p.x, p.y, p.z});
            fr.push_back(b.friction);
            re.push_back(b.restitution);
            ld.push_back(b.linearDamping);
            ad.push_back(b.angularDamping);
            gs.push_back(b.gravityScale);
            layer.push_back(b.layer);
            mask.push_back(b.mask);
            flags.push_back((b.dynamic ? NE_BODY_DYNAMIC : 0u) | (b.sleeping ? NE_BODY_SLEEPING : 0u) |
                            (b.kinematic ? NE_BODY_KINEMATIC : 0u) | (b.sensor ? NE_BODY_SENSOR : 0u) |
                            (b.ccd ? NE_BODY_CCD : 0u));
            no.push_back(static_cast<uint32_t>(nl.size()));
            nc.push_back(static_cast<uint32_t>(b.noCollide.size()));
            nl.insert(nl.end(), b.noCollide.begin(), b.noCollide.end());
            co.push_back(static_cast<uint32_t>(cs.size()));
            cc.push_back(static_cast<uint32_t>(b.children.size()));
            for (const ChildShape& c : b.children) {
                cs.push_back(static_cast<int32_t>(c.shape));
                cp.insert(cp.end(), {c.localPos.x, c.localPos.y, c.localPos.z});
                cr.insert(cr.end(), {c.localRot.w, c.localRot.x, c.localRot.y, c.localRot.z});
                crad.push_back(c.radius);
                chh.push_back(c.halfHeight);
                che.insert(che.end(), {c.halfExtents.x, c.halfExtents.y, c.halfExtents.z});
            }
            mi.push_back(static_cast<uint32_t>(marr.size()));
            if (b.shape == Shape::Mesh && b.mesh) {
                const MeshData& md = *b.mesh;
                MeshArrays a;
                a.src = &md;
                for (const V3& p : md.verts) a.verts.insert(a.verts.end(), {p.x, p.y, p.z});
                for (const MeshData::Tri& t3 : md.tris) a.tris.insert(a.tris.end(), {t3.a, t3.b, t3.c});
                a.order = md.order;
                for (const MeshData::Node& nd : md.nodes) {
                    a.lo.insert(a.lo.end(), {nd.lo.x, nd.lo.y, nd.lo.z});
                    a.hi.insert(a.hi.end(), {nd.hi.x, nd.hi.y, nd.hi.z});
                    a.left.push_back(nd.left); a.right.push_back(nd.right);
                    a.start.push_back(nd.start); a.count.push_back(nd.count);
                }
                marr.push_back(std::move(a));
            } else {
                mi.back() = 0;
            }
        }
        for (size_t k = 0; k < marr.size(); ++k) {
            const MeshArrays& a = marr[k];
            const MeshData& md = *a.src;
            NeMeshData m{};
            m.n_verts = static_cast<uint32_t>(md.verts.size());
            m.verts = a.verts.data();
            m.n_tris = static_cast<uint32_t>(md.tris.size());
            m.tris = a.tris.data();
            m.order = a.order.data();
            m.n_nodes = static_cast<uint32_t>(md.nodes.size());
            m.node_lo = a.lo.data(); m.node_hi = a.hi.data();
            m.node_left = a.left.data(); m.node_right = a.right.data();
            m.node_start = a.start.data(); m.node_count = a.count.data();
            meshes.push_back(m);
        }
        if (verts.empty()) verts.assign(3, 0.0);
        if (nl.empty()) nl.push_back(0);
        view.n = static_cast<uint32_t>(n);
        view.x = x.data(); view.q = q.data(); view.v = v.data(); view.w = w.data();
        view.force = f.data(); view.torque = t.data();
        view.inv_mass = im.data(); view.inv_inertia = ii.data();
        view.shape = shape.data(); view.radius = r.data(); view.half_height = hh.data(); view.half_extents = he.data();
        view.vert_offset = vo.data(); view.vert_count = vc.data(); view.verts = verts.data();
        view.n_verts = static_cast<uint32_t>(verts.size() / 3);
        view.friction = fr.data(); view.restitution = re.data();
        view.linear_damping = ld.data(); view.angular_damping = ad.data(); view.gravity_scale = gs.data();
        view.layer = layer.data(); view.mask = mask.data(); view.flags = flags.data();
        view.nocollide_offset = no.data(); view.nocollide_count = nc.data(); view.nocollide = nl.data();
        view.n_nocollide = static_cast<uint32_t>(nl.size());
        if (!cs.empty()) {
            view.child_offset = co.data(); view.child_count = cc.data();
            view.n_children = static_cast<uint32_t>(cs.size());
            view.child_shape = cs.data(); view.child_pos = cp.data(); view.child_rot = cr.data();
            view.child_radius = crad.data(); view.child_half_height = chh.data(); view.child_half_extents = che.data();
        }
        if (!meshes.empty()) {
            view.mesh_index = mi.data();
            view.n_meshes = static_cast<uint32_t>(meshes.size());
            view.meshes = meshes.data();
        }
    }
};

}  // namespace

World::World() = default;

World::~World() {
    if (dev_) ne_world_destroy(dev_);
}

void World::upload() {
    const NeWorldParams p = params_of(*this);
    if (!dev_) check(ne_world_create(&p, &dev_), "ne_world_create");
    else check(ne_world_set_params(dev_, &p), "ne_world_set_params");
    Packed pk(bodies);
    check(ne_world_upload(dev_, &pk.view), "ne_world_upload");
}

void World::syncFromDevice() {
    if (!dev_) return;
    const size_t n = bodies.size();
    std::vector<double> x(3 * n), q(4 * n), v(3 * n), w(3 * n), f(3 * n), t(3 * n);
    NeBodyArrays out{};
    out.n = static_cast<uint32_t>(n);
    out.x = x.data(); out.q = q.data(); out.v = v.data(); out.w = w.data(); out.force = f.data(); out.torque = t.data();
    check(ne_world_download(dev_, &out), "ne_world_download");
    for (size_t i = 0; i < n; ++i) {
        Body& b = bodies[i];
        b.prevX = b.x;
        b.prevQ = b.q;
        b.x = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        b.q = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
        b.v = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        b.w = {w[3 * i], w[3 * i + 1], w[3 * i + 2]};
        b.force = {f[3 * i], f[3 * i + 1], f[3 * i + 2]};
        b.torque = {t[3 * i], t[3 * i + 1], t[3 * i + 2]};
    }
    if (captureContacts) {
        uint64_t cnt = 0;
        NeContactArrays none{};
        check(ne_world_contacts(dev_, &none, 0, &cnt), "ne_world_contacts");
        std::vector<uint32_t> ci(cnt), cj(cnt);
        std::vector<double> pt(3 * cnt), nr(3 * cnt), dp(cnt);
        NeContactArrays ca{};
        ca.i = ci.data(); ca.j = cj.data(); ca.point = pt.data(); ca.normal = nr.data(); ca.depth = dp.data();
        check(ne_world_contacts(dev_, &ca, cnt, &cnt), "ne_world_contacts");
        debugContacts.clear();
        for (uint64_t k = 0; k < cnt; ++k)
            debugContacts.push_back({{pt[3 * k], pt[3 * k + 1], pt[3 * k + 2]},
                                     {nr[3 * k], nr[3 * k + 1], nr[3 * k + 2]}, dp[k], ci[k], cj[k]});
    }
}

void World::step() {
    upload();
    check(ne_world_step(dev_, 1), "ne_world_step");
    syncFromDevice();
}

void World::stepDevice(std::uint32_t n) {
    upload();
    check(ne_world_step(dev_, n), "ne_world_step");
}

void World::resetWarmCache() {
    if (dev_) check(ne_world_reset_warm_cache(dev_), "ne_world_reset_warm_cache");
}

V3 World::totalLinearMomentum() const {
    V3 p;
    for (const Body& b : bodies)
        if (b.invMass > 0.0) p += b.v * (1.0 / b.invMass);
    return p;
}

double World::totalKinetic() const {
    double e = 0.0;
    for (const Body& b : bodies) {
        if (!(b.invMass > 0.0)) continue;
        const double lin = 0.5 * (1.0 / b.invMass) * b.v.norm2();
        const V3 Ib{inv(b.invInertiaBody.x), inv(b.invInertiaBody.y), inv(b.invInertiaBody.z)};
        const V3 wb = b.q.inverseRotate(b.w);
        const V3 Lb{wb.x * Ib.x, wb.y * Ib.y, wb.z * Ib.z};
        e += lin + 0.5 * wb.dot(Lb);
    }
    return e;
}

// ---- PhysicsWorld -----------------------------------------------------------

BodyId PhysicsWorld::add(Body b) {
    const BodyId h = next_++;
    slot_[h] = w_.bodies.size();
    handle_.push_back(h);
    w_.bodies.push_back(std::move(b));
    return h;
}

BodyId PhysicsWorld::makeStatic(BodyId h) {
    if (Body* b = body(h)) {
        b->invMass = 0.0;
        b->invInertiaBody = {0, 0, 0};
        b->v = {};
        b->w = {};
        b->dynamic = false;
        b->kinematic = false;
    }
    return h;
}

BodyId PhysicsWorld::makeKinematic(BodyId h) {
    if (Body* b = body(h)) {
        b->invMass = 0.0;
        b->invInertiaBody = {0, 0, 0};
        b->dynamic = false;
        b->kinematic = true;
        b->sleeping = false;
    }
    return h;
}

// Swap-and-pop removal with noCollide index remapping (src/physics_world.hpp:143-165).
void PhysicsWorld::remove(BodyId h) {
    auto it = slot_.find(h);
    if (it == slot_.end()) return;
    const size_t s = it->second, last = w_.bodies.size() - 1;
    for (Body& b : w_.bodies) {
        auto& nc = b.noCollide;
        nc.erase(std::remove(nc.begin(), nc.end(), static_cast<uint32_t>(s)), nc.end());
        if (s != last)
            for (uint32_t& e : nc)
                if (e == static_cast<uint32_t>(last)) e = static_cast<uint32_t>(s);
    }
    if (s != last) {
        w_.bodies[s] = w_.bodies[last];
        const BodyId moved = handle_[last];
        handle_[s] = moved;
        slot_[moved] = s;
    }
    w_.bodies.pop_back();
    handle_.pop_back();
    slot_.erase(it);
}

}  // namespace ne
