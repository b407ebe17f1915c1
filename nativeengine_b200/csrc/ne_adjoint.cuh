// ne_adjoint.cuh -- one world's step() as a sequential program (forward, with
// an optional tape) and its hand-written adjoint (reverse mode).
//
// The forward is the reference's step (src/world.cpp:133-146) for one world,
// evaluated in the reference's order: integrate (world.cpp:373-411); every
// pair i < j that passes the filters and the conservative cull, through the
// narrowphase (detect.hpp:33-77, manifold.hpp:90-126) in sorted pair order;
// constraints with warm start (world.cpp:537-568); 8 sequential-impulse sweeps
// (world.cpp:572-612); position correction (contact.hpp:78-85); the warm cache
// (world.cpp:619-626); wrap (world.cpp:698-702).  Islands are independent, so
// one sequential pass over the world's contacts is the reference's global
// pass; every expression is the device kernels' (ne_step.cu), so the result
// is bit-identical to the device step and to the reference.
//
// The adjoint reverses that program: given the adjoint of the state after
// the step (x, q, v, w) and of the warm impulses it stores, it returns the
// adjoint of the state before the step, of the warm impulses it read, and
// accumulates the adjoints of the inverse masses, inverse inertias, world
// friction and world restitution.  The contact set, the clamps and every
// branch are those of the recomputed forward (a piecewise-smooth map is
// differentiated on the piece the trajectory is on).  Contact geometry
// (normal, point, depth as functions of both poses) is differentiated in
// forward mode with dual numbers through the same templated geometry; a
// box-box normal comes from EPA's final face, rebuilt from its box corners.
//
// Everything is __host__ __device__: the device kernel (ne_adjoint.cu) runs it
// one CTA per world (a Team of its threads); the host test build runs a Team
// of one.
#pragma once

#include "ne_dual.cuh"
#include "ne_step.cuh"

namespace neb {

// Dual-number geometry reads the FP64 vertex records.
template <> struct VertOf<Dual> { using type = D4; };

namespace adj {

// ---- state records -------------------------------------------------------

// Mutable state of one body (the step's input/output), host layout order.
struct St {
    V3 x;
    Q q;
    V3 v, w, f, t;
};

NE_HD St st_zero() {
    St s;
    s.x = s.v = s.w = s.f = s.t = mk(0.0, 0.0, 0.0);
    s.q = mkq(0.0, 0.0, 0.0, 0.0);
    return s;
}

// Constant data of one body (read from the device world's records).
struct Bc {
    double invM;
    V3 invI;
    double bound;
    double gs;           // gravity scale
    double lin, ang;     // damping
    double fric, rest;   // material (< 0: the world's)
    uint4 meta;
};

NE_HD V3 v3r(const D4& a) { return mk(a.x, a.y, a.z); }
NE_HD Q qr(const D4& a) { return mkq(a.x, a.y, a.z, a.w); }

NE_HD Bc load_bc(const DevWorld& d, uint32_t i) {
    Bc b;
    b.invM = d.pos[i].w;
    const D4 I = d.inert[i];
    b.invI = v3r(I);
    b.bound = I.w;
    const D4 g = d.geom[i], m = d.mat[i];
    b.gs = g.z;
    b.fric = m.x;
    b.rest = m.y;
    b.lin = m.z;
    b.ang = m.w;
    b.meta = d.meta[i];
    return b;
}

NE_HD bool mutable_(const Bc& b) { return (b.meta.y & kFlagMutable) != 0; }

NE_HD BodyG geom_of(const DevWorld& d, uint32_t i, const St& s) {
    BodyG b;
    b.x = s.x;
    b.q = s.q;
    b.he = v3r(d.ext[i]);
    const D4 g = d.geom[i];
    b.radius = g.x;
    b.half_height = g.y;
    const uint2 vr = d.vrng[i];
    b.verts = d.verts + vr.x;
    b.nverts = (int)vr.y;
    b.shape = (int)d.meta[i].x;
    return b;
}

// ---- forward pieces (the device kernels' arithmetic) -------------------------

// World::integrate() for one body (k_integrate).
NE_HD St integrate(const WorldP& W, const Bc& b, const St& s0) {
    St s = s0;
    const double dt = W.dt;
    if (b.meta.y & NE_BODY_KINEMATIC) {
        s.x = s.x + s.v * dt;
        s.q = integrate_orientation(s.q, s.w, dt);
    } else if (b.invM <= 0.0) {
    } else {
        s.v = s.v + (W.g * b.gs + s.f * b.invM) * dt;
        s.x = s.x + s.v * dt;
        V3 L = angular_momentum(s.q, b.invI, s.w);
        L = L + s.t * dt;
        const Q q0 = s.q;
        s.q = integrate_orientation(q0, s.w, dt);
        s.w = apply_inv_inertia(s.q, b.invI, L);
        if (b.lin > 0.0) s.v = s.v * (1.0 / (1.0 + b.lin * dt));
        if (b.ang > 0.0) s.w = s.w * (1.0 / (1.0 + b.ang * dt));
    }
    s.f = mk(0.0, 0.0, 0.0);
    s.t = s.f;
    return s;
}

NE_HD double combine(int mode, double x, double y) {
    switch (mode) {
        case NE_COMBINE_AVERAGE: return 0.5 * (x + y);
        case NE_COMBINE_MIN: return x < y ? x : y;
        case NE_COMBINE_MAX: return x > y ? x : y;
        case NE_COMBINE_MULTIPLY: return x * y;
        case NE_COMBINE_GEOMETRIC_MEAN: return sqrt((x > 0 ? x : 0) * (y > 0 ? y : 0));
    }
    return 0.5 * (x + y);
}

// d combine / d x and d y (on the branch taken).
NE_HD void combine_grad(int mode, double x, double y, double& gx, double& gy) {
    gx = gy = 0.0;
    switch (mode) {
        case NE_COMBINE_AVERAGE: gx = gy = 0.5; return;
        case NE_COMBINE_MIN: if (x < y) gx = 1.0; else gy = 1.0; return;
        case NE_COMBINE_MAX: if (x > y) gx = 1.0; else gy = 1.0; return;
        case NE_COMBINE_MULTIPLY: gx = y; gy = x; return;
        case NE_COMBINE_GEOMETRIC_MEAN: {
            const double a = x > 0 ? x : 0, c = y > 0 ? y : 0;
            const double s = sqrt(a * c);
            if (s > 0.0) {
                if (x > 0) gx = 0.5 * c / s;
                if (y > 0) gy = 0.5 * a / s;
            }
            return;
        }
    }
    gx = gy = 0.5;
}

// The filters and the conservative cull of the device broadphase (cull_keep).
NE_HD bool keep_pair(const DevWorld& d, const Domain& dom, uint32_t i, uint32_t j, const St& si, const St& sj,
                     const Bc& bi, const Bc& bj) {
    if (bi.invM + bj.invM <= 0.0) return false;
    const uint4 ma = bi.meta, mb = bj.meta;
    if (!((ma.w & (1u << (mb.z & 31u))) && (mb.w & (1u << (ma.z & 31u))))) return false;
    const uint2 nr = d.ncrng[i];
    for (uint32_t k = 0; k < nr.y; ++k)
        if (d.nc[nr.x + k] == j) return false;
    if ((ma.y | mb.y) & NE_BODY_SENSOR) return false;
    const int sa = (int)ma.x, sb = (int)mb.x;
    if (sa == SH_PLANE && sb == SH_PLANE) return false;
    if (sa == SH_PLANE || sb == SH_PLANE) return true;
    const V3 dd = min_image(dom, mk(sj.x.x - si.x.x, sj.x.y - si.x.y, sj.x.z - si.x.z));
    const double r = (bi.bound + bj.bound) * (1.0 + 1e-9) + 1e-9;
    if (norm2(dd) > r * r) return false;
    if (sa == SH_BOX || sb == SH_BOX) {
        const bool boxA = (sa == SH_BOX);
        const double rs = boxA ? bj.bound : bi.bound;
        const V3 rel = boxA ? dd : -dd;
        const Q qb = boxA ? si.q : sj.q;
        const V3 he = v3r(d.ext[boxA ? i : j]);
        const V3 l = inv_rotate(qb, rel);
        const double ex = fmax(fabs(l.x) - he.x, 0.0), ey = fmax(fabs(l.y) - he.y, 0.0),
                     ez = fmax(fabs(l.z) - he.z, 0.0);
        const double lim = rs * (1.0 + 1e-9) + 1e-9 * (1.0 + norm(he));
        if (ex * ex + ey * ey + ez * ez > lim * lim) return false;
    }
    return true;
}

// effMass (src/contact.hpp:28-33).
NE_HD double eff_mass(const Q& qa, const V3& ia, double ma, const Q& qb, const V3& ib, double mb, const V3& ra,
                      const V3& rb, const V3& u) {
    V3 angA = cross(apply_inv_inertia(qa, ia, cross(ra, u)), ra);
    V3 angB = cross(apply_inv_inertia(qb, ib, cross(rb, u)), rb);
    return ma + mb + dot(angA + angB, u);
}

// ---- contacts of one step ---------------------------------------------------

// Per-contact record (local body indices; reference order).
struct Con {
    uint32_t a, b, slot;     // local indices of the pair's bodies, slot
    V3 n, p;                 // normal b -> a, point
    double ov;               // depth
    V3 rA, rB;
    double restBias, mu, Kn;
    double nImp0;            // warm-start impulse read from the cache
    double nImp, tImp;       // impulses during / after the solve
    int warm_idx;            // index of the cache entry it was read from, or -1
    uint32_t own;            // team member that runs this contact's island
};

// Contact of a pair (the device narrowphase), plus EPA's final face for
// convex pairs (box corners rebuilt from it in the dual pass).
struct PairHit {
    int n;
    V3 normal;
    V3 point[4];
    double depth[4];
};

NE_HD PairHit pair_contacts(const BodyG& A, const BodyG& B, const Domain& dom, EpaScratch& S, int& flags) {
    PairHit h;
    h.n = 0;
    Contact c = detect_contact(A, B, dom, S, flags);
    if (!c.hit) return h;
    h.normal = c.normal;
    if (A.shape == SH_BOX && B.shape == SH_BOX) {
        Manifold m = box_box_manifold(A, B, c.normal, dom, flags);
        for (int k = 0; k < m.count; ++k) { h.point[k] = m.point[k]; h.depth[k] = m.depth[k]; }
        h.n = m.count;
    }
    if (h.n == 0) {
        h.point[0] = c.point;
        h.depth[0] = c.overlap;
        h.n = 1;
    }
    return h;
}

// ---- vector-Jacobian products of the math primitives -------------------------
// Convention: *_vjp(inputs..., out_bar, in_bars...) ADDS the input adjoints.

NE_HD void add(V3& a, const V3& b) { a = a + b; }
NE_HD void addq(Q& a, const Q& b) { a = qadd(a, b); }

// c = a x b
NE_HD void cross_vjp(const V3& a, const V3& b, const V3& cb, V3& ab, V3& bb) {
    add(ab, cross(b, cb));
    add(bb, cross(cb, a));
}

// r = rotate(q, v) = v + w t + qv x t,  t = 2 (qv x v)
NE_HD void rotate_vjp(const Q& q, const V3& v, const V3& rb, Q& qb, V3& vb) {
    const V3 qv = mk(q.x, q.y, q.z);
    const V3 t = 2.0 * cross(qv, v);
    add(vb, rb);
    qb.w += dot(rb, t);
    V3 tb = rb * q.w;
    V3 qvb = mk(0.0, 0.0, 0.0);
    cross_vjp(qv, t, rb, qvb, tb);
    // t = 2 (qv x v)
    cross_vjp(qv, v, tb * 2.0, qvb, vb);
    qb.x += qvb.x;
    qb.y += qvb.y;
    qb.z += qvb.z;
}

NE_HD void inv_rotate_vjp(const Q& q, const V3& v, const V3& rb, Q& qb, V3& vb) {
    Q cb = mkq(0.0, 0.0, 0.0, 0.0);
    rotate_vjp(qconj(q), v, rb, cb, vb);
    qb.w += cb.w;
    qb.x -= cb.x;
    qb.y -= cb.y;
    qb.z -= cb.z;
}

// o = apply_inv_inertia(q, I, u) = rotate(q, I * inv_rotate(q, u))
NE_HD void aii_vjp(const Q& q, const V3& I, const V3& u, const V3& ob, Q& qb, V3& Ib, V3& ub) {
    const V3 ubd = inv_rotate(q, u);
    const V3 sb = mk(ubd.x * I.x, ubd.y * I.y, ubd.z * I.z);
    V3 sbb = mk(0.0, 0.0, 0.0);
    rotate_vjp(q, sb, ob, qb, sbb);
    Ib.x += sbb.x * ubd.x;
    Ib.y += sbb.y * ubd.y;
    Ib.z += sbb.z * ubd.z;
    const V3 ubdb = mk(sbb.x * I.x, sbb.y * I.y, sbb.z * I.z);
    inv_rotate_vjp(q, u, ubdb, qb, ub);
}

// L = angular_momentum(q, invI, w) = rotate(q, Ib * inv_rotate(q, w)),
// Ib = 1 / invI (0 where invI == 0).
NE_HD void angmom_vjp(const Q& q, const V3& invI, const V3& w, const V3& Lb, Q& qb, V3& invIb, V3& wb) {
    const V3 Ib = mk(invI.x > 0 ? 1.0 / invI.x : 0.0, invI.y > 0 ? 1.0 / invI.y : 0.0,
                     invI.z > 0 ? 1.0 / invI.z : 0.0);
    const V3 wbd = inv_rotate(q, w);
    const V3 Lbd = mk(wbd.x * Ib.x, wbd.y * Ib.y, wbd.z * Ib.z);
    V3 Lbdb = mk(0.0, 0.0, 0.0);
    rotate_vjp(q, Lbd, Lb, qb, Lbdb);
    const double ib[3] = {Ib.x, Ib.y, Ib.z}, iv[3] = {invI.x, invI.y, invI.z};
    const double lb[3] = {Lbdb.x, Lbdb.y, Lbdb.z}, wv[3] = {wbd.x, wbd.y, wbd.z};
    double gI[3];
    for (int k = 0; k < 3; ++k) gI[k] = iv[k] > 0 ? -lb[k] * wv[k] * ib[k] * ib[k] : 0.0;
    invIb.x += gI[0];
    invIb.y += gI[1];
    invIb.z += gI[2];
    const V3 wbdb = mk(lb[0] * ib[0], lb[1] * ib[1], lb[2] * ib[2]);
    inv_rotate_vjp(q, w, wbdb, qb, wb);
}

// r = qmul(a, o)
NE_HD void qmul_vjp(const Q& a, const Q& o, const Q& rb, Q& ab, Q& ob) {
    ab.w += rb.w * o.w + rb.x * o.x + rb.y * o.y + rb.z * o.z;
    ab.x += -rb.w * o.x + rb.x * o.w - rb.y * o.z + rb.z * o.y;
    ab.y += -rb.w * o.y + rb.x * o.z + rb.y * o.w - rb.z * o.x;
    ab.z += -rb.w * o.z - rb.x * o.y + rb.y * o.x + rb.z * o.w;
    ob.w += rb.w * a.w + rb.x * a.x + rb.y * a.y + rb.z * a.z;
    ob.x += -rb.w * a.x + rb.x * a.w + rb.y * a.z - rb.z * a.y;
    ob.y += -rb.w * a.y - rb.x * a.z + rb.y * a.w + rb.z * a.x;
    ob.z += -rb.w * a.z + rb.x * a.y - rb.y * a.x + rb.z * a.w;
}

// q1 = integrate_orientation(q, w, dt) = normalise(q + qmul((0, w), q) * dt/2)
NE_HD void iorient_vjp(const Q& q, const V3& w, double dt, const Q& q1b, Q& qb, V3& wb) {
    const Q om = mkq(0.0, w.x, w.y, w.z);
    const Q qa = qadd(q, qscale(qmul(om, q), 0.5 * dt));
    const double n = sqrt(qa.w * qa.w + qa.x * qa.x + qa.y * qa.y + qa.z * qa.z);
    if (!(n > 1e-300)) return;
    const Q q1 = mkq(qa.w / n, qa.x / n, qa.y / n, qa.z / n);
    const double pr = q1.w * q1b.w + q1.x * q1b.x + q1.y * q1b.y + q1.z * q1b.z;
    const Q qab = mkq((q1b.w - q1.w * pr) / n, (q1b.x - q1.x * pr) / n, (q1b.y - q1.y * pr) / n,
                      (q1b.z - q1.z * pr) / n);
    addq(qb, qab);
    const Q mb = qscale(qab, 0.5 * dt);
    Q omb = mkq(0.0, 0.0, 0.0, 0.0);
    qmul_vjp(om, q, mb, omb, qb);
    wb.x += omb.x;
    wb.y += omb.y;
    wb.z += omb.z;
}

// Per-body adjoint accumulators beyond the state: inverse mass and inertia.
struct Pb {
    double invM;
    V3 invI;
};

// Body constants for the solver (post-integrate orientation).
struct Sk {
    Q q;
    V3 I;
    double m;
};

// K = eff_mass(...)
NE_HD void effmass_vjp(const Sk& A, const Sk& B, const V3& ra, const V3& rb, const V3& u, double Kb, Q& qAb,
                       Pb& pA, Q& qBb, Pb& pB, V3& rab, V3& rbb, V3& ub) {
    const V3 cA = cross(ra, u), cB = cross(rb, u);
    const V3 gA = apply_inv_inertia(A.q, A.I, cA), gB = apply_inv_inertia(B.q, B.I, cB);
    const V3 angA = cross(gA, ra), angB = cross(gB, rb);
    pA.invM += Kb;
    pB.invM += Kb;
    const V3 angb = u * Kb;
    add(ub, (angA + angB) * Kb);
    V3 gAb = mk(0.0, 0.0, 0.0), gBb = gAb, cAb = gAb, cBb = gAb;
    cross_vjp(gA, ra, angb, gAb, rab);
    cross_vjp(gB, rb, angb, gBb, rbb);
    aii_vjp(A.q, A.I, cA, gAb, qAb, pA.invI, cAb);
    aii_vjp(B.q, B.I, cB, gBb, qBb, pB.invI, cBb);
    cross_vjp(ra, u, cAb, rab, ub);
    cross_vjp(rb, u, cBb, rbb, ub);
}

// ---- the per-world program ------------------------------------------------------

// Scratch of one world (all arrays owned by the caller).
struct WScr {
    uint32_t b0, nb;                 // first body (global index), bodies
    uint32_t cap;                    // contact capacity
    St* s;                           // [nb] working state
    St* s0;                          // [nb] pre-step state (kept by the adjoint)
    St* s1;                          // [nb] post-integrate state (recorded)
    Con* con;                        // [cap]
    uint32_t ncon;
    const unsigned long long* wk_in; // warm cache read (sorted keys, one entry per contact)
    const double* wi_in;
    uint32_t nw_in;
    unsigned long long* wk_out;      // warm cache written ([cap])
    double* wi_out;
    uint32_t nw_out;
    double* tape;                    // [9 * cap * 14] pre-update states of phases 0-8, or null
    uint32_t* uf;                    // [nb] union-find parents (islands)
    int err;                         // bit 0 capacity, 1 unsupported, 2 narrowphase budget
};

// The threads that run one world: a warp on the device (lane, 32), one
// thread on the host (0, 1).  Work with no order constraint is split over the
// lanes; each island's solver updates run on one lane, in order.
struct Team {
    int lane, size;
    // Block teams (size > 32): shared scratch of kTeamScratch words; a warp
    // (size 32) or the host build (size 1) needs none.
    uint32_t* sm = nullptr;
    NE_HD void sync() const {
#ifdef __CUDA_ARCH__
        if (size > 32) __syncthreads(); else __syncwarp();
#endif
    }
    // Exclusive prefix of v over the lanes; *total = the sum (all lanes).
    NE_HD uint32_t scan(uint32_t v, uint32_t& total) const {
#ifdef __CUDA_ARCH__
        const int wl = lane & 31;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
            if (wl >= o) x += t;
        }
        if (size <= 32) {
            total = __shfl_sync(0xffffffffu, x, 31);
            return x - v;
        }
        const int w = lane >> 5, nw = size >> 5;
        if (wl == 31) sm[w] = x;
        __syncthreads();
        uint32_t before = 0, all = 0;
        for (int k = 0; k < nw; ++k) {
            if (k < w) before += sm[k];
            all += sm[k];
        }
        __syncthreads();
        total = all;
        return before + x - v;
#else
        total = v;
        return 0;
#endif
    }
    NE_HD int any_or(int v) const {
#ifdef __CUDA_ARCH__
        if (size > 32) return __syncthreads_or(v);
        for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
#endif
        return v;
    }
    // Sum over the lanes, in a fixed order (warp trees, then warps in order).
    NE_HD double sum(double v) const {
#ifdef __CUDA_ARCH__
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (size <= 32) return v;
        double* smd = reinterpret_cast<double*>(sm + 32);
        if ((lane & 31) == 0) smd[lane >> 5] = v;
        __syncthreads();
        double r = 0.0;
        for (int k = 0; k < (size >> 5); ++k) r += smd[k];
        __syncthreads();
        return r;
#else
        return v;
#endif
    }
};
// Shared scratch of a block team: 32 words for the scan, 32 doubles for the sum.
constexpr int kTeamScratch = 32 + 64;

NE_HD uint32_t uf_root(uint32_t* p, uint32_t x) {
    while (p[x] != x) x = p[x];
    return x;
}

constexpr int kTapeRec = 14;
constexpr int kErrCapacity = 1, kErrUnsupported = 2, kErrNumeric = 4;

NE_HD uint32_t lower_bound_key(const unsigned long long* a, uint32_t n, unsigned long long k) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo;
}

NE_HD void tape_put(double* t, const V3& vA, const V3& wA, const V3& vB, const V3& wB, double ix, double iy) {
    t[0] = vA.x; t[1] = vA.y; t[2] = vA.z; t[3] = wA.x; t[4] = wA.y; t[5] = wA.z;
    t[6] = vB.x; t[7] = vB.y; t[8] = vB.z; t[9] = wB.x; t[10] = wB.y; t[11] = wB.z;
    t[12] = ix; t[13] = iy;
}

NE_HD void tape_get(const double* t, V3& vA, V3& wA, V3& vB, V3& wB, double& ix, double& iy) {
    vA = mk(t[0], t[1], t[2]); wA = mk(t[3], t[4], t[5]);
    vB = mk(t[6], t[7], t[8]); wB = mk(t[9], t[10], t[11]);
    ix = t[12]; iy = t[13];
}

NE_HD Sk sk_of(const Bc& b, const St& s) {
    Sk k;
    k.q = s.q;
    k.I = b.invI;
    k.m = b.invM;
    return k;
}

NE_HD void apply_pair(V3& vA, V3& wA, V3& vB, V3& wB, const Sk& A, const Sk& B, const V3& ra, const V3& rb,
                      const V3& J) {
    vA = vA + J * A.m;
    wA = wA + apply_inv_inertia(A.q, A.I, cross(ra, J));
    vB = vB - J * B.m;
    wB = wB - apply_inv_inertia(B.q, B.I, cross(rb, J));
}

// One sequential-impulse update (ItemsF64::sweep) on explicit operands.
NE_HD void sweep_fwd(const Con& c, const Sk& A, const Sk& B, V3& vA, V3& wA, V3& vB, V3& wB, double& ix,
                     double& iy) {
    const V3 vc = (vA + cross(wA, c.rA)) - (vB + cross(wB, c.rB));
    const double vn = dot(vc, c.n);
    if (c.Kn > 1e-18) {
        double dj = (c.restBias - vn) / c.Kn;
        const double old = ix;
        ix = (old + dj > 0.0) ? old + dj : 0.0;
        dj = ix - old;
        apply_pair(vA, wA, vB, wB, A, B, c.rA, c.rB, c.n * dj);
    }
    if (c.mu > 0.0 && ix > 0.0) {
        const V3 vc2 = (vA + cross(wA, c.rA)) - (vB + cross(wB, c.rB));
        const V3 vt = vc2 - c.n * dot(vc2, c.n);
        const double vtl = norm(vt);
        if (vtl > 1e-12) {
            const V3 tg = vt / vtl;
            const double Kt = eff_mass(A.q, A.I, A.m, B.q, B.I, B.m, c.rA, c.rB, tg);
            if (Kt > 1e-18) {
                double djt = -vtl / Kt;
                const double maxF = c.mu * ix;
                const double old = iy;
                const double sum = old + djt;
                iy = (sum < -maxF) ? -maxF : (sum > maxF ? maxF : sum);
                djt = iy - old;
                apply_pair(vA, wA, vB, wB, A, B, c.rA, c.rB, tg * djt);
            }
        }
    }
}

// Adjoint accumulators of one contact's constants.
struct Cb {
    V3 n, rA, rB, p;
    double restBias, mu, Kn, ov;
    double ixb, iyb;     // running adjoints of the contact's normal / friction impulse
};

NE_HD Cb cb_zero() {
    Cb c;
    c.n = c.rA = c.rB = c.p = mk(0.0, 0.0, 0.0);
    c.restBias = c.mu = c.Kn = c.ov = 0.0;
    c.ixb = c.iyb = 0.0;
    return c;
}

// Reverse of apply_pair: given the adjoints of the updated velocities (which
// also flow to the velocities before), add the adjoint of J and of the
// constants.
NE_HD void apply_pair_vjp(const Sk& A, const Sk& B, const V3& ra, const V3& rb, const V3& J, const V3& vAb,
                          const V3& wAb, const V3& vBb, const V3& wBb, V3& Jb, Q& qAb, Pb& pA, Q& qBb, Pb& pB,
                          V3& rab, V3& rbb) {
    add(Jb, vAb * A.m - vBb * B.m);
    pA.invM += dot(vAb, J);
    pB.invM -= dot(vBb, J);
    V3 cAb = mk(0.0, 0.0, 0.0), cBb = cAb;
    aii_vjp(A.q, A.I, cross(ra, J), wAb, qAb, pA.invI, cAb);
    aii_vjp(B.q, B.I, cross(rb, J), -wBb, qBb, pB.invI, cBb);
    cross_vjp(ra, J, cAb, rab, Jb);
    cross_vjp(rb, J, cBb, rbb, Jb);
}

// Reverse of sweep_fwd from its taped inputs.  On entry the v/w/imp adjoints
// are those of the update's outputs; on exit, those of its inputs.
NE_HD void sweep_vjp(const Con& c, const Sk& A, const Sk& B, const double* tape, V3& vAb, V3& wAb, V3& vBb, V3& wBb,
                     double& ixb, double& iyb, Cb& cb, Q& qAb, Pb& pA, Q& qBb, Pb& pB) {
    V3 vA, wA, vB, wB;
    double ix, iy;
    tape_get(tape, vA, wA, vB, wB, ix, iy);
    // forward, keeping the intermediates
    const V3 vc = (vA + cross(wA, c.rA)) - (vB + cross(wB, c.rB));
    const double vn = dot(vc, c.n);
    const bool nact = c.Kn > 1e-18;
    double djn = 0.0, s = 0.0, dj2 = 0.0, ix1 = ix;
    V3 vA1 = vA, wA1 = wA, vB1 = vB, wB1 = wB, Jn = mk(0.0, 0.0, 0.0);
    if (nact) {
        djn = (c.restBias - vn) / c.Kn;
        s = ix + djn;
        ix1 = (s > 0.0) ? s : 0.0;
        dj2 = ix1 - ix;
        Jn = c.n * dj2;
        apply_pair(vA1, wA1, vB1, wB1, A, B, c.rA, c.rB, Jn);
    }
    bool fact = false;
    V3 vc2 = mk(0.0, 0.0, 0.0), vt = vc2, tg = vc2, Jt = vc2;
    double sN = 0, vtl = 0, Kt = 0, djt = 0, maxF = 0, sum = 0, djt2 = 0;
    if (c.mu > 0.0 && ix1 > 0.0) {
        vc2 = (vA1 + cross(wA1, c.rA)) - (vB1 + cross(wB1, c.rB));
        sN = dot(vc2, c.n);
        vt = vc2 - c.n * sN;
        vtl = norm(vt);
        if (vtl > 1e-12) {
            tg = vt / vtl;
            Kt = eff_mass(A.q, A.I, A.m, B.q, B.I, B.m, c.rA, c.rB, tg);
            if (Kt > 1e-18) {
                fact = true;
                djt = -vtl / Kt;
                maxF = c.mu * ix1;
                sum = iy + djt;
                const double iy1 = (sum < -maxF) ? -maxF : (sum > maxF ? maxF : sum);
                djt2 = iy1 - iy;
                Jt = tg * djt2;
            }
        }
    }
    // reverse: friction
    double ix1b = ixb;
    if (fact) {
        V3 Jtb = mk(0.0, 0.0, 0.0);
        apply_pair_vjp(A, B, c.rA, c.rB, Jt, vAb, wAb, vBb, wBb, Jtb, qAb, pA, qBb, pB, cb.rA, cb.rB);
        V3 tgb = Jtb * djt2;
        const double djt2b = dot(Jtb, tg);
        const double iy1b = iyb + djt2b;
        double oldb = -djt2b;
        double maxFb = 0.0, sumb = 0.0;
        if (sum < -maxF) maxFb -= iy1b;
        else if (sum > maxF) maxFb += iy1b;
        else sumb = iy1b;
        oldb += sumb;
        const double djtb = sumb;
        cb.mu += maxFb * ix1;
        ix1b += maxFb * c.mu;
        double vtlb = -djtb / Kt;
        const double Ktb = djtb * vtl / (Kt * Kt);
        effmass_vjp(A, B, c.rA, c.rB, tg, Ktb, qAb, pA, qBb, pB, cb.rA, cb.rB, tgb);
        V3 vtb = tgb / vtl;
        vtlb -= dot(tgb, vt) / (vtl * vtl);
        add(vtb, vt * (vtlb / vtl));
        V3 vc2b = vtb;
        cb.n = cb.n - vtb * sN;
        const double sNb = -dot(vtb, c.n);
        add(vc2b, c.n * sNb);
        add(cb.n, vc2 * sNb);
        add(vAb, vc2b);
        cross_vjp(wA1, c.rA, vc2b, wAb, cb.rA);
        vBb = vBb - vc2b;
        cross_vjp(wB1, c.rB, -vc2b, wBb, cb.rB);
        iyb = oldb;
    }
    // reverse: normal
    if (nact) {
        V3 Jb = mk(0.0, 0.0, 0.0);
        apply_pair_vjp(A, B, c.rA, c.rB, Jn, vAb, wAb, vBb, wBb, Jb, qAb, pA, qBb, pB, cb.rA, cb.rB);
        add(cb.n, Jb * dj2);
        const double dj2b = dot(Jb, c.n);
        const double ix1t = ix1b + dj2b;
        double oldb = -dj2b;
        const double sb = (s > 0.0) ? ix1t : 0.0;
        oldb += sb;
        const double djb = sb;
        cb.restBias += djb / c.Kn;
        const double vnb = -djb / c.Kn;
        cb.Kn -= djb * djn / c.Kn;
        const V3 vcb = c.n * vnb;
        add(cb.n, vc * vnb);
        add(vAb, vcb);
        cross_vjp(wA, c.rA, vcb, wAb, cb.rA);
        vBb = vBb - vcb;
        cross_vjp(wB, c.rB, -vcb, wBb, cb.rB);
        ixb = oldb;
    } else {
        ixb = ix1b;
    }
}

// Worlds the adjoint differentiates: no reflective walls (open or periodic),
// and every convex pair polyhedral (boxes and hulls: EPA's final face is exact
// there); spheres only against spheres and planes.
NE_HD bool backward_supported(const DevWorld& d, const WorldP& W, uint32_t b0, uint32_t b1) {
    if (!W.dom.periodic && !W.open_boundary) return false;
    bool curved = false, poly = false;
    for (uint32_t i = b0; i < b1; ++i) {
        const int s = (int)d.meta[i].x;
        if (d.meta[i].y & NE_BODY_KINEMATIC) return false;   // moving bodies shared by islands
        if (s == SH_CYLINDER || s == SH_CAPSULE || s == SH_MESH || s == SH_COMPOUND) return false;
        if (s == SH_SPHERE) curved = true;
        if (s == SH_BOX || s == SH_CONVEX) poly = true;
    }
    return !(curved && poly);
}

// One step of world [b0, b0+nb) in place on w.s, in the reference's order,
// run by team t (every member calls it with the same arguments; w.ncon,
// w.nw_out and w.err come out the same on every member).  Bodies and pairs
// are split over the members; contacts are appended in sorted pair order (a
// prefix over the members); the solver updates of an island run on one
// member, in the reference's order, so every body sees the reference's
// sequence.  With w.tape set, the post-integrate state and the input of every
// solver update (phases 0-8) are recorded for the adjoint.
NE_HD void fwd_step(const DevWorld& d, const WorldP& W, int warm, WScr& w, const Team& t) {
    const uint32_t nb = w.nb, b0 = w.b0;
    for (uint32_t b = t.lane; b < nb; b += t.size) {
        w.s[b] = integrate(W, load_bc(d, b0 + b), w.s[b]);
        if (w.tape) w.s1[b] = w.s[b];
        w.uf[b] = b;
    }
    t.sync();
    // Pairs in sorted order, narrowphase, constraint build (k_constraint_build).
    w.ncon = 0;
    int err = 0;
    EpaScratch S;
    for (uint32_t ia = 0; ia < nb; ++ia) {
        const Bc A = load_bc(d, b0 + ia);
        for (uint32_t ib0 = ia + 1; ib0 < nb; ib0 += t.size) {
            const uint32_t ib = ib0 + t.lane;
            PairHit h;
            h.n = 0;
            Bc B;
            if (ib < nb) {
                B = load_bc(d, b0 + ib);
                if (keep_pair(d, W.dom, b0 + ia, b0 + ib, w.s[ia], w.s[ib], A, B)) {
                    const BodyG ga = geom_of(d, b0 + ia, w.s[ia]), gb = geom_of(d, b0 + ib, w.s[ib]);
                    int fl = 0;
                    h = pair_contacts(ga, gb, W.dom, S, fl);
                    if (fl & 1) err |= kErrNumeric;
                }
            }
            uint32_t total;
            const uint32_t base = w.ncon + t.scan((uint32_t)h.n, total);
            if (w.ncon + total > w.cap) {
                w.err |= t.any_or(err) | kErrCapacity;
                return;
            }
            if (h.n > 0) {
                const double ea = A.rest < 0 ? W.restitution : A.rest, eb = B.rest < 0 ? W.restitution : B.rest;
                const double fa = A.fric < 0 ? W.friction : A.fric, fb = B.fric < 0 ? W.friction : B.fric;
                const double e = combine(W.rcomb, ea, eb);
                const double mu = combine(W.fcomb, fa, fb);
                const unsigned long long key = ((unsigned long long)(b0 + ia) << 32) | (unsigned long long)(b0 + ib);
                const uint32_t widx = warm ? lower_bound_key(w.wk_in, w.nw_in, key) : 0u;
                const St& sa = w.s[ia];
                const St& sb = w.s[ib];
                for (int k = 0; k < h.n; ++k) {
                    Con& c = w.con[base + k];
                    c.a = ia;
                    c.b = ib;
                    c.slot = (uint32_t)k;
                    c.n = h.normal;
                    c.p = h.point[k];
                    c.ov = h.depth[k];
                    c.rA = min_image(W.dom, c.p - sa.x);
                    c.rB = min_image(W.dom, c.p - sb.x);
                    const V3 vc = (sa.v + cross(sa.w, c.rA)) - (sb.v + cross(sb.w, c.rB));
                    const double vn = dot(vc, c.n);
                    c.restBias = (vn < -0.5) ? -e * vn : 0.0;
                    c.mu = mu;
                    c.nImp0 = 0.0;
                    c.warm_idx = -1;
                    if (warm && widx + k < w.nw_in && w.wk_in[widx + k] == key) {
                        c.nImp0 = w.wi_in[widx + k];
                        c.warm_idx = (int)(widx + k);
                    }
                    c.Kn = eff_mass(sa.q, A.invI, A.invM, sb.q, B.invI, B.invM, c.rA, c.rB, c.n);
                    c.nImp = c.nImp0;
                    c.tImp = 0.0;
                }
            }
            w.ncon += total;
        }
    }
    w.err |= t.any_or(err);
    t.sync();
    // Islands over the mutable bodies (union-find on member 0); each island
    // goes to the member root % size.
    const uint32_t nc = w.ncon;
    if (t.lane == 0) {
        for (uint32_t ci = 0; ci < nc; ++ci) {
            const Con& c = w.con[ci];
            if (!mutable_(load_bc(d, b0 + c.a)) || !mutable_(load_bc(d, b0 + c.b))) continue;
            const uint32_t ra = uf_root(w.uf, c.a), rb = uf_root(w.uf, c.b);
            if (ra != rb) w.uf[ra > rb ? ra : rb] = ra < rb ? ra : rb;
        }
    }
    t.sync();
    for (uint32_t ci = t.lane; ci < nc; ci += t.size) {
        Con& c = w.con[ci];
        const uint32_t body = mutable_(load_bc(d, b0 + c.a)) ? c.a : c.b;
        c.own = uf_root(w.uf, body) % (uint32_t)t.size;
    }
    t.sync();
    // Warm start, 8 sweeps (phases 0-8), on the post-integrate orientations;
    // then position correction (correct_item) and the warm cache.
    for (int ph = 0; ph <= 8; ++ph) {
        if (ph == 0 && !warm) continue;
        for (uint32_t ci = 0; ci < nc; ++ci) {
            Con& c = w.con[ci];
            if (c.own != (uint32_t)t.lane) continue;
            const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
            St& sa = w.s[c.a];
            St& sb = w.s[c.b];
            V3 vA = sa.v, wA = sa.w, vB = sb.v, wB = sb.w;
            if (w.tape) tape_put(w.tape + ((size_t)ph * w.cap + ci) * kTapeRec, vA, wA, vB, wB, c.nImp, c.tImp);
            const Sk kA = sk_of(A, sa), kB = sk_of(B, sb);
            if (ph == 0) {
                if (c.nImp0 == 0.0) continue;
                apply_pair(vA, wA, vB, wB, kA, kB, c.rA, c.rB, c.n * c.nImp0);
            } else {
                sweep_fwd(c, kA, kB, vA, wA, vB, wB, c.nImp, c.tImp);
            }
            if (mutable_(A)) { sa.v = vA; sa.w = wA; }
            if (mutable_(B)) { sb.v = vB; sb.w = wB; }
        }
    }
    for (uint32_t ci = 0; ci < nc; ++ci) {
        const Con& c = w.con[ci];
        if (c.own != (uint32_t)t.lane) continue;
        const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
        const double invSum = A.invM + B.invM;
        if (!(invSum <= 0.0 || c.ov <= 0.0)) {
            const V3 corr = c.n * (W.beta * c.ov / invSum);
            if (mutable_(A)) w.s[c.a].x = w.s[c.a].x + corr * A.invM;
            if (mutable_(B)) w.s[c.b].x = w.s[c.b].x - corr * B.invM;
        }
        if (warm) {
            w.wk_out[ci] = ((unsigned long long)(b0 + c.a) << 32) | (unsigned long long)(b0 + c.b);
            w.wi_out[ci] = c.nImp;
        }
    }
    w.nw_out = warm ? nc : 0;
    t.sync();
    // wrapPositions / applyWalls (world.cpp:698-702, 635-657; k_boundary).
    // The adjoint differentiates open and periodic worlds only.
    for (uint32_t b = t.lane; b < nb; b += t.size) {
        if (!(load_bc(d, b0 + b).invM > 0.0)) continue;
        St& s = w.s[b];
        if (W.dom.periodic) {
            s.x = wrap(W.dom, s.x);
            continue;
        }
        if (W.open_boundary) continue;
        BodyG g = geom_of(d, b0 + b, s);
        double px[3] = {s.x.x, s.x.y, s.x.z};
        double pv[3] = {s.v.x, s.v.y, s.v.z};
        const double h = W.dom.half;
        for (int axis = 0; axis < 3; ++axis) {
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                V3 outward = mk(axis == 0 ? double(sgn) : 0.0, axis == 1 ? double(sgn) : 0.0,
                                axis == 2 ? double(sgn) : 0.0);
                g.x = mk(px[0], px[1], px[2]);
                V3 sp = support_world(g, outward);
                double coord = (axis == 0 ? sp.x : axis == 1 ? sp.y : sp.z) * sgn;
                double pen = coord - h;
                if (pen > 0.0) {
                    px[axis] -= double(sgn) * pen;
                    if (pv[axis] * sgn > 0.0) pv[axis] = -W.restitution * pv[axis];
                }
            }
        }
        s.x = mk(px[0], px[1], px[2]);
        s.v = mk(pv[0], pv[1], pv[2]);
    }
    t.sync();
}

// ---- contact geometry in dual numbers -----------------------------------------

// Directions: x_a 0-2, q_a 3-6, x_b 7-9, q_b 10-13.
NE_HD BodyGT<Dual> dual_body(const BodyG& g, int base) {
    BodyGT<Dual> b;
    b.x = mk3<Dual>(Dual::seed(g.x.x, base), Dual::seed(g.x.y, base + 1), Dual::seed(g.x.z, base + 2));
    b.q = mkq4<Dual>(Dual::seed(g.q.w, base + 3), Dual::seed(g.q.x, base + 4), Dual::seed(g.q.y, base + 5),
                     Dual::seed(g.q.z, base + 6));
    b.he = mk3<Dual>(g.he.x, g.he.y, g.he.z);
    b.radius = g.radius;
    b.half_height = g.half_height;
    b.verts = g.verts;
    b.nverts = g.nverts;
    b.shape = g.shape;
    return b;
}

// The body-frame vertex whose world position is p (a support point of a box
// or a hull), rebuilt in duals.  Returns false for curved shapes.
NE_HD bool dual_vertex(const BodyG& g, const BodyGT<Dual>& D, const V3& p, Vec3<Dual>& out) {
    const V3 l = inv_rotate(g.q, p - g.x);
    V3 c;
    if (g.shape == SH_BOX) {
        c = mk(l.x >= 0 ? g.he.x : -g.he.x, l.y >= 0 ? g.he.y : -g.he.y, l.z >= 0 ? g.he.z : -g.he.z);
    } else if (g.shape == SH_CONVEX) {
        int best = 0;
        double bd = 1e300;
        for (int k = 0; k < g.nverts; ++k) {
            const V3 v = mk(g.verts[k].x, g.verts[k].y, g.verts[k].z);
            const double e = norm2(v - l);
            if (e < bd) { bd = e; best = k; }
        }
        c = mk(g.verts[best].x, g.verts[best].y, g.verts[best].z);
    } else {
        return false;
    }
    out = D.x + rotate(D.q, mk3<Dual>(c.x, c.y, c.z));
    return true;
}

struct PairDual {
    int n;
    Vec3<Dual> normal;
    Vec3<Dual> point[4];
    Dual depth[4];
};

// The contacts of pair (A, B) with their derivatives along both poses, taking
// the branches the FP64 evaluation took.  Returns false when the pair is not
// differentiable here (see backward_supported).
NE_HD bool pair_contacts_dual(const BodyG& A, const BodyG& B, const Domain& dom, EpaScratch& S, PairDual& out) {
    const BodyGT<Dual> DA = dual_body(A, 0), DB = dual_body(B, 7);
    out.n = 0;
    if (A.shape == SH_PLANE || B.shape == SH_PLANE) {
        const bool aPlane = A.shape == SH_PLANE;
        ContactT<Dual> t = aPlane ? plane_vs_convex(DB, DA, dom) : plane_vs_convex(DA, DB, dom);
        if (!t.hit) return true;
        out.normal = aPlane ? -t.normal : t.normal;
        out.point[0] = t.point;
        out.depth[0] = t.overlap;
        out.n = 1;
        return true;
    }
    if (A.shape == SH_SPHERE && B.shape == SH_SPHERE) {
        const Vec3<Dual> dd = min_image(dom, DA.x - DB.x);
        const Dual sumR = Dual(A.radius + B.radius), dist2 = norm2(dd);
        if (dist2 >= sumR * sumR || dist2 < Dual(1e-18)) return true;
        const Dual dist = sqrt(dist2);
        out.normal = dd / dist;
        out.depth[0] = sumR - dist;
        out.point[0] = DA.x - out.normal * Dual(A.radius);
        out.n = 1;
        return true;
    }
    if (A.shape == SH_SPHERE || B.shape == SH_SPHERE) return false;
    // Convex pair: EPA's final face, rebuilt from its vertices.
    SupV face[3];
    int fl = 0;
    Contact c = detect_contact(A, B, dom, S, fl, face);
    if (!c.hit) return true;
    const V3 shift = min_image_shift(A, B, dom);
    Vec3<Dual> fv[3], fa[3], fb[3];
    for (int k = 0; k < 3; ++k) {
        if (!dual_vertex(A, DA, face[k].a, fa[k])) return false;
        Vec3<Dual> bb;
        if (!dual_vertex(B, DB, face[k].b - shift, bb)) return false;
        fb[k] = bb + mk3<Dual>(shift.x, shift.y, shift.z);
        fv[k] = fa[k] - fb[k];
    }
    Vec3<Dual> nrm = cross(fv[1] - fv[0], fv[2] - fv[0]);
    const Dual L = norm(nrm);
    nrm = (L > 1e-18) ? nrm / L : mk3<Dual>(0.0, 0.0, 1.0);
    Dual dist = dot(nrm, fv[0]);
    if (dist < 0.0) { nrm = -nrm; dist = -dist; }
    out.normal = -nrm;
    if (A.shape == SH_BOX && B.shape == SH_BOX) {
        int f2 = 0;
        ManifoldT<Dual> m = box_box_manifold(DA, DB, out.normal, dom, f2);
        for (int k = 0; k < m.count; ++k) { out.point[k] = m.point[k]; out.depth[k] = m.depth[k]; }
        out.n = m.count;
        if (out.n > 0) return true;
    }
    // EPA's witness: barycentric coordinates of the origin's projection.
    const Vec3<Dual> proj = nrm * dist;
    const Vec3<Dual> v0 = fv[1] - fv[0], v1 = fv[2] - fv[0], v2 = proj - fv[0];
    const Dual d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    const Dual den = d00 * d11 - d01 * d01;
    Dual bv(0.0), bw(0.0);
    if (fabs(den) > 1e-18) {
        bv = (d11 * d20 - d01 * d21) / den;
        bw = (d00 * d21 - d01 * d20) / den;
    }
    const Dual bu = Dual(1.0) - bv - bw;
    const Vec3<Dual> onA = fa[0] * bu + fa[1] * bv + fa[2] * bw;
    const Vec3<Dual> onB = fb[0] * bu + fb[1] * bv + fb[2] * bw;
    out.point[0] = (onA + onB) * Dual(0.5);
    out.depth[0] = dist;
    out.n = 1;
    return true;
}

NE_HD void acc_dual(const Vec3<Dual>& v, const V3& vb, double* g) {
    for (int k = 0; k < kDualDirs; ++k) g[k] += vb.x * v.x.d[k] + vb.y * v.y.d[k] + vb.z * v.z.d[k];
}

// ---- the adjoint of one step ---------------------------------------------------

// On entry w.s holds the state before the step, sb[nb] the adjoint of the
// state after it, and wob[] the adjoint of the warm impulses the step stores
// (indexed like this step's contacts).  On exit sb holds the adjoint of the
// state before the step; wib[] (indexed like the warm cache read) and pb[nb]
// (inverse mass and inertia) are accumulated, and so are mub / eb (world
// friction / restitution, through the bodies that inherit them).  cbs[cap] is
// scratch.  The recomputed forward leaves w.s at the state after the step.
// Run by team t like fwd_step: the reverse of an island's updates runs on the
// member that ran them; adjoints of immovable bodies (which carry no
// gradient: zero inverse mass and inertia) go to a member-local sink, so no
// two members write the same memory.
NE_HD void bwd_step(const DevWorld& d, const WorldP& W, int warm, WScr& w, St* sb, const double* wob, double* wib,
                    Pb* pb, Cb* cbs, double& mub, double& eb, const Team& t) {
    const uint32_t nb = w.nb, b0 = w.b0;
    for (uint32_t b = t.lane; b < nb; b += t.size) w.s0[b] = w.s[b];
    t.sync();
    fwd_step(d, W, warm, w, t);
    if (w.err & (kErrCapacity | kErrUnsupported)) return;
    const uint32_t nc = w.ncon;
    for (uint32_t ci = t.lane; ci < nc; ci += t.size) {
        cbs[ci] = cb_zero();
        if (warm && wob) cbs[ci].ixb = wob[ci];
    }
    t.sync();
    const uint32_t me = (uint32_t)t.lane;
    St sink_s;
    Pb sink_p;
    double mub_l = 0.0, eb_l = 0.0;
    // Body adjoint / parameter accumulators of a contact's body (the sink for
    // an immovable one).
#define NE_ADJ_BODY(Bvar, li, S_, P_)                         \
    St* S_ = &sink_s;                                       \
    Pb* P_ = &sink_p;                                       \
    if (mutable_(Bvar)) { S_ = &sb[li]; P_ = &pb[li]; }      \
    else { sink_s = st_zero(); sink_p.invM = 0.0; sink_p.invI = mk(0.0, 0.0, 0.0); }
    // Position correction (x passes through; the correction's operands get adjoints).
    for (uint32_t ci = nc; ci-- > 0;) {
        const Con& c = w.con[ci];
        if (c.own != me) continue;
        const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
        const double invSum = A.invM + B.invM;
        if (invSum <= 0.0 || c.ov <= 0.0) continue;
        const double k = W.beta * c.ov / invSum;
        const V3 corr = c.n * k;
        V3 corrb = mk(0.0, 0.0, 0.0);
        double invSumb;
        if (mutable_(A)) {
            add(corrb, sb[c.a].x * A.invM);
            pb[c.a].invM += dot(sb[c.a].x, corr);
        }
        if (mutable_(B)) {
            corrb = corrb - sb[c.b].x * B.invM;
            pb[c.b].invM -= dot(sb[c.b].x, corr);
        }
        add(cbs[ci].n, corrb * k);
        const double kb = dot(corrb, c.n);
        cbs[ci].ov += kb * W.beta / invSum;
        invSumb = -kb * W.beta * c.ov / (invSum * invSum);
        if (mutable_(A)) pb[c.a].invM += invSumb;
        if (mutable_(B)) pb[c.b].invM += invSumb;
    }
    // Sweeps 8..1, then the warm start, in reverse order.
    for (int ph = 8; ph >= 0; --ph) {
        if (ph == 0 && !warm) break;
        for (uint32_t ci = nc; ci-- > 0;) {
            const Con& c = w.con[ci];
            if (c.own != me) continue;
            Cb& cb = cbs[ci];
            const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
            const Sk kA = sk_of(A, w.s1[c.a]), kB = sk_of(B, w.s1[c.b]);
            NE_ADJ_BODY(A, c.a, ba, pa)
            St sink_b;
            Pb sink_pb;
            St* bb = &sink_b;
            Pb* pbb = &sink_pb;
            if (mutable_(B)) { bb = &sb[c.b]; pbb = &pb[c.b]; }
            else { sink_b = st_zero(); sink_pb.invM = 0.0; sink_pb.invI = mk(0.0, 0.0, 0.0); }
            if (ph > 0) {
                sweep_vjp(c, kA, kB, w.tape + ((size_t)ph * w.cap + ci) * kTapeRec, ba->v, ba->w, bb->v, bb->w,
                          cb.ixb, cb.iyb, cb, ba->q, *pa, bb->q, *pbb);
                continue;
            }
            if (c.nImp0 == 0.0) continue;
            const V3 J = c.n * c.nImp0;
            V3 Jb = mk(0.0, 0.0, 0.0);
            apply_pair_vjp(kA, kB, c.rA, c.rB, J, ba->v, ba->w, bb->v, bb->w, Jb, ba->q, *pa, bb->q, *pbb, cb.rA,
                           cb.rB);
            add(cb.n, Jb * c.nImp0);
            cb.ixb += dot(Jb, c.n);
        }
    }
    // Constraint build: rA, rB, restitution bias, friction, Kn, warm impulse.
    for (uint32_t ci = 0; ci < nc; ++ci) {
        const Con& c = w.con[ci];
        if (c.own != me) continue;
        Cb& cb = cbs[ci];
        const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
        const St& sa = w.s1[c.a];
        const St& sbb = w.s1[c.b];
        NE_ADJ_BODY(A, c.a, ba, pa)
        St sink_b;
        Pb sink_pb;
        St* bb = &sink_b;
        Pb* pbb = &sink_pb;
        if (mutable_(B)) { bb = &sb[c.b]; pbb = &pb[c.b]; }
        else { sink_b = st_zero(); sink_pb.invM = 0.0; sink_pb.invI = mk(0.0, 0.0, 0.0); }
        if (warm && c.warm_idx >= 0 && wib) wib[c.warm_idx] += cb.ixb;
        // restitution bias from the pre-solve velocities
        const V3 vc = (sa.v + cross(sa.w, c.rA)) - (sbb.v + cross(sbb.w, c.rB));
        const double vn = dot(vc, c.n);
        if (vn < -0.5) {
            const double ea = A.rest < 0 ? W.restitution : A.rest, ebv = B.rest < 0 ? W.restitution : B.rest;
            const double e = combine(W.rcomb, ea, ebv);
            const double e_b = -vn * cb.restBias;
            double gx, gy;
            combine_grad(W.rcomb, ea, ebv, gx, gy);
            if (A.rest < 0) eb_l += e_b * gx;
            if (B.rest < 0) eb_l += e_b * gy;
            const double vnb = -e * cb.restBias;
            const V3 vcb = c.n * vnb;
            add(cb.n, vc * vnb);
            add(ba->v, vcb);
            cross_vjp(sa.w, c.rA, vcb, ba->w, cb.rA);
            bb->v = bb->v - vcb;
            cross_vjp(sbb.w, c.rB, -vcb, bb->w, cb.rB);
        }
        {
            const double fa = A.fric < 0 ? W.friction : A.fric, fb = B.fric < 0 ? W.friction : B.fric;
            double gx, gy;
            combine_grad(W.fcomb, fa, fb, gx, gy);
            if (A.fric < 0) mub_l += cb.mu * gx;
            if (B.fric < 0) mub_l += cb.mu * gy;
        }
        const Sk kA = sk_of(A, sa), kB = sk_of(B, sbb);
        effmass_vjp(kA, kB, c.rA, c.rB, c.n, cb.Kn, ba->q, *pa, bb->q, *pbb, cb.rA, cb.rB, cb.n);
        add(cb.p, cb.rA + cb.rB);
        ba->x = ba->x - cb.rA;
        bb->x = bb->x - cb.rB;
    }
    // Contact geometry: normal, points and depths as functions of both poses.
    {
        EpaScratch S;
        uint32_t ci = 0;
        int gerr = 0;
        while (ci < nc) {
            uint32_t cj = ci;
            while (cj < nc && w.con[cj].a == w.con[ci].a && w.con[cj].b == w.con[ci].b) ++cj;
            const Con& c = w.con[ci];
            if (c.own == me) {
                const BodyG ga = geom_of(d, b0 + c.a, w.s1[c.a]), gbd = geom_of(d, b0 + c.b, w.s1[c.b]);
                PairDual pd;
                if (!pair_contacts_dual(ga, gbd, W.dom, S, pd) || pd.n != (int)(cj - ci)) {
                    gerr = kErrUnsupported;
                } else {
                    double g[kDualDirs];
                    for (int k = 0; k < kDualDirs; ++k) g[k] = 0.0;
                    for (uint32_t k = ci; k < cj; ++k) {
                        const Cb& cb = cbs[k];
                        const int s = (int)(k - ci);
                        acc_dual(pd.normal, cb.n, g);
                        acc_dual(pd.point[s], cb.p, g);
                        for (int q = 0; q < kDualDirs; ++q) g[q] += cb.ov * pd.depth[s].d[q];
                    }
                    const Bc A = load_bc(d, b0 + c.a), B = load_bc(d, b0 + c.b);
                    if (mutable_(A)) {
                        add(sb[c.a].x, mk(g[0], g[1], g[2]));
                        addq(sb[c.a].q, mkq(g[3], g[4], g[5], g[6]));
                    }
                    if (mutable_(B)) {
                        add(sb[c.b].x, mk(g[7], g[8], g[9]));
                        addq(sb[c.b].q, mkq(g[10], g[11], g[12], g[13]));
                    }
                }
            }
            ci = cj;
        }
        w.err |= t.any_or(gerr);
        if (w.err & kErrUnsupported) return;
    }
#undef NE_ADJ_BODY
    t.sync();
    // Integration (World::integrate) per body.
    for (uint32_t b = t.lane; b < nb; b += t.size) {
        const Bc B = load_bc(d, b0 + b);
        const St& s0 = w.s0[b];
        St& g = sb[b];
        const double dt = W.dt;
        St o = st_zero();
        if (B.meta.y & NE_BODY_KINEMATIC) {
            // x1 = x + v dt; q1 = iorient(q, w); v, w unchanged
            o.x = g.x;
            o.v = g.v + g.x * dt;
            o.w = g.w;
            iorient_vjp(s0.q, s0.w, dt, g.q, o.q, o.w);
        } else if (B.invM <= 0.0) {
            o = g;
        } else {
            const double cl = (B.lin > 0.0) ? 1.0 / (1.0 + B.lin * dt) : 1.0;
            const double ca = (B.ang > 0.0) ? 1.0 / (1.0 + B.ang * dt) : 1.0;
            V3 v1b = g.v * cl;     // adjoint of the undamped v1
            const V3 w1b = g.w * ca;
            // recompute the forward intermediates
            const V3 L0 = angular_momentum(s0.q, B.invI, s0.w);
            const V3 L = L0 + s0.t * dt;
            const Q q1 = integrate_orientation(s0.q, s0.w, dt);
            Q q1b = g.q;
            V3 Lb = mk(0.0, 0.0, 0.0);
            aii_vjp(q1, B.invI, L, w1b, q1b, pb[b].invI, Lb);
            o.t = Lb * dt;
            angmom_vjp(s0.q, B.invI, s0.w, Lb, o.q, pb[b].invI, o.w);
            iorient_vjp(s0.q, s0.w, dt, q1b, o.q, o.w);
            o.x = g.x;
            add(v1b, g.x * dt);
            o.v = v1b;
            o.f = v1b * (B.invM * dt);
            pb[b].invM += dot(v1b, s0.f) * dt;
        }
        sb[b] = o;
    }
    t.sync();
    mub += t.sum(mub_l);
    eb += t.sum(eb_l);
}

}  // namespace adj

// ---- stepBackward launch ----------------------------------------------------------

constexpr uint32_t kAdjMaxBodies = 1024;

// Everything k_adj_world reads and writes (device pointers).  Body-indexed
// arrays use global body indices; contact-indexed ones give world w the range
// [coff[w], coff[w] + cap[w]) of CT entries.  Warm-cache slots: 0-1 the
// running caches, 2 .. 2+nck-1 the checkpoints, 2+nck .. 2+nck+K-1 the
// recomputed segment; slot s of world w lives at s*CT + coff[w] (counts at
// s*nworlds + w).
struct AdjArgs {
    DevWorld d;
    const WorldP* wp;
    const uint32_t* wbegin;        // [nworlds + 1]
    uint32_t nworlds, n;
    int warm;
    uint32_t nsteps, K, nck;
    const unsigned long long* wk0; // the device warm cache at the start
    const double* wi0;
    uint32_t nw0;
    const uint32_t* coff;          // [nworlds]
    const uint32_t* cap;           // [nworlds]
    uint32_t CT;
    adj::St *S, *S0, *S1, *SB;     // [n]
    uint32_t* UF;                  // [n] union-find scratch
    adj::St *CKS, *SEGS;           // [nck * n], [K * n]
    adj::Pb* PB;                   // [n]
    adj::Con* CON;                 // [CT]
    adj::Cb* CBS;                  // [CT]
    double* TAPE;                  // [9 * 14 * CT]
    unsigned long long* WK;        // [(2 + nck + K) * CT]
    double* WI;
    uint32_t* WN;                  // [(2 + nck + K) * nworlds]
    double *WOB, *WIB;             // [CT]
    const double *xbar, *vbar;     // [3n] or null
    double *gx, *gq, *gv, *gw;     // [3n] [4n] [3n] [3n] or null
    double *ginvm, *ginvi;         // [n] [3n]
    double *gmu, *ge;              // [nworlds]
    int* err;                      // [nworlds]
};

void launch_adjoint(const AdjArgs& a, cudaStream_t st);

}  // namespace neb
