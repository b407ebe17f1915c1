/* ne_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle's C restatement).
 *
 * A plain-C, single-threaded restatement of the reference's World::step()
 * (src/world.cpp:133-146) for the configurations the device path supports:
 * integrate (src/world.cpp:373-411), broadphasePairs (:424-501), collide
 * (:503-627) with detectContact (src/detect.hpp:33-77), GJK/EPA
 * (src/epa.hpp:28-158), the analytic contacts (src/narrowphase.hpp:34-155),
 * box-box clipping (src/manifold.hpp:55-126), and the boundary (:635-702).
 * Every expression keeps the reference's evaluation order, and growable
 * arrays stand where the reference grows std::vectors, so on x86-64 (no FMA
 * contraction) it reproduces the reference bit for bit; the CPU test suite
 * pins it to the reference compiled from its own sources.  Only the tests and
 * the benchmark's CPU-baseline leg may load it.  Joints, sleeping, CCD,
 * meshes and compounds are not restated (the device path refuses them too).
 */
#include "ne_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- vectors / quaternions (src/vmath.hpp:18-132) ---------------------- */

typedef struct { double x, y, z; } v3;
typedef struct { double w, x, y, z; } qt;

static v3 V(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static v3 vmul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 vdiv(v3 a, double s) { return V(a.x / s, a.y / s, a.z / s); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 vcross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static double vnorm2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static double vnorm(v3 a) { return sqrt(vnorm2(a)); }
static v3 vnormalized(v3 a) {
    double n = vnorm(a);
    return (n > 1e-300) ? V(a.x / n, a.y / n, a.z / n) : V(0, 0, 0);
}
static double comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

static qt Qn(double w, double x, double y, double z) { qt r; r.w = w; r.x = x; r.y = y; r.z = z; return r; }
static qt qmul(qt a, qt o) {
    return Qn(a.w * o.w - a.x * o.x - a.y * o.y - a.z * o.z, a.w * o.x + a.x * o.w + a.y * o.z - a.z * o.y,
              a.w * o.y - a.x * o.z + a.y * o.w + a.z * o.x, a.w * o.z + a.x * o.y - a.y * o.x + a.z * o.w);
}
static qt qnormalized(qt a) {
    double n = sqrt(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    return (n > 1e-300) ? Qn(a.w / n, a.x / n, a.y / n, a.z / n) : Qn(1, 0, 0, 0);
}
static v3 qrot(qt q, v3 v) {
    v3 qv = V(q.x, q.y, q.z);
    v3 t = vmul(vcross(qv, v), 2.0);
    return vadd(vadd(v, vmul(t, q.w)), vcross(qv, t));
}
static v3 qirot(qt q, v3 v) { return qrot(Qn(q.w, -q.x, -q.y, -q.z), v); }
static qt integrate_orientation(qt q, v3 w, double dt) {
    qt om = Qn(0.0, w.x, w.y, w.z);
    qt dq = qmul(om, q);
    double h = 0.5 * dt;
    dq = Qn(dq.w * h, dq.x * h, dq.y * h, dq.z * h);
    return qnormalized(Qn(q.w + dq.w, q.x + dq.x, q.y + dq.y, q.z + dq.z));
}

/* ---- bodies -------------------------------------------------------------- */

typedef struct {
    v3 x, v, w, force, torque;
    qt q;
    double invm;
    v3 invi;
    int shape;
    double radius, hh;
    v3 he;
    v3* verts;
    int nverts;
    double fric, rest, ldamp, adamp, gscale;
    uint32_t layer, mask, flags;
    uint32_t* nocol;
    int nnocol;
} Body;

static v3 inv_inertia_apply(const Body* b, v3 u) {   /* src/body.hpp:162-168 */
    v3 ub = qirot(b->q, u);
    v3 sb = V(ub.x * b->invi.x, ub.y * b->invi.y, ub.z * b->invi.z);
    return qrot(b->q, sb);
}

static v3 angular_momentum(const Body* b) {   /* src/body.hpp:195-202 */
    v3 Ib = V(b->invi.x > 0 ? 1.0 / b->invi.x : 0.0, b->invi.y > 0 ? 1.0 / b->invi.y : 0.0,
              b->invi.z > 0 ? 1.0 / b->invi.z : 0.0);
    v3 wb = qirot(b->q, b->w);
    v3 Lb = V(wb.x * Ib.x, wb.y * Ib.y, wb.z * Ib.z);
    return qrot(b->q, Lb);
}

static double bounding_radius(const Body* b) {   /* src/body.hpp:137-158 */
    if (b->shape == NE_SHAPE_SPHERE) return b->radius;
    if (b->shape == NE_SHAPE_BOX) return vnorm(b->he);
    if (b->shape == NE_SHAPE_CAPSULE) return b->hh + b->radius;
    if (b->shape == NE_SHAPE_PLANE || b->shape == NE_SHAPE_MESH) return 1e30;
    if (b->shape == NE_SHAPE_CONVEX) {
        double m = 0.0;
        for (int k = 0; k < b->nverts; ++k) {
            double r = vnorm(b->verts[k]);
            m = (m < r) ? r : m;
        }
        return m;
    }
    return sqrt(b->hh * b->hh + b->radius * b->radius);
}

/* ---- domain (src/box.hpp:24-41) ----------------------------------------- */

typedef struct { double half; int periodic; } Dom;

static v3 min_image(Dom d, v3 v) {
    if (!d.periodic) return v;
    double L = 2.0 * d.half;
    v.x -= L * floor(v.x / L + 0.5);
    v.y -= L * floor(v.y / L + 0.5);
    v.z -= L * floor(v.z / L + 0.5);
    return v;
}

static v3 wrap_pos(Dom d, v3 p) {
    if (!d.periodic) return p;
    double L = 2.0 * d.half;
    p.x -= L * floor((p.x + d.half) / L);
    p.y -= L * floor((p.y + d.half) / L);
    p.z -= L * floor((p.z + d.half) / L);
    return p;
}

/* ---- narrowphase --------------------------------------------------------- */

typedef struct { int hit; v3 normal, point; double overlap; } Contact;

static Contact no_contact(void) { Contact c; memset(&c, 0, sizeof c); return c; }

static v3 support(const Body* b, v3 d) {   /* src/gjk.hpp:17-46 */
    if (b->shape == NE_SHAPE_SPHERE) return vadd(b->x, vmul(vnormalized(d), b->radius));
    v3 db = qirot(b->q, d), sb;
    if (b->shape == NE_SHAPE_BOX) {
        sb = V(db.x >= 0 ? b->he.x : -b->he.x, db.y >= 0 ? b->he.y : -b->he.y, db.z >= 0 ? b->he.z : -b->he.z);
    } else if (b->shape == NE_SHAPE_CAPSULE) {
        double sy = (db.y >= 0.0) ? b->hh : -b->hh;
        sb = vadd(V(0.0, sy, 0.0), vmul(vnormalized(db), b->radius));
    } else if (b->shape == NE_SHAPE_CONVEX) {
        double best = -1e300;
        sb = V(0, 0, 0);
        for (int k = 0; k < b->nverts; ++k) {
            double dp = vdot(b->verts[k], db);
            if (dp > best) { best = dp; sb = b->verts[k]; }
        }
    } else {
        double sy = (db.y >= 0.0) ? b->hh : -b->hh;
        double rho = sqrt(db.x * db.x + db.z * db.z);
        sb = (rho > 1e-12) ? V(db.x / rho * b->radius, sy, db.z / rho * b->radius) : V(0.0, sy, 0.0);
    }
    return vadd(b->x, qrot(b->q, sb));
}

static Contact plane_vs_convex(const Body* other, const Body* plane, Dom dom) {
    Contact c = no_contact();
    v3 n = plane->he;
    v3 sp = support(other, vneg(n));
    v3 rel = min_image(dom, vsub(sp, plane->x));
    double pen = -vdot(n, rel);
    if (pen <= 0.0) return c;
    c.hit = 1; c.overlap = pen; c.normal = n;
    c.point = vadd(sp, vmul(n, 0.5 * pen));
    return c;
}

static Contact sphere_vs_cylinder(const Body* sph, const Body* cyl, Dom dom) {
    Contact c = no_contact();
    const double r = cyl->radius, h = cyl->hh, sr = sph->radius;
    v3 L = qirot(cyl->q, min_image(dom, vsub(sph->x, cyl->x)));
    double rho = sqrt(L.x * L.x + L.z * L.z);
    int inA = fabs(L.y) < h, inR = rho < r;
    v3 P, nl;
    if (inA && inR) {
        double dCap = h - fabs(L.y), dSide = r - rho;
        if (dSide < dCap) {
            double s = (rho > 1e-12) ? r / rho : 0.0;
            P = V(L.x * s, L.y, L.z * s);
            nl = (rho > 1e-12) ? V(L.x / rho, 0, L.z / rho) : V(1, 0, 0);
            c.overlap = sr + dSide;
        } else {
            double sy = (L.y >= 0) ? h : -h;
            P = V(L.x, sy, L.z);
            nl = V(0, (L.y >= 0) ? 1.0 : -1.0, 0);
            c.overlap = sr + dCap;
        }
        c.hit = 1;
    } else {
        double yc = (L.y > h) ? h : (L.y < -h ? -h : L.y);
        double rx = L.x, rz = L.z;
        if (rho > r) { double s = r / rho; rx *= s; rz *= s; }
        P = V(rx, yc, rz);
        v3 diff = vsub(L, P);
        double dist = vnorm(diff);
        if (dist >= sr) return c;
        c.hit = 1;
        c.overlap = sr - dist;
        nl = (dist > 1e-12) ? vdiv(diff, dist) : V(0, 1, 0);
    }
    c.normal = vnormalized(qrot(cyl->q, nl));
    c.point = vadd(cyl->x, qrot(cyl->q, P));
    return c;
}

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

static v3 closest_on_segment(v3 p, v3 a, v3 b) {
    v3 ab = vsub(b, a);
    double L2 = vnorm2(ab);
    if (L2 < 1e-18) return a;
    return vadd(a, vmul(ab, clampd(vdot(vsub(p, a), ab) / L2, 0.0, 1.0)));
}

static void closest_seg_seg(v3 p1, v3 q1, v3 p2, v3 q2, v3* c1, v3* c2) {
    v3 d1 = vsub(q1, p1), d2 = vsub(q2, p2), r = vsub(p1, p2);
    double a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    const double EPS = 1e-12;
    double s, t;
    if (a <= EPS && e <= EPS) { s = t = 0.0; }
    else if (a <= EPS) { s = 0.0; t = clampd(f / e, 0.0, 1.0); }
    else {
        double c = vdot(d1, r);
        if (e <= EPS) { t = 0.0; s = clampd(-c / a, 0.0, 1.0); }
        else {
            double b = vdot(d1, d2), denom = a * e - b * b;
            s = denom > EPS ? clampd((b * f - c * e) / denom, 0.0, 1.0) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) { t = 0.0; s = clampd(-c / a, 0.0, 1.0); }
            else if (t > 1.0) { t = 1.0; s = clampd((b - c) / a, 0.0, 1.0); }
        }
    }
    *c1 = vadd(p1, vmul(d1, s));
    *c2 = vadd(p2, vmul(d2, t));
}

static Contact capsule_vs_sphere(const Body* cap, const Body* sph, Dom dom) {
    Contact c = no_contact();
    v3 sc = vadd(cap->x, min_image(dom, vsub(sph->x, cap->x)));
    v3 axis = qrot(cap->q, V(0, 1, 0));
    v3 cp = closest_on_segment(sc, vsub(cap->x, vmul(axis, cap->hh)), vadd(cap->x, vmul(axis, cap->hh)));
    v3 e = vsub(sc, cp);
    double dist = vnorm(e), sumR = cap->radius + sph->radius;
    if (dist >= sumR) return c;
    v3 nrm = (dist > 1e-12) ? vdiv(e, dist) : V(0, 1, 0);
    c.hit = 1; c.overlap = sumR - dist; c.normal = vneg(nrm);
    c.point = vadd(cp, vmul(nrm, cap->radius));
    return c;
}

static Contact capsule_vs_capsule(const Body* A, const Body* B, Dom dom) {
    Contact c = no_contact();
    v3 axA = qrot(A->q, V(0, 1, 0)), axB = qrot(B->q, V(0, 1, 0));
    v3 bc = vadd(A->x, min_image(dom, vsub(B->x, A->x)));
    v3 pA, pB;
    closest_seg_seg(vsub(A->x, vmul(axA, A->hh)), vadd(A->x, vmul(axA, A->hh)), vsub(bc, vmul(axB, B->hh)),
                    vadd(bc, vmul(axB, B->hh)), &pA, &pB);
    v3 e = vsub(pB, pA);
    double dist = vnorm(e), sumR = A->radius + B->radius;
    if (dist >= sumR) return c;
    v3 nrm = (dist > 1e-12) ? vdiv(e, dist) : V(0, 1, 0);
    c.hit = 1; c.overlap = sumR - dist; c.normal = vneg(nrm);
    c.point = vadd(pA, vmul(nrm, A->radius));
    return c;
}

/* GJK returning an enclosing tetrahedron, EPA (src/epa.hpp:15-158). */
typedef struct { v3 v, a, b; } SupportV;
typedef struct { int a, b, c; v3 n; double dist; } Face;

static SupportV cso(const Body* A, const Body* B, v3 shift, v3 d) {
    SupportV s;
    s.a = support(A, d);
    s.b = vadd(support(B, vneg(d)), shift);
    s.v = vsub(s.a, s.b);
    return s;
}

static int gjk_tetra(const Body* A, const Body* B, v3 shift, SupportV tet[4]) {
    v3 d = V(1, 0, 0);
    SupportV s = cso(A, B, shift, d);
    if (vnorm2(s.v) < 1e-24) { d = V(0, 1, 0); s = cso(A, B, shift, d); }
    SupportV W[5];
    int n = 1;
    W[0] = s;
    d = vneg(s.v);
    for (int iter = 0; iter < 64; ++iter) {
        if (vnorm2(d) < 1e-24) d = V(1, 0, 0);
        SupportV p = cso(A, B, shift, d);
        if (vdot(p.v, d) <= 1e-12) return 0;
        for (int k = n; k > 0; --k) W[k] = W[k - 1];
        W[0] = p;
        ++n;
        v3 a = W[0].v, ao = vneg(a);
        if (n == 2) {
            v3 ab = vsub(W[1].v, a);
            d = vcross(vcross(ab, ao), ab);
            if (vnorm2(d) < 1e-24) d = V(ab.y, -ab.x, 0);
        } else if (n == 3) {
            v3 ab = vsub(W[1].v, a), ac = vsub(W[2].v, a), abc = vcross(ab, ac);
            if (vdot(abc, ao) > 0) d = abc;
            else { SupportV t = W[1]; W[1] = W[2]; W[2] = t; d = vneg(abc); }
            if (vnorm2(d) < 1e-24) return 0;
        } else {
            v3 ab = vsub(W[1].v, a), ac = vsub(W[2].v, a), ad = vsub(W[3].v, a);
            v3 abc = vcross(ab, ac), acd = vcross(ac, ad), adb = vcross(ad, ab);
            if (vdot(abc, ao) > 0) { n = 3; d = abc; }
            else if (vdot(acd, ao) > 0) { W[1] = W[2]; W[2] = W[3]; n = 3; d = acd; }
            else if (vdot(adb, ao) > 0) { SupportV w1 = W[1]; W[1] = W[3]; W[2] = w1; n = 3; d = adb; }
            else { for (int k = 0; k < 4; ++k) tet[k] = W[k]; return 1; }
        }
    }
    return 0;
}

typedef struct { void* p; int n, cap; size_t sz; } Vec;
static void vec_push(Vec* v, const void* x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 16; v->p = realloc(v->p, (size_t)v->cap * v->sz); }
    memcpy((char*)v->p + (size_t)v->n * v->sz, x, v->sz);
    ++v->n;
}

static Face make_face(const SupportV* vs, int i, int j, int k) {
    v3 n = vcross(vsub(vs[j].v, vs[i].v), vsub(vs[k].v, vs[i].v));
    double L = vnorm(n);
    n = (L > 1e-18) ? vdiv(n, L) : V(0, 0, 1);
    double dist = vdot(n, vs[i].v);
    if (dist < 0) { n = vneg(n); dist = -dist; int t = j; j = k; k = t; }
    Face f; f.a = i; f.b = j; f.c = k; f.n = n; f.dist = dist;
    return f;
}

static Contact epa_contact(const Body* A, const Body* B, v3 shift, const SupportV tet[4]) {
    Vec verts = {0, 0, 0, sizeof(SupportV)}, faces = {0, 0, 0, sizeof(Face)};
    Vec keep = {0, 0, 0, sizeof(Face)}, hz = {0, 0, 0, 2 * sizeof(int)};
    for (int k = 0; k < 4; ++k) vec_push(&verts, &tet[k]);
    SupportV* vs = (SupportV*)verts.p;
    Face f0 = make_face(vs, 0, 1, 2), f1 = make_face(vs, 0, 2, 3), f2 = make_face(vs, 0, 3, 1), f3 = make_face(vs, 1, 3, 2);
    vec_push(&faces, &f0); vec_push(&faces, &f1); vec_push(&faces, &f2); vec_push(&faces, &f3);
    Face best;
    memset(&best, 0, sizeof best);
    for (int iter = 0; iter < 64; ++iter) {
        Face* F = (Face*)faces.p;
        int ci = 0;
        for (int i = 1; i < faces.n; ++i) if (F[i].dist < F[ci].dist) ci = i;
        best = F[ci];
        SupportV p = cso(A, B, shift, best.n);
        double d = vdot(p.v, best.n);
        if (d - best.dist < 1e-7) break;
        int pidx = verts.n;
        vec_push(&verts, &p);
        vs = (SupportV*)verts.p;
        hz.n = 0; keep.n = 0;
        F = (Face*)faces.p;
        for (int fi = 0; fi < faces.n; ++fi) {
            const Face f = F[fi];
            if (vdot(f.n, vsub(p.v, vs[f.a].v)) > 1e-12) {
                int ed[3][2] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
                for (int q = 0; q < 3; ++q) {
                    int u = ed[q][0], w = ed[q][1], found = -1;
                    int* H = (int*)hz.p;
                    for (int e = 0; e < hz.n; ++e) if (H[2 * e] == w && H[2 * e + 1] == u) { found = e; break; }
                    if (found >= 0) {
                        memmove(H + 2 * found, H + 2 * found + 2, (size_t)(hz.n - found - 1) * 2 * sizeof(int));
                        --hz.n;
                    } else {
                        int pr[2] = {u, w};
                        vec_push(&hz, pr);
                    }
                }
            } else {
                vec_push(&keep, &f);
            }
        }
        faces.n = 0;
        for (int k = 0; k < keep.n; ++k) vec_push(&faces, (Face*)keep.p + k);
        int* H = (int*)hz.p;
        for (int e = 0; e < hz.n; ++e) { Face nf = make_face(vs, H[2 * e], H[2 * e + 1], pidx); vec_push(&faces, &nf); }
        if (faces.n == 0) break;
    }
    vs = (SupportV*)verts.p;
    const SupportV A0 = vs[best.a], B0 = vs[best.b], C0 = vs[best.c];
    v3 proj = vmul(best.n, best.dist);
    v3 v0 = vsub(B0.v, A0.v), v1 = vsub(C0.v, A0.v), v2 = vsub(proj, A0.v);
    double d00 = vdot(v0, v0), d01 = vdot(v0, v1), d11 = vdot(v1, v1), d20 = vdot(v2, v0), d21 = vdot(v2, v1);
    double den = d00 * d11 - d01 * d01, bv = 0, bw = 0;
    if (fabs(den) > 1e-18) { bv = (d11 * d20 - d01 * d21) / den; bw = (d00 * d21 - d01 * d20) / den; }
    double bu = 1.0 - bv - bw;
    v3 onA = vadd(vadd(vmul(A0.a, bu), vmul(B0.a, bv)), vmul(C0.a, bw));
    v3 onB = vadd(vadd(vmul(A0.b, bu), vmul(B0.b, bv)), vmul(C0.b, bw));
    Contact c;
    c.hit = 1; c.normal = vneg(best.n); c.overlap = best.dist; c.point = vmul(vadd(onA, onB), 0.5);
    free(verts.p); free(faces.p); free(keep.p); free(hz.p);
    return c;
}

static v3 min_image_shift(const Body* A, const Body* B, Dom dom) {
    v3 raw = vsub(B->x, A->x);
    return vsub(min_image(dom, raw), raw);
}

static Contact convex_contact(const Body* A, const Body* B, Dom dom) {
    v3 shift = min_image_shift(A, B, dom);
    SupportV tet[4];
    if (!gjk_tetra(A, B, shift, tet)) return no_contact();
    return epa_contact(A, B, shift, tet);
}

static Contact detect_contact(const Body* a, const Body* b, Dom dom) {   /* src/detect.hpp:33-77 */
    if (a->shape == NE_SHAPE_PLANE || b->shape == NE_SHAPE_PLANE) {
        if (a->shape == NE_SHAPE_PLANE && b->shape == NE_SHAPE_PLANE) return no_contact();
        const Body* plane = (a->shape == NE_SHAPE_PLANE) ? a : b;
        const Body* other = (a->shape == NE_SHAPE_PLANE) ? b : a;
        Contact t = plane_vs_convex(other, plane, dom);
        if (t.hit && a->shape == NE_SHAPE_PLANE) t.normal = vneg(t.normal);
        return t;
    }
    if (a->shape == NE_SHAPE_SPHERE && b->shape == NE_SHAPE_SPHERE) {
        Contact c = no_contact();
        v3 d = min_image(dom, vsub(a->x, b->x));
        double sumR = a->radius + b->radius, dist2 = vnorm2(d);
        if (dist2 >= sumR * sumR || dist2 < 1e-18) return c;
        double dist = sqrt(dist2);
        c.hit = 1; c.normal = vdiv(d, dist); c.overlap = sumR - dist;
        c.point = vsub(a->x, vmul(c.normal, a->radius));
        return c;
    }
    int aCyl = a->shape == NE_SHAPE_CYLINDER, bCyl = b->shape == NE_SHAPE_CYLINDER;
    if (a->shape == NE_SHAPE_SPHERE && bCyl) return sphere_vs_cylinder(a, b, dom);
    if (b->shape == NE_SHAPE_SPHERE && aCyl) {
        Contact t = sphere_vs_cylinder(b, a, dom);
        if (t.hit) t.normal = vneg(t.normal);
        return t;
    }
    int aCap = a->shape == NE_SHAPE_CAPSULE, bCap = b->shape == NE_SHAPE_CAPSULE;
    if (aCap && bCap) return capsule_vs_capsule(a, b, dom);
    if (aCap && b->shape == NE_SHAPE_SPHERE) return capsule_vs_sphere(a, b, dom);
    if (a->shape == NE_SHAPE_SPHERE && bCap) {
        Contact t = capsule_vs_sphere(b, a, dom);
        if (t.hit) t.normal = vneg(t.normal);
        return t;
    }
    return convex_contact(a, b, dom);
}

/* Box-box clipping manifold (src/manifold.hpp:55-126). */
typedef struct { v3 n, c, u, v; double eu, ev; v3 vert[4]; } BoxFace;

static v3 axis_vec(int a) { return a == 0 ? V(1, 0, 0) : (a == 1 ? V(0, 1, 0) : V(0, 0, 1)); }

static BoxFace box_face(const Body* b, v3 centre, int axis, int sign) {
    const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
    const double h[3] = {b->he.x, b->he.y, b->he.z};
    BoxFace f;
    f.n = qrot(b->q, vmul(axis_vec(axis), (double)sign));
    f.c = vadd(centre, vmul(f.n, h[axis]));
    f.u = qrot(b->q, axis_vec(t1)); f.eu = h[t1];
    f.v = qrot(b->q, axis_vec(t2)); f.ev = h[t2];
    f.vert[0] = vadd(vadd(f.c, vmul(f.u, f.eu)), vmul(f.v, f.ev));
    f.vert[1] = vadd(vsub(f.c, vmul(f.u, f.eu)), vmul(f.v, f.ev));
    f.vert[2] = vsub(vsub(f.c, vmul(f.u, f.eu)), vmul(f.v, f.ev));
    f.vert[3] = vsub(vadd(f.c, vmul(f.u, f.eu)), vmul(f.v, f.ev));
    return f;
}

static BoxFace best_face(const Body* b, v3 centre, v3 dir) {
    int ba = 0, bs = 1;
    double best = -1e30;
    for (int axis = 0; axis < 3; ++axis)
        for (int sign = -1; sign <= 1; sign += 2) {
            double a = vdot(qrot(b->q, vmul(axis_vec(axis), (double)sign)), dir);
            if (a > best) { best = a; ba = axis; bs = sign; }
        }
    return box_face(b, centre, ba, bs);
}

static int clip_plane(v3* poly, int m, v3* out, v3 pn, double off) {
    int o = 0;
    for (int i = 0; i < m; ++i) {
        v3 cur = poly[i], nxt = poly[(i + 1) % m];
        double dc = vdot(cur, pn) - off, dn = vdot(nxt, pn) - off;
        int inC = dc <= 0.0, inN = dn <= 0.0;
        if (inC) out[o++] = cur;
        if (inC != inN) { double t = dc / (dc - dn); out[o++] = vadd(cur, vmul(vsub(nxt, cur), t)); }
    }
    return o;
}

static int box_box_manifold(const Body* a, const Body* b, v3 n, Dom dom, v3 pts[4], double dep[4]) {
    v3 bShift = min_image_shift(a, b, dom);
    v3 bC = vadd(b->x, bShift);
    BoxFace fa = best_face(a, a->x, vneg(n)), fb = best_face(b, bC, n);
    double alignA = vdot(fa.n, vneg(n)), alignB = vdot(fb.n, n);
    int refA = alignA >= alignB;
    BoxFace ref = refA ? fa : fb;
    BoxFace inc = best_face(refA ? b : a, refA ? bC : a->x, vneg(ref.n));
    v3 buf[2][80];
    int np = 4;
    for (int k = 0; k < 4; ++k) buf[0][k] = inc.vert[k];
    np = clip_plane(buf[0], np, buf[1], ref.u, vdot(ref.c, ref.u) + ref.eu);
    np = clip_plane(buf[1], np, buf[0], vmul(ref.u, -1.0), -(vdot(ref.c, ref.u) - ref.eu));
    np = clip_plane(buf[0], np, buf[1], ref.v, vdot(ref.c, ref.v) + ref.ev);
    np = clip_plane(buf[1], np, buf[0], vmul(ref.v, -1.0), -(vdot(ref.c, ref.v) - ref.ev));
    int count = 0;
    for (int k = 0; k < np; ++k) {
        double sd = vdot(vsub(buf[0][k], ref.c), ref.n);
        if (sd > 0.01) continue;
        if (count >= 4) break;
        pts[count] = vsub(buf[0][k], vmul(ref.n, sd));
        dep[count] = -sd;
        ++count;
    }
    return count;
}

/* ---- the world ------------------------------------------------------------ */

typedef struct {
    uint32_t i, j;
    v3 n, rA, rB, point;
    double overlap, restBias, mu, nImp, tImp;
    uint64_t key;
    int slot;
} Con;

typedef struct {
    NeWorldParams p;
    int n;
    Body* B;
    v3* vpool;
    uint32_t* ncpool;
    /* warm cache: sorted (key, slot) -> nImp */
    uint64_t* wkey;
    int* wslot;
    double* wimp;
    int wn;
    /* last step */
    uint32_t *pi, *pj;
    uint64_t np;
    Con* cons;
    int ncons;
    uint32_t* label;
} World;

static double combine(int m, double a, double b) {   /* src/world.cpp:42-51 */
    switch (m) {
        case NE_COMBINE_AVERAGE: return 0.5 * (a + b);
        case NE_COMBINE_MIN: return a < b ? a : b;
        case NE_COMBINE_MAX: return a > b ? a : b;
        case NE_COMBINE_MULTIPLY: return a * b;
        case NE_COMBINE_GEOMETRIC_MEAN: return sqrt((a > 0 ? a : 0) * (b > 0 ? b : 0));
    }
    return 0.5 * (a + b);
}

static double eff_mass(const Body* a, const Body* b, v3 ra, v3 rb, v3 u) {   /* src/contact.hpp:28-33 */
    v3 angA = vcross(inv_inertia_apply(a, vcross(ra, u)), ra);
    v3 angB = vcross(inv_inertia_apply(b, vcross(rb, u)), rb);
    return a->invm + b->invm + vdot(vadd(angA, angB), u);
}

static void integrate(World* W) {   /* src/world.cpp:373-411 */
    const double dt = W->p.dt;
    const v3 g = V(W->p.gravity[0], W->p.gravity[1], W->p.gravity[2]);
    for (int k = 0; k < W->n; ++k) {
        Body* b = &W->B[k];
        if (b->flags & NE_BODY_KINEMATIC) {
            b->x = vadd(b->x, vmul(b->v, dt));
            b->q = integrate_orientation(b->q, b->w, dt);
        } else if (b->invm <= 0.0) {
        } else {
            b->v = vadd(b->v, vmul(vadd(vmul(g, b->gscale), vmul(b->force, b->invm)), dt));
            b->x = vadd(b->x, vmul(b->v, dt));
            v3 L = angular_momentum(b);
            L = vadd(L, vmul(b->torque, dt));
            b->q = integrate_orientation(b->q, b->w, dt);
            b->w = inv_inertia_apply(b, L);
            if (b->ldamp > 0.0) b->v = vmul(b->v, 1.0 / (1.0 + b->ldamp * dt));
            if (b->adamp > 0.0) b->w = vmul(b->w, 1.0 / (1.0 + b->adamp * dt));
        }
        b->force = V(0, 0, 0);
        b->torque = V(0, 0, 0);
    }
}

typedef struct { uint64_t key; uint32_t idx; } KeyIdx;
static int cmp_keyidx(const void* x, const void* y) {
    const KeyIdx *a = x, *b = y;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->idx < b->idx ? -1 : (a->idx > b->idx);
}
static int cmp_pair(const void* x, const void* y) {
    const uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return a < b ? -1 : (a > b);
}

static uint64_t cell_key(long x, long y, long z) {
    return (uint64_t)(x & 0x1FFFFF) | ((uint64_t)(y & 0x1FFFFF) << 21) | ((uint64_t)(z & 0x1FFFFF) << 42);
}

/* World::broadphasePairs (src/world.cpp:424-501): pairs as (i << 32 | j). */
static void broadphase(World* W) {
    const int n = W->n;
    Vec pairs = {0, 0, 0, sizeof(uint64_t)};
    double maxR = 0.0;
    int anyPlane = 0;
    for (int k = 0; k < n; ++k) {
        const Body* b = &W->B[k];
        if (b->shape == NE_SHAPE_PLANE || b->shape == NE_SHAPE_MESH) { anyPlane = 1; continue; }
        double r = bounding_radius(b);
        maxR = (maxR < r) ? r : maxR;
    }
    const double cell = 2.0 * maxR;
    if (W->p.force_brute_force || n < 64 || cell < 1e-9) {
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) { uint64_t pr = ((uint64_t)i << 32) | (uint32_t)j; vec_push(&pairs, &pr); }
    } else {
        long nc[3] = {1, 1, 1};
        const int per = W->p.periodic != 0;
        const double half = W->p.half;
        if (per) {
            double L = 2.0 * half;
            for (int a = 0; a < 3; ++a) { int m = (int)floor(L / cell); nc[a] = m < 1 ? 1 : m; }
        }
        KeyIdx* grid = malloc(sizeof(KeyIdx) * (size_t)(n ? n : 1));
        long (*cells)[3] = malloc(sizeof(long[3]) * (size_t)(n ? n : 1));
        int ng = 0;
        for (int i = 0; i < n; ++i) {
            const Body* b = &W->B[i];
            if (b->shape == NE_SHAPE_PLANE || b->shape == NE_SHAPE_MESH) continue;
            for (int a = 0; a < 3; ++a) {
                double c = comp(b->x, a);
                if (per) {
                    long k = (long)floor((c + half) / cell), m = nc[a];
                    cells[i][a] = ((k % m) + m) % m;
                } else {
                    cells[i][a] = (long)floor(c / cell);
                }
            }
            grid[ng].key = cell_key(cells[i][0], cells[i][1], cells[i][2]);
            grid[ng].idx = (uint32_t)i;
            ++ng;
        }
        qsort(grid, (size_t)ng, sizeof(KeyIdx), cmp_keyidx);
        for (int i = 0; i < n; ++i) {
            const Body* b = &W->B[i];
            if (b->shape == NE_SHAPE_PLANE || b->shape == NE_SHAPE_MESH) continue;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        long nx = cells[i][0] + dx, ny = cells[i][1] + dy, nz = cells[i][2] + dz;
                        if (per) {
                            nx = ((nx % nc[0]) + nc[0]) % nc[0];
                            ny = ((ny % nc[1]) + nc[1]) % nc[1];
                            nz = ((nz % nc[2]) + nc[2]) % nc[2];
                        }
                        uint64_t key = cell_key(nx, ny, nz);
                        int lo = 0, hi = ng;
                        while (lo < hi) { int mid = (lo + hi) / 2; if (grid[mid].key < key) lo = mid + 1; else hi = mid; }
                        for (int g = lo; g < ng && grid[g].key == key; ++g) {
                            uint32_t j = grid[g].idx;
                            if ((int)j == i) continue;
                            uint32_t a = (uint32_t)i < j ? (uint32_t)i : j, c = (uint32_t)i < j ? j : (uint32_t)i;
                            uint64_t pr = ((uint64_t)a << 32) | c;
                            vec_push(&pairs, &pr);
                        }
                    }
        }
        if (anyPlane) {
            for (int p = 0; p < n; ++p) {
                if (!(W->B[p].shape == NE_SHAPE_PLANE || W->B[p].shape == NE_SHAPE_MESH)) continue;
                for (int j = 0; j < n; ++j) {
                    if (j == p) continue;
                    uint32_t a = p < j ? (uint32_t)p : (uint32_t)j, c = p < j ? (uint32_t)j : (uint32_t)p;
                    uint64_t pr = ((uint64_t)a << 32) | c;
                    vec_push(&pairs, &pr);
                }
            }
        }
        free(grid);
        free(cells);
        qsort(pairs.p, (size_t)pairs.n, sizeof(uint64_t), cmp_pair);
        int u = 0;
        uint64_t* P = pairs.p;
        for (int k = 0; k < pairs.n; ++k)
            if (u == 0 || P[u - 1] != P[k]) P[u++] = P[k];
        pairs.n = u;
    }
    free(W->pi); free(W->pj);
    W->np = (uint64_t)pairs.n;
    W->pi = malloc(sizeof(uint32_t) * (size_t)(pairs.n ? pairs.n : 1));
    W->pj = malloc(sizeof(uint32_t) * (size_t)(pairs.n ? pairs.n : 1));
    for (int k = 0; k < pairs.n; ++k) {
        uint64_t pr = ((uint64_t*)pairs.p)[k];
        W->pi[k] = (uint32_t)(pr >> 32);
        W->pj[k] = (uint32_t)pr;
    }
    free(pairs.p);
}

static int warm_lookup(const World* W, uint64_t key, int slot, double* out) {
    int lo = 0, hi = W->wn;
    while (lo < hi) { int mid = (lo + hi) / 2; if (W->wkey[mid] < key) lo = mid + 1; else hi = mid; }
    for (int k = lo; k < W->wn && W->wkey[k] == key; ++k)
        if (W->wslot[k] == slot) { *out = W->wimp[k]; return 1; }
    return 0;
}

static void apply_impulse(Body* a, Body* b, v3 ra, v3 rb, v3 J) {
    a->v = vadd(a->v, vmul(J, a->invm));
    a->w = vadd(a->w, inv_inertia_apply(a, vcross(ra, J)));
    b->v = vsub(b->v, vmul(J, b->invm));
    b->w = vsub(b->w, inv_inertia_apply(b, vcross(rb, J)));
}

static uint32_t uf_find(uint32_t* parent, uint32_t x) {
    while (parent[x] != x) x = parent[x];
    return x;
}

/* World::collide (src/world.cpp:503-627). */
static void collide(World* W) {
    const Dom dom = {W->p.half, W->p.periodic};
    broadphase(W);
    Vec cons = {0, 0, 0, sizeof(Con)};
    Vec ipairs = {0, 0, 0, 2 * sizeof(uint32_t)};
    for (uint64_t pk = 0; pk < W->np; ++pk) {
        const uint32_t i = W->pi[pk], j = W->pj[pk];
        Body *a = &W->B[i], *b = &W->B[j];
        if (a->invm + b->invm <= 0.0) continue;
        if (!((a->mask & (1u << (b->layer & 31u))) && (b->mask & (1u << (a->layer & 31u))))) continue;
        int excluded = 0;
        for (int k = 0; k < a->nnocol; ++k) if (a->nocol[k] == j) excluded = 1;
        if (excluded) continue;
        if ((a->flags | b->flags) & NE_BODY_SENSOR) continue;
        Contact cs[4];
        int nc = 0;
        Contact c = detect_contact(a, b, dom);
        if (!c.hit) continue;
        if (a->shape == NE_SHAPE_BOX && b->shape == NE_SHAPE_BOX) {
            v3 pts[4];
            double dep[4];
            int m = box_box_manifold(a, b, c.normal, dom, pts, dep);
            for (int k = 0; k < m; ++k) { cs[k].hit = 1; cs[k].normal = c.normal; cs[k].point = pts[k]; cs[k].overlap = dep[k]; }
            nc = m;
        }
        if (nc == 0) { cs[0] = c; nc = 1; }
        const double ea = a->rest < 0 ? W->p.restitution : a->rest, eb = b->rest < 0 ? W->p.restitution : b->rest;
        const double fa = a->fric < 0 ? W->p.friction : a->fric, fb = b->fric < 0 ? W->p.friction : b->fric;
        const double e = combine(W->p.restitution_combine, ea, eb);
        const double mu = combine(W->p.friction_combine, fa, fb);
        if (a->invm > 0.0 && b->invm > 0.0) { uint32_t pr[2] = {i, j}; vec_push(&ipairs, pr); }
        const uint64_t key = ((uint64_t)i << 32) | j;
        for (int s = 0; s < nc; ++s) {
            Con k;
            memset(&k, 0, sizeof k);
            k.i = i; k.j = j; k.n = cs[s].normal; k.overlap = cs[s].overlap; k.mu = mu; k.point = cs[s].point;
            k.rA = min_image(dom, vsub(cs[s].point, a->x));
            k.rB = min_image(dom, vsub(cs[s].point, b->x));
            v3 vc = vsub(vadd(a->v, vcross(a->w, k.rA)), vadd(b->v, vcross(b->w, k.rB)));
            double vn = vdot(vc, k.n);
            k.restBias = (vn < -0.5) ? -e * vn : 0.0;
            k.key = key; k.slot = s;
            if (W->p.warm_start) warm_lookup(W, key, s, &k.nImp);
            vec_push(&cons, &k);
        }
    }
    Con* C = cons.p;
    const int m = cons.n;
    if (W->p.warm_start)
        for (int q = 0; q < m; ++q) {
            Con* k = &C[q];
            if (k->nImp == 0.0) continue;
            apply_impulse(&W->B[k->i], &W->B[k->j], k->rA, k->rB, vmul(k->n, k->nImp));
        }
    for (int it = 0; it < 8; ++it)
        for (int q = 0; q < m; ++q) {
            Con* k = &C[q];
            Body *a = &W->B[k->i], *b = &W->B[k->j];
            v3 vc = vsub(vadd(a->v, vcross(a->w, k->rA)), vadd(b->v, vcross(b->w, k->rB)));
            double vn = vdot(vc, k->n);
            double Kn = eff_mass(a, b, k->rA, k->rB, k->n);
            if (Kn > 1e-18) {
                double dj = (k->restBias - vn) / Kn;
                double old = k->nImp;
                k->nImp = (old + dj > 0.0) ? old + dj : 0.0;
                dj = k->nImp - old;
                apply_impulse(a, b, k->rA, k->rB, vmul(k->n, dj));
            }
            if (k->mu > 0.0 && k->nImp > 0.0) {
                v3 vc2 = vsub(vadd(a->v, vcross(a->w, k->rA)), vadd(b->v, vcross(b->w, k->rB)));
                v3 vt = vsub(vc2, vmul(k->n, vdot(vc2, k->n)));
                double vtl = vnorm(vt);
                if (vtl > 1e-12) {
                    v3 t = vdiv(vt, vtl);
                    double Kt = eff_mass(a, b, k->rA, k->rB, t);
                    if (Kt > 1e-18) {
                        double djt = -vtl / Kt;
                        double maxF = k->mu * k->nImp, old = k->tImp, sum = old + djt;
                        k->tImp = (sum < -maxF) ? -maxF : (sum > maxF ? maxF : sum);
                        djt = k->tImp - old;
                        apply_impulse(a, b, k->rA, k->rB, vmul(t, djt));
                    }
                }
            }
        }
    for (int q = 0; q < m; ++q) {   /* correctPenetration (src/contact.hpp:78-85) */
        Con* k = &C[q];
        Body *a = &W->B[k->i], *b = &W->B[k->j];
        double invSum = a->invm + b->invm;
        if (invSum <= 0.0 || k->overlap <= 0.0) continue;
        v3 corr = vmul(k->n, W->p.contact_beta * k->overlap / invSum);
        a->x = vadd(a->x, vmul(corr, a->invm));
        b->x = vsub(b->x, vmul(corr, b->invm));
    }
    if (W->p.warm_start) {
        free(W->wkey); free(W->wslot); free(W->wimp);
        W->wn = m;
        W->wkey = malloc(sizeof(uint64_t) * (size_t)(m ? m : 1));
        W->wslot = malloc(sizeof(int) * (size_t)(m ? m : 1));
        W->wimp = malloc(sizeof(double) * (size_t)(m ? m : 1));
        for (int q = 0; q < m; ++q) { W->wkey[q] = C[q].key; W->wslot[q] = C[q].slot; W->wimp[q] = C[q].nImp; }
    }
    free(W->cons);
    W->cons = C;
    W->ncons = m;
    /* island partition: union-find over the dyn-dyn pairs (src/world.cpp:332-343) */
    for (int k = 0; k < W->n; ++k) W->label[k] = (uint32_t)k;
    uint32_t* P = ipairs.p;
    for (int q = 0; q < ipairs.n; ++q) {
        uint32_t ra = uf_find(W->label, P[2 * q]), rb = uf_find(W->label, P[2 * q + 1]);
        if (ra == rb) continue;
        if (ra < rb) W->label[rb] = ra; else W->label[ra] = rb;
    }
    for (int k = 0; k < W->n; ++k) W->label[k] = uf_find(W->label, (uint32_t)k);
    free(ipairs.p);
}

static void boundary(World* W) {   /* src/world.cpp:635-657, 698-702 */
    const Dom dom = {W->p.half, W->p.periodic};
    if (W->p.periodic) {
        for (int k = 0; k < W->n; ++k)
            if (W->B[k].invm > 0.0) W->B[k].x = wrap_pos(dom, W->B[k].x);
        return;
    }
    if (W->p.open_boundary) return;
    const double h = W->p.half;
    for (int k = 0; k < W->n; ++k) {
        Body* b = &W->B[k];
        if (b->invm <= 0.0) continue;
        double* px[3] = {&b->x.x, &b->x.y, &b->x.z};
        double* pv[3] = {&b->v.x, &b->v.y, &b->v.z};
        for (int axis = 0; axis < 3; ++axis)
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                v3 outward = V(axis == 0 ? (double)sgn : 0.0, axis == 1 ? (double)sgn : 0.0, axis == 2 ? (double)sgn : 0.0);
                v3 sp = support(b, outward);
                double coord = comp(sp, axis) * sgn;
                double pen = coord - h;
                if (pen > 0.0) {
                    *px[axis] -= (double)sgn * pen;
                    if (*pv[axis] * sgn > 0.0) *pv[axis] = -W->p.restitution * *pv[axis];
                }
            }
    }
}

/* ---- entry points ------------------------------------------------------- */

static v3 rd3(const double* a, size_t i) { return V(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }

void* neport_create(const NeWorldParams* p, const NeBodyArrays* b) {
    World* W = calloc(1, sizeof(World));
    W->p = *p;
    W->n = (int)b->n;
    W->B = calloc((size_t)(W->n ? W->n : 1), sizeof(Body));
    W->vpool = malloc(sizeof(v3) * (size_t)(b->n_verts ? b->n_verts : 1));
    for (uint32_t k = 0; k < b->n_verts; ++k) W->vpool[k] = rd3(b->verts, k);
    W->ncpool = malloc(sizeof(uint32_t) * (size_t)(b->n_nocollide ? b->n_nocollide : 1));
    if (b->n_nocollide && b->nocollide) memcpy(W->ncpool, b->nocollide, sizeof(uint32_t) * b->n_nocollide);
    W->label = malloc(sizeof(uint32_t) * (size_t)(W->n ? W->n : 1));
    for (int i = 0; i < W->n; ++i) {
        Body* o = &W->B[i];
        o->x = rd3(b->x, i); o->v = rd3(b->v, i); o->w = rd3(b->w, i);
        o->q = Qn(b->q[4 * i], b->q[4 * i + 1], b->q[4 * i + 2], b->q[4 * i + 3]);
        o->force = b->force ? rd3(b->force, i) : V(0, 0, 0);
        o->torque = b->torque ? rd3(b->torque, i) : V(0, 0, 0);
        o->invm = b->inv_mass[i]; o->invi = rd3(b->inv_inertia, i);
        o->shape = b->shape[i]; o->radius = b->radius[i]; o->hh = b->half_height[i]; o->he = rd3(b->half_extents, i);
        if (o->shape == NE_SHAPE_CONVEX) { o->verts = W->vpool + b->vert_offset[i]; o->nverts = (int)b->vert_count[i]; }
        o->fric = b->friction[i]; o->rest = b->restitution[i]; o->ldamp = b->linear_damping[i];
        o->adamp = b->angular_damping[i]; o->gscale = b->gravity_scale[i];
        o->layer = b->layer[i]; o->mask = b->mask[i]; o->flags = b->flags[i];
        if (b->nocollide_count && b->nocollide_count[i]) {
            o->nocol = W->ncpool + b->nocollide_offset[i];
            o->nnocol = (int)b->nocollide_count[i];
        }
        W->label[i] = (uint32_t)i;
    }
    return W;
}

void neport_destroy(void* h) {
    World* W = h;
    if (!W) return;
    free(W->B); free(W->vpool); free(W->ncpool); free(W->wkey); free(W->wslot); free(W->wimp);
    free(W->pi); free(W->pj); free(W->cons); free(W->label);
    free(W);
}

void neport_set_params(void* h, const NeWorldParams* p) { ((World*)h)->p = *p; }

void neport_reset_warm_cache(void* h) { ((World*)h)->wn = 0; }

void neport_step(void* h, uint32_t nsteps) {
    World* W = h;
    for (uint32_t s = 0; s < nsteps; ++s) {
        integrate(W);
        collide(W);
        boundary(W);
    }
}

void neport_get_state(void* h, NeBodyArrays* out) {
    World* W = h;
    for (int i = 0; i < W->n && (uint32_t)i < out->n; ++i) {
        const Body* b = &W->B[i];
        if (out->x) { out->x[3 * i] = b->x.x; out->x[3 * i + 1] = b->x.y; out->x[3 * i + 2] = b->x.z; }
        if (out->q) { out->q[4 * i] = b->q.w; out->q[4 * i + 1] = b->q.x; out->q[4 * i + 2] = b->q.y; out->q[4 * i + 3] = b->q.z; }
        if (out->v) { out->v[3 * i] = b->v.x; out->v[3 * i + 1] = b->v.y; out->v[3 * i + 2] = b->v.z; }
        if (out->w) { out->w[3 * i] = b->w.x; out->w[3 * i + 1] = b->w.y; out->w[3 * i + 2] = b->w.z; }
    }
}

uint64_t neport_pairs(void* h, uint32_t* pi, uint32_t* pj, uint64_t cap) {
    World* W = h;
    for (uint64_t k = 0; k < W->np && k < cap; ++k) { pi[k] = W->pi[k]; pj[k] = W->pj[k]; }
    return W->np;
}

/* Contacts of the last step; the impulse is read back from the warm cache
 * (the reference keeps no other copy of it). */
uint64_t neport_contacts(void* h, NeContactArrays* out, uint64_t cap) {
    World* W = h;
    for (int k = 0; k < W->ncons && (uint64_t)k < cap; ++k) {
        const Con* c = &W->cons[k];
        out->i[k] = c->i; out->j[k] = c->j;
        if (out->slot) out->slot[k] = (uint32_t)c->slot;
        out->point[3 * k] = c->point.x; out->point[3 * k + 1] = c->point.y; out->point[3 * k + 2] = c->point.z;
        out->normal[3 * k] = c->n.x; out->normal[3 * k + 1] = c->n.y; out->normal[3 * k + 2] = c->n.z;
        out->depth[k] = c->overlap;
        if (out->n_imp) {
            double imp = 0.0;
            warm_lookup(W, c->key, c->slot, &imp);
            out->n_imp[k] = imp;
        }
        if (out->t_imp) out->t_imp[k] = 0.0;
    }
    return (uint64_t)W->ncons;
}

void neport_islands(void* h, uint32_t* label, uint32_t n) {
    World* W = h;
    for (uint32_t i = 0; i < n && (int)i < W->n; ++i) label[i] = W->label[i];
}
