// ne_geom.cuh -- narrowphase geometry on the device.
//
// Each routine restates one reference routine; the arithmetic is evaluated in
// the same order (see ne_math.cuh) and the data-dependent control flow (GJK
// simplex cases, EPA face order and horizon bookkeeping, Sutherland-Hodgman
// clipping) takes the same branches in the same order, with fixed-capacity
// arrays where the reference grows std::vectors.  A capacity overrun sets a flag
// the caller reports; it never writes out of bounds.
//
// The routines are templates over the real type R of the body geometry.
// R = double is the bit-exact path.  R = float is the batched FP32 form: the
// support mappings, the analytic pairs and the clipping run in FP32 in a
// body-relative frame, while the simplex and polytope arithmetic of GJK and
// EPA (search directions, containment and termination tests, face normals and
// distances, the barycentric witness) stays FP64 over the FP32 support
// points, which convert to double exactly.
#pragma once

#include "ne_math.cuh"

namespace neb {

enum : int {
    SH_SPHERE = 0, SH_CYLINDER = 1, SH_BOX = 2, SH_CAPSULE = 3,
    SH_CONVEX = 4, SH_PLANE = 5, SH_MESH = 6, SH_COMPOUND = 7
};

struct __align__(32) D4 {
    double x, y, z, w;
};

struct __align__(16) F4 {
    float x, y, z, w;
};

// Vertex record of a convex body: D4 in FP64, F4 in the FP32 form.
template <typename R> struct VertOf;
template <> struct VertOf<double> { using type = D4; };
template <> struct VertOf<float> { using type = F4; };

// Geometry view of one body, gathered from the device arrays.
template <typename R>
struct BodyGT {
    Vec3<R> x;
    Quat<R> q;
    Vec3<R> he;          // box half extents, or the plane's unit normal
    R radius;
    R half_height;
    const typename VertOf<R>::type* verts;   // convex vertices (body frame), x,y,z used
    int nverts;
    int shape;
};
using BodyG = BodyGT<double>;

template <typename R>
struct ContactT {
    int hit;
    Vec3<R> normal;      // b -> a
    Vec3<R> point;
    R overlap;
};
using Contact = ContactT<double>;

template <typename R>
NE_HD ContactT<R> no_contact_t() {
    ContactT<R> c;
    c.hit = 0;
    c.normal = mk3<R>(R(0), R(0), R(0));
    c.point = mk3<R>(R(0), R(0), R(0));
    c.overlap = R(0);
    return c;
}
NE_HD Contact no_contact() { return no_contact_t<double>(); }

// Bounding-sphere radius about the centre (src/body.hpp:137-158).  FP64.
NE_HD double bounding_radius(int shape, double radius, double half_height, const V3& he,
                             const D4* verts, int nverts) {
    if (shape == SH_SPHERE) return radius;
    if (shape == SH_BOX) return norm(he);
    if (shape == SH_CAPSULE) return half_height + radius;
    if (shape == SH_PLANE || shape == SH_MESH) return 1e30;
    if (shape == SH_CONVEX) {
        double m = 0.0;
        for (int k = 0; k < nverts; ++k) {
            double r = norm(mk(verts[k].x, verts[k].y, verts[k].z));
            m = (m < r) ? r : m;
        }
        return m;
    }
    return sqrt(half_height * half_height + radius * radius);   // cylinder
}

// Support mapping: farthest surface point along world direction d
// (src/gjk.hpp:17-46).
template <typename R>
NE_HD Vec3<R> support_world(const BodyGT<R>& b, const Vec3<R>& d) {
    if (b.shape == SH_SPHERE) return b.x + normalized(d) * b.radius;
    Vec3<R> db = inv_rotate(b.q, d);
    Vec3<R> sb;
    if (b.shape == SH_BOX) {
        sb = mk3<R>(db.x >= 0 ? b.he.x : -b.he.x, db.y >= 0 ? b.he.y : -b.he.y,
                    db.z >= 0 ? b.he.z : -b.he.z);
    } else if (b.shape == SH_CAPSULE) {
        R sy = (db.y >= R(0)) ? b.half_height : -b.half_height;
        sb = mk3<R>(R(0), sy, R(0)) + normalized(db) * b.radius;
    } else if (b.shape == SH_CONVEX) {
        R best = -Lim<R>::huge;
        sb = mk3<R>(R(0), R(0), R(0));
        for (int k = 0; k < b.nverts; ++k) {
            Vec3<R> v = mk3<R>(b.verts[k].x, b.verts[k].y, b.verts[k].z);
            R dp = dot(v, db);
            if (dp > best) { best = dp; sb = v; }
        }
    } else {   // cylinder, axis +Y, flat caps
        R sy = (db.y >= R(0)) ? b.half_height : -b.half_height;
        R rho = sqrt(db.x * db.x + db.z * db.z);
        sb = (rho > R(1e-12)) ? mk3<R>(db.x / rho * b.radius, sy, db.z / rho * b.radius) : mk3<R>(R(0), sy, R(0));
    }
    return b.x + rotate(b.q, sb);
}

// Half-space vs convex (src/detect.hpp:19-31): normal plane -> other.
template <typename R>
NE_HD ContactT<R> plane_vs_convex(const BodyGT<R>& other, const BodyGT<R>& plane, const Domain& dom) {
    ContactT<R> c = no_contact_t<R>();
    Vec3<R> n = plane.he;
    Vec3<R> sp = support_world(other, -n);
    Vec3<R> rel = min_image(dom, sp - plane.x);
    R pen = -dot(n, rel);
    if (pen <= R(0)) return c;
    c.hit = 1;
    c.overlap = pen;
    c.normal = n;
    c.point = sp + n * (R(0.5) * pen);
    return c;
}

// Sphere vs flat-cap cylinder (src/narrowphase.hpp:34-81): normal cyl -> sphere.
template <typename R>
NE_HD ContactT<R> sphere_vs_cylinder(const BodyGT<R>& sph, const BodyGT<R>& cyl, const Domain& dom) {
    ContactT<R> c = no_contact_t<R>();
    const R r = cyl.radius, h = cyl.half_height, sr = sph.radius;
    Vec3<R> rel = min_image(dom, sph.x - cyl.x);
    Vec3<R> L = inv_rotate(cyl.q, rel);
    R rho = sqrt(L.x * L.x + L.z * L.z);
    bool insideAxial = fabs(L.y) < h;
    bool insideRadial = rho < r;
    Vec3<R> Pl, nl;
    if (insideAxial && insideRadial) {
        R dCap = h - fabs(L.y);
        R dSide = r - rho;
        if (dSide < dCap) {
            R s = (rho > R(1e-12)) ? r / rho : R(0);
            Pl = mk3<R>(L.x * s, L.y, L.z * s);
            nl = (rho > R(1e-12)) ? mk3<R>(L.x / rho, R(0), L.z / rho) : mk3<R>(R(1), R(0), R(0));
            c.overlap = sr + dSide;
        } else {
            R sy = (L.y >= 0) ? h : -h;
            Pl = mk3<R>(L.x, sy, L.z);
            nl = mk3<R>(R(0), (L.y >= 0) ? R(1) : R(-1), R(0));
            c.overlap = sr + dCap;
        }
        c.hit = 1;
    } else {
        R yc = (L.y > h) ? h : (L.y < -h ? -h : L.y);
        R rx = L.x, rz = L.z;
        if (rho > r) { R s = r / rho; rx *= s; rz *= s; }
        Pl = mk3<R>(rx, yc, rz);
        Vec3<R> diff = L - Pl;
        R dist = norm(diff);
        if (dist >= sr) return c;
        c.hit = 1;
        c.overlap = sr - dist;
        nl = (dist > R(1e-12)) ? diff / dist : mk3<R>(R(0), R(1), R(0));
    }
    c.normal = normalized(rotate(cyl.q, nl));
    c.point = cyl.x + rotate(cyl.q, Pl);
    return c;
}

template <typename R>
NE_HD R np_clamp(R v, SameT<R> lo, SameT<R> hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename R>
NE_HD Vec3<R> closest_on_segment(const Vec3<R>& p, const Vec3<R>& a, const Vec3<R>& b) {
    Vec3<R> ab = b - a;
    R L2 = norm2(ab);
    if (L2 < R(1e-18)) return a;
    return a + ab * np_clamp<R>(dot(p - a, ab) / L2, R(0), R(1));
}

// Closest points between segments p1q1 and p2q2 (src/narrowphase.hpp:96-116).
template <typename R>
NE_HD void closest_seg_seg(const Vec3<R>& p1, const Vec3<R>& q1, const Vec3<R>& p2, const Vec3<R>& q2,
                           Vec3<R>& c1, Vec3<R>& c2) {
    Vec3<R> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    R a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    const R EPS = R(1e-12);
    R s, t;
    if (a <= EPS && e <= EPS) {
        s = t = R(0);
    } else if (a <= EPS) {
        s = R(0);
        t = np_clamp<R>(f / e, R(0), R(1));
    } else {
        R cc = dot(d1, r);
        if (e <= EPS) {
            t = R(0);
            s = np_clamp<R>(-cc / a, R(0), R(1));
        } else {
            R b = dot(d1, d2), denom = a * e - b * b;
            s = denom > EPS ? np_clamp<R>((b * f - cc * e) / denom, R(0), R(1)) : R(0);
            t = (b * s + f) / e;
            if (t < R(0)) { t = R(0); s = np_clamp<R>(-cc / a, R(0), R(1)); }
            else if (t > R(1)) { t = R(1); s = np_clamp<R>((b - cc) / a, R(0), R(1)); }
        }
    }
    c1 = p1 + d1 * s;
    c2 = p2 + d2 * t;
}

// Capsule (A) vs sphere (B) (src/narrowphase.hpp:120-135): normal B -> A.
template <typename R>
NE_HD ContactT<R> capsule_vs_sphere(const BodyGT<R>& cap, const BodyGT<R>& sph, const Domain& dom) {
    ContactT<R> c = no_contact_t<R>();
    Vec3<R> sc = cap.x + min_image(dom, sph.x - cap.x);
    Vec3<R> axis = rotate(cap.q, mk3<R>(R(0), R(1), R(0)));
    Vec3<R> cp = closest_on_segment(sc, cap.x - axis * cap.half_height, cap.x + axis * cap.half_height);
    Vec3<R> e = sc - cp;
    R dist = norm(e);
    R sumR = cap.radius + sph.radius;
    if (dist >= sumR) return c;
    Vec3<R> nrm = (dist > R(1e-12)) ? e / dist : mk3<R>(R(0), R(1), R(0));
    c.hit = 1;
    c.overlap = sumR - dist;
    c.normal = -nrm;
    c.point = cp + nrm * cap.radius;
    return c;
}

// Capsule vs capsule (src/narrowphase.hpp:138-155): normal B -> A.
template <typename R>
NE_HD ContactT<R> capsule_vs_capsule(const BodyGT<R>& A, const BodyGT<R>& B, const Domain& dom) {
    ContactT<R> c = no_contact_t<R>();
    Vec3<R> axA = rotate(A.q, mk3<R>(R(0), R(1), R(0))), axB = rotate(B.q, mk3<R>(R(0), R(1), R(0)));
    Vec3<R> bc = A.x + min_image(dom, B.x - A.x);
    Vec3<R> pA, pB;
    closest_seg_seg(A.x - axA * A.half_height, A.x + axA * A.half_height, bc - axB * B.half_height,
                    bc + axB * B.half_height, pA, pB);
    Vec3<R> e = pB - pA;
    R dist = norm(e);
    R sumR = A.radius + B.radius;
    if (dist >= sumR) return c;
    Vec3<R> nrm = (dist > R(1e-12)) ? e / dist : mk3<R>(R(0), R(1), R(0));
    c.hit = 1;
    c.overlap = sumR - dist;
    c.normal = -nrm;
    c.point = pA + nrm * A.radius;
    return c;
}

// ---- GJK + EPA (src/epa.hpp) ---------------------------------------------

// A Minkowski-difference vertex; v = a - b is recomputed on demand (same bits
// as the stored difference in the reference).
template <typename R>
struct SupVT {
    Vec3<R> a;   // support point on A
    Vec3<R> b;   // support point on B, shifted into A's image
};
using SupV = SupVT<double>;

template <typename R> NE_HD Vec3<R> sv(const SupVT<R>& s) { return s.a - s.b; }
// The same difference in FP64 (for R = float the operands convert exactly).
template <typename R> NE_HD V3 svd(const SupVT<R>& s) { return cvt<double>(s.a) - cvt<double>(s.b); }

template <typename R>
NE_HD SupVT<R> cso_support(const BodyGT<R>& A, const BodyGT<R>& B, const Vec3<R>& shift, const Vec3<R>& d) {
    SupVT<R> s;
    s.a = support_world(A, d);
    s.b = support_world(B, -d) + shift;
    return s;
}

// GJK returning an origin-enclosing tetrahedron (src/epa.hpp:28-64).  The
// simplex is kept newest-first, as the reference's front-inserting vector.
// The simplex arithmetic (search directions, region and termination tests) is
// FP64 over the support points, which convert exactly; only the support
// mappings run in R.  For R = double this is the reference's arithmetic
// unchanged; for R = float it keeps the near-degenerate containment tests
// exact enough that EPA never starts from a tetrahedron that misses the origin.
template <typename R>
NE_HD bool gjk_tetra(const BodyGT<R>& A, const BodyGT<R>& B, const Vec3<R>& shift, SupVT<R> tet[4]) {
    V3 d = mk(1.0, 0.0, 0.0);
    SupVT<R> s = cso_support(A, B, shift, cvt<R>(d));
    if (norm2(svd(s)) < 1e-24) { d = mk(0.0, 1.0, 0.0); s = cso_support(A, B, shift, cvt<R>(d)); }
    SupVT<R> W[4];
    int nw = 1;
    W[0] = s;
    d = -svd(s);
    for (int iter = 0; iter < 64; ++iter) {
        if (norm2(d) < 1e-24) d = mk(1.0, 0.0, 0.0);
        SupVT<R> p = cso_support(A, B, shift, cvt<R>(d));
        if (dot(svd(p), d) <= 1e-12) return false;
        for (int k = nw; k > 0; --k) W[k] = W[k - 1];
        W[0] = p;
        ++nw;
        const V3 a = svd(W[0]), ao = -a;
        if (nw == 2) {
            V3 ab = svd(W[1]) - a;
            d = cross(cross(ab, ao), ab);
            if (norm2(d) < 1e-24) d = mk(ab.y, -ab.x, 0.0);
        } else if (nw == 3) {
            V3 ab = svd(W[1]) - a, ac = svd(W[2]) - a;
            V3 abc = cross(ab, ac);
            if (dot(abc, ao) > 0) {
                d = abc;
            } else {
                SupVT<R> t = W[1]; W[1] = W[2]; W[2] = t;
                d = -abc;
            }
            if (norm2(d) < 1e-24) return false;
        } else {
            V3 b = svd(W[1]), c = svd(W[2]), dd = svd(W[3]);
            V3 ab = b - a, ac = c - a, ad = dd - a;
            V3 abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
            if (dot(abc, ao) > 0) {
                nw = 3; d = abc;                                   // {W0, W1, W2}
            } else if (dot(acd, ao) > 0) {
                W[1] = W[2]; W[2] = W[3]; nw = 3; d = acd;         // {W0, W2, W3}
            } else if (dot(adb, ao) > 0) {
                SupVT<R> w1 = W[1]; W[1] = W[3]; W[2] = w1; nw = 3; d = adb;   // {W0, W3, W1}
            } else {
                tet[0] = W[0]; tet[1] = W[1]; tet[2] = W[2]; tet[3] = W[3];
                return true;
            }
        }
    }
    return false;
}

// Fixed budgets for the expanding polytope.  Each EPA iteration adds one
// vertex (<= 4 + 64); the face list of a convex polytope with V vertices has
// at most 2V - 4 faces, so kEpaFaces leaves headroom for near-degenerate
// polytopes.  Overruns are reported, never written.
constexpr int kEpaVerts = 68;
constexpr int kEpaFaces = 192;
constexpr int kEpaHorizon = 96;

// EPA convergence: the reference's 1e-7 in FP64.  FP32 support points carry
// ~1e-7 relative rounding, so the FP32 form stops at 1e-6 (its faces and the
// test itself are still FP64).
template <typename R> struct EpaTol { static constexpr double conv = 1e-7; };
template <> struct EpaTol<float> { static constexpr double conv = 1e-6; };

struct EpaFace {
    V3 n;
    double dist;
    unsigned char a, b, c, pad;
};

template <typename R>
struct EpaScratchT {
    SupVT<R> verts[kEpaVerts];
    EpaFace faces[kEpaFaces];
    unsigned char hz[kEpaHorizon][2];
};
using EpaScratch = EpaScratchT<double>;

template <typename R>
NE_HD EpaFace epa_make_face(const SupVT<R>* verts, int i, int j, int k) {
    V3 vi = svd(verts[i]);
    V3 n = cross(svd(verts[j]) - vi, svd(verts[k]) - vi);
    double L = norm(n);
    n = (L > 1e-18) ? n / L : mk(0.0, 0.0, 1.0);
    double dist = dot(n, vi);
    if (dist < 0) { n = -n; dist = -dist; int t = j; j = k; k = t; }
    EpaFace f;
    f.n = n; f.dist = dist;
    f.a = (unsigned char)i; f.b = (unsigned char)j; f.c = (unsigned char)k; f.pad = 0;
    return f;
}

// EPA expansion + barycentric witness (src/epa.hpp:71-150).
// flags |= 1 on a budget overrun, |= 2 when the 64-iteration cap was reached.
// face_out (optional) receives the final face's three vertices, oriented so
// that their normal points away from the origin.
template <typename R>
NE_HD ContactT<R> epa_contact(const BodyGT<R>& A, const BodyGT<R>& B, const Vec3<R>& shift, const SupVT<R> tet[4],
                              EpaScratchT<R>& S, int& flags, SupVT<R>* face_out = nullptr) {
    SupVT<R>* verts = S.verts;
    EpaFace* faces = S.faces;
    int nv = 4, nf = 4;
    for (int k = 0; k < 4; ++k) verts[k] = tet[k];
    faces[0] = epa_make_face(verts, 0, 1, 2);
    faces[1] = epa_make_face(verts, 0, 2, 3);
    faces[2] = epa_make_face(verts, 0, 3, 1);
    faces[3] = epa_make_face(verts, 1, 3, 2);

    EpaFace best;
    best.n = mk(0.0, 0.0, 0.0); best.dist = 0.0; best.a = best.b = best.c = 0; best.pad = 0;
    int iter = 0;
    for (; iter < 64; ++iter) {
        int ci = 0;
        for (int i = 1; i < nf; ++i)
            if (faces[i].dist < faces[ci].dist) ci = i;
        best = faces[ci];
        SupVT<R> p = cso_support(A, B, shift, cvt<R>(best.n));
        V3 pv = svd(p);
        double d = dot(pv, best.n);
        if (d - best.dist < EpaTol<R>::conv) break;
        if (nv >= kEpaVerts) { flags |= 1; break; }
        const int pidx = nv;
        verts[nv++] = p;
        int nh = 0, nk = 0;
        bool over = false;
        for (int fi = 0; fi < nf; ++fi) {
            const EpaFace f = faces[fi];
            if (dot(f.n, pv - svd(verts[f.a])) > 1e-12) {
                const unsigned char ed[3][2] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
                for (int q = 0; q < 3; ++q) {
                    const unsigned char u = ed[q][0], w = ed[q][1];
                    int found = -1;
                    for (int e = 0; e < nh; ++e)
                        if (S.hz[e][0] == w && S.hz[e][1] == u) { found = e; break; }
                    if (found >= 0) {
                        for (int e = found; e + 1 < nh; ++e) { S.hz[e][0] = S.hz[e + 1][0]; S.hz[e][1] = S.hz[e + 1][1]; }
                        --nh;
                    } else if (nh < kEpaHorizon) {
                        S.hz[nh][0] = u; S.hz[nh][1] = w; ++nh;
                    } else {
                        over = true;
                    }
                }
            } else {
                faces[nk++] = f;   // nk <= fi: stable in-place compaction ("keep")
            }
        }
        nf = nk;
        if (over || nf + nh > kEpaFaces) { flags |= 1; break; }
        for (int e = 0; e < nh; ++e) faces[nf++] = epa_make_face(verts, S.hz[e][0], S.hz[e][1], pidx);
        if (nf == 0) break;
    }
    if (iter >= 64) flags |= 2;

    const SupVT<R>& A0 = verts[best.a];
    const SupVT<R>& B0 = verts[best.b];
    const SupVT<R>& C0 = verts[best.c];
    if (face_out) { face_out[0] = A0; face_out[1] = B0; face_out[2] = C0; }
    V3 proj = best.n * best.dist;
    V3 a0v = svd(A0);
    V3 v0 = svd(B0) - a0v, v1 = svd(C0) - a0v, v2 = proj - a0v;
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
    double d20 = dot(v2, v0), d21 = dot(v2, v1);
    double den = d00 * d11 - d01 * d01;
    double bv = 0, bw = 0;
    if (fabs(den) > 1e-18) {
        bv = (d11 * d20 - d01 * d21) / den;
        bw = (d00 * d21 - d01 * d20) / den;
    }
    double bu = 1.0 - bv - bw;
    V3 onA = cvt<double>(A0.a) * bu + cvt<double>(B0.a) * bv + cvt<double>(C0.a) * bw;
    V3 onB = cvt<double>(A0.b) * bu + cvt<double>(B0.b) * bv + cvt<double>(C0.b) * bw;
    ContactT<R> c;
    c.hit = 1;
    c.normal = cvt<R>(-best.n);
    c.overlap = (R)best.dist;
    c.point = cvt<R>((onA + onB) * 0.5);
    return c;
}

template <typename R>
NE_HD Vec3<R> min_image_shift(const BodyGT<R>& A, const BodyGT<R>& B, const Domain& dom) {
    Vec3<R> raw = B.x - A.x;
    return min_image(dom, raw) - raw;
}

template <typename R>
NE_HD ContactT<R> convex_contact(const BodyGT<R>& A, const BodyGT<R>& B, const Domain& dom, EpaScratchT<R>& S,
                                 int& flags, SupVT<R>* face_out = nullptr) {
    Vec3<R> shift = min_image_shift(A, B, dom);
    SupVT<R> tet[4];
    if (!gjk_tetra(A, B, shift, tet)) return no_contact_t<R>();
    return epa_contact(A, B, shift, tet, S, flags, face_out);
}

// Narrowphase dispatch (src/detect.hpp:33-77): normal b -> a.
template <typename R>
NE_HD ContactT<R> detect_contact(const BodyGT<R>& a, const BodyGT<R>& b, const Domain& dom, EpaScratchT<R>& S,
                                 int& flags, SupVT<R>* face_out = nullptr) {
    if (a.shape == SH_PLANE || b.shape == SH_PLANE) {
        if (a.shape == SH_PLANE && b.shape == SH_PLANE) return no_contact_t<R>();
        const BodyGT<R>& plane = (a.shape == SH_PLANE) ? a : b;
        const BodyGT<R>& other = (a.shape == SH_PLANE) ? b : a;
        ContactT<R> t = plane_vs_convex(other, plane, dom);
        if (t.hit && a.shape == SH_PLANE) t.normal = -t.normal;
        return t;
    }
    if (a.shape == SH_SPHERE && b.shape == SH_SPHERE) {
        ContactT<R> c = no_contact_t<R>();
        Vec3<R> d = min_image(dom, a.x - b.x);
        R sumR = a.radius + b.radius, dist2 = norm2(d);
        if (dist2 >= sumR * sumR || dist2 < R(1e-18)) return c;
        R dist = sqrt(dist2);
        c.hit = 1;
        c.normal = d / dist;
        c.overlap = sumR - dist;
        c.point = a.x - c.normal * a.radius;
        return c;
    }
    const bool aCyl = a.shape == SH_CYLINDER, bCyl = b.shape == SH_CYLINDER;
    if (a.shape == SH_SPHERE && bCyl) return sphere_vs_cylinder(a, b, dom);
    if (b.shape == SH_SPHERE && aCyl) {
        ContactT<R> t = sphere_vs_cylinder(b, a, dom);
        if (t.hit) t.normal = -t.normal;
        return t;
    }
    const bool aCap = a.shape == SH_CAPSULE, bCap = b.shape == SH_CAPSULE;
    if (aCap && bCap) return capsule_vs_capsule(a, b, dom);
    if (aCap && b.shape == SH_SPHERE) return capsule_vs_sphere(a, b, dom);
    if (a.shape == SH_SPHERE && bCap) {
        ContactT<R> t = capsule_vs_sphere(b, a, dom);
        if (t.hit) t.normal = -t.normal;
        return t;
    }
    return convex_contact(a, b, dom, S, flags, face_out);
}

// ---- box-box clipping manifold (src/manifold.hpp:16-126) -------------------

template <typename R>
struct ManifoldT {
    int count;
    Vec3<R> point[4];
    R depth[4];
};
using Manifold = ManifoldT<double>;

template <typename R>
struct BoxFaceT {
    Vec3<R> n, c, u, v;
    R eu, ev;
    Vec3<R> vert[4];
};

template <typename R>
NE_HD Vec3<R> axis_vec(int a) {
    return a == 0 ? mk3<R>(R(1), R(0), R(0)) : (a == 1 ? mk3<R>(R(0), R(1), R(0)) : mk3<R>(R(0), R(0), R(1)));
}

template <typename R>
NE_HD BoxFaceT<R> box_face(const BodyGT<R>& b, const Vec3<R>& centre, int axis, int sign) {
    const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
    const R h[3] = {b.he.x, b.he.y, b.he.z};
    BoxFaceT<R> f;
    f.n = rotate(b.q, axis_vec<R>(axis) * R(sign));
    f.c = centre + f.n * h[axis];
    f.u = rotate(b.q, axis_vec<R>(t1));
    f.eu = h[t1];
    f.v = rotate(b.q, axis_vec<R>(t2));
    f.ev = h[t2];
    f.vert[0] = f.c + f.u * f.eu + f.v * f.ev;
    f.vert[1] = f.c - f.u * f.eu + f.v * f.ev;
    f.vert[2] = f.c - f.u * f.eu - f.v * f.ev;
    f.vert[3] = f.c + f.u * f.eu - f.v * f.ev;
    return f;
}

template <typename R>
NE_HD BoxFaceT<R> best_face(const BodyGT<R>& b, const Vec3<R>& centre, const Vec3<R>& dir) {
    int bestAxis = 0, bestSign = 1;
    R best = R(-1e30);
    for (int axis = 0; axis < 3; ++axis)
        for (int sign = -1; sign <= 1; sign += 2) {
            R a = dot(rotate(b.q, axis_vec<R>(axis) * R(sign)), dir);
            if (a > best) { best = a; bestAxis = axis; bestSign = sign; }
        }
    return box_face(b, centre, bestAxis, bestSign);
}

constexpr int kClipCap = 32;

// Sutherland-Hodgman: keep the part of poly with p.pn <= off.
template <typename R>
NE_HD void clip_plane(Vec3<R>* poly, int& m, Vec3<R>* tmp, const Vec3<R>& pn, SameT<R> off, int& flags) {
    int o = 0;
    for (int i = 0; i < m; ++i) {
        const Vec3<R> cur = poly[i];
        const Vec3<R> nxt = poly[(i + 1) % m];
        R dc = dot(cur, pn) - off, dn = dot(nxt, pn) - off;
        bool inC = dc <= R(0), inN = dn <= R(0);
        if (inC) {
            if (o < kClipCap) tmp[o++] = cur; else flags |= 1;
        }
        if (inC != inN) {
            R t = dc / (dc - dn);
            if (o < kClipCap) tmp[o++] = cur + (nxt - cur) * t; else flags |= 1;
        }
    }
    for (int i = 0; i < o; ++i) poly[i] = tmp[i];
    m = o;
}

template <typename R>
NE_HD ManifoldT<R> box_box_manifold(const BodyGT<R>& a, const BodyGT<R>& b, const Vec3<R>& n, const Domain& dom,
                                    int& flags) {
    ManifoldT<R> m;
    m.count = 0;
    const Vec3<R> bShift = min_image_shift(a, b, dom);
    const Vec3<R> bC = b.x + bShift;
    BoxFaceT<R> fa = best_face(a, a.x, -n);
    BoxFaceT<R> fb = best_face(b, bC, n);
    R alignA = dot(fa.n, -n), alignB = dot(fb.n, n);
    const bool refA = alignA >= alignB;
    const BoxFaceT<R>& ref = refA ? fa : fb;
    const BodyGT<R>& incBody = refA ? b : a;
    const Vec3<R> incCentre = refA ? bC : a.x;
    BoxFaceT<R> inc = best_face(incBody, incCentre, -ref.n);

    Vec3<R> poly[kClipCap], tmp[kClipCap];
    int np = 4;
    for (int k = 0; k < 4; ++k) poly[k] = inc.vert[k];
    clip_plane(poly, np, tmp, ref.u, dot(ref.c, ref.u) + ref.eu, flags);
    clip_plane(poly, np, tmp, ref.u * R(-1), -(dot(ref.c, ref.u) - ref.eu), flags);
    clip_plane(poly, np, tmp, ref.v, dot(ref.c, ref.v) + ref.ev, flags);
    clip_plane(poly, np, tmp, ref.v * R(-1), -(dot(ref.c, ref.v) - ref.ev), flags);

    const R slop = R(0.01);
    for (int k = 0; k < np; ++k) {
        const Vec3<R> p = poly[k];
        R sd = dot(p - ref.c, ref.n);
        if (sd > slop) continue;
        if (m.count >= 4) break;
        m.point[m.count] = p - ref.n * sd;
        m.depth[m.count] = -sd;
        ++m.count;
    }
    return m;
}

}  // namespace neb
