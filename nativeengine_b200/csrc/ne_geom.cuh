// ne_geom.cuh -- narrowphase geometry on the device (FP64, bit-order faithful).
//
// Each routine restates one reference routine; the arithmetic is evaluated in
// the same order (see ne_math.cuh) and the data-dependent control flow (GJK
// simplex cases, EPA face order and horizon bookkeeping, Sutherland-Hodgman
// clipping) takes the same branches in the same order, with fixed-capacity
// arrays where the reference grows std::vectors.  A capacity overrun sets a flag
// the caller reports; it never writes out of bounds.
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

// Geometry view of one body, gathered from the device arrays.
struct BodyG {
    V3 x;
    Q q;
    V3 he;          // box half extents, or the plane's unit normal
    double radius;
    double half_height;
    const D4* verts;   // convex vertices (body frame), x,y,z used
    int nverts;
    int shape;
};

struct Contact {
    int hit;
    V3 normal;      // b -> a
    V3 point;
    double overlap;
};

NE_HD Contact no_contact() {
    Contact c;
    c.hit = 0;
    c.normal = mk(0.0, 0.0, 0.0);
    c.point = mk(0.0, 0.0, 0.0);
    c.overlap = 0.0;
    return c;
}

// Bounding-sphere radius about the centre (src/body.hpp:137-158).
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
NE_HD V3 support_world(const BodyG& b, const V3& d) {
    if (b.shape == SH_SPHERE) return b.x + normalized(d) * b.radius;
    V3 db = inv_rotate(b.q, d);
    V3 sb;
    if (b.shape == SH_BOX) {
        sb = mk(db.x >= 0 ? b.he.x : -b.he.x, db.y >= 0 ? b.he.y : -b.he.y,
                db.z >= 0 ? b.he.z : -b.he.z);
    } else if (b.shape == SH_CAPSULE) {
        double sy = (db.y >= 0.0) ? b.half_height : -b.half_height;
        sb = mk(0.0, sy, 0.0) + normalized(db) * b.radius;
    } else if (b.shape == SH_CONVEX) {
        double best = -1e300;
        sb = mk(0.0, 0.0, 0.0);
        for (int k = 0; k < b.nverts; ++k) {
            V3 v = mk(b.verts[k].x, b.verts[k].y, b.verts[k].z);
            double dp = dot(v, db);
            if (dp > best) { best = dp; sb = v; }
        }
    } else {   // cylinder, axis +Y, flat caps
        double sy = (db.y >= 0.0) ? b.half_height : -b.half_height;
        double rho = sqrt(db.x * db.x + db.z * db.z);
        sb = (rho > 1e-12) ? mk(db.x / rho * b.radius, sy, db.z / rho * b.radius) : mk(0.0, sy, 0.0);
    }
    return b.x + rotate(b.q, sb);
}

// Half-space vs convex (src/detect.hpp:19-31): normal plane -> other.
NE_HD Contact plane_vs_convex(const BodyG& other, const BodyG& plane, const Domain& dom) {
    Contact c = no_contact();
    V3 n = plane.he;
    V3 sp = support_world(other, -n);
    V3 rel = min_image(dom, sp - plane.x);
    double pen = -dot(n, rel);
    if (pen <= 0.0) return c;
    c.hit = 1;
    c.overlap = pen;
    c.normal = n;
    c.point = sp + n * (0.5 * pen);
    return c;
}

// Sphere vs flat-cap cylinder (src/narrowphase.hpp:34-81): normal cyl -> sphere.
NE_HD Contact sphere_vs_cylinder(const BodyG& sph, const BodyG& cyl, const Domain& dom) {
    Contact c = no_contact();
    const double r = cyl.radius, h = cyl.half_height, sr = sph.radius;
    V3 rel = min_image(dom, sph.x - cyl.x);
    V3 L = inv_rotate(cyl.q, rel);
    double rho = sqrt(L.x * L.x + L.z * L.z);
    bool insideAxial = fabs(L.y) < h;
    bool insideRadial = rho < r;
    V3 Pl, nl;
    if (insideAxial && insideRadial) {
        double dCap = h - fabs(L.y);
        double dSide = r - rho;
        if (dSide < dCap) {
            double s = (rho > 1e-12) ? r / rho : 0.0;
            Pl = mk(L.x * s, L.y, L.z * s);
            nl = (rho > 1e-12) ? mk(L.x / rho, 0.0, L.z / rho) : mk(1.0, 0.0, 0.0);
            c.overlap = sr + dSide;
        } else {
            double sy = (L.y >= 0) ? h : -h;
            Pl = mk(L.x, sy, L.z);
            nl = mk(0.0, (L.y >= 0) ? 1.0 : -1.0, 0.0);
            c.overlap = sr + dCap;
        }
        c.hit = 1;
    } else {
        double yc = (L.y > h) ? h : (L.y < -h ? -h : L.y);
        double rx = L.x, rz = L.z;
        if (rho > r) { double s = r / rho; rx *= s; rz *= s; }
        Pl = mk(rx, yc, rz);
        V3 diff = L - Pl;
        double dist = norm(diff);
        if (dist >= sr) return c;
        c.hit = 1;
        c.overlap = sr - dist;
        nl = (dist > 1e-12) ? diff / dist : mk(0.0, 1.0, 0.0);
    }
    c.normal = normalized(rotate(cyl.q, nl));
    c.point = cyl.x + rotate(cyl.q, Pl);
    return c;
}

NE_HD double np_clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

NE_HD V3 closest_on_segment(const V3& p, const V3& a, const V3& b) {
    V3 ab = b - a;
    double L2 = norm2(ab);
    if (L2 < 1e-18) return a;
    return a + ab * np_clamp(dot(p - a, ab) / L2, 0.0, 1.0);
}

// Closest points between segments p1q1 and p2q2 (src/narrowphase.hpp:96-116).
NE_HD void closest_seg_seg(const V3& p1, const V3& q1, const V3& p2, const V3& q2, V3& c1, V3& c2) {
    V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    const double EPS = 1e-12;
    double s, t;
    if (a <= EPS && e <= EPS) {
        s = t = 0.0;
    } else if (a <= EPS) {
        s = 0.0;
        t = np_clamp(f / e, 0.0, 1.0);
    } else {
        double cc = dot(d1, r);
        if (e <= EPS) {
            t = 0.0;
            s = np_clamp(-cc / a, 0.0, 1.0);
        } else {
            double b = dot(d1, d2), denom = a * e - b * b;
            s = denom > EPS ? np_clamp((b * f - cc * e) / denom, 0.0, 1.0) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) { t = 0.0; s = np_clamp(-cc / a, 0.0, 1.0); }
            else if (t > 1.0) { t = 1.0; s = np_clamp((b - cc) / a, 0.0, 1.0); }
        }
    }
    c1 = p1 + d1 * s;
    c2 = p2 + d2 * t;
}

// Capsule (A) vs sphere (B) (src/narrowphase.hpp:120-135): normal B -> A.
NE_HD Contact capsule_vs_sphere(const BodyG& cap, const BodyG& sph, const Domain& dom) {
    Contact c = no_contact();
    V3 sc = cap.x + min_image(dom, sph.x - cap.x);
    V3 axis = rotate(cap.q, mk(0.0, 1.0, 0.0));
    V3 cp = closest_on_segment(sc, cap.x - axis * cap.half_height, cap.x + axis * cap.half_height);
    V3 e = sc - cp;
    double dist = norm(e);
    double sumR = cap.radius + sph.radius;
    if (dist >= sumR) return c;
    V3 nrm = (dist > 1e-12) ? e / dist : mk(0.0, 1.0, 0.0);
    c.hit = 1;
    c.overlap = sumR - dist;
    c.normal = -nrm;
    c.point = cp + nrm * cap.radius;
    return c;
}

// Capsule vs capsule (src/narrowphase.hpp:138-155): normal B -> A.
NE_HD Contact capsule_vs_capsule(const BodyG& A, const BodyG& B, const Domain& dom) {
    Contact c = no_contact();
    V3 axA = rotate(A.q, mk(0.0, 1.0, 0.0)), axB = rotate(B.q, mk(0.0, 1.0, 0.0));
    V3 bc = A.x + min_image(dom, B.x - A.x);
    V3 pA, pB;
    closest_seg_seg(A.x - axA * A.half_height, A.x + axA * A.half_height, bc - axB * B.half_height,
                    bc + axB * B.half_height, pA, pB);
    V3 e = pB - pA;
    double dist = norm(e);
    double sumR = A.radius + B.radius;
    if (dist >= sumR) return c;
    V3 nrm = (dist > 1e-12) ? e / dist : mk(0.0, 1.0, 0.0);
    c.hit = 1;
    c.overlap = sumR - dist;
    c.normal = -nrm;
    c.point = pA + nrm * A.radius;
    return c;
}

// ---- GJK + EPA (src/epa.hpp) ---------------------------------------------

// A Minkowski-difference vertex; v = a - b is recomputed on demand (same bits
// as the stored difference in the reference).
struct SupV {
    V3 a;   // support point on A
    V3 b;   // support point on B, shifted into A's image
};

NE_HD V3 sv(const SupV& s) { return s.a - s.b; }

NE_HD SupV cso_support(const BodyG& A, const BodyG& B, const V3& shift, const V3& d) {
    SupV s;
    s.a = support_world(A, d);
    s.b = support_world(B, -d) + shift;
    return s;
}

// GJK returning an origin-enclosing tetrahedron (src/epa.hpp:28-64).  The
// simplex is kept newest-first, as the reference's front-inserting vector.
NE_HD bool gjk_tetra(const BodyG& A, const BodyG& B, const V3& shift, SupV tet[4]) {
    V3 d = mk(1.0, 0.0, 0.0);
    SupV s = cso_support(A, B, shift, d);
    if (norm2(sv(s)) < 1e-24) { d = mk(0.0, 1.0, 0.0); s = cso_support(A, B, shift, d); }
    SupV W[4];
    int nw = 1;
    W[0] = s;
    d = -sv(s);
    for (int iter = 0; iter < 64; ++iter) {
        if (norm2(d) < 1e-24) d = mk(1.0, 0.0, 0.0);
        SupV p = cso_support(A, B, shift, d);
        if (dot(sv(p), d) <= 1e-12) return false;
        for (int k = nw; k > 0; --k) W[k] = W[k - 1];
        W[0] = p;
        ++nw;
        const V3 a = sv(W[0]), ao = -a;
        if (nw == 2) {
            V3 ab = sv(W[1]) - a;
            d = cross(cross(ab, ao), ab);
            if (norm2(d) < 1e-24) d = mk(ab.y, -ab.x, 0.0);
        } else if (nw == 3) {
            V3 ab = sv(W[1]) - a, ac = sv(W[2]) - a;
            V3 abc = cross(ab, ac);
            if (dot(abc, ao) > 0) {
                d = abc;
            } else {
                SupV t = W[1]; W[1] = W[2]; W[2] = t;
                d = -abc;
            }
            if (norm2(d) < 1e-24) return false;
        } else {
            V3 b = sv(W[1]), c = sv(W[2]), dd = sv(W[3]);
            V3 ab = b - a, ac = c - a, ad = dd - a;
            V3 abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
            if (dot(abc, ao) > 0) {
                nw = 3; d = abc;                                   // {W0, W1, W2}
            } else if (dot(acd, ao) > 0) {
                W[1] = W[2]; W[2] = W[3]; nw = 3; d = acd;         // {W0, W2, W3}
            } else if (dot(adb, ao) > 0) {
                SupV w1 = W[1]; W[1] = W[3]; W[2] = w1; nw = 3; d = adb;   // {W0, W3, W1}
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

struct EpaFace {
    V3 n;
    double dist;
    unsigned char a, b, c, pad;
};

struct EpaScratch {
    SupV verts[kEpaVerts];
    EpaFace faces[kEpaFaces];
    unsigned char hz[kEpaHorizon][2];
};

NE_HD EpaFace epa_make_face(const SupV* verts, int i, int j, int k) {
    V3 vi = sv(verts[i]);
    V3 n = cross(sv(verts[j]) - vi, sv(verts[k]) - vi);
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
NE_HD Contact epa_contact(const BodyG& A, const BodyG& B, const V3& shift, const SupV tet[4],
                          EpaScratch& S, int& flags) {
    SupV* verts = S.verts;
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
        SupV p = cso_support(A, B, shift, best.n);
        V3 pv = sv(p);
        double d = dot(pv, best.n);
        if (d - best.dist < 1e-7) break;
        if (nv >= kEpaVerts) { flags |= 1; break; }
        const int pidx = nv;
        verts[nv++] = p;
        int nh = 0, nk = 0;
        bool over = false;
        for (int fi = 0; fi < nf; ++fi) {
            const EpaFace f = faces[fi];
            if (dot(f.n, pv - sv(verts[f.a])) > 1e-12) {
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

    const SupV& A0 = verts[best.a];
    const SupV& B0 = verts[best.b];
    const SupV& C0 = verts[best.c];
    V3 proj = best.n * best.dist;
    V3 a0v = sv(A0);
    V3 v0 = sv(B0) - a0v, v1 = sv(C0) - a0v, v2 = proj - a0v;
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
    double d20 = dot(v2, v0), d21 = dot(v2, v1);
    double den = d00 * d11 - d01 * d01;
    double bv = 0, bw = 0;
    if (fabs(den) > 1e-18) {
        bv = (d11 * d20 - d01 * d21) / den;
        bw = (d00 * d21 - d01 * d20) / den;
    }
    double bu = 1.0 - bv - bw;
    V3 onA = A0.a * bu + B0.a * bv + C0.a * bw;
    V3 onB = A0.b * bu + B0.b * bv + C0.b * bw;
    Contact c;
    c.hit = 1;
    c.normal = -best.n;
    c.overlap = best.dist;
    c.point = (onA + onB) * 0.5;
    return c;
}

NE_HD V3 min_image_shift(const BodyG& A, const BodyG& B, const Domain& dom) {
    V3 raw = B.x - A.x;
    return min_image(dom, raw) - raw;
}

NE_HD Contact convex_contact(const BodyG& A, const BodyG& B, const Domain& dom, EpaScratch& S,
                             int& flags) {
    V3 shift = min_image_shift(A, B, dom);
    SupV tet[4];
    if (!gjk_tetra(A, B, shift, tet)) return no_contact();
    return epa_contact(A, B, shift, tet, S, flags);
}

// Narrowphase dispatch (src/detect.hpp:33-77): normal b -> a.
NE_HD Contact detect_contact(const BodyG& a, const BodyG& b, const Domain& dom, EpaScratch& S,
                             int& flags) {
    if (a.shape == SH_PLANE || b.shape == SH_PLANE) {
        if (a.shape == SH_PLANE && b.shape == SH_PLANE) return no_contact();
        const BodyG& plane = (a.shape == SH_PLANE) ? a : b;
        const BodyG& other = (a.shape == SH_PLANE) ? b : a;
        Contact t = plane_vs_convex(other, plane, dom);
        if (t.hit && a.shape == SH_PLANE) t.normal = -t.normal;
        return t;
    }
    if (a.shape == SH_SPHERE && b.shape == SH_SPHERE) {
        Contact c = no_contact();
        V3 d = min_image(dom, a.x - b.x);
        double sumR = a.radius + b.radius, dist2 = norm2(d);
        if (dist2 >= sumR * sumR || dist2 < 1e-18) return c;
        double dist = sqrt(dist2);
        c.hit = 1;
        c.normal = d / dist;
        c.overlap = sumR - dist;
        c.point = a.x - c.normal * a.radius;
        return c;
    }
    const bool aCyl = a.shape == SH_CYLINDER, bCyl = b.shape == SH_CYLINDER;
    if (a.shape == SH_SPHERE && bCyl) return sphere_vs_cylinder(a, b, dom);
    if (b.shape == SH_SPHERE && aCyl) {
        Contact t = sphere_vs_cylinder(b, a, dom);
        if (t.hit) t.normal = -t.normal;
        return t;
    }
    const bool aCap = a.shape == SH_CAPSULE, bCap = b.shape == SH_CAPSULE;
    if (aCap && bCap) return capsule_vs_capsule(a, b, dom);
    if (aCap && b.shape == SH_SPHERE) return capsule_vs_sphere(a, b, dom);
    if (a.shape == SH_SPHERE && bCap) {
        Contact t = capsule_vs_sphere(b, a, dom);
        if (t.hit) t.normal = -t.normal;
        return t;
    }
    return convex_contact(a, b, dom, S, flags);
}

// ---- box-box clipping manifold (src/manifold.hpp:16-126) -------------------

struct Manifold {
    int count;
    V3 point[4];
    double depth[4];
};

struct BoxFace {
    V3 n, c, u, v;
    double eu, ev;
    V3 vert[4];
};

NE_HD V3 axis_vec(int a) {
    return a == 0 ? mk(1.0, 0.0, 0.0) : (a == 1 ? mk(0.0, 1.0, 0.0) : mk(0.0, 0.0, 1.0));
}

NE_HD BoxFace box_face(const BodyG& b, const V3& centre, int axis, int sign) {
    const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
    const double h[3] = {b.he.x, b.he.y, b.he.z};
    BoxFace f;
    f.n = rotate(b.q, axis_vec(axis) * double(sign));
    f.c = centre + f.n * h[axis];
    f.u = rotate(b.q, axis_vec(t1));
    f.eu = h[t1];
    f.v = rotate(b.q, axis_vec(t2));
    f.ev = h[t2];
    f.vert[0] = f.c + f.u * f.eu + f.v * f.ev;
    f.vert[1] = f.c - f.u * f.eu + f.v * f.ev;
    f.vert[2] = f.c - f.u * f.eu - f.v * f.ev;
    f.vert[3] = f.c + f.u * f.eu - f.v * f.ev;
    return f;
}

NE_HD BoxFace best_face(const BodyG& b, const V3& centre, const V3& dir) {
    int bestAxis = 0, bestSign = 1;
    double best = -1e30;
    for (int axis = 0; axis < 3; ++axis)
        for (int sign = -1; sign <= 1; sign += 2) {
            double a = dot(rotate(b.q, axis_vec(axis) * double(sign)), dir);
            if (a > best) { best = a; bestAxis = axis; bestSign = sign; }
        }
    return box_face(b, centre, bestAxis, bestSign);
}

constexpr int kClipCap = 32;

// Sutherland-Hodgman: keep the part of poly with p.pn <= off.
NE_HD void clip_plane(V3* poly, int& m, V3* tmp, const V3& pn, double off, int& flags) {
    int o = 0;
    for (int i = 0; i < m; ++i) {
        const V3 cur = poly[i];
        const V3 nxt = poly[(i + 1) % m];
        double dc = dot(cur, pn) - off, dn = dot(nxt, pn) - off;
        bool inC = dc <= 0.0, inN = dn <= 0.0;
        if (inC) {
            if (o < kClipCap) tmp[o++] = cur; else flags |= 1;
        }
        if (inC != inN) {
            double t = dc / (dc - dn);
            if (o < kClipCap) tmp[o++] = cur + (nxt - cur) * t; else flags |= 1;
        }
    }
    for (int i = 0; i < o; ++i) poly[i] = tmp[i];
    m = o;
}

NE_HD Manifold box_box_manifold(const BodyG& a, const BodyG& b, const V3& n, const Domain& dom,
                                int& flags) {
    Manifold m;
    m.count = 0;
    const V3 bShift = min_image_shift(a, b, dom);
    const V3 bC = b.x + bShift;
    BoxFace fa = best_face(a, a.x, -n);
    BoxFace fb = best_face(b, bC, n);
    double alignA = dot(fa.n, -n), alignB = dot(fb.n, n);
    const bool refA = alignA >= alignB;
    const BoxFace& ref = refA ? fa : fb;
    const BodyG& incBody = refA ? b : a;
    const V3 incCentre = refA ? bC : a.x;
    BoxFace inc = best_face(incBody, incCentre, -ref.n);

    V3 poly[kClipCap], tmp[kClipCap];
    int np = 4;
    for (int k = 0; k < 4; ++k) poly[k] = inc.vert[k];
    clip_plane(poly, np, tmp, ref.u, dot(ref.c, ref.u) + ref.eu, flags);
    clip_plane(poly, np, tmp, ref.u * -1.0, -(dot(ref.c, ref.u) - ref.eu), flags);
    clip_plane(poly, np, tmp, ref.v, dot(ref.c, ref.v) + ref.ev, flags);
    clip_plane(poly, np, tmp, ref.v * -1.0, -(dot(ref.c, ref.v) - ref.ev), flags);

    const double slop = 0.01;
    for (int k = 0; k < np; ++k) {
        const V3 p = poly[k];
        double sd = dot(p - ref.c, ref.n);
        if (sd > slop) continue;
        if (m.count >= 4) break;
        m.point[m.count] = p - ref.n * sd;
        m.depth[m.count] = -sd;
        ++m.count;
    }
    return m;
}

}  // namespace neb
