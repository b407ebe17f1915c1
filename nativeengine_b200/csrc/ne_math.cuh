// ne_math.cuh -- FP64 vector / quaternion arithmetic for the device step path.
//
// Every expression is written in the reference's evaluation order
// (src/vmath.hpp:18-132, src/box.hpp:24-41, src/body.hpp:162-202) and the
// library is compiled with --fmad=false, so each result is the same IEEE-754
// double the x86-64 reference computes (scalar SSE2, no contraction).  This is
// what makes pair lists, contacts, impulses and poses bit-comparable with the
// reference.  Do not "simplify" an expression here: reassociating a sum or
// fusing a multiply-add changes the last bit and breaks parity.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define NE_HD __host__ __device__ __forceinline__
#else
#define NE_HD inline
#ifndef __align__
#define __align__(n) __attribute__((aligned(n)))
#endif
#endif

namespace neb {

struct V3 {
    double x, y, z;
};

NE_HD V3 mk(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
NE_HD V3 operator+(const V3& a, const V3& b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
NE_HD V3 operator-(const V3& a, const V3& b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
NE_HD V3 operator-(const V3& a) { return mk(-a.x, -a.y, -a.z); }
NE_HD V3 operator*(const V3& a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
NE_HD V3 operator*(double s, const V3& a) { return mk(a.x * s, a.y * s, a.z * s); }
NE_HD V3 operator/(const V3& a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
NE_HD double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
NE_HD V3 cross(const V3& a, const V3& b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
NE_HD double norm2(const V3& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
NE_HD double norm(const V3& a) { return sqrt(norm2(a)); }
NE_HD V3 normalized(const V3& a) {
    double n = norm(a);
    return (n > 1e-300) ? mk(a.x / n, a.y / n, a.z / n) : mk(0.0, 0.0, 0.0);
}

// Quaternion (w, x, y, z), body -> world.
struct Q {
    double w, x, y, z;
};

NE_HD Q mkq(double w, double x, double y, double z) { Q r; r.w = w; r.x = x; r.y = y; r.z = z; return r; }
NE_HD Q qmul(const Q& a, const Q& o) {
    return mkq(a.w * o.w - a.x * o.x - a.y * o.y - a.z * o.z,
               a.w * o.x + a.x * o.w + a.y * o.z - a.z * o.y,
               a.w * o.y - a.x * o.z + a.y * o.w + a.z * o.x,
               a.w * o.z + a.x * o.y - a.y * o.x + a.z * o.w);
}
NE_HD Q qadd(const Q& a, const Q& o) { return mkq(a.w + o.w, a.x + o.x, a.y + o.y, a.z + o.z); }
NE_HD Q qscale(const Q& a, double s) { return mkq(a.w * s, a.x * s, a.y * s, a.z * s); }
NE_HD Q qnormalized(const Q& a) {
    double n = sqrt(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    return (n > 1e-300) ? mkq(a.w / n, a.x / n, a.y / n, a.z / n) : mkq(1.0, 0.0, 0.0, 0.0);
}
NE_HD Q qconj(const Q& a) { return mkq(a.w, -a.x, -a.y, -a.z); }

// v' = q v q*  as  t = 2 (q_vec x v);  v' = v + w t + q_vec x t.
NE_HD V3 rotate(const Q& q, const V3& v) {
    V3 qv = mk(q.x, q.y, q.z);
    V3 t = 2.0 * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
NE_HD V3 inv_rotate(const Q& q, const V3& v) { return rotate(qconj(q), v); }

// q_{n+1} = normalise(q + (omega_quat * q) * (dt/2)).
NE_HD Q integrate_orientation(const Q& q, const V3& omega, double dt) {
    Q omegaQ = mkq(0.0, omega.x, omega.y, omega.z);
    Q dq = qscale(qmul(omegaQ, q), 0.5 * dt);
    return qnormalized(qadd(q, dq));
}

// World-frame inverse inertia applied to u:  R diag(invI) R^T u.
NE_HD V3 apply_inv_inertia(const Q& q, const V3& invI, const V3& u) {
    V3 ub = inv_rotate(q, u);
    V3 sb = mk(ub.x * invI.x, ub.y * invI.y, ub.z * invI.z);
    return rotate(q, sb);
}

// World-frame angular momentum L = I_world w.
NE_HD V3 angular_momentum(const Q& q, const V3& invI, const V3& w) {
    V3 Ib = mk(invI.x > 0 ? 1.0 / invI.x : 0.0, invI.y > 0 ? 1.0 / invI.y : 0.0,
               invI.z > 0 ? 1.0 / invI.z : 0.0);
    V3 wb = inv_rotate(q, w);
    V3 Lb = mk(wb.x * Ib.x, wb.y * Ib.y, wb.z * Ib.z);
    return rotate(q, Lb);
}

// Cubic domain: minimum image and wrap (identity when not periodic).
struct Domain {
    double half;
    int periodic;
};

NE_HD V3 min_image(const Domain& d, V3 v) {
    if (!d.periodic) return v;
    const double L = 2.0 * d.half;
    v.x -= L * floor(v.x / L + 0.5);
    v.y -= L * floor(v.y / L + 0.5);
    v.z -= L * floor(v.z / L + 0.5);
    return v;
}

NE_HD V3 wrap(const Domain& d, V3 p) {
    if (!d.periodic) return p;
    const double L = 2.0 * d.half;
    p.x -= L * floor((p.x + d.half) / L);
    p.y -= L * floor((p.y + d.half) / L);
    p.z -= L * floor((p.z + d.half) / L);
    return p;
}

}  // namespace neb
