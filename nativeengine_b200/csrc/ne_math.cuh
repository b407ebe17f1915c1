// ne_math.cuh -- vector / quaternion arithmetic for the device step path.
//
// Everything is a template over the real type R.  With R = double every
// expression is written in the reference's evaluation order
// (src/vmath.hpp:18-132, src/box.hpp:24-41, src/body.hpp:162-202) and the
// FP64 kernels are compiled with --fmad=false, so each result is the same
// IEEE-754 double the x86-64 reference computes (scalar SSE2, no
// contraction).  This is what makes pair lists, contacts, impulses and poses
// bit-comparable with the reference.  Do not "simplify" an expression here:
// reassociating a sum or fusing a multiply-add changes the last bit and breaks
// parity.  Constants are written R(c), which is the same double for R = double.
// R = float is the batched FP32 form's narrowphase and solver arithmetic.
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

// Scalar arguments of the operators below are not deduced: R comes from the
// vector, and a literal or a wider scalar converts to it.
template <typename T>
struct Same {
    using type = T;
};
template <typename T>
using SameT = typename Same<T>::type;

// Underflow / overflow guards of the reference (1e-300, 1e300) and their
// FP32 counterparts.
template <typename R> struct Lim;
template <> struct Lim<double> {
    static constexpr double tiny = 1e-300;
    static constexpr double huge = 1e300;
};
template <> struct Lim<float> {
    static constexpr float tiny = 1e-30f;
    static constexpr float huge = 1e30f;
};

template <typename R>
struct Vec3 {
    R x, y, z;
};

// Quaternion (w, x, y, z), body -> world.
template <typename R>
struct Quat {
    R w, x, y, z;
};

using V3 = Vec3<double>;
using Q = Quat<double>;
using V3f = Vec3<float>;
using Qf = Quat<float>;

template <typename R>
NE_HD Vec3<R> mk3(SameT<R> x, SameT<R> y, SameT<R> z) { Vec3<R> r; r.x = x; r.y = y; r.z = z; return r; }
NE_HD V3 mk(double x, double y, double z) { return mk3<double>(x, y, z); }
template <typename R>
NE_HD Quat<R> mkq4(SameT<R> w, SameT<R> x, SameT<R> y, SameT<R> z) {
    Quat<R> r; r.w = w; r.x = x; r.y = y; r.z = z; return r;
}
NE_HD Q mkq(double w, double x, double y, double z) { return mkq4<double>(w, x, y, z); }

template <typename R> NE_HD Vec3<R> operator+(const Vec3<R>& a, const Vec3<R>& b) { return mk3<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename R> NE_HD Vec3<R> operator-(const Vec3<R>& a, const Vec3<R>& b) { return mk3<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename R> NE_HD Vec3<R> operator-(const Vec3<R>& a) { return mk3<R>(-a.x, -a.y, -a.z); }
template <typename R> NE_HD Vec3<R> operator*(const Vec3<R>& a, SameT<R> s) { return mk3<R>(a.x * s, a.y * s, a.z * s); }
template <typename R> NE_HD Vec3<R> operator*(SameT<R> s, const Vec3<R>& a) { return mk3<R>(a.x * s, a.y * s, a.z * s); }
template <typename R> NE_HD Vec3<R> operator/(const Vec3<R>& a, SameT<R> s) { return mk3<R>(a.x / s, a.y / s, a.z / s); }
template <typename R> NE_HD R dot(const Vec3<R>& a, const Vec3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> NE_HD Vec3<R> cross(const Vec3<R>& a, const Vec3<R>& b) {
    return mk3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename R> NE_HD R norm2(const Vec3<R>& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
template <typename R> NE_HD R norm(const Vec3<R>& a) { return sqrt(norm2(a)); }
template <typename R> NE_HD Vec3<R> normalized(const Vec3<R>& a) {
    R n = norm(a);
    return (n > Lim<R>::tiny) ? mk3<R>(a.x / n, a.y / n, a.z / n) : mk3<R>(R(0), R(0), R(0));
}

// Precision conversion (exact float -> double; rounding double -> float).
template <typename To, typename From> NE_HD Vec3<To> cvt(const Vec3<From>& a) {
    return mk3<To>((To)a.x, (To)a.y, (To)a.z);
}
template <typename To, typename From> NE_HD Quat<To> cvtq(const Quat<From>& a) {
    return mkq4<To>((To)a.w, (To)a.x, (To)a.y, (To)a.z);
}

template <typename R>
NE_HD Quat<R> qmul(const Quat<R>& a, const Quat<R>& o) {
    return mkq4<R>(a.w * o.w - a.x * o.x - a.y * o.y - a.z * o.z,
                   a.w * o.x + a.x * o.w + a.y * o.z - a.z * o.y,
                   a.w * o.y - a.x * o.z + a.y * o.w + a.z * o.x,
                   a.w * o.z + a.x * o.y - a.y * o.x + a.z * o.w);
}
template <typename R> NE_HD Quat<R> qadd(const Quat<R>& a, const Quat<R>& o) { return mkq4<R>(a.w + o.w, a.x + o.x, a.y + o.y, a.z + o.z); }
template <typename R> NE_HD Quat<R> qscale(const Quat<R>& a, SameT<R> s) { return mkq4<R>(a.w * s, a.x * s, a.y * s, a.z * s); }
template <typename R> NE_HD Quat<R> qnormalized(const Quat<R>& a) {
    R n = sqrt(a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z);
    return (n > Lim<R>::tiny) ? mkq4<R>(a.w / n, a.x / n, a.y / n, a.z / n) : mkq4<R>(R(1), R(0), R(0), R(0));
}
template <typename R> NE_HD Quat<R> qconj(const Quat<R>& a) { return mkq4<R>(a.w, -a.x, -a.y, -a.z); }

// v' = q v q*  as  t = 2 (q_vec x v);  v' = v + w t + q_vec x t.
template <typename R>
NE_HD Vec3<R> rotate(const Quat<R>& q, const Vec3<R>& v) {
    Vec3<R> qv = mk3<R>(q.x, q.y, q.z);
    Vec3<R> t = R(2) * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
template <typename R> NE_HD Vec3<R> inv_rotate(const Quat<R>& q, const Vec3<R>& v) { return rotate(qconj(q), v); }

// q_{n+1} = normalise(q + (omega_quat * q) * (dt/2)).  FP64 only.
NE_HD Q integrate_orientation(const Q& q, const V3& omega, double dt) {
    Q omegaQ = mkq(0.0, omega.x, omega.y, omega.z);
    Q dq = qscale(qmul(omegaQ, q), 0.5 * dt);
    return qnormalized(qadd(q, dq));
}

// World-frame inverse inertia applied to u:  R diag(invI) R^T u.
template <typename R>
NE_HD Vec3<R> apply_inv_inertia(const Quat<R>& q, const Vec3<R>& invI, const Vec3<R>& u) {
    Vec3<R> ub = inv_rotate(q, u);
    Vec3<R> sb = mk3<R>(ub.x * invI.x, ub.y * invI.y, ub.z * invI.z);
    return rotate(q, sb);
}

// World-frame angular momentum L = I_world w.  FP64 only.
NE_HD V3 angular_momentum(const Q& q, const V3& invI, const V3& w) {
    V3 Ib = mk(invI.x > 0 ? 1.0 / invI.x : 0.0, invI.y > 0 ? 1.0 / invI.y : 0.0,
               invI.z > 0 ? 1.0 / invI.z : 0.0);
    V3 wb = inv_rotate(q, w);
    V3 Lb = mk(wb.x * Ib.x, wb.y * Ib.y, wb.z * Ib.z);
    return rotate(q, Lb);
}

// Cubic domain: minimum image and wrap (identity when not periodic).  The
// FP32 form evaluates both in FP64 before converting to a body-relative frame.
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

// Body-relative frames of the FP32 form are already minimum images: the
// domain is never periodic there.
NE_HD V3f min_image(const Domain&, V3f v) { return v; }

NE_HD V3 wrap(const Domain& d, V3 p) {
    if (!d.periodic) return p;
    const double L = 2.0 * d.half;
    p.x -= L * floor((p.x + d.half) / L);
    p.y -= L * floor((p.y + d.half) / L);
    p.z -= L * floor((p.z + d.half) / L);
    return p;
}

}  // namespace neb
