// ne_dual.cuh -- forward-mode dual numbers for the contact-geometry Jacobians
// of the adjoint.
//
// A Dual carries a value and its derivatives along kDualDirs directions: the
// poses of the two bodies of a pair, (x_a, q_a, x_b, q_b) = 3 + 4 + 3 + 4.
// Instantiating the templated geometry of ne_geom.cuh with R = Dual gives the
// contact normal, point and depth together with their derivatives with respect
// to both poses: every branch is taken on the values, exactly as the FP64
// evaluation takes it, so the derivative is that of the branch the step used.
#pragma once

#include "ne_math.cuh"

namespace neb {

// The Dual overloads below must not hide the double ones for code in neb.
using ::sqrt;
using ::fabs;
using ::floor;

constexpr int kDualDirs = 14;

struct Dual {
    double v;
    double d[kDualDirs];
    NE_HD Dual() : v(0.0) {
        for (int k = 0; k < kDualDirs; ++k) d[k] = 0.0;
    }
    NE_HD Dual(double x) : v(x) {
        for (int k = 0; k < kDualDirs; ++k) d[k] = 0.0;
    }
    NE_HD Dual(int x) : v((double)x) {
        for (int k = 0; k < kDualDirs; ++k) d[k] = 0.0;
    }
    NE_HD static Dual seed(double x, int dir) {
        Dual r(x);
        r.d[dir] = 1.0;
        return r;
    }
};

NE_HD Dual operator+(const Dual& a, const Dual& b) {
    Dual r(a.v + b.v);
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
NE_HD Dual operator-(const Dual& a, const Dual& b) {
    Dual r(a.v - b.v);
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
NE_HD Dual operator-(const Dual& a) {
    Dual r(-a.v);
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = -a.d[k];
    return r;
}
NE_HD Dual operator*(const Dual& a, const Dual& b) {
    Dual r(a.v * b.v);
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
NE_HD Dual operator/(const Dual& a, const Dual& b) {
    Dual r(a.v / b.v);
    const double inv = 1.0 / b.v;
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
NE_HD Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
NE_HD Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
NE_HD Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }

NE_HD bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
NE_HD bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
NE_HD bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
NE_HD bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
NE_HD bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
NE_HD bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
NE_HD bool operator<(const Dual& a, double b) { return a.v < b; }
NE_HD bool operator>(const Dual& a, double b) { return a.v > b; }
NE_HD bool operator<=(const Dual& a, double b) { return a.v <= b; }
NE_HD bool operator>=(const Dual& a, double b) { return a.v >= b; }
NE_HD bool operator<(const Dual& a, int b) { return a.v < b; }
NE_HD bool operator>(const Dual& a, int b) { return a.v > b; }
NE_HD bool operator<=(const Dual& a, int b) { return a.v <= b; }
NE_HD bool operator>=(const Dual& a, int b) { return a.v >= b; }

NE_HD Dual sqrt(const Dual& a) {
    const double s = ::sqrt(a.v);
    Dual r(s);
    const double g = (s > 0.0) ? 0.5 / s : 0.0;
    for (int k = 0; k < kDualDirs; ++k) r.d[k] = a.d[k] * g;
    return r;
}
NE_HD Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }

template <> struct Lim<Dual> {
    static constexpr double tiny = 1e-300;
    static constexpr double huge = 1e300;
};

// Minimum image of a pair offset: a piecewise-constant shift, so its
// derivative is the identity on each piece.
NE_HD Vec3<Dual> min_image(const Domain& d, Vec3<Dual> v) {
    if (!d.periodic) return v;
    const double L = 2.0 * d.half;
    v.x = v.x - Dual(L * floor(v.x.v / L + 0.5));
    v.y = v.y - Dual(L * floor(v.y.v / L + 0.5));
    v.z = v.z - Dual(L * floor(v.z.v / L + 0.5));
    return v;
}

NE_HD V3 val(const Vec3<Dual>& a) { return mk(a.x.v, a.y.v, a.z.v); }

}  // namespace neb
