// ne/vmath.hpp -- value types of the host facade: the same public interface as
// the reference's ne::V3 / ne::Q (src/vmath.hpp:18-78), so code written
// against the reference compiles unchanged.  Host-side arithmetic only; the
// step runs on the device (libne_cuda.so).
#pragma once
#include <cmath>

namespace ne {

constexpr double PI = 3.14159265358979323846;

struct V3 {
    double x = 0.0, y = 0.0, z = 0.0;
    V3() = default;
    V3(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
    V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator-() const { return {-x, -y, -z}; }
    V3 operator*(double s) const { return {x * s, y * s, z * s}; }
    V3 operator/(double s) const { return {x / s, y / s, z / s}; }
    V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    double dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
    double norm2() const { return x * x + y * y + z * z; }
    double norm() const { return std::sqrt(norm2()); }
    V3 normalized() const {
        const double n = norm();
        return n > 1e-300 ? V3{x / n, y / n, z / n} : V3{0, 0, 0};
    }
};
inline V3 operator*(double s, const V3& v) { return v * s; }

// Quaternion (w, x, y, z), body -> world.
struct Q {
    double w = 1.0, x = 0.0, y = 0.0, z = 0.0;
    Q() = default;
    Q(double w_, double x_, double y_, double z_) : w(w_), x(x_), y(y_), z(z_) {}
    Q operator*(const Q& o) const {
        return {w * o.w - x * o.x - y * o.y - z * o.z, w * o.x + x * o.w + y * o.z - z * o.y,
                w * o.y - x * o.z + y * o.w + z * o.x, w * o.z + x * o.y - y * o.x + z * o.w};
    }
    double norm() const { return std::sqrt(w * w + x * x + y * y + z * z); }
    Q normalized() const {
        const double n = norm();
        return n > 1e-300 ? Q{w / n, x / n, y / n, z / n} : Q{1, 0, 0, 0};
    }
    Q conjugate() const { return {w, -x, -y, -z}; }
    V3 rotate(const V3& v) const {
        const V3 qv{x, y, z};
        const V3 t = 2.0 * qv.cross(v);
        return v + w * t + qv.cross(t);
    }
    V3 inverseRotate(const V3& v) const { return conjugate().rotate(v); }
};

}  // namespace ne
