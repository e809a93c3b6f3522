// CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// A plain scalar C++ restatement of the rigid-body hot path of the Rust
// crates bullet-math / bullet-collision / bullet-dynamics
// (CrazyboyQCD/bullet-physics). It exists to check the CUDA product path and
// to time a CPU baseline; nothing in the shipped library includes or links it.
// Every function names the reference file:line whose behaviour it restates.
//
// Precision is a template parameter (float mirrors the default `Real = f32`,
// double mirrors `--features f64`, crates/bullet-math/src/lib.rs:28-56).
//
// Third-party arithmetic: the reference delegates vector/quaternion/matrix
// arithmetic to glam 0.33.3 (not vendored in the reference tree). The
// formulas below are the textbook ones (Hamilton product, rotation
// v' = v(w^2 - |b|^2) + 2 b (b.v) + 2w (b x v), cofactor 3x3 inverse), so
// glam's exact operation order is not pinned bit-for-bit; parity is held to
// the reference's own test epsilons.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace oracle {

template <class R>
struct V3 {
    R x = 0, y = 0, z = 0;
    V3() = default;
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    static V3 splat(R v) { return V3(v, v, v); }
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    R& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator-() const { return V3(-x, -y, -z); }
    V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
    V3 operator*(const V3& o) const { return V3(x * o.x, y * o.y, z * o.z); }
    V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
    V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    V3& operator*=(R s) { x *= s; y *= s; z *= s; return *this; }
    R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const {
        return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    R length_squared() const { return dot(*this); }
    R length() const { return std::sqrt(length_squared()); }
    V3 normalize() const { return *this / length(); }
    V3 min(const V3& o) const { return V3(std::min(x, o.x), std::min(y, o.y), std::min(z, o.z)); }
    V3 max(const V3& o) const { return V3(std::max(x, o.x), std::max(y, o.y), std::max(z, o.z)); }
    V3 abs() const { return V3(std::fabs(x), std::fabs(y), std::fabs(z)); }
};

template <class R>
inline V3<R> operator*(R s, const V3<R>& v) { return v * s; }

template <class R>
struct Quat {
    R x = 0, y = 0, z = 0, w = 1;
    Quat() = default;
    Quat(R a, R b, R c, R d) : x(a), y(b), z(c), w(d) {}
    static Quat identity() { return Quat(0, 0, 0, 1); }
    V3<R> xyz() const { return V3<R>(x, y, z); }
    // Unit-quaternion inverse = conjugate.
    Quat inverse() const { return Quat(-x, -y, -z, w); }
    Quat operator*(const Quat& b) const {
        return Quat(w * b.x + x * b.w + y * b.z - z * b.y,
                    w * b.y - x * b.z + y * b.w + z * b.x,
                    w * b.z + x * b.y - y * b.x + z * b.w,
                    w * b.w - x * b.x - y * b.y - z * b.z);
    }
    Quat operator+(const Quat& b) const { return Quat(x + b.x, y + b.y, z + b.z, w + b.w); }
    R length_squared() const { return x * x + y * y + z * z + w * w; }
    Quat normalize() const {
        R l = std::sqrt(length_squared());
        return Quat(x / l, y / l, z / l, w / l);
    }
    // v' = v (w^2 - b.b) + b (2 b.v) + (b x v)(2w)
    V3<R> rotate(const V3<R>& v) const {
        V3<R> b(x, y, z);
        R b2 = b.dot(b);
        return v * (w * w - b2) + b * (v.dot(b) * R(2)) + b.cross(v) * (w * R(2));
    }
};

// Column-major 3x3.
template <class R>
struct M3 {
    V3<R> c0, c1, c2;
    M3() = default;
    M3(const V3<R>& a, const V3<R>& b, const V3<R>& c) : c0(a), c1(b), c2(c) {}
    static M3 diag(const V3<R>& d) {
        return M3(V3<R>(d.x, 0, 0), V3<R>(0, d.y, 0), V3<R>(0, 0, d.z));
    }
    static M3 from_quat(const Quat<R>& q) {
        R x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
        R xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
        R yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
        R wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
        return M3(V3<R>(R(1) - (yy + zz), xy + wz, xz - wy),
                  V3<R>(xy - wz, R(1) - (xx + zz), yz + wx),
                  V3<R>(xz + wy, yz - wx, R(1) - (xx + yy)));
    }
    const V3<R>& col(int i) const { return i == 0 ? c0 : (i == 1 ? c1 : c2); }
    V3<R> operator*(const V3<R>& v) const { return c0 * v.x + c1 * v.y + c2 * v.z; }
    M3 operator*(const M3& b) const { return M3((*this) * b.c0, (*this) * b.c1, (*this) * b.c2); }
    M3 operator+(const M3& b) const { return M3(c0 + b.c0, c1 + b.c1, c2 + b.c2); }
    M3 operator-(const M3& b) const { return M3(c0 - b.c0, c1 - b.c1, c2 - b.c2); }
    M3 operator*(R s) const { return M3(c0 * s, c1 * s, c2 * s); }
    M3 transpose() const {
        return M3(V3<R>(c0.x, c1.x, c2.x), V3<R>(c0.y, c1.y, c2.y), V3<R>(c0.z, c1.z, c2.z));
    }
    M3 inverse() const {
        V3<R> t0 = c1.cross(c2), t1 = c2.cross(c0), t2 = c0.cross(c1);
        R det = c2.dot(t2);
        R inv = R(1) / det;
        return M3(t0 * inv, t1 * inv, t2 * inv).transpose();
    }
};

// crates/bullet-math/src/spatial.rs:422-428
template <class R>
inline M3<R> skew(const V3<R>& t) {
    return M3<R>(V3<R>(0, t.z, -t.y), V3<R>(-t.z, 0, t.x), V3<R>(t.y, -t.x, 0));
}

// crates/bullet-math/src/util.rs:5-126
template <class R>
struct Aabb {
    V3<R> min, max;
    Aabb() = default;
    Aabb(const V3<R>& a, const V3<R>& b) : min(a), max(b) {}
    V3<R> center() const { return (min + max) * R(0.5); }
    V3<R> extents() const { return (max - min) * R(0.5); }
    // util.rs:28-38 — closed bounds: touching counts as overlapping.
    bool overlaps(const Aabb& o) const {
        return min.x <= o.max.x && min.y <= o.max.y && min.z <= o.max.z &&
               o.min.x <= max.x && o.min.y <= max.y && o.min.z <= max.z;
    }
    // util.rs:52-55
    Aabb expanded(R m) const { return Aabb(min - V3<R>::splat(m), max + V3<R>::splat(m)); }
};

// util.rs:133-141 — R * diag(inv) * R^T
template <class R>
inline M3<R> inertia_tensor_world(const V3<R>& inv_local, const Quat<R>& q) {
    M3<R> r = M3<R>::from_quat(q);
    return r * M3<R>::diag(inv_local) * r.transpose();
}

template <class R> struct Consts;
template <> struct Consts<float> {
    static constexpr float EPS = 1.1920929e-7f;            // f32::EPSILON
    static constexpr float EPA_EPSILON = 1e-4f;            // narrowphase/epa.rs:34-35
    static constexpr float EPA_PLANE_EPS = 1e-5f;          // epa.rs:40-41
    static constexpr float TAYLOR = 0.020833333f;          // body.rs:80-81
    static constexpr float FRAC_PI_4 = 0.785398163397448309615f;  // body.rs:72-73
    static constexpr float FRAC_1_SQRT_2 = 0.707106781186547524401f;
};
template <> struct Consts<double> {
    static constexpr double EPS = 2.220446049250313e-16;   // f64::EPSILON
    static constexpr double EPA_EPSILON = 1e-12;           // epa.rs:36-37
    static constexpr double EPA_PLANE_EPS = 1e-14;         // epa.rs:42-43
    static constexpr double TAYLOR = 0.020833333333;       // body.rs:82-83
    static constexpr double FRAC_PI_4 = 0.785398163397448309615;
    static constexpr double FRAC_1_SQRT_2 = 0.707106781186547524401;
};

}  // namespace oracle
