// Vector / quaternion / 3x3 arithmetic for the device kernels.
//
// The formulas are the textbook ones used by the reference's vector library
// (glam, called from crates/bullet-math/src/lib.rs:28-56): Hamilton product,
// rotation v' = v (w^2 - b.b) + 2 b (b.v) + 2 w (b x v), column-major 3x3
// with a cofactor inverse. Every operation is written out in a fixed order and
// the kernels are compiled without FMA contraction, so a kernel and a scalar
// CPU evaluation of the same expression round identically.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define BG_HD __host__ __device__ __forceinline__

namespace bgpu {

struct V3 {
    float x, y, z;
};

BG_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
BG_HD V3 splat(float s) { return V3{s, s, s}; }
BG_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
BG_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
BG_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
BG_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
BG_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
BG_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
BG_HD V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
BG_HD V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
BG_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
BG_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
BG_HD float len2(V3 a) { return dot(a, a); }
BG_HD float len(V3 a) { return sqrtf(len2(a)); }
BG_HD V3 normalize(V3 a) { return a / len(a); }
BG_HD V3 vmin(V3 a, V3 b) { return V3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
BG_HD V3 vmax(V3 a, V3 b) { return V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
BG_HD V3 vabs(V3 a) { return V3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
BG_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
BG_HD V3 from4(float4 f) { return V3{f.x, f.y, f.z}; }
BG_HD float4 to4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

struct Q {
    float x, y, z, w;
};
BG_HD Q q4(float4 f) { return Q{f.x, f.y, f.z, f.w}; }
BG_HD float4 to4(Q q) { return make_float4(q.x, q.y, q.z, q.w); }
BG_HD Q qinv(Q q) { return Q{-q.x, -q.y, -q.z, q.w}; }
BG_HD Q qmul(Q a, Q b) {
    return Q{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
             a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
BG_HD float qlen2(Q q) { return q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w; }
BG_HD V3 rotate(Q q, V3 v) {
    V3 b = V3{q.x, q.y, q.z};
    float b2 = dot(b, b);
    return v * (q.w * q.w - b2) + b * (dot(v, b) * 2.0f) + cross(b, v) * (q.w * 2.0f);
}

// Column-major 3x3: c0, c1, c2 are the columns.
struct M3 {
    V3 c0, c1, c2;
};
BG_HD V3 col(const M3& m, int i) { return i == 0 ? m.c0 : (i == 1 ? m.c1 : m.c2); }
BG_HD V3 mul(const M3& m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
BG_HD M3 mul(const M3& a, const M3& b) { return M3{mul(a, b.c0), mul(a, b.c1), mul(a, b.c2)}; }
BG_HD M3 transpose(const M3& m) {
    return M3{V3{m.c0.x, m.c1.x, m.c2.x}, V3{m.c0.y, m.c1.y, m.c2.y}, V3{m.c0.z, m.c1.z, m.c2.z}};
}
BG_HD M3 diag(V3 d) { return M3{V3{d.x, 0.f, 0.f}, V3{0.f, d.y, 0.f}, V3{0.f, 0.f, d.z}}; }
BG_HD M3 madd(const M3& a, const M3& b) { return M3{a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2}; }
BG_HD M3 msub(const M3& a, const M3& b) { return M3{a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2}; }
BG_HD M3 mscale(const M3& a, float s) { return M3{a.c0 * s, a.c1 * s, a.c2 * s}; }
BG_HD M3 from_quat(Q q) {
    float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    return M3{V3{1.0f - (yy + zz), xy + wz, xz - wy}, V3{xy - wz, 1.0f - (xx + zz), yz + wx},
              V3{xz + wy, yz - wx, 1.0f - (xx + yy)}};
}
BG_HD M3 inverse(const M3& m) {
    V3 t0 = cross(m.c1, m.c2), t1 = cross(m.c2, m.c0), t2 = cross(m.c0, m.c1);
    float det = dot(m.c2, t2);
    float inv = 1.0f / det;
    return transpose(M3{t0 * inv, t1 * inv, t2 * inv});
}
BG_HD M3 skew(V3 t) { return M3{V3{0.f, t.z, -t.y}, V3{-t.z, 0.f, t.x}, V3{t.y, -t.x, 0.f}}; }
// R * diag(inv) * R^T (the world inverse inertia).
BG_HD M3 inertia_world(V3 inv_local, Q q) {
    M3 r = from_quat(q);
    return mul(mul(r, diag(inv_local)), transpose(r));
}

BG_HD bool absdiff_le(V3 a, V3 b, float tol) {
    return fabsf(a.x - b.x) <= tol && fabsf(a.y - b.y) <= tol && fabsf(a.z - b.z) <= tol;
}

}  // namespace bgpu
