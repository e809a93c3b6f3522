// Shape table and support mappings (device side).
//
// Shape semantics follow crates/bullet-collision/src/shapes/: box margin 0.04
// with a componentwise-shrunk core (box_shape.rs:20-53), sphere core = centre
// and margin = radius (sphere.rs:18-26), capsule core = its Y segment and
// margin = radius (capsule.rs:27-69), hull margin 0 with a first-maximum
// vertex scan (convex_hull.rs:43-66), plane AABB of +-1e30 (plane.rs:32-40).
#pragma once
#include "bgpu_math.cuh"

namespace bgpu {

enum ShapeType : uint32_t { SHAPE_SPHERE = 0, SHAPE_BOX = 1, SHAPE_CAPSULE = 2, SHAPE_HULL = 3, SHAPE_PLANE = 4 };

// 64-byte shape record.
struct Shape {
    uint32_t type;
    float p0, p1, p2, p3;  // box: half extents; sphere: r; capsule: r, half height; plane: n.xyz, c
    uint32_t hull_off, hull_cnt;
    float margin;
    float cbt;             // contact-breaking threshold (shapes/mod.rs:388-392)
    float lmin[3], lmax[3];  // local AABB
    float pad;
};
static_assert(sizeof(Shape) == 64, "Shape record is 64 bytes");

// shapes/mod.rs:275-291 and the per-shape support_local.
__device__ __forceinline__ V3 support_local(const Shape& s, V3 d, const float4* __restrict__ hull) {
    switch (s.type) {
        case SHAPE_SPHERE: {
            float l = len(d);
            if (l > 0.0f) return d / l * s.p0;
            return V3{s.p0, 0.f, 0.f};
        }
        case SHAPE_BOX:
            return V3{d.x >= 0.0f ? s.p0 : -s.p0, d.y >= 0.0f ? s.p1 : -s.p1, d.z >= 0.0f ? s.p2 : -s.p2};
        case SHAPE_CAPSULE: {
            float l = len(d);
            if (l > 0.0f) {
                V3 tip = V3{0.f, d.y >= 0.0f ? s.p1 : -s.p1, 0.f};
                return tip + d / l * s.p0;
            }
            return V3{s.p0, s.p1, 0.f};
        }
        case SHAPE_HULL: {
            V3 best = V3{0.f, 0.f, 0.f};
            float bd = -INFINITY;
            for (uint32_t i = 0; i < s.hull_cnt; ++i) {
                float4 p4 = __ldg(&hull[s.hull_off + i]);
                V3 p = from4(p4);
                float dd = dot(p, d);
                if (dd > bd) { bd = dd; best = p; }
            }
            return best;
        }
        default:
            return V3{0.f, 0.f, 0.f};
    }
}

// shapes/mod.rs:305-319
__device__ __forceinline__ V3 core_support_local(const Shape& s, V3 d, const float4* __restrict__ hull) {
    switch (s.type) {
        case SHAPE_SPHERE: return V3{0.f, 0.f, 0.f};
        case SHAPE_BOX: {
            float hx = fmaxf(s.p0 - s.margin, 0.0f), hy = fmaxf(s.p1 - s.margin, 0.0f), hz = fmaxf(s.p2 - s.margin, 0.0f);
            return V3{d.x >= 0.0f ? hx : -hx, d.y >= 0.0f ? hy : -hy, d.z >= 0.0f ? hz : -hz};
        }
        case SHAPE_CAPSULE: return V3{0.f, d.y >= 0.0f ? s.p1 : -s.p1, 0.f};
        default: return support_local(s, d, hull);
    }
}

__device__ __forceinline__ V3 support_world(const Shape& s, V3 p, Q q, V3 dir, const float4* __restrict__ hull) {
    V3 ld = rotate(qinv(q), dir);
    return rotate(q, support_local(s, ld, hull)) + p;
}

__device__ __forceinline__ V3 core_support_world(const Shape& s, V3 p, Q q, V3 dir, const float4* __restrict__ hull) {
    V3 ld = rotate(qinv(q), dir);
    return rotate(q, core_support_local(s, ld, hull)) + p;
}

// shapes/mod.rs:350-375 (world AABB of a pose).
__device__ __forceinline__ void world_aabb(const Shape& s, V3 p, Q q, const float4* __restrict__ hull, V3& mn, V3& mx) {
    switch (s.type) {
        case SHAPE_SPHERE:
            mn = p - splat(s.p0);
            mx = p + splat(s.p0);
            return;
        case SHAPE_BOX: {
            mn = splat(INFINITY);
            mx = splat(-INFINITY);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                V3 c = V3{(i & 1) == 0 ? s.p0 : -s.p0, (i & 2) == 0 ? s.p1 : -s.p1, (i & 4) == 0 ? s.p2 : -s.p2};
                V3 w = rotate(q, c) + p;
                mn = vmin(mn, w);
                mx = vmax(mx, w);
            }
            return;
        }
        case SHAPE_CAPSULE: {
            V3 top = rotate(q, V3{0.f, s.p1, 0.f}) + p;
            V3 bot = rotate(q, V3{0.f, -s.p1, 0.f}) + p;
            V3 r = splat(s.p0);
            mn = vmin(top, bot) - r;
            mx = vmax(top, bot) + r;
            return;
        }
        case SHAPE_HULL: {  // support projections (shapes/mod.rs:448-469)
            Q qi = qinv(q);
            V3 ux = rotate(qi, V3{1.f, 0.f, 0.f}), uy = rotate(qi, V3{0.f, 1.f, 0.f}), uz = rotate(qi, V3{0.f, 0.f, 1.f});
            mn = V3{p.x + dot(support_local(s, -ux, hull), ux), p.y + dot(support_local(s, -uy, hull), uy),
                    p.z + dot(support_local(s, -uz, hull), uz)};
            mx = V3{p.x + dot(support_local(s, ux, hull), ux), p.y + dot(support_local(s, uy, hull), uy),
                    p.z + dot(support_local(s, uz, hull), uz)};
            return;
        }
        default:
            mn = splat(-1e30f);
            mx = splat(1e30f);
            return;
    }
}

}  // namespace bgpu
