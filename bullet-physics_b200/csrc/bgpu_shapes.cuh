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

enum ShapeType : uint32_t { SHAPE_SPHERE = 0, SHAPE_BOX = 1, SHAPE_CAPSULE = 2, SHAPE_HULL = 3, SHAPE_PLANE = 4,
                            SHAPE_MESH = 5 };

// Static triangle mesh (triangle_mesh.rs, with its BVH from bvh.rs; heightfields are built into
// one). The record keeps the BVH in the hull array: node k at float4 hull_off + 2k as
// (min.xyz, a) and (max.xyz, b), with a = start | 1 << 31, b = count for a leaf and a = left,
// b = right for an internal node (a, b as uint bits), hull_cnt nodes in the reference's
// pre-order. The triangles follow in the BVH's permutation order: slot k holds three float4
// vertices at tri_base + 3k (p0's bits), the triangle's own index in the first one's w bits;
// p1's bits hold the triangle count. Local bounds in lmin / lmax; margin 0.
constexpr uint32_t MESH_LEAF = 1u << 31;

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

__host__ __device__ __forceinline__ uint32_t mesh_tri_base(const Shape& s) {
    uint32_t u;
    memcpy(&u, &s.p0, 4);
    return u;
}
__host__ __device__ __forceinline__ uint32_t mesh_ntris(const Shape& s) {
    uint32_t u;
    memcpy(&u, &s.p1, 4);
    return u;
}

// util.rs:106-126 (Aabb::transformed): the eight corners of a box's centre +- extents, rotated
// and moved, wrapped in an axis-aligned box.
__device__ __forceinline__ void aabb_transformed(V3 lmin, V3 lmax, V3 p, Q q, V3& mn, V3& mx) {
    const V3 c = (lmin + lmax) * 0.5f, e = (lmax - lmin) * 0.5f;
    mn = splat(INFINITY);
    mx = splat(-INFINITY);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const V3 corner = V3{(i & 1) == 0 ? c.x + e.x : c.x - e.x, (i & 2) == 0 ? c.y + e.y : c.y - e.y,
                             (i & 4) == 0 ? c.z + e.z : c.z - e.z};
        const V3 w = rotate(q, corner) + p;
        mn = vmin(mn, w);
        mx = vmax(mx, w);
    }
}

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
        case SHAPE_MESH:  // triangle_mesh.rs:213-216
            aabb_transformed(V3{s.lmin[0], s.lmin[1], s.lmin[2]}, V3{s.lmax[0], s.lmax[1], s.lmax[2]}, p, q, mn, mx);
            return;
        default:
            mn = splat(-1e30f);
            mx = splat(1e30f);
            return;
    }
}

}  // namespace bgpu
