// CCD swept-sphere clamp (step.rs:1068-1155, :1210-1214; convex_sweep.rs:37-214, :263-295;
// gjk.rs:864-1044). One block per body that has CCD settings: the block's threads stride over
// the bodies of its world, keep those that pass the collision filters (no-contact-response
// targets, joint-suppressed pairs, group/mask) and whose broad-phase proxy touches the swept box,
// and cast a sphere against each; the block's smallest hit fraction is the clamp. A second
// kernel, after the position integration, pulls each clamped body back along its step motion.
// The reference scans every body for every CCD body as well; the cast itself (a ternary search
// for the closest approach, then bisection, each probe a GJK point distance) matches its
// arithmetic step for step.
#include <cstdio>
#include <cstdlib>
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

// A GJK simplex of up to four points, in the order the closest-feature tests keep them.
struct Simplex {
    V3 p[4];
    int n;
};

__device__ __forceinline__ void keep1(Simplex& s, V3 a) { s.p[0] = a; s.n = 1; }
__device__ __forceinline__ void keep2(Simplex& s, V3 a, V3 b) { s.p[0] = a; s.p[1] = b; s.n = 2; }
__device__ __forceinline__ void keep3(Simplex& s, V3 a, V3 b, V3 c) { s.p[0] = a; s.p[1] = b; s.p[2] = c; s.n = 3; }

// gjk.rs:889-906
__device__ __forceinline__ V3 closest_segment(V3 a, V3 b, Simplex& keep) {
    const V3 ab = b - a;
    if (len2(ab) == 0.0f) { keep1(keep, a); return a; }
    const float t = -dot(a, ab) / len2(ab);
    if (t <= 0.0f) { keep1(keep, a); return a; }
    if (t >= 1.0f) { keep1(keep, b); return b; }
    keep2(keep, b, a);
    return a + ab * t;
}

// gjk.rs:911-989, a degenerate triangle: the closest of its three edges. A call of its own
// (rarely taken), so the common path keeps the simplex in registers.
__device__ __noinline__ V3 closest_triangle_edges(V3 a, V3 b, V3 c, Simplex& keep) {
    Simplex kab, kbc, kca;
    const V3 qab = closest_segment(a, b, kab), qbc = closest_segment(b, c, kbc), qca = closest_segment(c, a, kca);
    if (len2(qab) <= len2(qbc) && len2(qab) <= len2(qca)) { keep = kab; return qab; }
    if (len2(qbc) <= len2(qca)) { keep = kbc; return qbc; }
    keep = kca;
    return qca;
}

// gjk.rs:911-989
__device__ __forceinline__ V3 closest_triangle(V3 a, V3 b, V3 c, Simplex& keep) {
    const V3 ab = b - a, ac = c - a, ap = -a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { keep1(keep, a); return a; }
    const V3 bp = -b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { keep1(keep, b); return b; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        if (d1 == d3) { keep1(keep, a); return a; }
        const float v = d1 / (d1 - d3);
        keep2(keep, b, a);
        return a + ab * v;
    }
    const V3 cp = -c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { keep1(keep, c); return c; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        if (d2 == d6) { keep1(keep, a); return a; }
        const float w = d2 / (d2 - d6);
        keep2(keep, c, a);
        return a + ac * w;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        if ((d4 - d3) + (d5 - d6) == 0.0f) { keep1(keep, b); return b; }
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        keep2(keep, c, b);
        return b + (c - b) * w;
    }
    const float sum = va + vb + vc;
    if (sum <= 0.0f || isnan(sum)) return closest_triangle_edges(a, b, c, keep);
    const float denom = 1.0f / sum;
    const float v = vb * denom, w = vc * denom;
    keep3(keep, c, b, a);
    return a + ab * v + ac * w;
}

// gjk.rs:994-1044, coplanar points: the closest of the four faces, the first of equal ones (a
// call of its own, rarely taken).
__device__ __noinline__ V3 closest_coplanar(V3 a, V3 b, V3 c, V3 d, Simplex& keep) {
    const V3 f[4][3] = {{a, b, c}, {a, b, d}, {a, c, d}, {b, c, d}};
    V3 best = V3{0.0f, 0.0f, 0.0f};
    Simplex best_keep;
    best_keep.n = 0;
    for (int k = 0; k < 4; ++k) {
        Simplex kk;
        const V3 q = closest_triangle(f[k][0], f[k][1], f[k][2], kk);
        if (k == 0 || len2(q) < len2(best)) { best = q; best_keep = kk; }
    }
    keep = best_keep;
    return best;
}

// gjk.rs:994-1044
__device__ __forceinline__ V3 closest_tetrahedron(V3 a, V3 b, V3 c, V3 d, Simplex& keep) {
    const V3 ao = -a, ab = b - a, ac = c - a, ad = d - a;
    if (fabsf(dot(cross(ab, ac), ad)) < 1e-12f) return closest_coplanar(a, b, c, d, keep);
    const V3 abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
    const V3 bo = -b;
    const V3 bcd = cross(c - b, d - b);
    if (dot(abc, ao) * dot(abc, ad) < 0.0f) return closest_triangle(a, b, c, keep);
    if (dot(acd, ao) * dot(acd, ab) < 0.0f) return closest_triangle(a, c, d, keep);
    if (dot(adb, ao) * dot(adb, ac) < 0.0f) return closest_triangle(a, d, b, keep);
    if (dot(bcd, bo) * dot(bcd, a - b) < 0.0f) return closest_triangle(b, c, d, keep);
    keep.p[0] = a; keep.p[1] = b; keep.p[2] = c; keep.p[3] = d; keep.n = 4;
    return V3{0.0f, 0.0f, 0.0f};
}

// gjk.rs:864-885
__device__ __forceinline__ V3 closest_origin(Simplex& s) {
    Simplex keep;
    V3 v;
    switch (s.n) {
        case 0: return V3{0.0f, 0.0f, 0.0f};
        case 1: return s.p[0];
        case 2: v = closest_segment(s.p[0], s.p[1], keep); break;
        case 3: v = closest_triangle(s.p[0], s.p[1], s.p[2], keep); break;
        default: v = closest_tetrahedron(s.p[0], s.p[1], s.p[2], s.p[3], keep); break;
    }
    s = keep;
    return v;
}

// The target inflated by the swept sphere (convex_sweep.rs:107-125): its support point along d.
struct Inflated {
    Shape s;
    V3 pos;
    Q ori;
    float radius;
    const float4* hull;
    __device__ __forceinline__ V3 support(V3 d) const {
        const V3 sphere = len2(d) > 1e-12f ? d / len(d) * radius : V3{0.0f, 0.0f, 0.0f};
        return support_world(s, pos, ori, d, hull) + sphere;
    }
};

// convex_sweep.rs:72-103: squared distance from `point` to the inflated target and the unit
// direction from the target toward the point (zero when inside or touching).
__device__ __forceinline__ float point_distance(const Inflated& t, V3 point, V3& dir) {
    auto mink = [&](V3 v) { return point - t.support(-v); };
    V3 v = point;
    if (len2(v) < 1e-12f) v = V3{1.0f, 0.0f, 0.0f};
    Simplex s;
    s.p[0] = mink(v);
    s.n = 1;
    v = s.p[0];
    for (int it = 0; it < 64; ++it) {
        if (len2(v) < 1e-10f) { dir = V3{0.0f, 0.0f, 0.0f}; return 0.0f; }
        const V3 w = mink(-v);
        bool repeat = false;  // the simplex already holds w (constant indices keep s in registers)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < s.n && len2(s.p[k] - w) < 1e-12f) repeat = true;
        if (repeat) { dir = v / len(v); return len2(v); }
        if (s.n >= 4) break;  // unreachable: a kept tetrahedron means v == 0, which returned above
        switch (s.n) {
            case 1: s.p[1] = w; break;
            case 2: s.p[2] = w; break;
            default: s.p[3] = w; break;
        }
        ++s.n;
        v = closest_origin(s);
    }
    if (len2(v) < 1e-10f) { dir = V3{0.0f, 0.0f, 0.0f}; return 0.0f; }
    dir = v / len(v);
    return len2(v);
}

__device__ __forceinline__ float point_distance2(const Inflated& t, V3 p) {
    V3 d;
    return point_distance(t, p, d);
}

// convex_sweep.rs:155-214 (sweep_with_dist), the fraction only
__device__ bool sweep_convex(V3 from, V3 dir, float length, const Inflated& t, float& fraction) {
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 40; ++it) {
        const float m1 = lo + (hi - lo) / 3.0f;
        const float m2 = hi - (hi - lo) / 3.0f;
        if (point_distance2(t, from + dir * (m1 * length)) < point_distance2(t, from + dir * (m2 * length))) hi = m2;
        else lo = m1;
    }
    const float s_min = (lo + hi) * 0.5f;
    if (point_distance2(t, from + dir * (s_min * length)) > 1e-8f) return false;
    float low = 0.0f, high = s_min;
    for (int it = 0; it < 60; ++it) {
        const float mid = (low + high) * 0.5f;
        if (point_distance2(t, from + dir * (mid * length)) <= 1e-8f) high = mid;
        else low = mid;
    }
    fraction = (low + high) * 0.5f;
    return true;
}

// convex_sweep.rs:217-262 (point_triangle_distance): squared distance to the triangle and the
// vector from its closest point to `p`.
__device__ float point_triangle_distance(V3 p, V3 a, V3 b, V3 c, V3& dv) {
    const V3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { dv = p - a; return len2(dv); }
    const V3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { dv = p - b; return len2(dv); }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        dv = p - (a + ab * v);
        return len2(dv);
    }
    const V3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { dv = p - c; return len2(dv); }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        dv = p - (a + ac * w);
        return len2(dv);
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        dv = p - (b + (c - b) * w);
        return len2(dv);
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    dv = p - (a + ab * v + ac * w);
    return len2(dv);
}

// convex_sweep.rs:131-151 (sweep_triangle) distance: zero inside the inflated triangle.
__device__ __forceinline__ float tri_inflated_distance2(V3 p, V3 a, V3 b, V3 c, float radius) {
    V3 dv;
    const float q = point_triangle_distance(p, a, b, c, dv);
    if (q <= radius * radius) return 0.0f;
    const float d = sqrtf(q);
    return (d - radius) * (d - radius);
}

// convex_sweep.rs:155-214 (sweep_with_dist) against one triangle, the fraction only.
__device__ bool sweep_triangle(V3 from, V3 dir, float length, float radius, V3 a, V3 b, V3 c, float& fraction) {
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 40; ++it) {
        const float m1 = lo + (hi - lo) / 3.0f;
        const float m2 = hi - (hi - lo) / 3.0f;
        if (tri_inflated_distance2(from + dir * (m1 * length), a, b, c, radius) <
            tri_inflated_distance2(from + dir * (m2 * length), a, b, c, radius))
            hi = m2;
        else
            lo = m1;
    }
    const float s_min = (lo + hi) * 0.5f;
    if (tri_inflated_distance2(from + dir * (s_min * length), a, b, c, radius) > 1e-8f) return false;
    float low = 0.0f, high = s_min;
    for (int it = 0; it < 60; ++it) {
        const float mid = (low + high) * 0.5f;
        if (tri_inflated_distance2(from + dir * (mid * length), a, b, c, radius) <= 1e-8f) high = mid;
        else low = mid;
    }
    fraction = (low + high) * 0.5f;
    return true;
}

// convex_sweep.rs:305-345 (sweep_mesh): the segment in the mesh frame, the BVH candidates of its
// swept box (bgpu_shapes.cuh's mesh layout), the smallest per-triangle fraction.
__device__ bool sweep_mesh(V3 from, V3 to, float radius, const Shape& ms, V3 pos, Q ori,
                           const float4* __restrict__ hull, uint32_t* status, float& fraction) {
    const Q inv = qinv(ori);
    const V3 lf = rotate(inv, from - pos), lt = rotate(inv, to - pos);
    const V3 delta = lt - lf;
    const float length = len(delta);
    if (length <= 1.1920929e-7f) return false;
    const V3 dir = delta / length;
    const V3 r = V3{radius, radius, radius};
    const V3 bmin = vmin(lf, lt) - r, bmax = vmax(lf, lt) + r;
    const uint32_t tri_base = mesh_tri_base(ms);
    bool any = false;
    float best = 1.0f;
    uint32_t stack[64];
    int sp = 0;
    if (ms.hull_cnt) stack[sp++] = 0;
    while (sp > 0) {
        const uint32_t k = stack[--sp];
        const float4 n0 = hull[ms.hull_off + 2 * k], n1 = hull[ms.hull_off + 2 * k + 1];
        if (!(n0.x <= bmax.x && n0.y <= bmax.y && n0.z <= bmax.z && bmin.x <= n1.x && bmin.y <= n1.y && bmin.z <= n1.z))
            continue;
        const uint32_t na = __float_as_uint(n0.w), nb = __float_as_uint(n1.w);
        if (!(na & MESH_LEAF)) {
            if (sp + 2 > 64) {
                atomicOr(status, ST_TRAVERSAL_STACK);
                continue;
            }
            stack[sp++] = na;
            stack[sp++] = nb;
            continue;
        }
        const uint32_t start = na & ~MESH_LEAF;
        for (uint32_t slot = start; slot < start + nb; ++slot) {
            const uint32_t o = tri_base + 3 * slot;
            float f;
            if (sweep_triangle(lf, dir, length, radius, from4(hull[o]), from4(hull[o + 1]), from4(hull[o + 2]), f) &&
                (!any || f < best)) {
                best = f;
                any = true;
            }
        }
    }
    if (any) fraction = best;
    return any;
}

// convex_sweep.rs:263-295 (sweep_plane), the fraction only
__device__ bool sweep_plane(V3 from, V3 dir, float length, float radius, const Shape& s, Q ori, float& fraction) {
    const V3 n = rotate(ori, V3{s.p0, s.p1, s.p2});
    const float dn0 = dot(n, from) - s.p3;
    if (fabsf(dn0) <= radius) { fraction = 0.0f; return true; }
    const float dd = dot(n, dir * length);
    if (dd >= 0.0f) return false;
    const float sign = dn0 > 0.0f ? 1.0f : -1.0f;
    const float f = (sign * radius - dn0) / dd;
    if (!(f >= 0.0f && f <= 1.0f)) return false;
    fraction = f;
    return true;
}

__device__ bool key_suppressed(const uint64_t* keys, uint32_t n, uint64_t k) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && keys[lo] == k;
}

__device__ __forceinline__ bool body_active(uint32_t act) {
    return act == ACT_ACTIVE || act == ACT_WANTS_DEACTIVATION || act == ACT_DISABLE_DEACTIVATION;
}

// One warp per CCD body. Candidates that pass the filters and the proxy-box pretest are kept in
// shared memory with a lower bound on their hit fraction; casts then run a warp-wide wave at a
// time in that order, and stop once the next bound is not below the best hit. Two facts keep the
// result equal to casting every candidate: the inflated target lies inside the ball of radius
// bound + swept radius about its position, so a segment that misses that ball (by more than the
// 1e-4 distance the cast accepts as touching, plus rounding) is a miss; and a hit's fraction is at
// least where the segment enters that ball. Overflowing the candidate buffer falls back to casting
// every candidate.
constexpr int CCD_THREADS = 32;
constexpr int CCD_CAP = 256;
constexpr uint32_t CCD_TREE_CAP = 1024;          // tree hits per CCD body before the world scan
constexpr uint32_t TREE_LEAF_REF = 0x80000000u;  // leaf children in the broad-phase node records
constexpr uint32_t CCD_WARP_CAST_MAX = 6;        // candidates left for which casts take the whole warp

struct CcdCtx {
    V3 from, to, dir;
    float length, radius;
    uint32_t* status;
};

__device__ __forceinline__ float cast_one(const BodyDev& b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                          const CcdCtx& c, uint32_t j) {
    const Shape& sj = shapes[b.info[j].x];
    float f;
    bool hit;
    if (sj.type == SHAPE_PLANE) {
        hit = sweep_plane(c.from, c.dir, c.length, c.radius, sj, q4(b.quat[j]), f);
    } else if (sj.type == SHAPE_MESH) {
        hit = sweep_mesh(c.from, c.to, c.radius, sj, from4(b.pos[j]), q4(b.quat[j]), hull, c.status, f);
    } else {
        Inflated t{sj, from4(b.pos[j]), q4(b.quat[j]), c.radius, hull};
        hit = sweep_convex(c.from, c.dir, c.length, t, f);
    }
    return hit ? f : 1.0f;
}

// The cast of one candidate by a whole warp, with the same result as sweep_convex: the
// ternary search's decisions depend only on the probes, so each round evaluates every probe of
// the next 4 levels of its decision tree at once (15 nodes x 2 probes on lanes 0-29) and then
// follows the taken path; the bisection likewise 5 levels per round (31 probes). A node's
// (lo, hi) is replayed from the round's root with the same operations as the sequential loop,
// so every probe point, and the fraction, is bit-identical to sweep_convex's.
__device__ __forceinline__ void replay_ternary(float& l, float& h, uint32_t node) {
    uint32_t path = 0, depth = 0;  // bit t: the branch taken at depth t + 1 (collected leaf first)
    for (uint32_t x = node; x > 0; x = (x - 1) >> 1) {
        path = (path << 1) | ((x & 1u) ? 0u : 1u);  // odd child: d(m1) < d(m2) (hi = m2)
        ++depth;
    }
    for (uint32_t t = 0; t < depth; ++t) {
        const float m1 = l + (h - l) / 3.0f;
        const float m2 = h - (h - l) / 3.0f;
        if (((path >> t) & 1u) == 0u) h = m2;
        else l = m1;
    }
}

__device__ __forceinline__ void replay_bisect(float& l, float& h, uint32_t node) {
    uint32_t path = 0, depth = 0;
    for (uint32_t x = node; x > 0; x = (x - 1) >> 1) {
        path = (path << 1) | ((x & 1u) ? 0u : 1u);  // odd child: d(mid) <= 1e-8 (high = mid)
        ++depth;
    }
    for (uint32_t t = 0; t < depth; ++t) {
        const float mid = (l + h) * 0.5f;
        if (((path >> t) & 1u) == 0u) h = mid;
        else l = mid;
    }
}

// td / bd: levels of the ternary / bisection decision tree evaluated per round (td levels:
// 2 (2^td - 1) probes; bd levels: 2^bd - 1 probes), on a segment of g lanes (the warp split into
// 32 / g segments that search side by side, each its own target; 2 (2^td - 1) <= g and
// 2^bd - 1 <= g). Every lane of the warp calls this with the same g, td and bd; the control flow
// is uniform across the warp (a segment whose closest approach misses still runs the bisection
// rounds if another segment's hits, and ignores them).
__device__ bool sweep_convex_seg(V3 from, V3 dir, float length, const Inflated& t, float& fraction, uint32_t td,
                                 uint32_t bd, uint32_t g) {
    const uint32_t sl = (threadIdx.x & 31u) % g;  // lane within the segment
    float lo = 0.0f, hi = 1.0f;
    for (uint32_t done = 0; done < 40;) {  // 40 ternary steps
        const uint32_t depth = min(td, 40u - done);
        const uint32_t probes = 2u * ((1u << depth) - 1u);
        float v = 0.0f;
        if (sl < probes) {
            float l = lo, h = hi;
            replay_ternary(l, h, sl >> 1);
            const float m = (sl & 1u) ? h - (h - l) / 3.0f : l + (h - l) / 3.0f;
            v = point_distance2(t, from + dir * (m * length));
        }
        uint32_t n = 0;
        for (uint32_t d = 0; d < depth; ++d) {
            const float d1 = __shfl_sync(0xffffffffu, v, int(2 * n), int(g));
            const float d2 = __shfl_sync(0xffffffffu, v, int(2 * n + 1), int(g));
            const float m1 = lo + (hi - lo) / 3.0f;
            const float m2 = hi - (hi - lo) / 3.0f;
            if (d1 < d2) { hi = m2; n = 2 * n + 1; }
            else { lo = m1; n = 2 * n + 2; }
        }
        done += depth;
    }
    const float s_min = (lo + hi) * 0.5f;
    const bool hit = !(point_distance2(t, from + dir * (s_min * length)) > 1e-8f);
    if (!__any_sync(0xffffffffu, hit)) return false;
    float low = 0.0f, high = s_min;
    for (uint32_t done = 0; done < 60;) {  // 60 bisection steps
        const uint32_t depth = min(bd, 60u - done);
        float v = 0.0f;
        if (sl < (1u << depth) - 1u) {
            float l = low, h = high;
            replay_bisect(l, h, sl);
            v = point_distance2(t, from + dir * (((l + h) * 0.5f) * length));
        }
        uint32_t n = 0;
        for (uint32_t d = 0; d < depth; ++d) {
            const float dm = __shfl_sync(0xffffffffu, v, int(n), int(g));
            const float mid = (low + high) * 0.5f;
            if (dm <= 1e-8f) { high = mid; n = 2 * n + 1; }
            else { low = mid; n = 2 * n + 2; }
        }
        done += depth;
    }
    fraction = (low + high) * 0.5f;
    return hit;
}

// cast_one for the whole warp (every lane returns the fraction): convex targets through
// sweep_convex_seg on the whole warp; planes and meshes by lane 0, broadcast.
__device__ __forceinline__ float cast_warp(const BodyDev& b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                           const CcdCtx& c, uint32_t j, uint32_t td, uint32_t bd) {
    const Shape& sj = shapes[b.info[j].x];
    if (sj.type == SHAPE_PLANE || sj.type == SHAPE_MESH) {
        float f = 1.0f;
        if ((threadIdx.x & 31u) == 0u) f = cast_one(b, shapes, hull, c, j);
        return __shfl_sync(0xffffffffu, f, 0);
    }
    Inflated t{sj, from4(b.pos[j]), q4(b.quat[j]), c.radius, hull};
    float f;
    return sweep_convex_seg(c.from, c.dir, c.length, t, f, td, bd, 32u) ? f : 1.0f;
}

__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// step.rs:1068-1155: the clamp fraction of CCD list entry blockIdx.x (1 when not clamped).
__global__ void __launch_bounds__(CCD_THREADS) k_ccd_sweep(BodyDev b, const Shape* __restrict__ shapes,
                                                           const float4* __restrict__ hull, const uint32_t* __restrict__ ids,
                                                           const float2* __restrict__ par, uint32_t n,
                                                           const uint32_t* __restrict__ world_off,
                                                           const uint32_t* __restrict__ world_of,
                                                           const uint64_t* __restrict__ suppressed, uint32_t nsuppressed,
                                                           float dt, float* clamp, uint32_t* status,
                                                           const float4* __restrict__ tree_rec,
                                                           const uint32_t* __restrict__ tree_leaf, int tree_m,
                                                           const uint32_t* __restrict__ unb, uint32_t nunb,
                                                           uint32_t depths) {
    __shared__ uint32_t cand[CCD_CAP], sorted[CCD_CAP];
    __shared__ uint32_t tlist[CCD_TREE_CAP];
    __shared__ uint32_t ntl;
    __shared__ float lb[CCD_CAP], slb[CCD_CAP];
    __shared__ uint32_t ncand;
    const uint32_t k = blockIdx.x, lane = threadIdx.x;
    const uint32_t i = ids[k];
    const float threshold = par[k].x, radius = par[k].y;
    const uint4 info = b.info[i];
    const Shape& si = shapes[info.x];
    const V3 from = from4(b.pos[i]);
    const V3 to = from + from4(b.linvel[i]) * dt;
    bool eligible = body_active(info.z) && !(info.y & (BF_STATIC | BF_KINEMATIC)) && threshold > 0.0f && radius > 0.0f &&
                    si.type != SHAPE_PLANE;
    eligible = eligible && !(len2(to - from) <= threshold * threshold);
    if (!eligible) {
        if (lane == 0) clamp[k] = 1.0f;
        return;
    }
    const V3 smin = vmin(from, to) - V3{radius, radius, radius}, smax = vmax(from, to) + V3{radius, radius, radius};
    const V3 delta = to - from;
    CcdCtx c;
    c.length = len(delta);
    c.dir = delta / c.length;
    c.from = from;
    c.to = to;
    c.radius = radius;
    c.status = status;
    // convex_sweep.rs:45-50: a vanishing motion casts nothing
    if (c.length <= 1.1920929e-7f) {
        if (lane == 0) clamp[k] = 1.0f;
        return;
    }
    const uint32_t gi = info.w & 0xFFFFu, mi = info.w >> 16;
    uint32_t lo = 0, hi = n;
    if (world_of) { lo = world_off[world_of[i]]; hi = world_off[world_of[i] + 1]; }
    // The targets: in a plain world, the step's broad-phase tree gives the proxies whose boxes
    // touch the swept box (the same closed test as the scan below, so the same set), plus the
    // proxies kept out of the tree (planes, meshes); in a batch, or when the list overflows,
    // every body of the world.
    const bool use_tree = tree_rec && !world_of && tree_m >= 1;
    if (lane == 0) {
        ncand = 0;
        ntl = 0;
        if (use_tree) {
            uint32_t cnt = 0;
            auto push = [&](uint32_t j) {
                if (cnt < CCD_TREE_CAP) tlist[cnt] = j;
                ++cnt;
            };
            const float4 qmin = make_float4(smin.x, smin.y, smin.z, 0.0f), qmax = make_float4(smax.x, smax.y, smax.z, 0.0f);
            auto touch = [&](float4 a, float4 b) {
                return a.x <= qmax.x && a.y <= qmax.y && a.z <= qmax.z && qmin.x <= b.x && qmin.y <= b.y && qmin.z <= b.z;
            };
            if (tree_m == 1) {
                push(tree_leaf[0]);
            } else {
                uint32_t stack[64];
                int sp = 0;
                stack[sp++] = 0u;
                while (sp > 0 && cnt <= CCD_TREE_CAP) {
                    const float4* r = tree_rec + size_t(stack[--sp]) * 4;
                    const float4 a = r[0], bb = r[1], cc = r[2], d = r[3];
                    const uint32_t ref[2] = {__float_as_uint(a.w), __float_as_uint(bb.w)};
                    const bool hit[2] = {touch(a, bb), touch(cc, d)};
                    for (int q = 0; q < 2; ++q) {
                        if (!hit[q]) continue;
                        if (ref[q] & TREE_LEAF_REF) push(ref[q] & ~TREE_LEAF_REF);
                        else if (sp < 64) stack[sp++] = ref[q];
                        else atomicOr(status, ST_TRAVERSAL_STACK);
                    }
                }
            }
            for (uint32_t u = 0; u < nunb; ++u) push(unb[u]);
            ntl = cnt;
        }
    }
    __syncthreads();
    const bool from_tree = use_tree && ntl <= CCD_TREE_CAP;
    const uint32_t nsrc = from_tree ? ntl : hi - lo;
    float best = 1.0f;
    for (uint32_t s = lane; s < nsrc; s += CCD_THREADS) {
        const uint32_t j = from_tree ? tlist[s] : lo + s;
        if (j == i) continue;
        const uint4 oj = b.info[j];
        if (oj.y & BF_NO_RESPONSE) continue;
        const uint32_t gj = oj.w & 0xFFFFu, mj = oj.w >> 16;
        if ((gi & mj) == 0 || (gj & mi) == 0) continue;
        const float4 amin = b.aabb_min[j], amax = b.aabb_max[j];
        // Aabb::overlaps (util.rs:28-38), closed on every axis
        if (!(amin.x <= smax.x && amin.y <= smax.y && amin.z <= smax.z && smin.x <= amax.x && smin.y <= amax.y &&
              smin.z <= amax.z))
            continue;
        if (nsuppressed) {
            const uint64_t key = (uint64_t(min(i, j)) << 32) | max(i, j);
            if (key_suppressed(suppressed, nsuppressed, key)) continue;
        }
        const Shape& sj = shapes[oj.x];
        if (sj.type == SHAPE_PLANE) {  // analytic and cheap: cast now
            best = fminf(best, cast_one(b, shapes, hull, c, j));
            continue;
        }
        // bounding ball of the inflated target, widened by the touch distance and rounding
        const V3 cj = from4(b.pos[j]);
        const float bound = len(vmax(vabs(V3{sj.lmin[0], sj.lmin[1], sj.lmin[2]}), vabs(V3{sj.lmax[0], sj.lmax[1], sj.lmax[2]})));
        const float slack = 1e-3f + 1e-5f * (len(cj) + len(from) + c.length);
        const float rr = bound + radius + slack;
        const V3 m = from - cj;
        const float bb = dot(m, c.dir);
        const float tca = fminf(fmaxf(-bb, 0.0f), c.length);
        if (len2(m + c.dir * tca) > rr * rr) continue;  // the segment misses the ball: no hit
        const float cc = len2(m) - rr * rr;
        float lower = 0.0f;
        if (cc > 0.0f) {
            const float disc = fmaxf(bb * bb - cc, 0.0f);
            lower = fmaxf((-bb - sqrtf(disc)) / c.length - 1e-6f - slack / c.length, 0.0f);
        }
        const uint32_t slot = atomicAdd(&ncand, 1u);
        if (slot < CCD_CAP) {
            cand[slot] = j;
            lb[slot] = lower;
        }
    }
    best = warp_min(best);
    __syncthreads();
    const uint32_t nc = ncand;
    if (nc > CCD_CAP) {
        // too many candidates for the buffer: cast every candidate that passes the same tests
        float mine = best;
        for (uint32_t s = lane; s < nsrc; s += CCD_THREADS) {
            const uint32_t j = from_tree ? tlist[s] : lo + s;
            if (j == i) continue;
            const uint4 oj = b.info[j];
            if ((oj.y & BF_NO_RESPONSE) || shapes[oj.x].type == SHAPE_PLANE) continue;
            const uint32_t gj = oj.w & 0xFFFFu, mj = oj.w >> 16;
            if ((gi & mj) == 0 || (gj & mi) == 0) continue;
            const float4 amin = b.aabb_min[j], amax = b.aabb_max[j];
            if (!(amin.x <= smax.x && amin.y <= smax.y && amin.z <= smax.z && smin.x <= amax.x && smin.y <= amax.y &&
                  smin.z <= amax.z))
                continue;
            if (nsuppressed && key_suppressed(suppressed, nsuppressed, (uint64_t(min(i, j)) << 32) | max(i, j))) continue;
            mine = fminf(mine, cast_one(b, shapes, hull, c, j));
        }
        best = warp_min(mine);
    } else {
        // order the candidates by their lower bound (rank by counting; ties by slot)
        for (uint32_t s = lane; s < nc; s += CCD_THREADS) {
            uint32_t r = 0;
            const float v = lb[s];
            for (uint32_t t = 0; t < nc; ++t) r += (lb[t] < v || (lb[t] == v && t < s)) ? 1u : 0u;
            sorted[r] = cand[s];
            slb[r] = v;
        }
        __syncthreads();
        // Few candidates: one at a time with the whole warp (23 probe latencies a cast); many:
        // a candidate per lane (141 probe latencies for up to 32 casts).
        // Up to 4 candidates whose bounds are below best side by side, one warp segment each (the
        // extra casts cannot lower best below the sequential result: a cast's fraction is never
        // below its bound), with shallower trees the narrower the segment.
        uint32_t s0 = 0;
        while (s0 < nc && nc - s0 <= CCD_WARP_CAST_MAX) {
            if (!(slb[s0] < best)) break;  // every later candidate hits no sooner than best
            uint32_t r = 1;
            bool mesh = shapes[b.info[sorted[s0]].x].type == SHAPE_MESH;
            while (r < 4 && s0 + r < nc && slb[s0 + r] < best) {
                mesh = mesh || shapes[b.info[sorted[s0 + r]].x].type == SHAPE_MESH;
                ++r;
            }
            if (mesh || r == 1) {
                best = fminf(best, cast_warp(b, shapes, hull, c, sorted[s0], depths & 0xffu, depths >> 8));
                ++s0;
                continue;
            }
            const uint32_t g = r >= 4 ? 8u : 16u, segs = 32u / g, use = min(segs, r);
            const uint32_t seg = lane / g;
            const uint32_t j = sorted[s0 + (seg < use ? seg : 0u)];
            const Shape& sj = shapes[b.info[j].x];
            Inflated tj{sj, from4(b.pos[j]), q4(b.quat[j]), c.radius, hull};
            float f = 1.0f;
            const bool hitj = sweep_convex_seg(c.from, c.dir, c.length, tj, f, g == 8u ? 2u : 3u, g == 8u ? 3u : 4u, g);
            best = fminf(best, warp_min(hitj && seg < use ? f : 1.0f));
            s0 += use;
        }
        for (uint32_t w0 = s0; w0 < nc; w0 += CCD_THREADS) {
            if (!(slb[w0] < best)) break;
            const uint32_t s = w0 + lane;
            float f = 1.0f;
            if (s < nc && slb[s] < best) f = cast_one(b, shapes, hull, c, sorted[s]);
            best = fminf(best, warp_min(f));
        }
    }
    if (lane == 0) clamp[k] = best;
}

// step.rs:1210-1214, after the position integration (which leaves the velocities unchanged).
__global__ void k_ccd_apply(BodyDev b, const uint32_t* __restrict__ ids, const float* __restrict__ clamp, uint32_t m,
                            float dt) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const float c = clamp[k];
    if (!(c < 1.0f)) return;
    const uint32_t i = ids[k];
    const V3 p = from4(b.pos[i]);
    const V3 from = p - from4(b.linvel[i]) * dt;
    b.pos[i] = to4(from + (p - from) * c, 0.0f);
}

}  // namespace

void launch_ccd_sweep(const BodyDev& b, const Shape* shapes, const float4* hull, const uint32_t* ids, const float2* par,
                      uint32_t m, uint32_t n, const uint32_t* world_off, const uint32_t* world_of,
                      const uint64_t* suppressed, uint32_t nsuppressed, float dt, float* clamp, uint32_t* status,
                      const float4* tree_rec, const uint32_t* tree_leaf, int tree_m, const uint32_t* unb,
                      uint32_t nunb, cudaStream_t s) {
    if (m == 0) return;
    // Speculation depths of the whole-warp casts (ternary | bisection << 8). On ccd_rain (2,048
    // casting bodies) the deepest trees measured fastest: 14.9 ms per step at (4, 5) against
    // 16.5 at (3, 4), 18.2 at (2, 3) and 22.2 at (1, 2). BGPU_CCD_DEPTH="t,b" overrides them,
    // for measurement.
    uint32_t td = 4u, bd = 5u;
    static int env_td = -1, env_bd = -1;
    if (env_td < 0) {
        env_td = env_bd = 0;
        if (const char* e = std::getenv("BGPU_CCD_DEPTH")) std::sscanf(e, "%d,%d", &env_td, &env_bd);
    }
    if (env_td >= 1 && env_td <= 4) td = uint32_t(env_td);
    if (env_bd >= 1 && env_bd <= 5) bd = uint32_t(env_bd);
    k_ccd_sweep<<<m, CCD_THREADS, 0, s>>>(b, shapes, hull, ids, par, n, world_off, world_of, suppressed, nsuppressed,
                                          dt, clamp, status, tree_rec, tree_leaf, tree_m, unb, nunb, td | (bd << 8));
}

void launch_ccd_apply(const BodyDev& b, const uint32_t* ids, const float* clamp, uint32_t m, float dt, cudaStream_t s) {
    if (m == 0) return;
    k_ccd_apply<<<(m + 127) / 128, 128, 0, s>>>(b, ids, clamp, m, dt);
}

}  // namespace bgpu
