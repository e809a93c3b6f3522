// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_math.hpp).
// Shapes restated from crates/bullet-collision/src/shapes/{mod,box_shape,
// sphere,capsule,convex_hull,plane,triangle_mesh,bvh,heightfield}.rs.
#pragma once
#include <algorithm>
#include <array>
#include <memory>
#include "oracle_math.hpp"

namespace oracle {

enum ShapeType : uint32_t { SHAPE_SPHERE = 0, SHAPE_BOX = 1, SHAPE_CAPSULE = 2, SHAPE_HULL = 3, SHAPE_PLANE = 4,
                            SHAPE_MESH = 5 };

// util.rs:106-126 (Aabb::transformed): the eight corners of centre +- extents, rotated and moved.
template <class R>
Aabb<R> aabb_transformed(const Aabb<R>& a, const V3<R>& p, const Quat<R>& q) {
    V3<R> c = a.center(), e = a.extents();
    V3<R> mn = V3<R>::splat(std::numeric_limits<R>::infinity());
    V3<R> mx = V3<R>::splat(-std::numeric_limits<R>::infinity());
    for (int i = 0; i < 8; ++i) {
        V3<R> corner((i & 1) == 0 ? c.x + e.x : c.x - e.x, (i & 2) == 0 ? c.y + e.y : c.y - e.y,
                     (i & 4) == 0 ? c.z + e.z : c.z - e.z);
        V3<R> w = q.rotate(corner) + p;
        mn = mn.min(w);
        mx = mx.max(w);
    }
    return Aabb<R>(mn, mx);
}

// Static triangle mesh (triangle_mesh.rs:34-123) with its BVH (bvh.rs:16-206): nodes in
// pre-order, internal nodes with a child pair, leaves with a range of the triangle
// permutation; longest-axis median split of the triangle centres, at most 4 per leaf.
template <class R>
struct MeshData {
    struct Node {
        Aabb<R> aabb;
        bool leaf = true;
        uint32_t a = 0, b = 0;  // leaf: start, count; internal: left, right
    };
    std::vector<V3<R>> vertices;
    std::vector<std::array<uint32_t, 3>> indices;
    std::vector<Node> nodes;
    std::vector<uint32_t> tri_order;
    std::vector<Aabb<R>> tri_aabbs;
    Aabb<R> local_bounds;

    V3<R> tri_vertex(uint32_t t, int k) const { return vertices[indices[t][k]]; }
    V3<R> center(uint32_t t) const {  // bvh.rs:248-251
        return (tri_vertex(t, 0) + tri_vertex(t, 1) + tri_vertex(t, 2)) * (R(1) / R(3));
    }
    // bvh.rs:210-225
    Aabb<R> slice_aabb(uint32_t start, uint32_t count) const {
        bool have = false;
        Aabb<R> a{V3<R>(), V3<R>()};
        for (uint32_t k = start; k < start + count; ++k)
            for (int v = 0; v < 3; ++v) {
                V3<R> p = tri_vertex(tri_order[k], v);
                if (!have) { a = Aabb<R>(p, p); have = true; }
                else a = Aabb<R>(a.min.min(p), a.max.max(p));
            }
        return a;
    }
    // bvh.rs:171-203
    uint32_t build_node(uint32_t start, uint32_t count) {
        Aabb<R> aabb = slice_aabb(start, count);
        uint32_t index = uint32_t(nodes.size());
        Node nd;
        nd.aabb = aabb;
        nd.leaf = true;
        nd.a = start;
        nd.b = count;
        nodes.push_back(nd);
        if (count <= 4) return index;
        V3<R> e = aabb.extents();  // bvh.rs:255-268 longest_axis: first strict maximum
        int axis = 0;
        R mx = e.x;
        if (e.y > mx) { axis = 1; mx = e.y; }
        if (e.z > mx) axis = 2;
        auto comp = [&](uint32_t t) { V3<R> c = center(t); return axis == 0 ? c.x : (axis == 1 ? c.y : c.z); };
        std::stable_sort(tri_order.begin() + start, tri_order.begin() + start + count,
                         [&](uint32_t x, uint32_t y) { return comp(x) < comp(y); });
        uint32_t mid = count / 2;
        uint32_t left = build_node(start, mid);
        uint32_t right = build_node(start + mid, count - mid);
        nodes[index].leaf = false;
        nodes[index].a = left;
        nodes[index].b = right;
        return index;
    }
    void build() {
        tri_order.resize(indices.size());
        for (uint32_t t = 0; t < tri_order.size(); ++t) tri_order[t] = t;
        nodes.clear();
        build_node(0, uint32_t(indices.size()));
        tri_aabbs.clear();
        for (uint32_t t = 0; t < indices.size(); ++t) {  // triangle_mesh.rs:98-112
            V3<R> a = tri_vertex(t, 0), b = tri_vertex(t, 1), c = tri_vertex(t, 2);
            tri_aabbs.push_back(Aabb<R>(a.min(b.min(c)), a.max(b.max(c))));
            local_bounds = t == 0 ? tri_aabbs[0] : Aabb<R>(local_bounds.min.min(tri_aabbs[t].min),
                                                           local_bounds.max.max(tri_aabbs[t].max));
        }
        if (indices.empty()) local_bounds = Aabb<R>(V3<R>(), V3<R>());
    }
    // bvh.rs:45-66: stack walk (left pushed first, so the right child pops first).
    void triangles_in_aabb(const Aabb<R>& q, std::vector<uint32_t>& out) const {
        out.clear();
        if (nodes.empty()) return;
        std::vector<uint32_t> stack{0u};
        while (!stack.empty()) {
            uint32_t k = stack.back();
            stack.pop_back();
            const Node& n = nodes[k];
            if (!n.aabb.overlaps(q)) continue;
            if (!n.leaf) {
                stack.push_back(n.a);
                stack.push_back(n.b);
            } else {
                for (uint32_t i = n.a; i < n.a + n.b; ++i) out.push_back(tri_order[i]);
            }
        }
    }
};

// manifold.rs:8
template <class R> constexpr R CONTACT_BREAKING_THRESHOLD = R(0.02);

template <class R>
struct Shape {
    ShapeType type = SHAPE_SPHERE;
    V3<R> half;            // box half extents
    R radius = 0;          // sphere / capsule
    R half_height = 0;     // capsule (segment along local Y)
    V3<R> normal;          // plane
    R constant = 0;        // plane
    std::vector<V3<R>> points;  // hull
    Aabb<R> hull_bounds;        // convex_hull.rs:22-34
    std::shared_ptr<MeshData<R>> mesh;            // triangle mesh / heightfield (static only)
    std::shared_ptr<std::vector<Shape>> tri_hulls;  // triangle_mesh.rs:94-104: 3-vertex hulls

    static Shape sphere(R r) { Shape s; s.type = SHAPE_SPHERE; s.radius = r; return s; }
    static Shape box(const V3<R>& h) { Shape s; s.type = SHAPE_BOX; s.half = h; return s; }
    static Shape capsule(R r, R hh) { Shape s; s.type = SHAPE_CAPSULE; s.radius = r; s.half_height = hh; return s; }
    // plane.rs:17-23 — the normal is normalized on construction.
    static Shape plane(const V3<R>& n, R c) { Shape s; s.type = SHAPE_PLANE; s.normal = n.normalize(); s.constant = c; return s; }
    static Shape hull(const std::vector<V3<R>>& pts) {
        Shape s; s.type = SHAPE_HULL; s.points = pts;
        V3<R> mn = V3<R>::splat(std::numeric_limits<R>::infinity());
        V3<R> mx = V3<R>::splat(-std::numeric_limits<R>::infinity());
        for (auto& p : pts) { mn = mn.min(p); mx = mx.max(p); }
        if (pts.empty()) { mn = V3<R>(); mx = V3<R>(); }
        s.hull_bounds = Aabb<R>(mn, mx);
        return s;
    }

    // triangle_mesh.rs:85-123 (one part): vertices, triangles, BVH, per-triangle hulls and boxes.
    static Shape triangle_mesh(const std::vector<V3<R>>& v, const std::vector<std::array<uint32_t, 3>>& idx) {
        Shape s;
        s.type = SHAPE_MESH;
        s.mesh = std::make_shared<MeshData<R>>();
        s.mesh->vertices = v;
        s.mesh->indices = idx;
        s.mesh->build();
        s.tri_hulls = std::make_shared<std::vector<Shape>>();
        for (uint32_t t = 0; t < idx.size(); ++t)
            s.tri_hulls->push_back(hull({s.mesh->tri_vertex(t, 0), s.mesh->tri_vertex(t, 1), s.mesh->tri_vertex(t, 2)}));
        return s;
    }
    // heightfield.rs:84-140: a width x depth row-major grid centred on the origin, heights
    // offset by the min/max midpoint, two triangles per cell. options: bit 0 flip quad edges,
    // bit 1 diamond subdivision, bit 2 zigzag subdivision, bit 3 flip winding; up axis in bits 4-5
    // (0 Y, the default; 1 X; 2 Z).
    static Shape heightfield(const std::vector<R>& h, uint32_t width, uint32_t depth, const V3<R>& cell,
                             uint32_t options) {
        R mn = std::numeric_limits<R>::infinity(), mx = -std::numeric_limits<R>::infinity();
        for (R x : h) { mn = std::min(mn, x); mx = std::max(mx, x); }
        R mid = (mn + mx) * R(0.5);
        const uint32_t up = (options >> 4) & 3u;
        std::vector<V3<R>> v;
        for (uint32_t y = 0; y < depth; ++y)
            for (uint32_t x = 0; x < width; ++x) {
                R hh = h[size_t(y) * width + x] - mid;
                R u = (R(x) - R(width - 1) * R(0.5)) * cell.x;
                R w = (R(y) - R(depth - 1) * R(0.5)) * cell.z;
                v.push_back(up == 1 ? V3<R>(hh, u, w) : (up == 2 ? V3<R>(u, w, hh) : V3<R>(u, hh, w)));
            }
        const bool flip_edges = options & 1u, diamond = options & 2u, zigzag = options & 4u, flip_wind = options & 8u;
        auto wind = [&](std::array<uint32_t, 3> t) {
            return flip_wind ? std::array<uint32_t, 3>{t[2], t[1], t[0]} : t;
        };
        std::vector<std::array<uint32_t, 3>> idx;
        for (uint32_t y = 0; y + 1 < depth; ++y)
            for (uint32_t x = 0; x + 1 < width; ++x) {
                uint32_t v00 = y * width + x, v10 = v00 + 1, v01 = v00 + width, v11 = v01 + 1;
                bool flipped = flip_edges || (diamond && ((y + x) & 1u) == 0) || (zigzag && (y & 1u) == 0);
                if (flipped) {
                    idx.push_back(wind({v00, v01, v11}));
                    idx.push_back(wind({v00, v11, v10}));
                } else {
                    idx.push_back(wind({v00, v01, v10}));
                    idx.push_back(wind({v10, v01, v11}));
                }
            }
        return triangle_mesh(v, idx);
    }

    bool is_convex() const { return type != SHAPE_PLANE && type != SHAPE_MESH; }

    // shapes/mod.rs:236-251; box_shape.rs:20-22 (0.04); sphere.rs:18-20 (r);
    // capsule.rs:27-29 (r); convex_hull.rs:43-45 (0); plane.rs:26-28 (0).
    R margin() const {
        switch (type) {
            case SHAPE_SPHERE: return radius;
            case SHAPE_BOX: return R(0.04);
            case SHAPE_CAPSULE: return radius;
            default: return R(0);
        }
    }

    // shapes/mod.rs:255-271 and the per-shape local_aabb.
    Aabb<R> local_aabb() const {
        switch (type) {
            case SHAPE_SPHERE: return Aabb<R>(V3<R>::splat(-radius), V3<R>::splat(radius));
            case SHAPE_BOX: return Aabb<R>(-half, half);
            case SHAPE_CAPSULE: {
                V3<R> r(radius, half_height + radius, radius);
                return Aabb<R>(-r, r);
            }
            case SHAPE_HULL: return hull_bounds;
            case SHAPE_MESH: return mesh->local_bounds;  // triangle_mesh.rs:209-211
            default: return Aabb<R>(V3<R>::splat(R(-1e30)), V3<R>::splat(R(1e30)));
        }
    }

    // shapes/mod.rs:275-291
    V3<R> support_local(const V3<R>& d) const {
        switch (type) {
            case SHAPE_SPHERE: {  // sphere.rs:35-42
                R len = d.length();
                if (len > R(0)) return d / len * radius;
                return V3<R>(radius, 0, 0);
            }
            case SHAPE_BOX:  // box_shape.rs:30-37
                return V3<R>(d.x >= R(0) ? half.x : -half.x, d.y >= R(0) ? half.y : -half.y,
                             d.z >= R(0) ? half.z : -half.z);
            case SHAPE_CAPSULE: {  // capsule.rs:38-54
                R len = d.length();
                if (len > R(0)) {
                    V3<R> tip(0, d.y >= R(0) ? half_height : -half_height, 0);
                    return tip + d / len * radius;
                }
                return V3<R>(radius, half_height, 0);
            }
            case SHAPE_HULL: {  // convex_hull.rs:55-66 (first strict maximum)
                V3<R> best;
                R best_dot = -std::numeric_limits<R>::infinity();
                for (auto& p : points) {
                    R dd = p.dot(d);
                    if (dd > best_dot) { best_dot = dd; best = p; }
                }
                return best;
            }
            default: return V3<R>();
        }
    }

    // shapes/mod.rs:305-319
    V3<R> core_support_local(const V3<R>& d) const {
        switch (type) {
            case SHAPE_SPHERE: return V3<R>();  // sphere.rs:24-26
            case SHAPE_BOX: {                  // box_shape.rs:42-53
                V3<R> h(std::max(half.x - margin(), R(0)), std::max(half.y - margin(), R(0)),
                        std::max(half.z - margin(), R(0)));
                return V3<R>(d.x >= R(0) ? h.x : -h.x, d.y >= R(0) ? h.y : -h.y, d.z >= R(0) ? h.z : -h.z);
            }
            case SHAPE_CAPSULE:  // capsule.rs:59-69
                return V3<R>(0, d.y >= R(0) ? half_height : -half_height, 0);
            default: return support_local(d);
        }
    }

    // shapes/mod.rs:323-332
    V3<R> support_world(const V3<R>& p, const Quat<R>& q, const V3<R>& dir) const {
        V3<R> ld = q.inverse().rotate(dir);
        return q.rotate(support_local(ld)) + p;
    }
    // shapes/mod.rs:337-346
    V3<R> core_support_world(const V3<R>& p, const Quat<R>& q, const V3<R>& dir) const {
        V3<R> ld = q.inverse().rotate(dir);
        return q.rotate(core_support_local(ld)) + p;
    }

    // shapes/mod.rs:350-375
    Aabb<R> world_aabb(const V3<R>& p, const Quat<R>& q) const {
        switch (type) {
            case SHAPE_SPHERE:  // sphere.rs:45-48
                return Aabb<R>(p - V3<R>::splat(radius), p + V3<R>::splat(radius));
            case SHAPE_BOX: {  // box_shape.rs:57-72
                V3<R> mn = V3<R>::splat(std::numeric_limits<R>::infinity());
                V3<R> mx = V3<R>::splat(-std::numeric_limits<R>::infinity());
                for (int i = 0; i < 8; ++i) {
                    V3<R> c((i & 1) == 0 ? half.x : -half.x, (i & 2) == 0 ? half.y : -half.y,
                            (i & 4) == 0 ? half.z : -half.z);
                    V3<R> w = q.rotate(c) + p;
                    mn = mn.min(w);
                    mx = mx.max(w);
                }
                return Aabb<R>(mn, mx);
            }
            case SHAPE_CAPSULE: {  // capsule.rs:74-79
                V3<R> top = q.rotate(V3<R>(0, half_height, 0)) + p;
                V3<R> bot = q.rotate(V3<R>(0, -half_height, 0)) + p;
                V3<R> r = V3<R>::splat(radius);
                return Aabb<R>(top.min(bot) - r, top.max(bot) + r);
            }
            case SHAPE_HULL: {  // convex_hull.rs:70-72 + shapes/mod.rs:448-469
                Quat<R> qi = q.inverse();
                V3<R> ux = qi.rotate(V3<R>(1, 0, 0)), uy = qi.rotate(V3<R>(0, 1, 0)),
                      uz = qi.rotate(V3<R>(0, 0, 1));
                V3<R> mn(p.x + support_local(-ux).dot(ux), p.y + support_local(-uy).dot(uy),
                         p.z + support_local(-uz).dot(uz));
                V3<R> mx(p.x + support_local(ux).dot(ux), p.y + support_local(uy).dot(uy),
                         p.z + support_local(uz).dot(uz));
                return Aabb<R>(mn, mx);
            }
            case SHAPE_MESH: return aabb_transformed(mesh->local_bounds, p, q);  // triangle_mesh.rs:213-216
            default: return local_aabb();  // plane.rs:38-40
        }
    }

    // shapes/mod.rs:388-392
    R contact_breaking_threshold() const {
        Aabb<R> a = local_aabb();
        R disc = (a.max - a.min).length() * R(0.5) + a.center().length();
        return disc * CONTACT_BREAKING_THRESHOLD<R>;
    }

    // shapes/mod.rs:396-412
    V3<R> local_inertia(R mass) const {
        switch (type) {
            case SHAPE_SPHERE: return V3<R>::splat(R(0.4) * mass * radius * radius);  // sphere.rs:52-54
            case SHAPE_BOX: {  // box_shape.rs:76-84
                R m = mass / R(3);
                return V3<R>(m * (half.y * half.y + half.z * half.z), m * (half.x * half.x + half.z * half.z),
                             m * (half.x * half.x + half.y * half.y));
            }
            case SHAPE_CAPSULE: {  // capsule.rs:84-98
                const R PI = R(3.14159265358979323846);
                R h = R(2) * half_height;
                R r2 = radius * radius;
                R h2 = h * h;
                R v_cyl = PI * r2 * h;
                R v_sph = R(4) / R(3) * PI * r2 * radius;
                R v = v_cyl + v_sph;
                R m_cyl = mass * v_cyl / v;
                R m_sph = mass * v_sph / v;
                R ixx = m_cyl * (R(3) * r2 + h2) / R(12) + m_sph * (R(0.4) * r2 + R(0.25) * h2);
                R iyy = m_cyl * r2 / R(2) + m_sph * R(0.4) * r2;
                return V3<R>(ixx, iyy, ixx);
            }
            case SHAPE_HULL: {  // convex_hull.rs:78-86
                V3<R> h = hull_bounds.extents();
                R m = mass / R(3);
                return V3<R>(m * (h.y * h.y + h.z * h.z), m * (h.x * h.x + h.z * h.z), m * (h.x * h.x + h.y * h.y));
            }
            default: return V3<R>();
        }
    }
};

}  // namespace oracle
