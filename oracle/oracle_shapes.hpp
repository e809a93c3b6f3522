// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_math.hpp).
// Shapes restated from crates/bullet-collision/src/shapes/{mod,box_shape,
// sphere,capsule,convex_hull,plane}.rs.
#pragma once
#include "oracle_math.hpp"

namespace oracle {

enum ShapeType : uint32_t { SHAPE_SPHERE = 0, SHAPE_BOX = 1, SHAPE_CAPSULE = 2, SHAPE_HULL = 3, SHAPE_PLANE = 4 };

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

    bool is_convex() const { return type != SHAPE_PLANE; }

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
