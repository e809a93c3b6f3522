// CPU oracle — TEST INFRASTRUCTURE ONLY: the CCD swept-sphere clamp.
//
// Restates:
//   crates/bullet-collision/src/narrowphase/convex_sweep.rs:37-59 (swept_sphere_cast),
//     :72-103 (point_convex_distance, GJK distance from a point), :107-125 (sweep_convex),
//     :155-214 (sweep_with_dist: ternary search for the closest approach, then bisection for
//     the first fraction inside the inflated target), :263-295 (sweep_plane), :355-357;
//   crates/bullet-collision/src/narrowphase/gjk.rs:864-1044 (closest_origin on a point,
//     segment, triangle or tetrahedron simplex, keeping the closest feature);
//   crates/bullet-dynamics/src/world/step.rs:1068-1155 (the per-body clamp fraction) and
//     :1210-1214 (the clamp applied after the position integration).
// Triangle meshes and heightfields are not shapes of this build, so sweep_mesh has no
// counterpart here.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>
#include "oracle_math.hpp"
#include "oracle_shapes.hpp"

namespace oracle {

template <class R>
struct SweepHit {
    R fraction = 1;
    V3<R> normal, point;
};

// gjk.rs:889-906
template <class R>
V3<R> closest_origin_segment(const V3<R>& a, const V3<R>& b, std::vector<V3<R>>& keep) {
    V3<R> ab = b - a;
    if (ab.length_squared() == R(0)) { keep = {a}; return a; }
    R t = -a.dot(ab) / ab.length_squared();
    if (t <= R(0)) { keep = {a}; return a; }
    if (t >= R(1)) { keep = {b}; return b; }
    keep = {b, a};
    return a + ab * t;
}

// gjk.rs:911-989
template <class R>
V3<R> closest_origin_triangle(const V3<R>& a, const V3<R>& b, const V3<R>& c, std::vector<V3<R>>& keep) {
    V3<R> ab = b - a, ac = c - a, ap = -a;
    R d1 = ab.dot(ap), d2 = ac.dot(ap);
    if (d1 <= R(0) && d2 <= R(0)) { keep = {a}; return a; }
    V3<R> bp = -b;
    R d3 = ab.dot(bp), d4 = ac.dot(bp);
    if (d3 >= R(0) && d4 <= d3) { keep = {b}; return b; }
    R vc = d1 * d4 - d3 * d2;
    if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
        if (d1 == d3) { keep = {a}; return a; }
        R v = d1 / (d1 - d3);
        keep = {b, a};
        return a + ab * v;
    }
    V3<R> cp = -c;
    R d5 = ab.dot(cp), d6 = ac.dot(cp);
    if (d6 >= R(0) && d5 <= d6) { keep = {c}; return c; }
    R vb = d5 * d2 - d1 * d6;
    if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
        if (d2 == d6) { keep = {a}; return a; }
        R w = d2 / (d2 - d6);
        keep = {c, a};
        return a + ac * w;
    }
    R va = d3 * d6 - d5 * d4;
    if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
        if ((d4 - d3) + (d5 - d6) == R(0)) { keep = {b}; return b; }
        R w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        keep = {c, b};
        return b + (c - b) * w;
    }
    R sum = va + vb + vc;
    if (sum <= R(0) || std::isnan(sum)) {
        std::vector<V3<R>> kab, kbc, kca;
        V3<R> qab = closest_origin_segment(a, b, kab);
        V3<R> qbc = closest_origin_segment(b, c, kbc);
        V3<R> qca = closest_origin_segment(c, a, kca);
        if (qab.length_squared() <= qbc.length_squared() && qab.length_squared() <= qca.length_squared()) {
            keep = kab;
            return qab;
        }
        if (qbc.length_squared() <= qca.length_squared()) { keep = kbc; return qbc; }
        keep = kca;
        return qca;
    }
    R denom = R(1) / sum;
    R v = vb * denom, w = vc * denom;
    keep = {c, b, a};
    return a + ab * v + ac * w;
}

// gjk.rs:994-1044
template <class R>
V3<R> closest_origin_tetrahedron(const V3<R>& a, const V3<R>& b, const V3<R>& c, const V3<R>& d,
                                 std::vector<V3<R>>& keep) {
    V3<R> ao = -a, ab = b - a, ac = c - a, ad = d - a;
    if (std::fabs(ab.cross(ac).dot(ad)) < R(1e-12)) {
        // coplanar: the closest of the four faces (the first of equal ones, like min_by)
        const V3<R> f[4][3] = {{a, b, c}, {a, b, d}, {a, c, d}, {b, c, d}};
        V3<R> best;
        std::vector<V3<R>> best_keep;
        for (int k = 0; k < 4; ++k) {
            std::vector<V3<R>> kk;
            V3<R> q = closest_origin_triangle(f[k][0], f[k][1], f[k][2], kk);
            if (k == 0 || q.length_squared() < best.length_squared()) { best = q; best_keep = kk; }
        }
        keep = best_keep;
        return best;
    }
    V3<R> abc = ab.cross(ac), acd = ac.cross(ad), adb = ad.cross(ab);
    V3<R> bo = -b;
    V3<R> bcd = (c - b).cross(d - b);
    if (abc.dot(ao) * abc.dot(ad) < R(0)) return closest_origin_triangle(a, b, c, keep);
    if (acd.dot(ao) * acd.dot(ab) < R(0)) return closest_origin_triangle(a, c, d, keep);
    if (adb.dot(ao) * adb.dot(ac) < R(0)) return closest_origin_triangle(a, d, b, keep);
    if (bcd.dot(bo) * bcd.dot(a - b) < R(0)) return closest_origin_triangle(b, c, d, keep);
    keep = {a, b, c, d};
    return V3<R>();
}

// gjk.rs:864-885
template <class R>
V3<R> closest_origin(std::vector<V3<R>>& s) {
    std::vector<V3<R>> keep;
    V3<R> v;
    switch (s.size()) {
        case 0: return V3<R>();
        case 1: return s[0];
        case 2: v = closest_origin_segment(s[0], s[1], keep); break;
        case 3: v = closest_origin_triangle(s[0], s[1], s[2], keep); break;
        default: v = closest_origin_tetrahedron(s[0], s[1], s[2], s[3], keep); break;
    }
    s = keep;
    return v;
}

// convex_sweep.rs:72-103: squared distance from `point` to the support-mapped shape and the unit
// direction from the shape toward the point (zero when inside or touching).
template <class R, class F>
void point_convex_distance(const F& support, const V3<R>& point, R& d2, V3<R>& dir) {
    auto mink = [&](const V3<R>& v) { return point - support(-v); };
    V3<R> v = point;
    if (v.length_squared() < R(1e-12)) v = V3<R>(1, 0, 0);
    std::vector<V3<R>> simplex{mink(v)};
    v = simplex[0];
    for (int it = 0; it < 64; ++it) {
        if (v.length_squared() < R(1e-10)) { d2 = 0; dir = V3<R>(); return; }
        V3<R> w = mink(-v);
        for (const V3<R>& p : simplex)
            if ((p - w).length_squared() < R(1e-12)) { d2 = v.length_squared(); dir = v / v.length(); return; }
        simplex.push_back(w);
        v = closest_origin(simplex);
    }
    if (v.length_squared() < R(1e-10)) { d2 = 0; dir = V3<R>(); return; }
    d2 = v.length_squared();
    dir = v / v.length();
}

// convex_sweep.rs:155-214
template <class R, class F>
bool sweep_with_dist(const V3<R>& from, const V3<R>& dir, R length, R radius, const F& dist, SweepHit<R>& hit) {
    auto dist2 = [&](const V3<R>& p) { R d2; V3<R> v; dist(p, d2, v); return d2; };
    R lo = 0, hi = 1;
    for (int it = 0; it < 40; ++it) {
        R m1 = lo + (hi - lo) / R(3);
        R m2 = hi - (hi - lo) / R(3);
        if (dist2(from + dir * (m1 * length)) < dist2(from + dir * (m2 * length))) hi = m2;
        else lo = m1;
    }
    R s_min = (lo + hi) * R(0.5);
    R d_min2 = dist2(from + dir * (s_min * length));
    if (d_min2 > R(1e-8)) return false;
    R low = 0, high = s_min;
    for (int it = 0; it < 60; ++it) {
        R mid = (low + high) * R(0.5);
        if (dist2(from + dir * (mid * length)) <= R(1e-8)) high = mid;
        else low = mid;
    }
    R fraction = (low + high) * R(0.5);
    V3<R> probe = from + dir * std::max((fraction - R(2e-4)) * length, R(0));
    R d2;
    V3<R> v;
    dist(probe, d2, v);
    V3<R> normal = v.length_squared() > R(1e-12) ? v / v.length() : -dir;
    V3<R> entry = from + dir * (fraction * length);
    hit.fraction = fraction;
    hit.normal = normal;
    hit.point = entry - normal * radius;
    return true;
}

// convex_sweep.rs:263-295 (plane: normal n in the body frame, constant c)
template <class R>
bool sweep_plane(const V3<R>& from, const V3<R>& dir, R length, R radius, const V3<R>& normal, R constant,
                 const Quat<R>& ori, SweepHit<R>& hit) {
    V3<R> n = ori.rotate(normal);
    R dn0 = n.dot(from) - constant;
    if (std::fabs(dn0) <= radius) {
        hit.fraction = 0;
        hit.normal = dn0 >= R(0) ? n : -n;
        hit.point = from - n * dn0;
        return true;
    }
    R dd = n.dot(dir * length);
    if (dd >= R(0)) return false;
    R sign = dn0 > R(0) ? R(1) : R(-1);
    R fraction = (sign * radius - dn0) / dd;
    if (!(fraction >= R(0) && fraction <= R(1))) return false;
    V3<R> nn = sign > R(0) ? n : -n;
    V3<R> entry = from + (dir * length) * fraction;
    hit.fraction = fraction;
    hit.normal = nn;
    hit.point = entry - nn * radius;
    return true;
}

// convex_sweep.rs:217-262 (point_triangle_distance): squared distance from `point` to the
// triangle and the vector from its closest point to `point`.
template <class R>
R point_triangle_distance(const V3<R>& point, const V3<R>& a, const V3<R>& b, const V3<R>& c, V3<R>& dv) {
    V3<R> ab = b - a, ac = c - a, ap = point - a;
    R d1 = ab.dot(ap), d2 = ac.dot(ap);
    if (d1 <= R(0) && d2 <= R(0)) { dv = point - a; return dv.length_squared(); }
    V3<R> bp = point - b;
    R d3 = ab.dot(bp), d4 = ac.dot(bp);
    if (d3 >= R(0) && d4 <= d3) { dv = point - b; return dv.length_squared(); }
    R vc = d1 * d4 - d3 * d2;
    if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
        R v = d1 / (d1 - d3);
        V3<R> q = a + ab * v;
        dv = point - q;
        return dv.length_squared();
    }
    V3<R> cp = point - c;
    R d5 = ab.dot(cp), d6 = ac.dot(cp);
    if (d6 >= R(0) && d5 <= d6) { dv = point - c; return dv.length_squared(); }
    R vb = d5 * d2 - d1 * d6;
    if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
        R w = d2 / (d2 - d6);
        V3<R> q = a + ac * w;
        dv = point - q;
        return dv.length_squared();
    }
    R va = d3 * d6 - d5 * d4;
    if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
        R w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        V3<R> q = b + (c - b) * w;
        dv = point - q;
        return dv.length_squared();
    }
    R denom = R(1) / (va + vb + vc);
    R v = vb * denom, w = vc * denom;
    V3<R> q = a + ab * v + ac * w;
    dv = point - q;
    return dv.length_squared();
}

// convex_sweep.rs:131-151 (sweep_triangle)
template <class R>
bool sweep_triangle(const V3<R>& from, const V3<R>& dir, R length, R radius, const V3<R>& a, const V3<R>& b,
                    const V3<R>& c, SweepHit<R>& hit) {
    auto dist = [&](const V3<R>& p, R& d2, V3<R>& v) {
        V3<R> dv;
        R q = point_triangle_distance(p, a, b, c, dv);
        if (q <= radius * radius) { d2 = 0; v = V3<R>(); return; }
        R d = std::sqrt(q);
        d2 = (d - radius) * (d - radius);
        v = dv / d;
    };
    return sweep_with_dist(from, dir, length, radius, dist, hit);
}

// convex_sweep.rs:305-345 (sweep_mesh): in the mesh frame, the BVH candidates of the swept box,
// the closest per-triangle hit.
template <class R>
bool sweep_mesh(const V3<R>& from, const V3<R>& to, R radius, const MeshData<R>& mesh, const V3<R>& pos,
                const Quat<R>& ori, SweepHit<R>& hit) {
    Quat<R> inv = ori.inverse();
    V3<R> lf = inv.rotate(from - pos), lt = inv.rotate(to - pos);
    V3<R> delta = lt - lf;
    R length = delta.length();
    if (length <= std::numeric_limits<R>::epsilon()) return false;
    V3<R> dir = delta / length;
    V3<R> rr = V3<R>::splat(radius);
    Aabb<R> box(lf.min(lt) - rr, lf.max(lt) + rr);
    std::vector<uint32_t> cand;
    mesh.triangles_in_aabb(box, cand);
    bool any = false;
    SweepHit<R> best;
    for (uint32_t t : cand) {
        SweepHit<R> h;
        if (sweep_triangle(lf, dir, length, radius, mesh.tri_vertex(t, 0), mesh.tri_vertex(t, 1), mesh.tri_vertex(t, 2), h) &&
            (!any || h.fraction < best.fraction)) {
            best = h;
            any = true;
        }
    }
    if (!any) return false;
    hit.fraction = best.fraction;
    hit.normal = ori.rotate(best.normal);
    hit.point = ori.rotate(best.point) + pos;
    return true;
}

// convex_sweep.rs:37-59 + :107-125: a sphere of `radius` cast from `from` to `to` against a shape
// at (pos, ori).
template <class R, class S>
bool swept_sphere_cast(const V3<R>& from, const V3<R>& to, R radius, const S& shape, const V3<R>& pos,
                       const Quat<R>& ori, SweepHit<R>& hit) {
    V3<R> delta = to - from;
    R length = delta.length();
    if (length <= std::numeric_limits<R>::epsilon()) return false;
    V3<R> dir = delta / length;
    if (shape.type == SHAPE_MESH) return sweep_mesh(from, to, radius, *shape.mesh, pos, ori, hit);
    if (!shape.is_convex()) return sweep_plane(from, dir, length, radius, shape.normal, shape.constant, ori, hit);
    auto support = [&](const V3<R>& d) {
        V3<R> sphere = d.length_squared() > R(1e-12) ? d / d.length() * radius : V3<R>();
        return shape.support_world(pos, ori, d) + sphere;
    };
    auto dist = [&](const V3<R>& p, R& d2, V3<R>& v) { point_convex_distance<R>(support, p, d2, v); };
    return sweep_with_dist(from, dir, length, radius, dist, hit);
}

}  // namespace oracle
