// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_math.hpp).
// Narrowphase restated from crates/bullet-collision/src/narrowphase/
// {mod,sphere,plane,box_box,gjk,epa,convex_convex}.rs.
#pragma once
#include "oracle_shapes.hpp"

namespace oracle {

// manifold.rs:12-41
template <class R>
struct ContactPoint {
    V3<R> position, normal;
    R penetration = 0;
    R normal_impulse = 0;
    R tangent_impulse[2] = {0, 0};
    uint32_t lifetime = 0;
    ContactPoint() = default;
    ContactPoint(const V3<R>& p, const V3<R>& n, R pen) : position(p), normal(n), penetration(pen) {}
};

template <class R>
struct Manifold {
    std::vector<ContactPoint<R>> points;
    // manifold.rs:68-73
    void flip() { for (auto& p : points) p.normal = -p.normal; }
};

// narrowphase/mod.rs:53-57
template <class R>
inline R pair_threshold(const Shape<R>& a, const Shape<R>& b) {
    return std::min(a.contact_breaking_threshold(), b.contact_breaking_threshold());
}

// sphere.rs:10-32 — no margin band.
template <class R>
bool sphere_sphere(const Shape<R>& sa, const V3<R>& pa, const Shape<R>& sb, const V3<R>& pb, Manifold<R>& out) {
    V3<R> delta = pb - pa;
    R dist_sq = delta.length_squared();
    R rs = sa.radius + sb.radius;
    if (dist_sq >= rs * rs) return false;
    R dist = std::sqrt(dist_sq);
    V3<R> n = dist > R(1e-12) ? delta / dist : V3<R>(0, 1, 0);
    R pen = rs - dist;
    V3<R> pos = pa + n * (sa.radius - pen * R(0.5));
    out.points.push_back(ContactPoint<R>(pos, n, pen));
    return true;
}

template <class R> inline R signum(R v) { return std::signbit(v) ? R(-1) : R(1); }

// sphere.rs:38-82 — normal points from the box to the sphere.
template <class R>
bool sphere_box(const Shape<R>& s, const V3<R>& ps, const Shape<R>& b, const V3<R>& pb, const Quat<R>& ob,
                R threshold, Manifold<R>& out) {
    V3<R> local = ob.inverse().rotate(ps - pb);
    V3<R> h = b.half;
    V3<R> cl(std::min(std::max(local.x, -h.x), h.x), std::min(std::max(local.y, -h.y), h.y),
             std::min(std::max(local.z, -h.z), h.z));
    V3<R> delta = local - cl;
    R dist_sq = delta.length_squared();
    R cd = s.radius + threshold;
    if (dist_sq >= cd * cd) return false;
    R dist = std::sqrt(dist_sq);
    V3<R> nl;
    R pen;
    if (dist > R(1e-12)) {
        nl = delta / dist;
        pen = s.radius - dist;
    } else {
        R dx = h.x - std::fabs(local.x), dy = h.y - std::fabs(local.y), dz = h.z - std::fabs(local.z);
        R d;
        if (dx <= dy && dx <= dz) { nl = V3<R>(signum(local.x), 0, 0); d = dx; }
        else if (dy <= dz) { nl = V3<R>(0, signum(local.y), 0); d = dy; }
        else { nl = V3<R>(0, 0, signum(local.z)); d = dz; }
        pen = s.radius + d;
    }
    out.points.push_back(ContactPoint<R>(ob.rotate(cl) + pb, ob.rotate(nl), pen));
    return true;
}

// plane.rs:19-56 — one deepest point, band contacts (negative penetration).
template <class R>
bool plane_convex(const Shape<R>& plane, const V3<R>& pp, const Quat<R>& qp, const Shape<R>& cvx, const V3<R>& pc,
                  const Quat<R>& qc, R threshold, Manifold<R>& out) {
    V3<R> n = qp.rotate(plane.normal);
    R c = plane.constant + n.dot(pp);
    V3<R> normal = n.dot(pc - pp) >= R(0) ? n : -n;
    if (!(normal.x == n.x && normal.y == n.y && normal.z == n.z)) c = -c;
    V3<R> deepest = cvx.support_world(pc, qc, -normal);
    R depth = c - normal.dot(deepest);
    if (depth < -threshold) return false;
    out.points.push_back(ContactPoint<R>(deepest, normal, depth));
    return true;
}

// ---------------------------------------------------------------- box-box
// box_box.rs:31-48
template <class R>
inline void line_closest_approach(const V3<R>& pa, const V3<R>& ua, const V3<R>& pb, const V3<R>& ub, R& alpha, R& beta) {
    V3<R> p = pb - pa;
    R uaub = ua.dot(ub);
    R q1 = ua.dot(p);
    R q2 = -ub.dot(p);
    R d = R(1) - uaub * uaub;
    if (d <= R(1e-4)) { alpha = 0; beta = 0; return; }
    d = R(1) / d;
    alpha = (q1 + uaub * q2) * d;
    beta = (uaub * q1 + q2) * d;
}

template <class R>
struct ClipPoly { R pts[8][2]; int len = 0; };

// box_box.rs:92-111
template <class R>
inline void clip_poly(const ClipPoly<R>& src, int axis, R sign, R h, ClipPoly<R>& out) {
    int n = src.len;
    out.len = 0;
    for (int i = 0; i < n; ++i) {
        const R* cur = src.pts[i];
        const R* nxt = src.pts[(i + 1) % n];
        bool cin = sign * cur[axis] < h;
        bool nin = sign * nxt[axis] < h;
        if (cin) { out.pts[out.len][0] = cur[0]; out.pts[out.len][1] = cur[1]; out.len++; }
        if (cin != nin) {
            R t = (sign * h - cur[axis]) / (nxt[axis] - cur[axis]);
            R p[2];
            p[axis] = sign * h;
            p[1 - axis] = cur[1 - axis] + (nxt[1 - axis] - cur[1 - axis]) * t;
            out.pts[out.len][0] = p[0]; out.pts[out.len][1] = p[1]; out.len++;
        }
    }
}

// box_box.rs:116-124
template <class R>
inline ClipPoly<R> intersect_rect_quad(const R h[2], const R quad[4][2]) {
    ClipPoly<R> buf, tmp;
    for (int i = 0; i < 4; ++i) { buf.pts[i][0] = quad[i][0]; buf.pts[i][1] = quad[i][1]; }
    buf.len = 4;
    clip_poly(buf, 0, R(-1), h[0], tmp);
    clip_poly(tmp, 0, R(1), h[0], buf);
    clip_poly(buf, 1, R(-1), h[1], tmp);
    clip_poly(tmp, 1, R(1), h[1], buf);
    return buf;
}

// box_box.rs:131-174 — deepest (last max) + farthest, stable descending sort.
template <class R>
inline int cull_points(const V3<R>* pts, const R* deps, int n, int maxc, V3<R>* opts, R* odeps) {
    if (n <= maxc) {
        for (int i = 0; i < n; ++i) { opts[i] = pts[i]; odeps[i] = deps[i]; }
        return n;
    }
    int i0 = 0;
    R dd = deps[0];
    for (int i = 1; i < n; ++i) if (deps[i] >= dd) { i0 = i; dd = deps[i]; }
    int ri[8]; R rd[8]; int rn = 0;
    for (int i = 0; i < n; ++i) if (i != i0) { ri[rn] = i; rd[rn] = (pts[i] - pts[i0]).length_squared(); rn++; }
    for (int j = 1; j < rn; ++j) {
        int ki = ri[j]; R kd = rd[j]; int k = j;
        while (k > 0 && rd[k - 1] < kd) { ri[k] = ri[k - 1]; rd[k] = rd[k - 1]; --k; }
        ri[k] = ki; rd[k] = kd;
    }
    opts[0] = pts[i0]; odeps[0] = deps[i0];
    int m = 1;
    for (int t = 0; t < maxc - 1 && t < rn; ++t) { opts[m] = pts[ri[t]]; odeps[m] = deps[ri[t]]; ++m; }
    return m;
}

// box_box.rs:178-528 (ODE dBoxBox2 as adapted by the reference).
template <class R>
bool box_box(const Shape<R>& a, const V3<R>& pa, const Quat<R>& oa, const Shape<R>& b, const V3<R>& pb,
             const Quat<R>& ob, Manifold<R>& out) {
    const R EPSILON = R(1e-6), FUDGE = R(1.05);
    M3<R> r1 = M3<R>::from_quat(oa), r2 = M3<R>::from_quat(ob);
    V3<R> ha = a.half, hb = b.half;
    V3<R> p1 = pa, p2 = pb;
    V3<R> p = p2 - p1;
    V3<R> pp = r1.transpose() * p;
    M3<R> r = r1.transpose() * r2;
    R r11 = r.c0.x, r12 = r.c1.x, r13 = r.c2.x;
    R r21 = r.c0.y, r22 = r.c1.y, r23 = r.c2.y;
    R r31 = r.c0.z, r32 = r.c1.z, r33 = r.c2.z;
    R q11 = std::fabs(r11), q12 = std::fabs(r12), q13 = std::fabs(r13);
    R q21 = std::fabs(r21), q22 = std::fabs(r22), q23 = std::fabs(r23);
    R q31 = std::fabs(r31), q32 = std::fabs(r32), q33 = std::fabs(r33);

    R s = -std::numeric_limits<R>::infinity();
    bool invert_normal = false;
    int code = 0;
    bool from_r2 = false, is_cross = false;
    int normal_axis = 0;
    V3<R> normal_c;

    auto tst_face = [&](R e1, R e2, bool fr2, int ax, int cc) -> bool {
        R s2 = std::fabs(e1) - e2;
        if (s2 > R(0)) return false;
        if (s2 > s) { s = s2; is_cross = false; from_r2 = fr2; normal_axis = ax; invert_normal = e1 < R(0); code = cc; }
        return true;
    };
    auto tst_cross = [&](R e1, R e2, R n1, R n2, R n3, int cc) -> bool {
        R s2 = std::fabs(e1) - e2;
        if (s2 > EPSILON) return false;
        R l = std::sqrt(n1 * n1 + n2 * n2 + n3 * n3);
        if (l > EPSILON) {
            s2 = s2 / l;
            if (s2 * FUDGE > s) {
                s = s2; is_cross = true; normal_c = V3<R>(n1 / l, n2 / l, n3 / l); invert_normal = e1 < R(0); code = cc;
            }
        }
        return true;
    };

    if (!tst_face(pp.x, ha.x + hb.x * q11 + hb.y * q12 + hb.z * q13, false, 0, 1)) return false;
    if (!tst_face(pp.y, ha.y + hb.x * q21 + hb.y * q22 + hb.z * q23, false, 1, 2)) return false;
    if (!tst_face(pp.z, ha.z + hb.x * q31 + hb.y * q32 + hb.z * q33, false, 2, 3)) return false;
    if (!tst_face(r2.c0.dot(p), ha.x * q11 + ha.y * q21 + ha.z * q31 + hb.x, true, 0, 4)) return false;
    if (!tst_face(r2.c1.dot(p), ha.x * q12 + ha.y * q22 + ha.z * q32 + hb.y, true, 1, 5)) return false;
    if (!tst_face(r2.c2.dot(p), ha.x * q13 + ha.y * q23 + ha.z * q33 + hb.z, true, 2, 6)) return false;

    const R f2 = R(1e-5);
    q11 += f2; q12 += f2; q13 += f2; q21 += f2; q22 += f2; q23 += f2; q31 += f2; q32 += f2; q33 += f2;

    if (!tst_cross(pp.z * r21 - pp.y * r31, ha.y * q31 + ha.z * q21 + hb.y * q13 + hb.z * q12, R(0), -r31, r21, 7)) return false;
    if (!tst_cross(pp.z * r22 - pp.y * r32, ha.y * q32 + ha.z * q22 + hb.x * q13 + hb.z * q11, R(0), -r32, r22, 8)) return false;
    if (!tst_cross(pp.z * r23 - pp.y * r33, ha.y * q33 + ha.z * q23 + hb.x * q12 + hb.y * q11, R(0), -r33, r23, 9)) return false;
    if (!tst_cross(pp.x * r31 - pp.z * r11, ha.x * q31 + ha.z * q11 + hb.y * q23 + hb.z * q22, r31, R(0), -r11, 10)) return false;
    if (!tst_cross(pp.x * r32 - pp.z * r12, ha.x * q32 + ha.z * q12 + hb.x * q23 + hb.z * q21, r32, R(0), -r12, 11)) return false;
    if (!tst_cross(pp.x * r33 - pp.z * r13, ha.x * q33 + ha.z * q13 + hb.x * q22 + hb.y * q21, r33, R(0), -r13, 12)) return false;
    if (!tst_cross(pp.y * r11 - pp.x * r21, ha.x * q21 + ha.y * q11 + hb.y * q33 + hb.z * q32, -r21, r11, R(0), 13)) return false;
    if (!tst_cross(pp.y * r12 - pp.x * r22, ha.x * q22 + ha.y * q12 + hb.x * q33 + hb.z * q31, -r22, r12, R(0), 14)) return false;
    if (!tst_cross(pp.y * r13 - pp.x * r23, ha.x * q23 + ha.y * q13 + hb.x * q32 + hb.y * q31, -r23, r13, R(0), 15)) return false;

    V3<R> normal_sat = is_cross ? r1 * normal_c : (from_r2 ? r2.col(normal_axis) : r1.col(normal_axis));
    if (invert_normal) normal_sat = -normal_sat;
    R depth = -s;

    if (code > 6) {  // box_box.rs:402-423 edge-edge
        V3<R> qa = p1;
        for (int j = 0; j < 3; ++j) {
            V3<R> c = r1.col(j);
            R sign = normal_sat.dot(c) > R(0) ? R(1) : R(-1);
            qa += c * (sign * ha[j]);
        }
        V3<R> qb = p2;
        for (int j = 0; j < 3; ++j) {
            V3<R> c = r2.col(j);
            R sign = normal_sat.dot(c) > R(0) ? R(-1) : R(1);
            qb += c * (sign * hb[j]);
        }
        V3<R> ua = r1.col((code - 7) / 3), ub = r2.col((code - 7) % 3);
        R alpha, beta;
        line_closest_approach(qa, ua, qb, ub, alpha, beta);
        qb += ub * beta;
        out.points.push_back(ContactPoint<R>(qb, normal_sat, depth));
        return true;
    }

    // box_box.rs:426-527 face-face
    const M3<R>& ra = code <= 3 ? r1 : r2;
    const M3<R>& rb = code <= 3 ? r2 : r1;
    V3<R> pa_ref = code <= 3 ? p1 : p2;
    V3<R> pb_inc = code <= 3 ? p2 : p1;
    V3<R> sa = code <= 3 ? ha : hb;
    V3<R> sb = code <= 3 ? hb : ha;
    V3<R> normal2 = code <= 3 ? normal_sat : -normal_sat;
    V3<R> nr = rb.transpose() * normal2;
    V3<R> anr = nr.abs();
    int lanr, a1, a2;
    if (anr.y > anr.x) {
        if (anr.y > anr.z) { lanr = 1; a1 = 0; a2 = 2; } else { lanr = 2; a1 = 0; a2 = 1; }
    } else if (anr.x > anr.z) { lanr = 0; a1 = 1; a2 = 2; } else { lanr = 2; a1 = 0; a2 = 1; }

    V3<R> center = nr[lanr] < R(0) ? (pb_inc - pa_ref + rb.col(lanr) * sb[lanr])
                                     : (pb_inc - pa_ref - rb.col(lanr) * sb[lanr]);
    int code_n = code <= 3 ? code - 1 : code - 4;
    int code1, code2;
    if (code_n == 0) { code1 = 1; code2 = 2; } else if (code_n == 1) { code1 = 0; code2 = 2; } else { code1 = 0; code2 = 1; }

    R c1 = center.dot(ra.col(code1));
    R c2 = center.dot(ra.col(code2));
    R m11 = ra.col(code1).dot(rb.col(a1));
    R m12 = ra.col(code1).dot(rb.col(a2));
    R m21 = ra.col(code2).dot(rb.col(a1));
    R m22 = ra.col(code2).dot(rb.col(a2));
    R k1 = m11 * sb[a1], k2 = m21 * sb[a1], k3 = m12 * sb[a2], k4 = m22 * sb[a2];
    R quad[4][2] = {{c1 - k1 - k3, c2 - k2 - k4}, {c1 - k1 + k3, c2 - k2 + k4},
                    {c1 + k1 + k3, c2 + k2 + k4}, {c1 + k1 - k3, c2 + k2 - k4}};
    R rect[2] = {sa[code1], sa[code2]};
    ClipPoly<R> ret = intersect_rect_quad(rect, quad);
    if (ret.len == 0) return false;

    R det1 = R(1) / (m11 * m22 - m12 * m21);
    m11 *= det1; m12 *= det1; m21 *= det1; m22 *= det1;
    V3<R> pts[8]; R deps[8]; int np = 0;
    for (int i = 0; i < ret.len; ++i) {
        R rx = ret.pts[i][0], ry = ret.pts[i][1];
        R kk1 = m22 * (rx - c1) - m12 * (ry - c2);
        R kk2 = -m21 * (rx - c1) + m11 * (ry - c2);
        V3<R> point = center + rb.col(a1) * kk1 + rb.col(a2) * kk2;
        R dep = sa[code_n] - normal2.dot(point);
        if (dep >= R(0)) { pts[np] = point; deps[np] = dep; ++np; }
    }
    if (np == 0) return false;
    V3<R> cp[4]; R cd[4];
    int nc = cull_points(pts, deps, np, 4, cp, cd);
    for (int i = 0; i < nc; ++i) {
        V3<R> pos = cp[i] + pa_ref;
        if (code > 3) pos += normal_sat * cd[i];
        out.points.push_back(ContactPoint<R>(pos, normal_sat, cd[i]));
    }
    return true;
}

// ---------------------------------------------------------------- GJK
// gjk.rs:137-140
template <class R> struct SupportVertex { V3<R> w, p_b; };

template <class R>
struct GjkOutcome {
    int kind = 0;  // 0 separated, 1 band, 2 overlap
    R distance = 0;
    V3<R> normal, point_on_b;
    V3<R> simplex[4];
    int simplex_len = 0;
};

template <class R>
struct Closest { bool inside = false; V3<R> v, p_b; };

// gjk.rs:366-394
template <class R>
Closest<R> reduce_segment(SupportVertex<R>* buf, int& len) {
    SupportVertex<R> a = buf[1], b = buf[0];
    V3<R> ab = b.w - a.w;
    R denom = ab.length_squared();
    Closest<R> c;
    if (denom < R(1e-24)) { len = 1; buf[0] = a; c.v = a.w; c.p_b = a.p_b; return c; }
    R t = -a.w.dot(ab) / denom;
    if (t <= R(0)) { len = 1; buf[0] = a; c.v = a.w; c.p_b = a.p_b; }
    else if (t >= R(1)) { len = 1; buf[0] = b; c.v = b.w; c.p_b = b.p_b; }
    else { len = 2; buf[0] = a; buf[1] = b; c.v = a.w + ab * t; c.p_b = a.p_b + (b.p_b - a.p_b) * t; }
    return c;
}

// gjk.rs:399-477
template <class R>
V3<R> closest_triangle_bary(const SupportVertex<R>& a, const SupportVertex<R>& b, const SupportVertex<R>& c, R wts[3]) {
    V3<R> ab = b.w - a.w, ac = c.w - a.w, ap = -a.w;
    R d1 = ab.dot(ap), d2 = ac.dot(ap);
    if (d1 <= R(0) && d2 <= R(0)) { wts[0] = 1; wts[1] = 0; wts[2] = 0; return a.w; }
    V3<R> bp = -b.w;
    R d3 = ab.dot(bp), d4 = ac.dot(bp);
    if (d3 >= R(0) && d4 <= d3) { wts[0] = 0; wts[1] = 1; wts[2] = 0; return b.w; }
    R vc = d1 * d4 - d3 * d2;
    if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
        if (d1 == d3) { wts[0] = 1; wts[1] = 0; wts[2] = 0; return a.w; }
        R t = d1 / (d1 - d3);
        wts[0] = R(1) - t; wts[1] = t; wts[2] = 0;
        return a.w + ab * t;
    }
    V3<R> cp = -c.w;
    R d5 = ab.dot(cp), d6 = ac.dot(cp);
    if (d6 >= R(0) && d5 <= d6) { wts[0] = 0; wts[1] = 0; wts[2] = 1; return c.w; }
    R vb = d5 * d2 - d1 * d6;
    if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
        if (d2 == d6) { wts[0] = 1; wts[1] = 0; wts[2] = 0; return a.w; }
        R t = d2 / (d2 - d6);
        wts[0] = R(1) - t; wts[1] = 0; wts[2] = t;
        return a.w + ac * t;
    }
    R va = d3 * d6 - d5 * d4;
    if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
        if ((d4 - d3) + (d5 - d6) == R(0)) { wts[0] = 0; wts[1] = 1; wts[2] = 0; return b.w; }
        R t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        wts[0] = 0; wts[1] = R(1) - t; wts[2] = t;
        return b.w + (c.w - b.w) * t;
    }
    R sum = va + vb + vc;
    if (sum <= R(0) || std::isnan(sum)) {
        R la = a.w.length_squared(), lb = b.w.length_squared(), lc = c.w.length_squared();
        if (la <= lb && la <= lc) { wts[0] = 1; wts[1] = 0; wts[2] = 0; return a.w; }
        if (lb <= lc) { wts[0] = 0; wts[1] = 1; wts[2] = 0; return b.w; }
        wts[0] = 0; wts[1] = 0; wts[2] = 1; return c.w;
    }
    R denom = R(1) / sum;
    R v = vb * denom, w = vc * denom;
    wts[0] = R(1) - v - w; wts[1] = v; wts[2] = w;
    return a.w + ab * v + ac * w;
}

// gjk.rs:479-499
template <class R>
Closest<R> reduce_triangle(SupportVertex<R>* buf, int& len) {
    SupportVertex<R> a = buf[2], b = buf[1], c = buf[0];
    R w[3];
    V3<R> v = closest_triangle_bary(a, b, c, w);
    SupportVertex<R> kept[4] = {a, a, a, a};
    SupportVertex<R> src[3] = {a, b, c};
    int n = 0;
    for (int i = 0; i < 3; ++i) if (w[i] > R(0)) kept[n++] = src[i];
    if (n == 0) { n = 1; kept[0] = a; }
    for (int i = 0; i < n; ++i) buf[i] = kept[i];
    len = n;
    Closest<R> r;
    r.v = v;
    r.p_b = a.p_b * w[0] + b.p_b * w[1] + c.p_b * w[2];
    return r;
}

// gjk.rs:571-583
template <class R>
Closest<R> triangle_step(SupportVertex<R>* buf, int& len, SupportVertex<R> a, SupportVertex<R> b, SupportVertex<R> c) {
    buf[0] = c; buf[1] = b; buf[2] = a; len = 3;
    return reduce_triangle(buf, len);
}

// gjk.rs:501-567
template <class R>
Closest<R> reduce_tetrahedron(SupportVertex<R>* buf, int& len) {
    SupportVertex<R> a = buf[3], b = buf[2], c = buf[1], d = buf[0];
    V3<R> ab = b.w - a.w, ac = c.w - a.w, ad = d.w - a.w;
    if (std::fabs(ab.cross(ac).dot(ad)) < R(1e-12)) {
        SupportVertex<R> faces[4][3] = {{a, b, c}, {a, b, d}, {a, c, d}, {b, c, d}};
        int bf = 0;
        R bw[3];
        V3<R> bv = closest_triangle_bary(faces[0][0], faces[0][1], faces[0][2], bw);
        R best_v2 = std::numeric_limits<R>::infinity();
        for (int f = 1; f < 4; ++f) {
            R cw[3];
            V3<R> cv = closest_triangle_bary(faces[f][0], faces[f][1], faces[f][2], cw);
            R v2 = cv.length_squared();
            if (v2 < best_v2) { best_v2 = v2; bv = cv; bw[0] = cw[0]; bw[1] = cw[1]; bw[2] = cw[2]; bf = f; }
        }
        SupportVertex<R> kept[4] = {buf[0], buf[0], buf[0], buf[0]};
        int n = 0;
        for (int i = 0; i < 3; ++i) if (bw[i] > R(0)) kept[n++] = faces[bf][i];
        if (n == 0) { n = 1; kept[0] = faces[bf][0]; }
        V3<R> pb = faces[bf][0].p_b * bw[0] + faces[bf][1].p_b * bw[1] + faces[bf][2].p_b * bw[2];
        for (int i = 0; i < n; ++i) buf[i] = kept[i];
        len = n;
        Closest<R> r; r.v = bv; r.p_b = pb;
        return r;
    }
    V3<R> abc = ab.cross(ac), acd = ac.cross(ad), adb = ad.cross(ab);
    V3<R> ao = -a.w, bo = -b.w;
    V3<R> bcd = (c.w - b.w).cross(d.w - b.w);
    if (abc.dot(ao) * abc.dot(ad) < R(0)) return triangle_step(buf, len, a, b, c);
    if (acd.dot(ao) * acd.dot(ab) < R(0)) return triangle_step(buf, len, a, c, d);
    if (adb.dot(ao) * adb.dot(ac) < R(0)) return triangle_step(buf, len, a, d, b);
    if (bcd.dot(bo) * bcd.dot(a.w - b.w) < R(0)) return triangle_step(buf, len, b, c, d);
    Closest<R> r; r.inside = true;
    return r;
}

template <class R>
Closest<R> reduce(SupportVertex<R>* buf, int& len) {
    if (len == 1) { Closest<R> c; c.v = buf[0].w; c.p_b = buf[0].p_b; return c; }
    if (len == 2) return reduce_segment(buf, len);
    if (len == 3) return reduce_triangle(buf, len);
    return reduce_tetrahedron(buf, len);
}

// gjk.rs:668-680
template <class R>
V3<R> perpendicular(const V3<R>& v) {
    V3<R> helper = std::fabs(v.x) < R(0.9) ? V3<R>(1, 0, 0) : V3<R>(0, 1, 0);
    V3<R> perp = v.cross(helper);
    if (perp.length_squared() > R(0)) return perp.normalize();
    V3<R> alt = std::fabs(v.x) < R(0.9) ? V3<R>(0, 1, 0) : V3<R>(1, 0, 0);
    perp = v.cross(alt);
    if (perp.length_squared() > R(0)) return perp.normalize();
    return V3<R>(0, 0, 1);
}

// gjk.rs:18-52 — pts[0] is the most recent vertex.
template <class R>
struct Simplex {
    V3<R> pts[4];
    int len = 0;
    void add(const V3<R>& v) {
        for (int i = len; i > 0; --i) pts[i] = pts[i - 1];
        pts[0] = v;
        ++len;
    }
    void set(std::initializer_list<V3<R>> l) {
        int i = 0;
        for (auto& v : l) pts[i++] = v;
        len = i;
    }
};

template <class R>
V3<R> toward_origin(const V3<R>& n, const V3<R>& t) { return n.dot(t) < R(0) ? -n : n; }

// gjk.rs:636-655
template <class R>
bool solve_segment(Simplex<R>& s, V3<R>& dir) {
    V3<R> a = s.pts[1], b = s.pts[0];
    V3<R> ab = b - a, ao = -a;
    if (ab.dot(ao) > R(0)) {
        V3<R> cr = ab.cross(ao);
        if (cr.length_squared() > ab.length_squared() * ao.length_squared() * R(1e-10)) dir = cr.cross(ab);
        else dir = perpendicular(ab);
    } else {
        s.set({a});
        dir = ao;
    }
    return false;
}

// gjk.rs:784-803
template <class R>
bool shrink_or_normal(Simplex<R>& s, V3<R>& dir, const V3<R>& closest, const V3<R>& normal, const V3<R>& n0, const V3<R>& n1) {
    R span2 = 0;
    for (int i = 0; i < s.len; ++i) span2 = std::max(span2, s.pts[i].length_squared());
    if (closest.length_squared() < span2 * R(1e-12)) dir = normal;
    else { s.set({n0, n1}); dir = -closest; }
    return false;
}

// gjk.rs:687-772
template <class R>
bool solve_triangle(Simplex<R>& s, V3<R>& dir) {
    V3<R> a = s.pts[2], b = s.pts[1], c = s.pts[0];
    V3<R> ab = b - a, ac = c - a;
    V3<R> normal = ab.cross(ac);
    V3<R> ap = -a;
    R d1 = ab.dot(ap), d2 = ac.dot(ap);
    if (d1 <= R(0) && d2 <= R(0)) { s.set({a}); dir = -a; return false; }
    V3<R> bp = -b;
    R d3 = ab.dot(bp), d4 = ac.dot(bp);
    if (d3 >= R(0) && d4 <= d3) { s.set({b}); dir = -b; return false; }
    R vc = d1 * d4 - d3 * d2;
    if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
        R v = d1 == d3 ? R(0) : d1 / (d1 - d3);
        return shrink_or_normal(s, dir, a + ab * v, normal, b, a);
    }
    V3<R> cp = -c;
    R d5 = ab.dot(cp), d6 = ac.dot(cp);
    if (d6 >= R(0) && d5 <= d6) { s.set({c}); dir = -c; return false; }
    R vb = d5 * d2 - d1 * d6;
    if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
        R w = d2 == d6 ? R(0) : d2 / (d2 - d6);
        return shrink_or_normal(s, dir, a + ac * w, normal, c, a);
    }
    R va = d3 * d6 - d5 * d4;
    if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
        R w = (d4 - d3) + (d5 - d6) == R(0) ? R(0) : (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return shrink_or_normal(s, dir, b + (c - b) * w, normal, c, b);
    }
    R sum = va + vb + vc;
    if (sum <= R(0) || std::isnan(sum)) { dir = normal; return false; }
    R denom = R(1) / sum;
    R v = vb * denom, w = vc * denom;
    V3<R> closest = a + ab * v + ac * w;
    R span2 = std::max(std::max(a.length_squared(), b.length_squared()), c.length_squared());
    if (closest.length_squared() < span2 * R(1e-12)) dir = normal;
    else dir = -closest;
    return false;
}

// gjk.rs:807-848
template <class R>
bool solve_tetrahedron(Simplex<R>& s, V3<R>& dir) {
    V3<R> a = s.pts[3], b = s.pts[2], c = s.pts[1], d = s.pts[0];
    V3<R> ab = b - a, ac = c - a, ad = d - a, ao = -a, bo = -b;
    V3<R> abc = ab.cross(ac), acd = ac.cross(ad), adb = ad.cross(ab);
    V3<R> bcd = (b - c).cross(d - c);
    if (abc.dot(ao) * abc.dot(ad) < R(0)) { s.set({c, b, a}); dir = toward_origin(abc, ao); return false; }
    if (acd.dot(ao) * acd.dot(ab) < R(0)) { s.set({d, c, a}); dir = toward_origin(acd, ao); return false; }
    if (adb.dot(ao) * adb.dot(ac) < R(0)) { s.set({d, b, a}); dir = toward_origin(adb, ao); return false; }
    if (bcd.dot(bo) * bcd.dot(a - b) < R(0)) { s.set({d, c, b}); dir = toward_origin(bcd, bo); return false; }
    return true;
}

template <class R>
bool solve_simplex(Simplex<R>& s, V3<R>& dir) {
    if (s.len == 2) return solve_segment(s, dir);
    if (s.len == 3) return solve_triangle(s, dir);
    if (s.len == 4) return solve_tetrahedron(s, dir);
    dir = -s.pts[0];
    return false;
}

// gjk.rs:299-342 — strict origin-enclosing walk over the core supports.
template <class R, class F>
bool enclosing_walk(F support, const V3<R>& fallback, bool has_seed, const V3<R>& seed, Simplex<R>& s) {
    V3<R> init = (has_seed && seed.length_squared() > R(1e-12)) ? seed : fallback;
    s.len = 0;
    s.add(support(init));
    V3<R> dir = -s.pts[0];
    for (int it = 0; it < 64; ++it) {
        R d2 = dir.length_squared();
        if (d2 <= R(0) || std::isnan(d2)) dir = perpendicular(s.pts[0]);
        V3<R> a = support(dir);
        if (a.dot(dir) < R(0)) return false;
        s.add(a);
        if (solve_simplex(s, dir)) return true;
        V3<R> ref = s.len >= 2 ? s.pts[0] - s.pts[s.len - 1] : s.pts[0];
        if (dir.length_squared() < ref.length_squared() * R(1e-12)) dir = perpendicular(ref);
    }
    return false;
}

template <class R>
inline bool abs_diff_eq(const V3<R>& a, const V3<R>& b, R tol) {
    return std::fabs(a.x - b.x) <= tol && std::fabs(a.y - b.y) <= tol && std::fabs(a.z - b.z) <= tol;
}

// gjk.rs:171-288 — distance walk over the margin cores.
template <class R>
GjkOutcome<R> gjk_contact(const Shape<R>& sa, const V3<R>& pa, const Quat<R>& qa, const Shape<R>& sb, const V3<R>& pb,
                          const Quat<R>& qb, bool has_seed, const V3<R>& seed, R threshold) {
    const R TOUCH_TOLERANCE2 = R(1e-12), REL_ERROR2 = R(1e-6);
    R margin_a = sa.margin(), margin_b = sb.margin();
    R margin_sum = margin_a + margin_b;
    auto support = [&](const V3<R>& d) {
        SupportVertex<R> v;
        V3<R> p_a = sa.core_support_world(pa, qa, d);
        V3<R> p_b = sb.core_support_world(pb, qb, -d);
        v.w = p_a - p_b;
        v.p_b = p_b;
        return v;
    };
    V3<R> center_dir = pb - pa;
    V3<R> fallback = center_dir.length_squared() > R(1e-12) ? center_dir : V3<R>(1, 0, 0);
    V3<R> init = (has_seed && seed.length_squared() > R(1e-12)) ? seed : fallback;
    SupportVertex<R> first = support(init);
    SupportVertex<R> buf[4] = {first, first, first, first};
    int len = 1;
    V3<R> dir = -first.w;
    R touch2 = TOUCH_TOLERANCE2 * std::max(first.w.length_squared(), R(1));
    GjkOutcome<R> out;
    for (int it = 0; it < 64; ++it) {
        Closest<R> cl = reduce(buf, len);
        if (cl.inside) {
            out.kind = 2;
            for (int i = 0; i < 4; ++i) out.simplex[i] = buf[i].w;
            out.simplex_len = 4;
            return out;
        }
        V3<R> v = cl.v;
        R v2 = v.length_squared();
        if (v2 < touch2) {
            Simplex<R> s;
            bool ok = enclosing_walk<R>([&](const V3<R>& d) { return support(d).w; }, fallback, true, dir, s);
            if (ok && s.len == 4) {
                out.kind = 2;
                for (int i = 0; i < 4; ++i) out.simplex[i] = s.pts[i];
                out.simplex_len = 4;
            } else {
                out.kind = 0;
            }
            return out;
        }
        dir = -v;
        SupportVertex<R> w = support(dir);
        R delta = v.dot(w.w);
        R band = margin_sum + threshold;
        if (delta > R(0) && delta * delta > v2 * band * band) { out.kind = 0; return out; }
        bool dup = false;
        for (int i = 0; i < len; ++i) if (abs_diff_eq(w.w, buf[i].w, R(1e-6))) dup = true;
        if (dup || delta >= v2 * (R(1) - REL_ERROR2)) {
            R core_distance = std::sqrt(v2);
            R distance = core_distance - margin_sum;
            if (distance < threshold) {
                V3<R> n = dir / core_distance;
                out.kind = 1;
                out.distance = distance;
                out.normal = n;
                out.point_on_b = cl.p_b - n * margin_b;
                return out;
            }
            out.kind = 0;
            return out;
        }
        buf[len] = w;
        ++len;
    }
    out.kind = 0;
    return out;
}

// ---------------------------------------------------------------- EPA
template <class R>
struct EpaFace { int a, b, c; V3<R> normal; R distance, plane_distance; };

// epa.rs:281-303
template <class R>
bool edge_distance(const V3<R>& pa, const V3<R>& pb, const V3<R>& normal, R& out) {
    V3<R> ba = pb - pa;
    V3<R> n_ab = ba.cross(normal);
    if (pa.dot(n_ab) < R(0)) {
        R ba_l2 = ba.length_squared();
        R a_dot_ba = pa.dot(ba), b_dot_ba = pb.dot(ba);
        if (a_dot_ba > R(0)) out = pa.length();
        else if (b_dot_ba < R(0)) out = pb.length();
        else {
            R a_dot_b = pa.dot(pb);
            out = std::sqrt(std::max((pa.length_squared() * pb.length_squared() - a_dot_b * a_dot_b) / ba_l2, R(0)));
        }
        return true;
    }
    return false;
}

// epa.rs:262-275
template <class R>
R face_distance(const V3<R>& n, const V3<R>& pa, const V3<R>& pb, const V3<R>& pc) {
    R d;
    if (edge_distance(pa, pb, n, d)) return d;
    if (edge_distance(pb, pc, n, d)) return d;
    if (edge_distance(pc, pa, n, d)) return d;
    return pa.dot(n);
}

template <class R>
inline bool face_visible(const EpaFace<R>& f, const V3<R>& p) {
    return f.normal.dot(p) - f.plane_distance > Consts<R>::EPA_PLANE_EPS;  // epa.rs:396-398
}

// epa.rs:309-388 — atomic two-phase expansion.
template <class R>
bool epa_expand(std::vector<EpaFace<R>>& faces, const std::vector<V3<R>>& verts,
                std::vector<std::pair<int, int>>& boundary, const V3<R>& np, int nidx) {
    boundary.clear();
    bool any = false;
    for (auto& f : faces) {
        if (!face_visible(f, np)) continue;
        any = true;
        int es[3][2] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
        for (auto& e : es) {
            int u = e[0], v = e[1];
            int pos = -1;
            for (size_t i = 0; i < boundary.size(); ++i)
                if (boundary[i].first == v && boundary[i].second == u) { pos = int(i); break; }
            if (pos >= 0) { boundary[pos] = boundary.back(); boundary.pop_back(); }  // swap_remove
            else boundary.push_back({u, v});
        }
    }
    if (!any) return true;
    for (auto& e : boundary) {
        V3<R> cr = (verts[e.second] - verts[e.first]).cross(np - verts[e.first]);
        if (cr.length() < R(1e-12)) return false;
    }
    faces.erase(std::remove_if(faces.begin(), faces.end(), [&](const EpaFace<R>& f) { return face_visible(f, np); }),
                faces.end());
    for (auto& e : boundary) {
        int u = e.first, v = e.second;
        V3<R> cr = (verts[v] - verts[u]).cross(np - verts[u]);
        R l = cr.length();
        V3<R> n = cr / l;
        EpaFace<R> f;
        f.a = u; f.b = v; f.c = nidx;
        f.normal = n;
        f.distance = face_distance(n, verts[u], verts[v], np);
        f.plane_distance = n.dot(verts[u]);
        faces.push_back(f);
    }
    boundary.clear();
    return true;
}

// epa.rs:212-224 — first minimum of |distance|.
template <class R>
int epa_find_best(const std::vector<EpaFace<R>>& faces) {
    int best = 0;
    for (size_t i = 1; i < faces.size(); ++i)
        if (std::fabs(faces[i].distance) < std::fabs(faces[best].distance)) best = int(i);
    return best;
}

// epa.rs:127-205. Returns status: 0 converged, 1 degenerate, 2 iteration limit, 3 vertex limit.
template <class R, class F>
int epa_penetration(const V3<R> simplex[4], F support, V3<R>& normal, R& depth) {
    std::vector<V3<R>> verts(simplex, simplex + 4);
    std::vector<EpaFace<R>> faces;
    std::vector<std::pair<int, int>> boundary;
    const int quads[4][4] = {{0, 1, 2, 3}, {0, 3, 1, 2}, {0, 2, 3, 1}, {1, 3, 2, 0}};
    for (auto& q : quads) {  // epa.rs:226-256
        int a = q[0], b = q[1], c = q[2], opp = q[3];
        V3<R> n = (simplex[b] - simplex[a]).cross(simplex[c] - simplex[a]);
        if (n.dot(simplex[opp] - simplex[a]) > R(0)) { n = -n; std::swap(b, c); }
        R l = n.length();
        if (l < R(1e-12)) continue;
        n = n / l;
        EpaFace<R> f;
        f.a = a; f.b = b; f.c = c; f.normal = n;
        f.plane_distance = n.dot(simplex[a]);
        f.distance = face_distance(n, simplex[a], simplex[b], simplex[c]);
        faces.push_back(f);
    }
    if (faces.empty()) { normal = V3<R>(); depth = 0; return 1; }
    int status = 2;
    const V3<R> dirs[6] = {V3<R>(1, 0, 0), V3<R>(-1, 0, 0), V3<R>(0, 1, 0), V3<R>(0, -1, 0), V3<R>(0, 0, 1), V3<R>(0, 0, -1)};
    for (auto& d : dirs) {
        int idx = int(verts.size());
        V3<R> p = support(d);
        verts.push_back(p);
        if (!epa_expand(faces, verts, boundary, p, idx)) { status = 1; break; }
    }
    // epa.rs:174-201: the refinement loop runs even after a rejected seeding
    // expansion (the `break` above only leaves the seeding loop).
    for (int it = 0; it < 255; ++it) {
        int bi = epa_find_best(faces);
        V3<R> bn = faces[bi].normal;
        R bd = faces[bi].distance;
        V3<R> np = support(bn);
        R wdist = bn.dot(np) - bd;
        if (wdist <= Consts<R>::EPA_EPSILON) { normal = bn; depth = bd; return 0; }
        if (verts.size() >= 128) { status = 3; break; }
        int nidx = int(verts.size());
        verts.push_back(np);
        if (!epa_expand(faces, verts, boundary, np, nidx)) { status = 1; break; }
    }
    int bi = epa_find_best(faces);
    normal = faces[bi].normal;
    depth = faces[bi].distance;
    return status;
}

// convex_convex.rs:30-155
template <class R>
bool convex_convex(const Shape<R>& sa, const V3<R>& pa, const Quat<R>& qa, const Shape<R>& sb, const V3<R>& pb,
                   const Quat<R>& qb, bool has_seed, const V3<R>& seed, R threshold, Manifold<R>& out,
                   int* gjk_kind = nullptr) {
    GjkOutcome<R> g = gjk_contact(sa, pa, qa, sb, pb, qb, has_seed, seed, threshold);
    if (gjk_kind) *gjk_kind = g.kind;
    if (g.kind == 0) return false;
    if (g.kind == 1) {
        out.points.push_back(ContactPoint<R>(g.point_on_b, g.normal, -g.distance));
        return true;
    }
    auto support = [&](const V3<R>& d) { return sa.core_support_world(pa, qa, d) - sb.core_support_world(pb, qb, -d); };
    V3<R> n;
    R core_depth;
    epa_penetration<R>(g.simplex, support, n, core_depth);
    if (core_depth <= R(0)) return false;
    R depth = core_depth + sa.margin() + sb.margin();
    V3<R> point_a = sa.support_world(pa, qa, n);
    out.points.push_back(ContactPoint<R>(point_a - n * depth, n, depth));
    return true;
}

// manifold.rs:80-108 (ContactManifold::reduce): the deepest point first (stable sort by
// penetration, deepest first), then greedily the candidate farthest from the kept points.
template <class R>
void reduce_manifold(Manifold<R>& m, size_t max) {
    if (m.points.size() <= max) return;
    std::vector<ContactPoint<R>> cand = m.points;
    std::stable_sort(cand.begin(), cand.end(),
                     [](const ContactPoint<R>& a, const ContactPoint<R>& b) { return a.penetration > b.penetration; });
    std::vector<ContactPoint<R>> kept{cand[0]};
    std::vector<char> used(cand.size(), 0);
    used[0] = 1;
    while (kept.size() < max) {
        size_t best = 0;
        R best_sep = -std::numeric_limits<R>::infinity();
        for (size_t i = 0; i < cand.size(); ++i) {
            if (used[i]) continue;
            R sep = std::numeric_limits<R>::infinity();
            for (auto& q : kept) sep = std::min(sep, (cand[i].position - q.position).length_squared());
            if (sep > best_sep) { best_sep = sep; best = i; }
        }
        kept.push_back(cand[best]);
        used[best] = 1;
    }
    m.points = kept;
}

// convex_mesh.rs:236-253 (segment_closest_point_sq)
template <class R>
R segment_closest_point_sq(const V3<R>& from, const V3<R>& to, const V3<R>& p, V3<R>& nearest) {
    V3<R> v = to - from;
    R t = v.dot(p - from);
    if (t > R(0)) {
        R dvv = v.dot(v);
        if (t < dvv) t /= dvv;
        else t = R(1);
    } else {
        t = R(0);
    }
    nearest = from + v * t;
    return (p - nearest).length_squared();
}

// convex_mesh.rs:257-268 (point_in_triangle)
template <class R>
bool point_in_triangle(const V3<R>& p, const V3<R>& v1, const V3<R>& v2, const V3<R>& v3, const V3<R>& n) {
    V3<R> e1 = v2 - v1, e2 = v3 - v2, e3 = v1 - v3;
    R r1 = e1.cross(n).dot(p - v1), r2 = e2.cross(n).dot(p - v2), r3 = e3.cross(n).dot(p - v3);
    return (r1 > R(0) && r2 > R(0) && r3 > R(0)) || (r1 <= R(0) && r2 <= R(0) && r3 <= R(0));
}

// convex_mesh.rs:160-232 (sphere_triangle_contact): point on the triangle, normal toward the
// sphere centre, penetration radius - distance.
template <class R>
bool sphere_triangle_contact(const V3<R>& center, R radius, R threshold, const V3<R>& a, const V3<R>& b,
                             const V3<R>& c, V3<R>& point, V3<R>& normal_out, R& pen) {
    const R rwt = radius + threshold;
    V3<R> normal = (b - a).cross(c - a);
    R l2 = normal.length_squared();
    if (l2 < Consts<R>::EPS * Consts<R>::EPS) return false;
    normal = normal * (R(1) / std::sqrt(l2));
    R dist = normal.dot(center - a);
    if (dist < R(0)) {
        dist = -dist;
        normal = -normal;
    }
    if (dist >= rwt) return false;
    V3<R> cp;
    if (point_in_triangle(center, a, b, c, normal)) {
        cp = center - normal * dist;
    } else {
        R min_d = rwt * rwt;
        bool found = false;
        const V3<R>* ends[3][2] = {{&a, &b}, {&b, &c}, {&c, &a}};
        for (auto& e : ends) {
            V3<R> on;
            R d = segment_closest_point_sq(*e[0], *e[1], center, on);
            if (d < min_d) { min_d = d; cp = on; found = true; }
        }
        if (!found) return false;
    }
    V3<R> to_c = center - cp;
    R d2 = to_c.length_squared();
    if (d2 >= rwt * rwt) return false;
    point = cp;
    if (d2 > Consts<R>::EPS) {
        R d = std::sqrt(d2);
        normal_out = to_c * (R(1) / d);
        pen = radius - d;
    } else {
        normal_out = normal;
        pen = radius;
    }
    return true;
}

// convex_mesh.rs:26-153: the convex's world AABB swept into the mesh frame picks candidate
// triangles from the BVH; each candidate whose own AABB overlaps goes through the sphere
// detector or convex_convex against the triangle as a three-vertex hull; at most four points
// survive (reduce). Normals point from the convex to the mesh. (The internal-edge fix runs
// only for meshes whose edge info was generated, which nothing here does.)
template <class R>
bool convex_mesh(const Shape<R>& cv, const V3<R>& pc, const Quat<R>& qc, const Shape<R>& ms, const V3<R>& pm,
                 const Quat<R>& qm, bool has_seed, const V3<R>& seed, R threshold, Manifold<R>& out) {
    Aabb<R> cw = cv.world_aabb(pc, qc);
    Quat<R> inv_m = qm.inverse();
    V3<R> lmin = V3<R>::splat(std::numeric_limits<R>::infinity());
    V3<R> lmax = V3<R>::splat(-std::numeric_limits<R>::infinity());
    V3<R> c = cw.center(), e = cw.extents();
    for (int i = 0; i < 8; ++i) {
        V3<R> corner((i & 1) == 0 ? c.x + e.x : c.x - e.x, (i & 2) == 0 ? c.y + e.y : c.y - e.y,
                     (i & 4) == 0 ? c.z + e.z : c.z - e.z);
        V3<R> p = inv_m.rotate(corner - pm);
        lmin = lmin.min(p);
        lmax = lmax.max(p);
    }
    Aabb<R> query(lmin, lmax);
    const MeshData<R>& md = *ms.mesh;
    std::vector<uint32_t> cand;
    md.triangles_in_aabb(query, cand);
    out.points.clear();
    if (cv.type == SHAPE_SPHERE) {
        V3<R> center = inv_m.rotate(pc - pm);
        for (uint32_t t : cand) {
            if (!md.tri_aabbs[t].overlaps(query)) continue;
            V3<R> pt, nl;
            R pen;
            if (sphere_triangle_contact(center, cv.radius, threshold, md.tri_vertex(t, 0), md.tri_vertex(t, 1),
                                        md.tri_vertex(t, 2), pt, nl, pen))
                out.points.push_back(ContactPoint<R>(pm + qm.rotate(pt), qm.rotate(-nl), pen));
        }
    } else {
        for (uint32_t t : cand) {
            if (!md.tri_aabbs[t].overlaps(query)) continue;
            Manifold<R> m;
            if (convex_convex(cv, pc, qc, (*ms.tri_hulls)[t], pm, qm, has_seed, seed, threshold, m))
                for (auto& pt : m.points) out.points.push_back(pt);
        }
    }
    if (out.points.empty()) return false;
    reduce_manifold(out, 4);
    return true;
}

// narrowphase/mod.rs:63-286 (rigid convex/plane subset plus convex-vs-static-mesh: no compounds;
// mesh-mesh and plane-mesh pairs are two static bodies here, which the pair pass never collides).
template <class R>
bool collide(const Shape<R>& sa, const V3<R>& pa, const Quat<R>& qa, const Shape<R>& sb, const V3<R>& pb,
             const Quat<R>& qb, bool has_seed, const V3<R>& seed, Manifold<R>& out) {
    R thr = pair_threshold(sa, sb);
    out.points.clear();
    if (sa.type == SHAPE_PLANE && sb.type == SHAPE_PLANE) return false;
    if (sa.type == SHAPE_MESH || sb.type == SHAPE_MESH) {  // mod.rs:102-243
        if (sa.type == SHAPE_MESH && sb.is_convex()) {
            bool r = convex_mesh(sb, pb, qb, sa, pa, qa, has_seed, seed, thr, out);
            if (r) out.flip();
            return r;
        }
        if (sb.type == SHAPE_MESH && sa.is_convex()) return convex_mesh(sa, pa, qa, sb, pb, qb, has_seed, seed, thr, out);
        return false;
    }
    if (sa.type == SHAPE_PLANE) return plane_convex(sa, pa, qa, sb, pb, qb, thr, out);
    if (sb.type == SHAPE_PLANE) {
        bool r = plane_convex(sb, pb, qb, sa, pa, qa, thr, out);
        if (r) out.flip();
        return r;
    }
    if (sa.type == SHAPE_SPHERE && sb.type == SHAPE_SPHERE) return sphere_sphere(sa, pa, sb, pb, out);
    if (sa.type == SHAPE_SPHERE && sb.type == SHAPE_BOX) {
        bool r = sphere_box(sa, pa, sb, pb, qb, thr, out);
        if (r) out.flip();
        return r;
    }
    if (sa.type == SHAPE_BOX && sb.type == SHAPE_SPHERE) return sphere_box(sb, pb, sa, pa, qa, thr, out);
    if (sa.type == SHAPE_BOX && sb.type == SHAPE_BOX) return box_box(sa, pa, qa, sb, pb, qb, out);
    return convex_convex(sa, pa, qa, sb, pb, qb, has_seed, seed, thr, out);
}

}  // namespace oracle
