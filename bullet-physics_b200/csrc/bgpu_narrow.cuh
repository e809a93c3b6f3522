// Narrowphase contact generation (device side).
//
// Behaviour follows crates/bullet-collision/src/narrowphase/: shape-pair
// dispatch (mod.rs:63-286), sphere-sphere without a band (sphere.rs:10-32),
// sphere-box with the pair band (sphere.rs:38-82), plane-convex deepest point
// with the band (plane.rs:19-56), ODE-style box-box SAT with face clipping
// (box_box.rs:178-528), and the generic convex path: GJK distance walk on the
// margin cores (gjk.rs:171-288) with EPA on deep overlap (epa.rs:127-398,
// convex_convex.rs:30-155). Normals point from body A to body B; each point's
// position is the witness on B.
#pragma once
#include "bgpu_shapes.cuh"

namespace bgpu {

struct Manifold {
    int n;
    V3 pos[4];
    V3 nrm[4];
    float pen[4];
};

__device__ __forceinline__ void mf_push(Manifold& m, V3 p, V3 n, float pen) {
    if (m.n < 4) { m.pos[m.n] = p; m.nrm[m.n] = n; m.pen[m.n] = pen; m.n++; }
}
__device__ __forceinline__ void mf_flip(Manifold& m) {
    for (int i = 0; i < m.n; ++i) m.nrm[i] = -m.nrm[i];
}

// sphere.rs:10-32
__device__ __forceinline__ bool sphere_sphere(float ra, V3 pa, float rb, V3 pb, Manifold& out) {
    V3 delta = pb - pa;
    float d2 = len2(delta);
    float rs = ra + rb;
    if (d2 >= rs * rs) return false;
    float d = sqrtf(d2);
    V3 n = d > 1e-12f ? delta / d : V3{0.f, 1.f, 0.f};
    float pen = rs - d;
    mf_push(out, pa + n * (ra - pen * 0.5f), n, pen);
    return true;
}

__device__ __forceinline__ float signum_f(float v) { return signbit(v) ? -1.0f : 1.0f; }

// sphere.rs:38-82 — normal from the box to the sphere.
__device__ __forceinline__ bool sphere_box(float r, V3 ps, V3 h, V3 pb, Q ob, float thr, Manifold& out) {
    V3 local = rotate(qinv(ob), ps - pb);
    V3 cl = V3{fminf(fmaxf(local.x, -h.x), h.x), fminf(fmaxf(local.y, -h.y), h.y), fminf(fmaxf(local.z, -h.z), h.z)};
    V3 delta = local - cl;
    float d2 = len2(delta);
    float cd = r + thr;
    if (d2 >= cd * cd) return false;
    float d = sqrtf(d2);
    V3 nl;
    float pen;
    if (d > 1e-12f) {
        nl = delta / d;
        pen = r - d;
    } else {
        float dx = h.x - fabsf(local.x), dy = h.y - fabsf(local.y), dz = h.z - fabsf(local.z);
        float dd;
        if (dx <= dy && dx <= dz) { nl = V3{signum_f(local.x), 0.f, 0.f}; dd = dx; }
        else if (dy <= dz) { nl = V3{0.f, signum_f(local.y), 0.f}; dd = dy; }
        else { nl = V3{0.f, 0.f, signum_f(local.z)}; dd = dz; }
        pen = r + dd;
    }
    mf_push(out, rotate(ob, cl) + pb, rotate(ob, nl), pen);
    return true;
}

// plane.rs:19-56
__device__ __forceinline__ bool plane_convex(const Shape& pl, V3 pp, Q qp, const Shape& cv, V3 pc, Q qc, float thr,
                                             const float4* __restrict__ hull, Manifold& out) {
    V3 n = rotate(qp, V3{pl.p0, pl.p1, pl.p2});
    float c = pl.p3 + dot(n, pp);
    V3 normal = dot(n, pc - pp) >= 0.0f ? n : -n;
    if (!(normal.x == n.x && normal.y == n.y && normal.z == n.z)) c = -c;
    V3 deepest = support_world(cv, pc, qc, -normal, hull);
    float depth = c - dot(normal, deepest);
    if (depth < -thr) return false;
    mf_push(out, deepest, normal, depth);
    return true;
}

// ------------------------------------------------------------------ box-box (box_box.rs)
struct ClipPoly {
    float x[8], y[8];
    int n;
};

__device__ __forceinline__ void clip_poly(const ClipPoly& src, int axis, float sign, float h, ClipPoly& out) {
    int n = src.n;
    out.n = 0;
    for (int i = 0; i < n; ++i) {
        int j = (i + 1) % n;
        float cur[2] = {src.x[i], src.y[i]};
        float nxt[2] = {src.x[j], src.y[j]};
        bool cin = sign * cur[axis] < h;
        bool nin = sign * nxt[axis] < h;
        if (cin && out.n < 8) { out.x[out.n] = cur[0]; out.y[out.n] = cur[1]; out.n++; }
        if (cin != nin && out.n < 8) {
            float t = (sign * h - cur[axis]) / (nxt[axis] - cur[axis]);
            float p[2];
            p[axis] = sign * h;
            p[1 - axis] = cur[1 - axis] + (nxt[1 - axis] - cur[1 - axis]) * t;
            out.x[out.n] = p[0]; out.y[out.n] = p[1]; out.n++;
        }
    }
}

// box_box's arrays (clip polygons, clipped points, cull order), indexed at runtime. The kernels
// keep one per thread in shared memory, where a runtime index costs no local-memory traffic. 83
// words: an odd stride puts the 32 lanes' copies of a field in 32 different banks.
struct BoxBoxScratch {
    ClipPoly buf, tmp;
    V3 pts[8];
    float deps[8];
    float rd[8];
    int ri[8];
    int pad;
};
static_assert(sizeof(BoxBoxScratch) % 8 == 4, "odd word stride");

static __device__ __noinline__ bool box_box(V3 ha, V3 p1, Q oa, V3 hb, V3 p2, Q ob, Manifold& out,
                                            BoxBoxScratch& S) {
    const float EPS = 1e-6f, FUDGE = 1.05f;
    M3 r1 = from_quat(oa), r2 = from_quat(ob);
    V3 p = p2 - p1;
    V3 pp = mul(transpose(r1), p);
    M3 r = mul(transpose(r1), r2);
    float r11 = r.c0.x, r12 = r.c1.x, r13 = r.c2.x;
    float r21 = r.c0.y, r22 = r.c1.y, r23 = r.c2.y;
    float r31 = r.c0.z, r32 = r.c1.z, r33 = r.c2.z;
    float q11 = fabsf(r11), q12 = fabsf(r12), q13 = fabsf(r13);
    float q21 = fabsf(r21), q22 = fabsf(r22), q23 = fabsf(r23);
    float q31 = fabsf(r31), q32 = fabsf(r32), q33 = fabsf(r33);

    float s = -INFINITY;
    bool invert = false, from_r2 = false, is_cross = false;
    int code = 0, axis = 0;
    V3 nc = V3{0.f, 0.f, 0.f};

#define BG_TST_FACE(e1, e2, fr2, ax, cc)                                                   \
    {                                                                                      \
        float _e1 = (e1);                                                                  \
        float s2 = fabsf(_e1) - (e2);                                                      \
        if (s2 > 0.0f) return false;                                                       \
        if (s2 > s) { s = s2; is_cross = false; from_r2 = (fr2); axis = (ax); invert = _e1 < 0.0f; code = (cc); } \
    }
#define BG_TST_CROSS(e1, e2, n1, n2, n3, cc)                                               \
    {                                                                                      \
        float _e1 = (e1);                                                                  \
        float s2 = fabsf(_e1) - (e2);                                                      \
        if (s2 > EPS) return false;                                                        \
        float _n1 = (n1), _n2 = (n2), _n3 = (n3);                                          \
        float l = sqrtf(_n1 * _n1 + _n2 * _n2 + _n3 * _n3);                                \
        if (l > EPS) {                                                                     \
            s2 = s2 / l;                                                                   \
            if (s2 * FUDGE > s) { s = s2; is_cross = true; nc = V3{_n1 / l, _n2 / l, _n3 / l}; invert = _e1 < 0.0f; code = (cc); } \
        }                                                                                  \
    }

    BG_TST_FACE(pp.x, ha.x + hb.x * q11 + hb.y * q12 + hb.z * q13, false, 0, 1)
    BG_TST_FACE(pp.y, ha.y + hb.x * q21 + hb.y * q22 + hb.z * q23, false, 1, 2)
    BG_TST_FACE(pp.z, ha.z + hb.x * q31 + hb.y * q32 + hb.z * q33, false, 2, 3)
    BG_TST_FACE(dot(r2.c0, p), ha.x * q11 + ha.y * q21 + ha.z * q31 + hb.x, true, 0, 4)
    BG_TST_FACE(dot(r2.c1, p), ha.x * q12 + ha.y * q22 + ha.z * q32 + hb.y, true, 1, 5)
    BG_TST_FACE(dot(r2.c2, p), ha.x * q13 + ha.y * q23 + ha.z * q33 + hb.z, true, 2, 6)

    const float f2 = 1e-5f;
    q11 += f2; q12 += f2; q13 += f2; q21 += f2; q22 += f2; q23 += f2; q31 += f2; q32 += f2; q33 += f2;

    BG_TST_CROSS(pp.z * r21 - pp.y * r31, ha.y * q31 + ha.z * q21 + hb.y * q13 + hb.z * q12, 0.0f, -r31, r21, 7)
    BG_TST_CROSS(pp.z * r22 - pp.y * r32, ha.y * q32 + ha.z * q22 + hb.x * q13 + hb.z * q11, 0.0f, -r32, r22, 8)
    BG_TST_CROSS(pp.z * r23 - pp.y * r33, ha.y * q33 + ha.z * q23 + hb.x * q12 + hb.y * q11, 0.0f, -r33, r23, 9)
    BG_TST_CROSS(pp.x * r31 - pp.z * r11, ha.x * q31 + ha.z * q11 + hb.y * q23 + hb.z * q22, r31, 0.0f, -r11, 10)
    BG_TST_CROSS(pp.x * r32 - pp.z * r12, ha.x * q32 + ha.z * q12 + hb.x * q23 + hb.z * q21, r32, 0.0f, -r12, 11)
    BG_TST_CROSS(pp.x * r33 - pp.z * r13, ha.x * q33 + ha.z * q13 + hb.x * q22 + hb.y * q21, r33, 0.0f, -r13, 12)
    BG_TST_CROSS(pp.y * r11 - pp.x * r21, ha.x * q21 + ha.y * q11 + hb.y * q33 + hb.z * q32, -r21, r11, 0.0f, 13)
    BG_TST_CROSS(pp.y * r12 - pp.x * r22, ha.x * q22 + ha.y * q12 + hb.x * q33 + hb.z * q31, -r22, r12, 0.0f, 14)
    BG_TST_CROSS(pp.y * r13 - pp.x * r23, ha.x * q23 + ha.y * q13 + hb.x * q32 + hb.y * q31, -r23, r13, 0.0f, 15)
#undef BG_TST_FACE
#undef BG_TST_CROSS

    V3 nsat = is_cross ? mul(r1, nc) : (from_r2 ? col(r2, axis) : col(r1, axis));
    if (invert) nsat = -nsat;
    float depth = -s;

    if (code > 6) {  // box_box.rs:402-423
        V3 qa = p1;
        for (int j = 0; j < 3; ++j) {
            V3 c = col(r1, j);
            float sg = dot(nsat, c) > 0.0f ? 1.0f : -1.0f;
            qa += c * (sg * comp(ha, j));
        }
        V3 qb = p2;
        for (int j = 0; j < 3; ++j) {
            V3 c = col(r2, j);
            float sg = dot(nsat, c) > 0.0f ? -1.0f : 1.0f;
            qb += c * (sg * comp(hb, j));
        }
        V3 ua = col(r1, (code - 7) / 3), ub = col(r2, (code - 7) % 3);
        // line_closest_approach (box_box.rs:31-48); only beta moves the B witness.
        V3 pd = qb - qa;
        float uaub = dot(ua, ub);
        float qq1 = dot(ua, pd);
        float qq2 = -dot(ub, pd);
        float d = 1.0f - uaub * uaub;
        float beta = 0.0f;
        if (!(d <= 1e-4f)) {
            d = 1.0f / d;
            beta = (uaub * qq1 + qq2) * d;
        }
        qb += ub * beta;
        mf_push(out, qb, nsat, depth);
        return true;
    }

    const M3& ra = code <= 3 ? r1 : r2;
    const M3& rb = code <= 3 ? r2 : r1;
    V3 pa_ref = code <= 3 ? p1 : p2;
    V3 pb_inc = code <= 3 ? p2 : p1;
    V3 sa = code <= 3 ? ha : hb;
    V3 sb = code <= 3 ? hb : ha;
    V3 normal2 = code <= 3 ? nsat : -nsat;
    V3 nr = mul(transpose(rb), normal2);
    V3 anr = vabs(nr);
    int lanr, a1, a2;
    if (anr.y > anr.x) {
        if (anr.y > anr.z) { lanr = 1; a1 = 0; a2 = 2; } else { lanr = 2; a1 = 0; a2 = 1; }
    } else if (anr.x > anr.z) { lanr = 0; a1 = 1; a2 = 2; } else { lanr = 2; a1 = 0; a2 = 1; }

    V3 center = comp(nr, lanr) < 0.0f ? (pb_inc - pa_ref + col(rb, lanr) * comp(sb, lanr))
                                      : (pb_inc - pa_ref - col(rb, lanr) * comp(sb, lanr));
    int code_n = code <= 3 ? code - 1 : code - 4;
    int code1, code2;
    if (code_n == 0) { code1 = 1; code2 = 2; } else if (code_n == 1) { code1 = 0; code2 = 2; } else { code1 = 0; code2 = 1; }
    float c1 = dot(center, col(ra, code1));
    float c2 = dot(center, col(ra, code2));
    float m11 = dot(col(ra, code1), col(rb, a1));
    float m12 = dot(col(ra, code1), col(rb, a2));
    float m21 = dot(col(ra, code2), col(rb, a1));
    float m22 = dot(col(ra, code2), col(rb, a2));
    float k1 = m11 * comp(sb, a1), k2 = m21 * comp(sb, a1), k3 = m12 * comp(sb, a2), k4 = m22 * comp(sb, a2);

    ClipPoly& buf = S.buf;
    ClipPoly& tmp = S.tmp;
    buf.x[0] = c1 - k1 - k3; buf.y[0] = c2 - k2 - k4;
    buf.x[1] = c1 - k1 + k3; buf.y[1] = c2 - k2 + k4;
    buf.x[2] = c1 + k1 + k3; buf.y[2] = c2 + k2 + k4;
    buf.x[3] = c1 + k1 - k3; buf.y[3] = c2 + k2 - k4;
    buf.n = 4;
    float rect0 = comp(sa, code1), rect1 = comp(sa, code2);
    clip_poly(buf, 0, -1.0f, rect0, tmp);
    clip_poly(tmp, 0, 1.0f, rect0, buf);
    clip_poly(buf, 1, -1.0f, rect1, tmp);
    clip_poly(tmp, 1, 1.0f, rect1, buf);
    if (buf.n == 0) return false;

    float det1 = 1.0f / (m11 * m22 - m12 * m21);
    m11 *= det1; m12 *= det1; m21 *= det1; m22 *= det1;
    V3* pts = S.pts;
    float* deps = S.deps;
    int np = 0;
    for (int i = 0; i < buf.n; ++i) {
        float rx = buf.x[i], ry = buf.y[i];
        float kk1 = m22 * (rx - c1) - m12 * (ry - c2);
        float kk2 = -m21 * (rx - c1) + m11 * (ry - c2);
        V3 point = center + col(rb, a1) * kk1 + col(rb, a2) * kk2;
        float dep = comp(sa, code_n) - dot(normal2, point);
        if (dep >= 0.0f) { pts[np] = point; deps[np] = dep; ++np; }
    }
    if (np == 0) return false;

    // cull_points (box_box.rs:131-174): deepest (last maximum) + farthest, stable.
    int sel[4];
    int nsel;
    if (np <= 4) {
        nsel = np;
        for (int i = 0; i < np; ++i) sel[i] = i;
    } else {
        int i0 = 0;
        float dd = deps[0];
        for (int i = 1; i < np; ++i) if (deps[i] >= dd) { i0 = i; dd = deps[i]; }
        int* ri = S.ri;
        float* rd = S.rd;
        int rn = 0;
        for (int i = 0; i < np; ++i) if (i != i0) { ri[rn] = i; rd[rn] = len2(pts[i] - pts[i0]); rn++; }
        for (int j = 1; j < rn; ++j) {
            int ki = ri[j];
            float kd = rd[j];
            int k = j;
            while (k > 0 && rd[k - 1] < kd) { ri[k] = ri[k - 1]; rd[k] = rd[k - 1]; --k; }
            ri[k] = ki; rd[k] = kd;
        }
        sel[0] = i0;
        nsel = 1;
        for (int t = 0; t < 3 && t < rn; ++t) sel[nsel++] = ri[t];
    }
    for (int t = 0; t < nsel; ++t) {
        V3 pos = pts[sel[t]] + pa_ref;
        if (code > 3) pos += nsat * deps[sel[t]];
        mf_push(out, pos, nsat, deps[sel[t]]);
    }
    return true;
}

// ------------------------------------------------------------------ GJK (gjk.rs)
struct SV {
    V3 w, pb;
};

struct GjkResult {
    int kind;  // 0 separated, 1 band, 2 overlap
    float distance;
    V3 normal, point_on_b;
    V3 simplex[4];
};

struct ConvexPair {
    const Shape* sa;
    const Shape* sb;
    V3 pa, pb;
    Q qa, qb;
    const float4* hull;
    __device__ SV support(V3 d) const {
        SV v;
        V3 p_a = core_support_world(*sa, pa, qa, d, hull);
        V3 p_b = core_support_world(*sb, pb, qb, -d, hull);
        v.w = p_a - p_b;
        v.pb = p_b;
        return v;
    }
};

// gjk.rs:399-477
__device__ __forceinline__ V3 closest_triangle_bary(const SV& a, const SV& b, const SV& c, float* w) {
    V3 ab = b.w - a.w, ac = c.w - a.w, ap = -a.w;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { w[0] = 1.f; w[1] = 0.f; w[2] = 0.f; return a.w; }
    V3 bp = -b.w;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { w[0] = 0.f; w[1] = 1.f; w[2] = 0.f; return b.w; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        if (d1 == d3) { w[0] = 1.f; w[1] = 0.f; w[2] = 0.f; return a.w; }
        float t = d1 / (d1 - d3);
        w[0] = 1.0f - t; w[1] = t; w[2] = 0.f;
        return a.w + ab * t;
    }
    V3 cp = -c.w;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { w[0] = 0.f; w[1] = 0.f; w[2] = 1.f; return c.w; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        if (d2 == d6) { w[0] = 1.f; w[1] = 0.f; w[2] = 0.f; return a.w; }
        float t = d2 / (d2 - d6);
        w[0] = 1.0f - t; w[1] = 0.f; w[2] = t;
        return a.w + ac * t;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        if ((d4 - d3) + (d5 - d6) == 0.0f) { w[0] = 0.f; w[1] = 1.f; w[2] = 0.f; return b.w; }
        float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        w[0] = 0.f; w[1] = 1.0f - t; w[2] = t;
        return b.w + (c.w - b.w) * t;
    }
    float sum = va + vb + vc;
    if (sum <= 0.0f || isnan(sum)) {
        float la = len2(a.w), lb = len2(b.w), lc = len2(c.w);
        if (la <= lb && la <= lc) { w[0] = 1.f; w[1] = 0.f; w[2] = 0.f; return a.w; }
        if (lb <= lc) { w[0] = 0.f; w[1] = 1.f; w[2] = 0.f; return b.w; }
        w[0] = 0.f; w[1] = 0.f; w[2] = 1.f;
        return c.w;
    }
    float denom = 1.0f / sum;
    float v = vb * denom, ww = vc * denom;
    w[0] = 1.0f - v - ww; w[1] = v; w[2] = ww;
    return a.w + ab * v + ac * ww;
}

struct Closest {
    bool inside;
    V3 v, pb;
};

// The GJK simplex is four named points B0..B3 (B0 oldest; the array form buf[i] of the
// reference maps to Bi): with constant indices only, it stays in registers through the loop.

// gjk.rs:479-499: the closest point of triangle (a, b, c) = (B2, B1, B0); the points with a
// positive barycentric weight are kept, in the order a, b, c, as B0, B1, ...
__device__ __forceinline__ Closest reduce_triangle(SV& B0, SV& B1, SV& B2, int& n) {
    const SV a = B2, b = B1, c = B0;
    float w[3];
    const V3 v = closest_triangle_bary(a, b, c, w);
    const bool fa = w[0] > 0.0f, fb = w[1] > 0.0f, fc = w[2] > 0.0f;
    int k = int(fa) + int(fb) + int(fc);
    if (k == 0) {
        k = 1;
        B0 = a;
    } else {
        const SV k0 = fa ? a : (fb ? b : c);
        const SV k1 = fa ? (fb ? b : c) : c;
        B0 = k0;
        if (k > 1) B1 = k1;
        if (k > 2) B2 = c;
    }
    n = k;
    Closest r;
    r.inside = false;
    r.v = v;
    r.pb = a.pb * w[0] + b.pb * w[1] + c.pb * w[2];
    return r;
}

// gjk.rs:354-567, four coplanar points (a, b, c, d) = (B3, B2, B1, B0): the closest of the
// four faces. Rarely taken, so a call of its own; its kept points come back by value.
struct CoplanarReduced {
    SV k[3];
    int n;
    Closest r;
};

static __device__ __noinline__ CoplanarReduced gjk_reduce_coplanar(SV a, SV b, SV c, SV d, SV first) {
    SV faces[4][3] = {{a, b, c}, {a, b, d}, {a, c, d}, {b, c, d}};
    int bf = 0;
    float bw[3];
    V3 bv = closest_triangle_bary(faces[0][0], faces[0][1], faces[0][2], bw);
    float best_v2 = INFINITY;
    for (int f = 1; f < 4; ++f) {
        float cw[3];
        V3 cv = closest_triangle_bary(faces[f][0], faces[f][1], faces[f][2], cw);
        float v2 = len2(cv);
        if (v2 < best_v2) { best_v2 = v2; bv = cv; bw[0] = cw[0]; bw[1] = cw[1]; bw[2] = cw[2]; bf = f; }
    }
    CoplanarReduced out;
    out.k[0] = out.k[1] = out.k[2] = first;
    int k = 0;
    for (int i = 0; i < 3; ++i) if (bw[i] > 0.0f) out.k[k++] = faces[bf][i];
    if (k == 0) { k = 1; out.k[0] = faces[bf][0]; }
    out.n = k;
    out.r.inside = false;
    out.r.v = bv;
    out.r.pb = faces[bf][0].pb * bw[0] + faces[bf][1].pb * bw[1] + faces[bf][2].pb * bw[2];
    return out;
}

// gjk.rs:354-567
__device__ __forceinline__ Closest gjk_reduce(SV& B0, SV& B1, SV& B2, SV& B3, int& n) {
    Closest r;
    r.inside = false;
    if (n == 1) { r.v = B0.w; r.pb = B0.pb; return r; }
    if (n == 2) {  // gjk.rs:366-394
        const SV a = B1, b = B0;
        V3 ab = b.w - a.w;
        float denom = len2(ab);
        if (denom < 1e-24f) { n = 1; B0 = a; r.v = a.w; r.pb = a.pb; return r; }
        float t = -dot(a.w, ab) / denom;
        if (t <= 0.0f) { n = 1; B0 = a; r.v = a.w; r.pb = a.pb; }
        else if (t >= 1.0f) { n = 1; B0 = b; r.v = b.w; r.pb = b.pb; }
        else { n = 2; B0 = a; B1 = b; r.v = a.w + ab * t; r.pb = a.pb + (b.pb - a.pb) * t; }
        return r;
    }
    if (n == 3) return reduce_triangle(B0, B1, B2, n);
    const SV a = B3, b = B2, c = B1, d = B0;
    V3 ab = b.w - a.w, ac = c.w - a.w, ad = d.w - a.w;
    if (fabsf(dot(cross(ab, ac), ad)) < 1e-12f) {
        const CoplanarReduced cr = gjk_reduce_coplanar(a, b, c, d, B0);
        B0 = cr.k[0];
        if (cr.n > 1) B1 = cr.k[1];
        if (cr.n > 2) B2 = cr.k[2];
        n = cr.n;
        return cr.r;
    }
    V3 abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
    V3 ao = -a.w, bo = -b.w;
    V3 bcd = cross(c.w - b.w, d.w - b.w);
    if (dot(abc, ao) * dot(abc, ad) < 0.0f) { B0 = c; B1 = b; B2 = a; n = 3; return reduce_triangle(B0, B1, B2, n); }
    if (dot(acd, ao) * dot(acd, ab) < 0.0f) { B0 = d; B1 = c; B2 = a; n = 3; return reduce_triangle(B0, B1, B2, n); }
    if (dot(adb, ao) * dot(adb, ac) < 0.0f) { B0 = b; B1 = d; B2 = a; n = 3; return reduce_triangle(B0, B1, B2, n); }
    if (dot(bcd, bo) * dot(bcd, a.w - b.w) < 0.0f) { B0 = d; B1 = c; B2 = b; n = 3; return reduce_triangle(B0, B1, B2, n); }
    r.inside = true;
    return r;
}

// gjk.rs:668-680
__device__ __forceinline__ V3 perpendicular(V3 v) {
    V3 helper = fabsf(v.x) < 0.9f ? V3{1.f, 0.f, 0.f} : V3{0.f, 1.f, 0.f};
    V3 perp = cross(v, helper);
    if (len2(perp) > 0.0f) return normalize(perp);
    V3 alt = fabsf(v.x) < 0.9f ? V3{0.f, 1.f, 0.f} : V3{1.f, 0.f, 0.f};
    perp = cross(v, alt);
    if (len2(perp) > 0.0f) return normalize(perp);
    return V3{0.f, 0.f, 1.f};
}

__device__ __forceinline__ V3 toward_origin(V3 n, V3 t) { return dot(n, t) < 0.0f ? -n : n; }

// Strict enclosing walk (gjk.rs:299-342, 624-848). pts[0] is the newest vertex.
static __device__ __noinline__ bool enclosing_walk(const ConvexPair& cp, V3 fallback, V3 seed, V3* pts) {
    int n = 0;
    V3 init = len2(seed) > 1e-12f ? seed : fallback;
    pts[0] = cp.support(init).w;
    n = 1;
    V3 dir = -pts[0];
    for (int it = 0; it < 64; ++it) {
        float d2 = len2(dir);
        if (d2 <= 0.0f || isnan(d2)) dir = perpendicular(pts[0]);
        V3 a = cp.support(dir).w;
        if (dot(a, dir) < 0.0f) return false;
        for (int i = n; i > 0; --i) pts[i] = pts[i - 1];
        pts[0] = a;
        ++n;
        bool enclosed = false;
        if (n == 2) {  // gjk.rs:636-655
            V3 sa = pts[1], sb = pts[0];
            V3 ab = sb - sa, ao = -sa;
            if (dot(ab, ao) > 0.0f) {
                V3 cr = cross(ab, ao);
                if (len2(cr) > len2(ab) * len2(ao) * 1e-10f) dir = cross(cr, ab);
                else dir = perpendicular(ab);
            } else { pts[0] = sa; n = 1; dir = ao; }
        } else if (n == 3) {  // gjk.rs:687-772
            V3 ta = pts[2], tb = pts[1], tc = pts[0];
            V3 ab = tb - ta, ac = tc - ta;
            V3 normal = cross(ab, ac);
            V3 ap = -ta;
            float d1 = dot(ab, ap), d2v = dot(ac, ap);
            float span2 = fmaxf(fmaxf(len2(ta), len2(tb)), len2(tc));
            bool done = false;
            if (d1 <= 0.0f && d2v <= 0.0f) { pts[0] = ta; n = 1; dir = -ta; done = true; }
            float d3 = 0.f, d4 = 0.f, d5 = 0.f, d6 = 0.f, vc = 0.f, vb = 0.f;
            if (!done) {
                V3 bp = -tb;
                d3 = dot(ab, bp); d4 = dot(ac, bp);
                if (d3 >= 0.0f && d4 <= d3) { pts[0] = tb; n = 1; dir = -tb; done = true; }
            }
            if (!done) {
                vc = d1 * d4 - d3 * d2v;
                if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
                    float v = d1 == d3 ? 0.0f : d1 / (d1 - d3);
                    V3 closest = ta + ab * v;
                    if (len2(closest) < span2 * 1e-12f) dir = normal;
                    else { pts[0] = tb; pts[1] = ta; n = 2; dir = -closest; }
                    done = true;
                }
            }
            if (!done) {
                V3 cpv = -tc;
                d5 = dot(ab, cpv); d6 = dot(ac, cpv);
                if (d6 >= 0.0f && d5 <= d6) { pts[0] = tc; n = 1; dir = -tc; done = true; }
            }
            if (!done) {
                vb = d5 * d2v - d1 * d6;
                if (vb <= 0.0f && d2v >= 0.0f && d6 <= 0.0f) {
                    float w = d2v == d6 ? 0.0f : d2v / (d2v - d6);
                    V3 closest = ta + ac * w;
                    if (len2(closest) < span2 * 1e-12f) dir = normal;
                    else { pts[0] = tc; pts[1] = ta; n = 2; dir = -closest; }
                    done = true;
                }
            }
            if (!done) {
                float va = d3 * d6 - d5 * d4;
                if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
                    float w = (d4 - d3) + (d5 - d6) == 0.0f ? 0.0f : (d4 - d3) / ((d4 - d3) + (d5 - d6));
                    V3 closest = tb + (tc - tb) * w;
                    if (len2(closest) < span2 * 1e-12f) dir = normal;
                    else { pts[0] = tc; pts[1] = tb; n = 2; dir = -closest; }
                    done = true;
                }
                if (!done) {
                    float sum = va + vb + vc;
                    if (sum <= 0.0f || isnan(sum)) dir = normal;
                    else {
                        float denom = 1.0f / sum;
                        float v = vb * denom, w = vc * denom;
                        V3 closest = ta + ab * v + ac * w;
                        if (len2(closest) < span2 * 1e-12f) dir = normal;
                        else dir = -closest;
                    }
                }
            }
        } else if (n == 4) {  // gjk.rs:807-848
            V3 a4 = pts[3], b4 = pts[2], c4 = pts[1], d4v = pts[0];
            V3 ab = b4 - a4, ac = c4 - a4, ad = d4v - a4, ao = -a4, bo = -b4;
            V3 abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
            V3 bcd = cross(b4 - c4, d4v - c4);
            if (dot(abc, ao) * dot(abc, ad) < 0.0f) { pts[0] = c4; pts[1] = b4; pts[2] = a4; n = 3; dir = toward_origin(abc, ao); }
            else if (dot(acd, ao) * dot(acd, ab) < 0.0f) { pts[0] = d4v; pts[1] = c4; pts[2] = a4; n = 3; dir = toward_origin(acd, ao); }
            else if (dot(adb, ao) * dot(adb, ac) < 0.0f) { pts[0] = d4v; pts[1] = b4; pts[2] = a4; n = 3; dir = toward_origin(adb, ao); }
            else if (dot(bcd, bo) * dot(bcd, a4 - b4) < 0.0f) { pts[0] = d4v; pts[1] = c4; pts[2] = b4; n = 3; dir = toward_origin(bcd, bo); }
            else enclosed = true;
        } else {
            dir = -pts[0];
        }
        if (enclosed) return n == 4;
        V3 ref = n >= 2 ? pts[0] - pts[n - 1] : pts[0];
        if (len2(dir) < len2(ref) * 1e-12f) dir = perpendicular(ref);
    }
    return false;
}

// gjk.rs:171-288
static __device__ __noinline__ GjkResult gjk_contact(const ConvexPair& cp, bool has_seed, V3 seed, float thr) {
    const float TOUCH2 = 1e-12f, REL2 = 1e-6f;
    float ma = cp.sa->margin, mb = cp.sb->margin;
    float msum = ma + mb;
    V3 cdir = cp.pb - cp.pa;
    V3 fallback = len2(cdir) > 1e-12f ? cdir : V3{1.f, 0.f, 0.f};
    V3 init = (has_seed && len2(seed) > 1e-12f) ? seed : fallback;
    SV first = cp.support(init);
    SV B0 = first, B1 = first, B2 = first, B3 = first;
    int n = 1;
    V3 dir = -first.w;
    float touch2 = TOUCH2 * fmaxf(len2(first.w), 1.0f);
    GjkResult out;
    out.kind = 0;
    for (int it = 0; it < 64; ++it) {
        Closest cl = gjk_reduce(B0, B1, B2, B3, n);
        if (cl.inside) {
            out.kind = 2;
            out.simplex[0] = B0.w;
            out.simplex[1] = B1.w;
            out.simplex[2] = B2.w;
            out.simplex[3] = B3.w;
            return out;
        }
        V3 v = cl.v;
        float v2 = len2(v);
        if (v2 < touch2) {
            V3 pts[5];
            if (enclosing_walk(cp, fallback, dir, pts)) {
                out.kind = 2;
                for (int i = 0; i < 4; ++i) out.simplex[i] = pts[i];
            } else {
                out.kind = 0;
            }
            return out;
        }
        dir = -v;
        SV w = cp.support(dir);
        float delta = dot(v, w.w);
        float band = msum + thr;
        if (delta > 0.0f && delta * delta > v2 * band * band) { out.kind = 0; return out; }
        bool dup = absdiff_le(w.w, B0.w, 1e-6f);
        if (n > 1 && absdiff_le(w.w, B1.w, 1e-6f)) dup = true;
        if (n > 2 && absdiff_le(w.w, B2.w, 1e-6f)) dup = true;
        if (n > 3 && absdiff_le(w.w, B3.w, 1e-6f)) dup = true;
        if (dup || delta >= v2 * (1.0f - REL2)) {
            float cd = sqrtf(v2);
            float distance = cd - msum;
            if (distance < thr) {
                V3 nn = dir / cd;
                out.kind = 1;
                out.distance = distance;
                out.normal = nn;
                out.point_on_b = cl.pb - nn * mb;
                return out;
            }
            out.kind = 0;
            return out;
        }
        if (n == 1) B1 = w;
        else if (n == 2) B2 = w;
        else B3 = w;
        ++n;
    }
    out.kind = 0;
    return out;
}

// ------------------------------------------------------------------ EPA (epa.rs)
constexpr int EPA_MAX_VERTS = 128;
constexpr int EPA_MAX_FACES = 384;
constexpr int EPA_MAX_EDGES = 384;
constexpr float EPA_EPSILON = 1e-4f;    // epa.rs:34-35
constexpr float EPA_PLANE_EPS = 1e-5f;  // epa.rs:40-41

struct EpaFace {
    V3 n;
    float dist, pdist;
    uint8_t a, b, c, pad;
};

struct EpaScratch {
    V3 v[EPA_MAX_VERTS];
    EpaFace f[EPA_MAX_FACES];
    uint8_t eu[EPA_MAX_EDGES], ev[EPA_MAX_EDGES];
};

// epa.rs:281-303
__device__ __forceinline__ bool edge_distance(V3 pa, V3 pb, V3 n, float& out) {
    V3 ba = pb - pa;
    V3 nab = cross(ba, n);
    if (dot(pa, nab) < 0.0f) {
        float ba_l2 = len2(ba);
        float adb = dot(pa, ba), bdb = dot(pb, ba);
        if (adb > 0.0f) out = len(pa);
        else if (bdb < 0.0f) out = len(pb);
        else {
            float ab = dot(pa, pb);
            out = sqrtf(fmaxf((len2(pa) * len2(pb) - ab * ab) / ba_l2, 0.0f));
        }
        return true;
    }
    return false;
}

// epa.rs:262-275
__device__ __forceinline__ float face_distance(V3 n, V3 pa, V3 pb, V3 pc) {
    float d;
    if (edge_distance(pa, pb, n, d)) return d;
    if (edge_distance(pb, pc, n, d)) return d;
    if (edge_distance(pc, pa, n, d)) return d;
    return dot(pa, n);
}

__device__ __forceinline__ bool face_visible(const EpaFace& f, V3 p) { return dot(f.n, p) - f.pdist > EPA_PLANE_EPS; }

// epa.rs:309-388 — two-phase atomic expansion. Returns 0 ok, 1 degenerate (hull untouched),
// 2 capacity exceeded (hull untouched).
static __device__ __noinline__ int epa_expand(EpaScratch& s, int& nf, V3 np, int nidx) {
    int ne = 0;
    bool any = false;
    for (int fi = 0; fi < nf; ++fi) {
        const EpaFace& f = s.f[fi];
        if (!face_visible(f, np)) continue;
        any = true;
        int es[3][2] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
        for (int e = 0; e < 3; ++e) {
            int u = es[e][0], v = es[e][1];
            int pos = -1;
            for (int i = 0; i < ne; ++i) if (s.eu[i] == v && s.ev[i] == u) { pos = i; break; }
            if (pos >= 0) { s.eu[pos] = s.eu[ne - 1]; s.ev[pos] = s.ev[ne - 1]; --ne; }
            else {
                if (ne >= EPA_MAX_EDGES) return 2;
                s.eu[ne] = uint8_t(u); s.ev[ne] = uint8_t(v); ++ne;
            }
        }
    }
    if (!any) return 0;
    for (int i = 0; i < ne; ++i) {
        V3 cr = cross(s.v[s.ev[i]] - s.v[s.eu[i]], np - s.v[s.eu[i]]);
        if (len(cr) < 1e-12f) return 1;
    }
    int kept = 0;
    for (int fi = 0; fi < nf; ++fi) if (!face_visible(s.f[fi], np)) ++kept;
    if (kept + ne > EPA_MAX_FACES) return 2;
    int w = 0;
    for (int fi = 0; fi < nf; ++fi) {
        if (face_visible(s.f[fi], np)) continue;
        if (w != fi) s.f[w] = s.f[fi];
        ++w;
    }
    nf = w;
    for (int i = 0; i < ne; ++i) {
        int u = s.eu[i], v = s.ev[i];
        V3 cr = cross(s.v[v] - s.v[u], np - s.v[u]);
        float l = len(cr);
        V3 n = cr / l;
        EpaFace f;
        f.n = n;
        f.dist = face_distance(n, s.v[u], s.v[v], np);
        f.pdist = dot(n, s.v[u]);
        f.a = uint8_t(u); f.b = uint8_t(v); f.c = uint8_t(nidx); f.pad = 0;
        s.f[nf++] = f;
    }
    return 0;
}

__device__ __forceinline__ int epa_best(const EpaScratch& s, int nf) {
    int b = 0;
    for (int i = 1; i < nf; ++i) if (fabsf(s.f[i].dist) < fabsf(s.f[b].dist)) b = i;
    return b;
}

// epa.rs:127-205. Returns status bits: 1 = a buffer capacity was hit (result is the intact hull's best face).
static __device__ __noinline__ int epa_penetration(const ConvexPair& cp, const V3* simplex, EpaScratch& s, V3& normal, float& depth) {
    for (int i = 0; i < 4; ++i) s.v[i] = simplex[i];
    int nv = 4, nf = 0;
    const int quads[4][4] = {{0, 1, 2, 3}, {0, 3, 1, 2}, {0, 2, 3, 1}, {1, 3, 2, 0}};
    for (int qi = 0; qi < 4; ++qi) {
        int a = quads[qi][0], b = quads[qi][1], c = quads[qi][2], opp = quads[qi][3];
        V3 n = cross(simplex[b] - simplex[a], simplex[c] - simplex[a]);
        if (dot(n, simplex[opp] - simplex[a]) > 0.0f) { n = -n; int t = b; b = c; c = t; }
        float l = len(n);
        if (l < 1e-12f) continue;
        n = n / l;
        EpaFace f;
        f.n = n;
        f.pdist = dot(n, simplex[a]);
        f.dist = face_distance(n, simplex[a], simplex[b], simplex[c]);
        f.a = uint8_t(a); f.b = uint8_t(b); f.c = uint8_t(c); f.pad = 0;
        s.f[nf++] = f;
    }
    if (nf == 0) { normal = V3{0.f, 0.f, 0.f}; depth = 0.0f; return 0; }
    int status = 0;
    const V3 dirs[6] = {{1.f, 0.f, 0.f}, {-1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, -1.f, 0.f}, {0.f, 0.f, 1.f}, {0.f, 0.f, -1.f}};
    for (int d = 0; d < 6; ++d) {
        V3 p = cp.support(dirs[d]).w;
        int idx = nv;
        s.v[nv++] = p;
        int r = epa_expand(s, nf, p, idx);
        if (r == 2) status |= 1;
        if (r != 0) break;
    }
    for (int it = 0; it < 255; ++it) {
        int bi = epa_best(s, nf);
        V3 bn = s.f[bi].n;
        float bd = s.f[bi].dist;
        V3 np = cp.support(bn).w;
        float wdist = dot(bn, np) - bd;
        if (wdist <= EPA_EPSILON) { normal = bn; depth = bd; return status; }
        if (nv >= EPA_MAX_VERTS) break;
        int nidx = nv;
        s.v[nv++] = np;
        int r = epa_expand(s, nf, np, nidx);
        if (r == 2) status |= 1;
        if (r != 0) break;
    }
    int bi = epa_best(s, nf);
    normal = s.f[bi].n;
    depth = s.f[bi].dist;
    return status;
}

}  // namespace bgpu
