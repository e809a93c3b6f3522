// Pair pass of the step (crates/bullet-dynamics/src/world/step.rs:439-854):
// per broad-phase pair, the group/mask filter, the persistent-manifold
// lookup, the refresh-versus-redetect gate, the narrow phase, the merge of a
// fresh detection into the cached manifold, and the solver-row preparation
// (sequential_impulse.rs:339-550). Three kernels: classify+refresh (one
// thread per pair), narrow phase (analytic routes, then GJK/EPA on its own
// compacted list so EPA's scratch only costs where it runs), and
// capture+refresh+rows for the pairs that were re-detected.
#include <cub/cub.cuh>
#include <cooperative_groups.h>
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

constexpr float REDETECT_SPEED_SQUARED = 0.08f * 0.08f;  // world.rs:62
constexpr float REDRIFT_T = 0.005f;                       // manifold.rs:149-151
constexpr float REDRIFT_ANGLE = 0.01f;

struct Pt {
    V3 la, lb, n;
    float pen, imp;
    uint32_t life;
    uint32_t src;  // index of the point in the entry it was loaded from (0xff: new); not stored
};

struct Entry {
    V3 dpa, dpb;
    Q dqa, dqb;
    float thr;
    uint32_t meta;
    Pt p[4];
    __device__ int count() const { return int(meta & 7u); }
};

__device__ __forceinline__ Entry load_entry(const float4* __restrict__ e) {
    Entry E;
    float4 a = __ldg(&e[0]), b = __ldg(&e[1]), c = __ldg(&e[2]), d = __ldg(&e[3]);
    E.dpa = from4(a);
    E.thr = a.w;
    E.dqa = q4(b);
    E.dpb = from4(c);
    E.meta = __float_as_uint(c.w);
    E.dqb = q4(d);
    int n = E.count();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= n) break;
        float4 x = __ldg(&e[4 + 3 * k]), y = __ldg(&e[5 + 3 * k]), z = __ldg(&e[6 + 3 * k]);
        E.p[k].la = from4(x); E.p[k].pen = x.w;
        E.p[k].lb = from4(y); E.p[k].imp = y.w;
        E.p[k].n = from4(z); E.p[k].life = __float_as_uint(z.w);
        E.p[k].src = uint32_t(k);
    }
    return E;
}

// The point loops below run to a constant bound with a guard, so every E.p / Out index is a
// compile-time constant after unrolling and the arrays stay in registers (a runtime index
// would put them in local memory).
__device__ __forceinline__ void store_entry(float4* e, const Entry& E) {
    e[0] = to4(E.dpa, E.thr);
    e[1] = to4(E.dqa);
    e[2] = to4(E.dpb, __uint_as_float(E.meta));
    e[3] = to4(E.dqb);
    const int n = E.count();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= n) break;
        e[4 + 3 * k] = to4(E.p[k].la, E.p[k].pen);
        e[5 + 3 * k] = to4(E.p[k].lb, E.p[k].imp);
        e[6 + 3 * k] = to4(E.p[k].n, __uint_as_float(E.p[k].life));
    }
}

__device__ __forceinline__ void store_meta_only(float4* e, uint32_t meta) {
    e[2] = make_float4(0.f, 0.f, 0.f, __uint_as_float(meta));
}

__device__ __forceinline__ float rotation_angle(Q q) { return 2.0f * acosf(fminf(fmaxf(q.w, -1.0f), 1.0f)); }

// manifold.rs:287-304
__device__ __forceinline__ bool needs_redetect(const Entry& E, V3 pa, Q qa, V3 pb, Q qb) {
    if (!(E.meta & META_INIT)) return true;
    V3 drift = (pb - E.dpb) - (pa - E.dpa);
    if (len2(drift) > REDRIFT_T * REDRIFT_T) return true;
    Q ra = qmul(qa, qinv(E.dqa));
    Q rb = qmul(qb, qinv(E.dqb));
    return rotation_angle(ra) + rotation_angle(rb) > REDRIFT_ANGLE;
}

struct Out {
    int n;
    V3 pos[4], nrm[4];
    float pen[4], imp[4];
    uint32_t src[4];  // the loaded entry's index of the point each row comes from (0xff: new point)
};

// manifold.rs:246-282: a point survives while its penetration stays above -thr and its lateral
// drift below thr. The survivors keep their order (out k addresses surviving point k); they are
// not moved here: K marks them, and store_entry_kept / emit_rows_kept write them compacted to
// global memory, so no runtime index touches E.p and the entry stays in registers.
struct Kept {
    bool k[4];
    V3 wb[4];  // the survivor's world point on B
    int n;
};

__device__ __forceinline__ void refresh(Entry& E, V3 pa, Q qa, V3 pb, Q qb, Kept& K) {
    const float thr = E.thr, thr_sq = thr * thr;
    const int n = E.count();
    K.n = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        K.k[k] = false;
        K.wb[k] = V3{0.0f, 0.0f, 0.0f};
        if (k < n) {
            Pt& p = E.p[k];
            const V3 wa = pa + rotate(qa, p.la);
            const V3 wb = pb + rotate(qb, p.lb);
            const V3 d = wa - wb;
            const float pen = dot(d, p.n);
            if (!(pen < -thr)) {
                const V3 lat = d - p.n * pen;
                if (!(len2(lat) > thr_sq)) {
                    p.pen = pen;
                    p.life += 1;
                    K.wb[k] = wb;
                    K.k[k] = true;
                    ++K.n;
                }
            }
        }
    }
}

// The refreshed entry: header, count = survivors, survivors in order.
__device__ __forceinline__ void store_entry_kept(float4* e, const Entry& E, const Kept& K) {
    e[0] = to4(E.dpa, E.thr);
    e[1] = to4(E.dqa);
    e[2] = to4(E.dpb, __uint_as_float((E.meta & ~7u) | uint32_t(K.n)));
    e[3] = to4(E.dqb);
    int s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!K.k[k]) continue;
        e[4 + 3 * s] = to4(E.p[k].la, E.p[k].pen);
        e[5 + 3 * s] = to4(E.p[k].lb, E.p[k].imp);
        e[6 + 3 * s] = to4(E.p[k].n, __uint_as_float(E.p[k].life));
        ++s;
    }
}

__device__ __forceinline__ int32_t total_key(float v) {
    int32_t b = __float_as_int(v);
    return b ^ int32_t(uint32_t(b >> 31) >> 1);
}

// manifold.rs:326-376. pts holds the up to 8 candidate points of this thread (the cached ones,
// then the new ones that match none), pts[k * stride]: k_capture keeps them in shared memory,
// where a runtime index costs nothing.
__device__ __forceinline__ void capture(Entry& E, const Manifold& m, V3 pa, Q qa, V3 pb, Q qb, float thr, Pt* pts,
                                        uint32_t stride) {
    E.thr = thr;
    Q ia = qinv(qa), ib = qinv(qb);
    float thr_sq = thr * thr;
    auto P = [&](int k) -> Pt& { return pts[size_t(k) * stride]; };
    int n = E.count();
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (k < n) P(k) = E.p[k];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (c >= m.n) break;
        V3 wb = m.pos[c];
        V3 wa = m.pos[c] + m.nrm[c] * m.pen[c];
        Pt pt;
        pt.la = rotate(ia, wa - pa);
        pt.lb = rotate(ib, wb - pb);
        pt.n = m.nrm[c];
        pt.pen = m.pen[c];
        pt.imp = 0.0f;
        pt.life = 0;
        pt.src = 0xffu;
        bool matched = false;
        for (int k = 0; k < n; ++k) {
            Pt& q = P(k);
            if (len2(q.la - pt.la) < thr_sq && dot(q.n, pt.n) >= 0.9f) {
                pt.imp = q.imp;
                pt.src = q.src;
                q = pt;
                matched = true;
                break;
            }
        }
        if (!matched) P(n++) = pt;
    }
    if (n > 4) {  // stable descending sort by penetration (total order), keep four
        for (int a = 1; a < n; ++a) {
            Pt v = P(a);
            int32_t kv = total_key(v.pen);
            int b = a;
            while (b > 0 && total_key(P(b - 1).pen) < kv) { P(b) = P(b - 1); --b; }
            P(b) = v;
        }
        n = 4;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (k < n) E.p[k] = P(k);
    E.dpa = pa; E.dqa = qa; E.dpb = pb; E.dqb = qb;
    E.meta = (E.meta & ~7u) | uint32_t(n) | META_INIT | META_VALID;
}

__device__ __forceinline__ M3 load_iw(const float4* __restrict__ iw, uint32_t i, float& inv_mass) {
    float4 a = iw[3 * i], b = iw[3 * i + 1], c = iw[3 * i + 2];
    inv_mass = c.y;
    return M3{V3{a.x, a.y, a.z}, V3{a.w, b.x, b.y}, V3{b.z, b.w, c.x}};
}

// sequential_impulse.rs:655-673
__device__ __forceinline__ float effective_mass(float ima, float imb, V3 aa, V3 ab, V3 ra, V3 rb, V3 d) {
    float k = ima + imb + dot(d, cross(aa, ra)) + dot(d, cross(ab, rb));
    return k > 0.0f ? 1.0f / k : 0.0f;
}

// step.rs:750-764 + sequential_impulse.rs:339-550: one prepared row per refreshed point.
// rec_row_src (adjoint recording, else null) receives, per row, the old cache position * 4 + point
// index that supplied its warm-start impulse (old: the pair's old cache position, or -1).
struct RowCtx {
    float ima, imb;
    M3 iwa, iwb;
    V3 posa, posb;
    float4 ma, mb;
};

__device__ __forceinline__ RowCtx row_ctx(const BodyDev& b, uint32_t i, uint32_t j) {
    RowCtx c;
    c.iwa = load_iw(b.iw, i, c.ima);
    c.iwb = load_iw(b.iw, j, c.imb);
    c.posa = from4(b.pos[i]);
    c.posb = from4(b.pos[j]);
    c.ma = b.material[i];
    c.mb = b.material[j];
    return c;
}

__device__ __forceinline__ void emit_row(const RowCtx& c, const StepParams& sp, V3 pos, V3 n, float pen,
                                         float imp_cached, float4* r) {
    const SolverParams& info = sp.info;
    const float inv_dt = sp.inv_dt;
    const float ima = c.ima, imb = c.imb;
    const M3& iwa = c.iwa;
    const M3& iwb = c.iwb;
    float imp = imp_cached * info.warmstarting_factor;
    V3 t1, t2;
    tangent_basis_dev(n, t1, t2);
    V3 ra = pos - c.posa;
    V3 rb = pos - c.posb;
    V3 ana = mul(iwa, cross(ra, n)), anb = mul(iwb, cross(rb, n));
    V3 a1a = mul(iwa, cross(ra, t1)), a1b = mul(iwb, cross(rb, t1));
    V3 a2a = mul(iwa, cross(ra, t2)), a2b = mul(iwb, cross(rb, t2));
    float nm = effective_mass(ima, imb, ana, anb, ra, rb, n);
    float t1m = effective_mass(ima, imb, a1a, a1b, ra, rb, t1);
    float t2m = effective_mass(ima, imb, a2a, a2b, ra, rb, t2);
    float friction = c.ma.x * c.mb.x;
    float restitution = c.ma.y * c.mb.y;
    float erp = info.erp2;
    float ncfm = 0.0f;
    float cfm_global = info.global_cfm * inv_dt;
    if (cfm_global != 0.0f || info.sor != 1.0f) {
        float kk = nm > 0.0f ? 1.0f / nm : 0.0f;
        nm = kk + cfm_global > 0.0f ? info.sor / (kk + cfm_global) : 0.0f;
        ncfm = cfm_global * nm;
    }
    if (info.sor != 1.0f) { t1m *= info.sor; t2m *= info.sor; }
    float span = fmaxf(pen - info.linear_slop, 0.0f);
    float separation = fminf(pen, 0.0f);
    bool split = info.split_impulse != 0 && pen > -info.split_impulse_penetration_threshold;
    float baum = split ? 0.0f : erp * inv_dt * span;
    float sepb = separation < 0.0f ? separation * inv_dt : 0.0f;
    float rhs = split ? pen * erp * inv_dt * nm : 0.0f;
    r[0] = to4(n, friction);
    r[1] = to4(ra, baum);
    r[2] = to4(rb, sepb);
    r[3] = make_float4(imp, 0.0f, 0.0f, restitution);
    r[4] = make_float4(nm, t1m, t2m, ncfm);
    r[5] = make_float4(rhs, 0.0f, split ? 1.0f : 0.0f, pen);
}

// Rows of explicit contact points (the stand-alone row preparation).
__device__ __forceinline__ void emit_rows(const BodyDev& b, uint32_t i, uint32_t j, const Out& o, const StepParams& sp,
                                          float4* __restrict__ rows, uint32_t* __restrict__ row_count, uint32_t p,
                                          uint32_t* rec_row_src, int64_t old) {
    const RowCtx c = row_ctx(b, i, j);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= o.n) break;
        emit_row(c, sp, o.pos[k], o.nrm[k], o.pen[k], o.imp[k], rows + (size_t(p) * 4 + k) * ROW_F4);
        if (rec_row_src)
            rec_row_src[size_t(p) * 4 + k] = (old >= 0 && o.src[k] < 4u) ? uint32_t(old) * 4u + o.src[k] : REC_NONE;
    }
    row_count[p] = uint32_t(o.n);
}

// Rows of an entry's refreshed survivors, in order.
__device__ __forceinline__ void emit_rows_kept(const BodyDev& b, uint32_t i, uint32_t j, const Entry& E, const Kept& K,
                                               const StepParams& sp, float4* __restrict__ rows,
                                               uint32_t* __restrict__ row_count, uint32_t p, uint32_t* rec_row_src,
                                               int64_t old) {
    const RowCtx c = row_ctx(b, i, j);
    int s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!K.k[k]) continue;
        emit_row(c, sp, K.wb[k], E.p[k].n, E.p[k].pen, E.p[k].imp, rows + (size_t(p) * 4 + s) * ROW_F4);
        if (rec_row_src)
            rec_row_src[size_t(p) * 4 + s] =
                (old >= 0 && E.p[k].src < 4u) ? uint32_t(old) * 4u + E.p[k].src : REC_NONE;
        ++s;
    }
    row_count[p] = uint32_t(K.n);
}

__device__ __forceinline__ uint32_t route_of(uint32_t ta, uint32_t tb) {
    if (ta == SHAPE_PLANE && tb == SHAPE_PLANE) return NP_NONE;
    if (ta == SHAPE_MESH || tb == SHAPE_MESH) {  // mod.rs:102-243: convex vs mesh only (meshes are static here)
        const uint32_t other = ta == SHAPE_MESH ? tb : ta;
        return (other == SHAPE_MESH || other == SHAPE_PLANE) ? NP_NONE : NP_MESH;
    }
    if (ta == SHAPE_PLANE) return NP_PLANE_A;
    if (tb == SHAPE_PLANE) return NP_PLANE_B;
    if (ta == SHAPE_SPHERE && tb == SHAPE_SPHERE) return NP_SPHERE_SPHERE;
    if (ta == SHAPE_SPHERE && tb == SHAPE_BOX) return NP_SPHERE_BOX;
    if (ta == SHAPE_BOX && tb == SHAPE_SPHERE) return NP_BOX_SPHERE;
    if (ta == SHAPE_BOX && tb == SHAPE_BOX) return NP_BOX_BOX;
    return NP_CONVEX;
}

// Position of k in the sorted keys[0, n), or -1. The search starts with a galloping
// probe around `guess` (from step to step a pair keeps nearly the same rank among the
// sorted pairs, so the key is usually a few places away) and ends with a binary search
// of the bracket it found: a few dependent loads instead of log2(n).
__device__ __forceinline__ int64_t find_key(const uint64_t* __restrict__ keys, uint32_t n, uint64_t k, uint32_t guess) {
    if (n == 0) return -1;
    uint32_t lo, hi;  // the answer (first index with keys[i] >= k) lies in [lo, hi]
    const uint32_t g = guess < n ? guess : n - 1;
    if (keys[g] < k) {
        lo = g + 1;
        uint32_t step = 1;
        hi = n;
        while (lo + step - 1 < n) {
            const uint32_t probe = lo + step - 1;
            if (keys[probe] >= k) { hi = probe; break; }
            lo = probe + 1;
            step <<= 1;
        }
    } else {
        hi = g;
        uint32_t step = 1;
        lo = 0;
        while (hi >= step) {
            const uint32_t probe = hi - step;
            if (keys[probe] < k) { lo = probe + 1; break; }
            hi = probe;
            step <<= 1;
        }
    }
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == k) ? int64_t(lo) : -1;
}


__device__ __forceinline__ bool active_state(uint32_t a) {
    return a == ACT_ACTIVE || a == ACT_WANTS_DEACTIVATION || a == ACT_DISABLE_DEACTIVATION;
}

// One atomicAdd per distinct route among the calling lanes of a warp.
__device__ __forceinline__ uint32_t claim_route_slot(uint32_t* counts, uint32_t route) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, route);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = uint32_t(__ffs(int(peers)) - 1);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&counts[route], uint32_t(__popc(int(peers))));
    base = __shfl_sync(peers, base, int(leader));
    return base + uint32_t(__popc(peers & ((1u << lane) - 1u)));
}

// Position t of the detection lists (the analytic routes in route order, then the
// convex list) -> pair id. counts = the scalars from ROUTE_COUNT0 (index = route).
__device__ __forceinline__ uint32_t detect_list_pair(const uint32_t* __restrict__ list, const uint32_t* counts,
                                                     uint32_t npairs, uint32_t t, uint32_t last_route) {
    for (uint32_t r = NP_PLANE_A; r <= last_route; ++r) {
        if (t < counts[r]) return list[size_t(r - 1) * npairs + t];
        t -= counts[r];
    }
    return 0xffffffffu;
}

// step.rs:645-799, classify + refresh path. Scalars: [0] analytic list count, [1] convex list count.
__global__ void k_classify(BodyDev b, const Shape* __restrict__ shapes, const uint64_t* __restrict__ pairs,
                           uint32_t npairs, const uint64_t* __restrict__ old_keys, const float4* __restrict__ old_entries,
                           const uint32_t* __restrict__ old_count_ptr, StepParams sp, PairDataDev pd) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    uint64_t key = pairs[p];
    uint32_t i = key_lo(key), j = key_hi(key);
    uint4 ia = b.info[i], ib = b.info[j];
    float4* ne = pd.entries + size_t(p) * ENTRY_F4;
    pd.row_count[p] = 0;
    pd.detect_n[p] = 0;
    uint32_t ga = ia.w & 0xffffu, mka = ia.w >> 16, gb = ib.w & 0xffffu, mkb = ib.w >> 16;
    // step.rs:645-651: pairs linked by a joint with disable_collisions are skipped like
    // group/mask rejects.
    const bool suppressed = sp.nsuppressed && find_key(sp.suppressed, sp.nsuppressed, key, 0) >= 0;
    if (suppressed || (ga & mkb) == 0 || (gb & mka) == 0) {
        pd.status[p] = PS_NONE;
        store_meta_only(ne, 0u);
        return;
    }
    uint32_t old_count = *old_count_ptr;
    const uint32_t guess = uint32_t((uint64_t(p) * old_count) / npairs);
    int64_t old = old_count ? find_key(old_keys, old_count, key, guess) : -1;
    if (old >= 0) pd.old_owned[old] = 1u;
    bool act_a = active_state(ia.z), act_b = active_state(ib.z);
    bool sk_a = (ia.y & (BF_STATIC | BF_KINEMATIC)) != 0, sk_b = (ib.y & (BF_STATIC | BF_KINEMATIC)) != 0;
    if ((!act_a && !act_b) || (sk_a && sk_b)) {
        // step.rs:677-715: a sleeping island / immovable pair keeps its manifold verbatim.
        pd.status[p] = PS_KEEP;
        if (old >= 0) {
            const float4* oe = old_entries + size_t(old) * ENTRY_F4;
            for (int t = 0; t < ENTRY_F4; ++t) ne[t] = __ldg(&oe[t]);
        } else {
            store_meta_only(ne, 0u);
        }
        return;
    }
    bool no_response = ((ia.y | ib.y) & BF_NO_RESPONSE) != 0;
    V3 pa = from4(b.pred[i]), pb = from4(b.pred[j]);
    Q qa = q4(b.quat[i]), qb = q4(b.quat[j]);
    bool fast = b.settled[i] > REDETECT_SPEED_SQUARED || b.settled[j] > REDETECT_SPEED_SQUARED;
    Entry E;
    E.meta = 0;
    if (old >= 0) E = load_entry(old_entries + size_t(old) * ENTRY_F4);
    Kept K;
    K.n = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) K.k[k] = k < E.count();  // no refresh: the loaded points as they are
    if (old >= 0 && !needs_redetect(E, pa, qa, pb, qb)) {
        refresh(E, pa, qa, pb, qb, K);
        bool deep = false;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (K.k[k] && E.p[k].pen > sp.info.linear_slop) deep = true;
        if (!fast || !deep) {
            store_entry_kept(ne, E, K);
            if (!no_response) emit_rows_kept(b, i, j, E, K, sp, pd.rows, pd.row_count, p, pd.rec.row_src, old);
            pd.status[p] = PS_SERVED;
            return;
        }
    } else {
        K.n = E.count();
    }
    if (old >= 0) store_entry_kept(ne, E, K);
    else store_meta_only(ne, 0u);
    if (pd.rec.pt_src) {  // where the stored points came from, for the capture pass
        pd.rec.pair_old[p] = old >= 0 ? uint32_t(old) : REC_NONE;
        uint32_t packed = 0xffffffffu;  // byte s: the source of stored point s
        int s = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (old >= 0 && K.k[k]) {
                packed = (packed & ~(0xffu << (8 * s))) | ((E.p[k].src & 0xffu) << (8 * s));
                ++s;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) pd.rec.pt_src[size_t(p) * 4 + k] = uint8_t(packed >> (8 * k));
    }
    uint32_t route = route_of(shapes[ia.x].type, shapes[ib.x].type);
    pd.status[p] = PS_DETECT | (route << 8);
    if (route == NP_NONE) return;
    // One list per route (route r in [(r - 1) P, r P), P = npairs), so that the narrow
    // phase's warps run one shape routine each instead of every route their lanes hold.
    const uint32_t slot = claim_route_slot(&pd.scalars[ROUTE_COUNT0], route);
    pd.route_list[size_t(route - 1) * npairs + slot] = p;
}

// narrowphase/mod.rs:63-286 for one pair; returns the manifold (positions on B, normals A->B).
__device__ __forceinline__ void collide_analytic(uint32_t route, const Shape& sa, V3 pa, Q qa, const Shape& sb, V3 pb,
                                                 Q qb, const float4* __restrict__ hull, Manifold& m, BoxBoxScratch& bbs) {
    float thr = fminf(sa.cbt, sb.cbt);
    m.n = 0;
    switch (route) {
        case NP_PLANE_A: plane_convex(sa, pa, qa, sb, pb, qb, thr, hull, m); break;
        case NP_PLANE_B:
            if (plane_convex(sb, pb, qb, sa, pa, qa, thr, hull, m)) mf_flip(m);
            break;
        case NP_SPHERE_SPHERE: sphere_sphere(sa.p0, pa, sb.p0, pb, m); break;
        case NP_SPHERE_BOX:
            if (sphere_box(sa.p0, pa, V3{sb.p0, sb.p1, sb.p2}, pb, qb, thr, m)) mf_flip(m);
            break;
        case NP_BOX_SPHERE: sphere_box(sb.p0, pb, V3{sa.p0, sa.p1, sa.p2}, pa, qa, thr, m); break;
        case NP_BOX_BOX: box_box(V3{sa.p0, sa.p1, sa.p2}, pa, qa, V3{sb.p0, sb.p1, sb.p2}, pb, qb, m, bbs); break;
        default: break;
    }
}

// convex_convex.rs:30-155
__device__ __noinline__ void collide_convex(const Shape& sa, V3 pa, Q qa, const Shape& sb, V3 pb, Q qb, bool has_seed,
                                            V3 seed, const float4* __restrict__ hull, EpaScratch& scratch, Manifold& m,
                                            uint32_t* status) {
    m.n = 0;
    float thr = fminf(sa.cbt, sb.cbt);
    ConvexPair cp;
    cp.sa = &sa; cp.sb = &sb; cp.pa = pa; cp.pb = pb; cp.qa = qa; cp.qb = qb; cp.hull = hull;
    GjkResult g = gjk_contact(cp, has_seed, seed, thr);
    if (g.kind == 0) return;
    if (g.kind == 1) {
        mf_push(m, g.point_on_b, g.normal, -g.distance);
        return;
    }
    V3 n;
    float core_depth;
    if (epa_penetration(cp, g.simplex, scratch, n, core_depth)) atomicOr(status, ST_EPA_CAPACITY);
    if (core_depth <= 0.0f) return;
    float depth = core_depth + sa.margin + sb.margin;
    V3 point_a = support_world(sa, pa, qa, n, hull);
    mf_push(m, point_a - n * depth, n, depth);
}

// ---------------------------------------------------------------- convex vs static mesh
// narrowphase/convex_mesh.rs:26-153. The convex's world AABB, swept into the mesh frame, picks
// candidate triangles from the mesh BVH (bvh.rs:45-66, the same stack walk: left pushed first,
// so the right child is visited first); each candidate whose own AABB overlaps the query runs
// the sphere detector (spheres) or convex_convex against the triangle as a three-vertex hull;
// the points then reduce to four (manifold.rs:80-108). Normals point from the convex to the mesh.
constexpr int MESH_MAX_CAND = 64;   // candidate points per pair (more: ST_MESH_CANDIDATES)
constexpr int MESH_STACK = 64;      // BVH walk depth

// convex_mesh.rs:236-253
__device__ __forceinline__ float seg_closest_sq(V3 from, V3 to, V3 p, V3& nearest) {
    const V3 v = to - from;
    float t = dot(v, p - from);
    if (t > 0.0f) {
        const float dvv = dot(v, v);
        if (t < dvv) t /= dvv;
        else t = 1.0f;
    } else {
        t = 0.0f;
    }
    nearest = from + v * t;
    return len2(p - nearest);
}

// convex_mesh.rs:160-232: point on the triangle, normal toward the centre, radius - distance.
__device__ __forceinline__ bool sphere_triangle(V3 center, float radius, float threshold, V3 a, V3 b, V3 c, V3& point,
                                                V3& normal_out, float& pen) {
    const float rwt = radius + threshold;
    V3 normal = cross(b - a, c - a);
    const float l2 = len2(normal);
    const float eps = 1.1920929e-7f;  // f32::EPSILON
    if (l2 < eps * eps) return false;
    normal = normal * (1.0f / sqrtf(l2));
    float dist = dot(normal, center - a);
    if (dist < 0.0f) {
        dist = -dist;
        normal = -normal;
    }
    if (dist >= rwt) return false;
    V3 cp;
    // convex_mesh.rs:257-268 point_in_triangle
    const float r1 = dot(cross(b - a, normal), center - a), r2 = dot(cross(c - b, normal), center - b),
                r3 = dot(cross(a - c, normal), center - c);
    if ((r1 > 0.0f && r2 > 0.0f && r3 > 0.0f) || (r1 <= 0.0f && r2 <= 0.0f && r3 <= 0.0f)) {
        cp = center - normal * dist;
    } else {
        float min_d = rwt * rwt;
        bool found = false;
        V3 on;
        float d = seg_closest_sq(a, b, center, on);
        if (d < min_d) { min_d = d; cp = on; found = true; }
        d = seg_closest_sq(b, c, center, on);
        if (d < min_d) { min_d = d; cp = on; found = true; }
        d = seg_closest_sq(c, a, center, on);
        if (d < min_d) { min_d = d; cp = on; found = true; }
        if (!found) return false;
    }
    const V3 to_c = center - cp;
    const float d2 = len2(to_c);
    if (d2 >= rwt * rwt) return false;
    point = cp;
    if (d2 > eps) {
        const float d = sqrtf(d2);
        normal_out = to_c * (1.0f / d);
        pen = radius - d;
    } else {
        normal_out = normal;
        pen = radius;
    }
    return true;
}

struct MeshCandidates {
    int n;
    V3 pos[MESH_MAX_CAND];
    V3 nrm[MESH_MAX_CAND];
    float pen[MESH_MAX_CAND];
};

// manifold.rs:80-108: deepest first (stable), then greedily the farthest from the kept points.
__device__ __forceinline__ void reduce_to_manifold(const MeshCandidates& c, Manifold& m) {
    m.n = 0;
    if (c.n <= 4) {
        for (int i = 0; i < c.n; ++i) mf_push(m, c.pos[i], c.nrm[i], c.pen[i]);
        return;
    }
    uint8_t ord[MESH_MAX_CAND];
    for (int i = 0; i < c.n; ++i) {  // stable insertion sort by penetration, deepest first
        int j = i;
        while (j > 0 && c.pen[ord[j - 1]] < c.pen[i]) {
            ord[j] = ord[j - 1];
            --j;
        }
        ord[j] = uint8_t(i);
    }
    uint64_t used = 1ull;  // bit s: sorted position s taken
    int kept[4] = {ord[0], 0, 0, 0};
    int nk = 1;
    while (nk < 4) {
        int best = 0;
        float best_sep = -INFINITY;
        for (int s = 0; s < c.n; ++s) {
            if (used & (1ull << s)) continue;
            float sep = INFINITY;
            for (int q = 0; q < nk; ++q) sep = fminf(sep, len2(c.pos[ord[s]] - c.pos[kept[q]]));
            if (sep > best_sep) { best_sep = sep; best = s; }
        }
        kept[nk++] = ord[best];
        used |= 1ull << best;
    }
    for (int q = 0; q < 4; ++q) mf_push(m, c.pos[kept[q]], c.nrm[kept[q]], c.pen[kept[q]]);
}

__device__ __noinline__ void collide_mesh(const Shape& cv, V3 pc, Q qc, const Shape& ms, V3 pm, Q qm, bool has_seed,
                                          V3 seed, const float4* __restrict__ hull, EpaScratch& scratch, Manifold& m,
                                          uint32_t* status) {
    m.n = 0;
    const float thr = fminf(cv.cbt, ms.cbt);
    V3 wmn, wmx;
    world_aabb(cv, pc, qc, hull, wmn, wmx);
    const Q inv_m = qinv(qm);
    const V3 c = (wmn + wmx) * 0.5f, e = (wmx - wmn) * 0.5f;
    V3 lmin = splat(INFINITY), lmax = splat(-INFINITY);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const V3 corner = V3{(i & 1) == 0 ? c.x + e.x : c.x - e.x, (i & 2) == 0 ? c.y + e.y : c.y - e.y,
                             (i & 4) == 0 ? c.z + e.z : c.z - e.z};
        const V3 p = rotate(inv_m, corner - pm);
        lmin = vmin(lmin, p);
        lmax = vmax(lmax, p);
    }
    auto overlaps = [&](V3 a0, V3 a1) {  // util.rs:28-38, closed
        return a0.x <= lmax.x && a0.y <= lmax.y && a0.z <= lmax.z && lmin.x <= a1.x && lmin.y <= a1.y && lmin.z <= a1.z;
    };
    const bool sphere = cv.type == SHAPE_SPHERE;
    const V3 center = rotate(inv_m, pc - pm);
    const uint32_t tri_base = mesh_tri_base(ms);
    Shape tri;  // the candidate triangle as a three-vertex hull (margin 0)
    tri.type = SHAPE_HULL;
    tri.hull_cnt = 3;
    tri.margin = 0.0f;
    tri.cbt = thr;
    MeshCandidates cand;
    cand.n = 0;
    uint32_t stack[MESH_STACK];
    int sp = 0;
    if (ms.hull_cnt) stack[sp++] = 0;
    while (sp > 0) {
        const uint32_t k = stack[--sp];
        const float4 n0 = hull[ms.hull_off + 2 * k], n1 = hull[ms.hull_off + 2 * k + 1];
        if (!overlaps(from4(n0), from4(n1))) continue;
        const uint32_t na = __float_as_uint(n0.w), nb = __float_as_uint(n1.w);
        if (!(na & MESH_LEAF)) {
            if (sp + 2 > MESH_STACK) {
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
            const V3 a = from4(hull[o]), b = from4(hull[o + 1]), cc = from4(hull[o + 2]);
            if (!overlaps(vmin(a, vmin(b, cc)), vmax(a, vmax(b, cc)))) continue;  // triangle_mesh.rs:98-112 boxes
            V3 pt, nl;
            float pen;
            bool hit = false;
            if (sphere) {
                if (sphere_triangle(center, cv.p0, thr, a, b, cc, pt, nl, pen)) {
                    pt = pm + rotate(qm, pt);
                    nl = rotate(qm, -nl);
                    hit = true;
                }
            } else {
                tri.hull_off = o;
                Manifold one;
                collide_convex(cv, pc, qc, tri, pm, qm, has_seed, seed, hull, scratch, one, status);
                if (one.n) {
                    pt = one.pos[0];
                    nl = one.nrm[0];
                    pen = one.pen[0];
                    hit = true;
                }
            }
            if (!hit) continue;
            if (cand.n == MESH_MAX_CAND) {
                atomicOr(status, ST_MESH_CANDIDATES);
                continue;
            }
            cand.pos[cand.n] = pt;
            cand.nrm[cand.n] = nl;
            cand.pen[cand.n] = pen;
            ++cand.n;
        }
    }
    reduce_to_manifold(cand, m);
}

// One pair on the mesh route: the convex side against the mesh side (mod.rs:200-243); with the
// mesh first the manifold is flipped.
__device__ __forceinline__ void collide_mesh_pair(const Shape& sa, V3 pa, Q qa, const Shape& sb, V3 pb, Q qb,
                                                  bool has_seed, V3 seed, const float4* __restrict__ hull,
                                                  EpaScratch& scratch, Manifold& m, uint32_t* status) {
    if (sa.type == SHAPE_MESH) {
        collide_mesh(sb, pb, qb, sa, pa, qa, has_seed, seed, hull, scratch, m, status);
        mf_flip(m);
    } else {
        collide_mesh(sa, pa, qa, sb, pb, qb, has_seed, seed, hull, scratch, m, status);
    }
}

// A detection with points goes to the capture list; one without drops the pair's manifold
// here (step.rs:800-853: an empty detection removes it), so the capture pass only runs
// where there is something to merge.
__device__ __forceinline__ void store_detection(PairDataDev& pd, uint32_t p, uint32_t npairs, const Manifold& m) {
    float4* d = pd.detect + size_t(p) * 8;
    for (int k = 0; k < m.n; ++k) {
        d[2 * k] = to4(m.pos[k], m.pen[k]);
        d[2 * k + 1] = to4(m.nrm[k], 0.0f);
    }
    pd.detect_n[p] = uint32_t(m.n);
    if (m.n == 0) {
        store_meta_only(pd.entries + size_t(p) * ENTRY_F4, 0u);
        return;
    }
    cooperative_groups::coalesced_group g = cooperative_groups::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(&pd.scalars[CAPTURE_COUNT], g.size());
    base = g.shfl(base, 0);
    pd.route_list[size_t(CAPTURE_LIST) * npairs + base + g.thread_rank()] = p;
}

__device__ __forceinline__ bool entry_seed(const float4* __restrict__ e, V3& s) {
    float4 c = e[2];
    uint32_t meta = __float_as_uint(c.w);
    if (!(meta & META_VALID) || (meta & 7u) == 0) return false;
    float4 z = e[6];
    V3 n = from4(z);
    if (len2(n) > 0.5f) { s = n; return true; }
    return false;
}

constexpr uint32_t NARROW_ANALYTIC_TB = 128;

__global__ __launch_bounds__(NARROW_ANALYTIC_TB) void k_narrow_analytic(BodyDev b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                  const uint64_t* __restrict__ pairs, uint32_t npairs, PairDataDev pd) {
    __shared__ BoxBoxScratch s_bbs[NARROW_ANALYTIC_TB];
    uint32_t counts[NP_CONVEX + 1];
    uint32_t cnt = 0;
#pragma unroll
    for (uint32_t r = 0; r <= NP_CONVEX; ++r) {
        counts[r] = pd.scalars[ROUTE_COUNT0 + r];
        if (r >= NP_PLANE_A && r < NP_CONVEX) cnt += counts[r];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) pd.scalars[0] = cnt;  // analytic detections (step statistics)
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        uint32_t p = detect_list_pair(pd.route_list, counts, npairs, t, NP_BOX_BOX);
        uint64_t key = pairs[p];
        uint32_t i = key_lo(key), j = key_hi(key);
        uint4 ia = b.info[i], ib = b.info[j];
        Shape sa = shapes[ia.x], sb = shapes[ib.x];
        Manifold m;
        collide_analytic(pd.status[p] >> 8, sa, from4(b.pred[i]), q4(b.quat[i]), sb, from4(b.pred[j]), q4(b.quat[j]),
                         hull, m, s_bbs[threadIdx.x]);
        store_detection(pd, p, npairs, m);
    }
}

__global__ void k_narrow_convex(BodyDev b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                const uint64_t* __restrict__ pairs, uint32_t npairs, PairDataDev pd, uint32_t* status) {
    uint32_t cnt = pd.scalars[ROUTE_COUNT0 + NP_CONVEX];
    if (blockIdx.x == 0 && threadIdx.x == 0) pd.scalars[1] = cnt;  // convex detections (step statistics)
    EpaScratch scratch;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        uint32_t p = pd.route_list[size_t(NP_CONVEX - 1) * npairs + t];
        uint64_t key = pairs[p];
        uint32_t i = key_lo(key), j = key_hi(key);
        uint4 ia = b.info[i], ib = b.info[j];
        Shape sa = shapes[ia.x], sb = shapes[ib.x];
        V3 seed = V3{0.f, 0.f, 0.f};
        bool has_seed = entry_seed(pd.entries + size_t(p) * ENTRY_F4, seed);
        Manifold m;
        collide_convex(sa, from4(b.pred[i]), q4(b.quat[i]), sb, from4(b.pred[j]), q4(b.quat[j]), has_seed, seed, hull,
                       scratch, m, status);
        store_detection(pd, p, npairs, m);
    }
}

// The mesh route of the pair pass: one warp per pair. Lane 0 walks the mesh BVH and lists the
// candidate triangles (those whose own box overlaps the query) in walk order; the lanes run the
// per-triangle detectors side by side; lane 0 then keeps the hits in candidate order and reduces
// them (the same points, in the same order, as collide_mesh's single pass).
constexpr int MESH_WARPS = 4;
constexpr int MESH_MAX_TRIS = 128;  // candidate triangles per pair (more: ST_MESH_CANDIDATES)

__global__ void __launch_bounds__(32 * MESH_WARPS) k_narrow_mesh(BodyDev b, const Shape* __restrict__ shapes,
                                                                 const float4* __restrict__ hull,
                                                                 const uint64_t* __restrict__ pairs, uint32_t npairs,
                                                                 PairDataDev pd, uint32_t* status) {
    __shared__ uint32_t s_slot[MESH_WARPS][MESH_MAX_TRIS];
    __shared__ float4 s_pt[MESH_WARPS][MESH_MAX_TRIS], s_nr[MESH_WARPS][MESH_MAX_TRIS];
    __shared__ uint32_t s_n[MESH_WARPS];
    const uint32_t cnt = pd.scalars[ROUTE_COUNT0 + NP_MESH];
    if (blockIdx.x == 0 && threadIdx.x == 0) pd.scalars[1] += cnt;  // with the convex detections (statistics)
    const uint32_t wi = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    EpaScratch scratch;
    for (uint32_t t = blockIdx.x * MESH_WARPS + wi; t < cnt; t += gridDim.x * MESH_WARPS) {
        const uint32_t p = pd.route_list[size_t(NP_MESH - 1) * npairs + t];
        const uint64_t key = pairs[p];
        const uint32_t i = key_lo(key), j = key_hi(key);
        const Shape sa = shapes[b.info[i].x], sb = shapes[b.info[j].x];
        const bool mesh_a = sa.type == SHAPE_MESH;
        const Shape& cv = mesh_a ? sb : sa;
        const Shape& ms = mesh_a ? sa : sb;
        const uint32_t ic = mesh_a ? j : i, im = mesh_a ? i : j;
        const V3 pc = from4(b.pred[ic]), pm = from4(b.pred[im]);
        const Q qc = q4(b.quat[ic]), qm = q4(b.quat[im]);
        V3 seed = V3{0.f, 0.f, 0.f};
        const bool has_seed = entry_seed(pd.entries + size_t(p) * ENTRY_F4, seed);
        const float thr = fminf(cv.cbt, ms.cbt);
        const uint32_t tri_base = mesh_tri_base(ms);
        if (lane == 0) {  // convex_mesh.rs:37-60 query box, bvh.rs:45-66 walk, triangle box filter
            V3 wmn, wmx;
            world_aabb(cv, pc, qc, hull, wmn, wmx);
            const Q inv_m = qinv(qm);
            const V3 c = (wmn + wmx) * 0.5f, e = (wmx - wmn) * 0.5f;
            V3 lmin = splat(INFINITY), lmax = splat(-INFINITY);
            for (int k = 0; k < 8; ++k) {
                const V3 corner = V3{(k & 1) == 0 ? c.x + e.x : c.x - e.x, (k & 2) == 0 ? c.y + e.y : c.y - e.y,
                                     (k & 4) == 0 ? c.z + e.z : c.z - e.z};
                const V3 q = rotate(inv_m, corner - pm);
                lmin = vmin(lmin, q);
                lmax = vmax(lmax, q);
            }
            auto overlaps = [&](V3 a0, V3 a1) {
                return a0.x <= lmax.x && a0.y <= lmax.y && a0.z <= lmax.z && lmin.x <= a1.x && lmin.y <= a1.y &&
                       lmin.z <= a1.z;
            };
            uint32_t nc = 0;
            uint32_t stack[MESH_STACK];
            int sp = 0;
            if (ms.hull_cnt) stack[sp++] = 0;
            while (sp > 0) {
                const uint32_t k = stack[--sp];
                const float4 n0 = hull[ms.hull_off + 2 * k], n1 = hull[ms.hull_off + 2 * k + 1];
                if (!overlaps(from4(n0), from4(n1))) continue;
                const uint32_t na = __float_as_uint(n0.w), nb = __float_as_uint(n1.w);
                if (!(na & MESH_LEAF)) {
                    if (sp + 2 > MESH_STACK) {
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
                    const V3 ta = from4(hull[o]), tb = from4(hull[o + 1]), tc = from4(hull[o + 2]);
                    if (!overlaps(vmin(ta, vmin(tb, tc)), vmax(ta, vmax(tb, tc)))) continue;
                    if (nc == MESH_MAX_TRIS) {
                        atomicOr(status, ST_MESH_CANDIDATES);
                        continue;
                    }
                    s_slot[wi][nc++] = slot;
                }
            }
            s_n[wi] = nc;
        }
        __syncwarp();
        const uint32_t nc = s_n[wi];
        const bool sphere = cv.type == SHAPE_SPHERE;
        const V3 center = rotate(qinv(qm), pc - pm);
        Shape tri;
        tri.type = SHAPE_HULL;
        tri.hull_cnt = 3;
        tri.margin = 0.0f;
        tri.cbt = thr;
        for (uint32_t k = lane; k < nc; k += 32) {
            const uint32_t o = tri_base + 3 * s_slot[wi][k];
            V3 pt = V3{0.f, 0.f, 0.f}, nl = V3{0.f, 0.f, 0.f};
            float pen = 0.0f;
            bool hit = false;
            if (sphere) {
                if (sphere_triangle(center, cv.p0, thr, from4(hull[o]), from4(hull[o + 1]), from4(hull[o + 2]), pt, nl,
                                    pen)) {
                    pt = pm + rotate(qm, pt);
                    nl = rotate(qm, -nl);
                    hit = true;
                }
            } else {
                tri.hull_off = o;
                Manifold one;
                collide_convex(cv, pc, qc, tri, pm, qm, has_seed, seed, hull, scratch, one, status);
                if (one.n) {
                    pt = one.pos[0];
                    nl = one.nrm[0];
                    pen = one.pen[0];
                    hit = true;
                }
            }
            s_pt[wi][k] = to4(pt, pen);
            s_nr[wi][k] = to4(nl, hit ? 1.0f : 0.0f);
        }
        __syncwarp();
        if (lane == 0) {
            MeshCandidates cand;
            cand.n = 0;
            for (uint32_t k = 0; k < nc; ++k) {
                const float4 nr = s_nr[wi][k];
                if (nr.w == 0.0f) continue;
                if (cand.n == MESH_MAX_CAND) {
                    atomicOr(status, ST_MESH_CANDIDATES);
                    break;
                }
                const float4 pt = s_pt[wi][k];
                cand.pos[cand.n] = from4(pt);
                cand.pen[cand.n] = pt.w;
                cand.nrm[cand.n] = from4(nr);
                ++cand.n;
            }
            Manifold m;
            reduce_to_manifold(cand, m);
            if (mesh_a) mf_flip(m);
            store_detection(pd, p, npairs, m);
        }
        __syncwarp();  // the warp's shared lists are reused by its next pair
    }
}

// step.rs:800-853: merge the detection into the manifold, refresh, emit rows; or drop the manifold.
__device__ __forceinline__ void capture_one(const BodyDev& b, const Shape* __restrict__ shapes, const uint64_t* __restrict__ pairs,
                                            const StepParams& sp, PairDataDev& pd, uint32_t p, Pt* pts, uint32_t stride) {
    uint64_t key = pairs[p];
    uint32_t i = key_lo(key), j = key_hi(key);
    float4* ne = pd.entries + size_t(p) * ENTRY_F4;
    const uint32_t n = pd.detect_n[p];  // > 0: the capture list holds detections with points
    Manifold m;
    m.n = int(n);
    const float4* d = pd.detect + size_t(p) * 8;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        if (k >= n) break;
        float4 a = d[2 * k], c = d[2 * k + 1];
        m.pos[k] = from4(a); m.pen[k] = a.w; m.nrm[k] = from4(c);
    }
    uint4 ia = b.info[i], ib = b.info[j];
    Entry E;
    uint32_t meta = __float_as_uint(ne[2].w);
    if (meta & META_VALID) {
        E = load_entry(ne);
        if (pd.rec.pt_src)
            for (int k = 0; k < E.count(); ++k) E.p[k].src = pd.rec.pt_src[size_t(p) * 4 + k];
    } else {
        E.meta = 0;
        E.thr = 0.02f;
    }
    V3 pa = from4(b.pred[i]), pb = from4(b.pred[j]);
    Q qa = q4(b.quat[i]), qb = q4(b.quat[j]);
    float thr = fminf(shapes[ia.x].cbt, shapes[ib.x].cbt);
    capture(E, m, pa, qa, pb, qb, thr, pts, stride);
    Kept K;
    refresh(E, pa, qa, pb, qb, K);
    store_entry_kept(ne, E, K);
    if (((ia.y | ib.y) & BF_NO_RESPONSE) == 0) {
        const int64_t old = pd.rec.pair_old ? (pd.rec.pair_old[p] == REC_NONE ? -1 : int64_t(pd.rec.pair_old[p])) : -1;
        emit_rows_kept(b, i, j, E, K, sp, pd.rows, pd.row_count, p, pd.rec.row_src, old);
    }
}

constexpr uint32_t CAPTURE_TB = 64;

__global__ void __launch_bounds__(CAPTURE_TB) k_capture(BodyDev b, const Shape* __restrict__ shapes,
                                                        const uint64_t* __restrict__ pairs, uint32_t npairs,
                                                        StepParams sp, PairDataDev pd) {
    __shared__ Pt s_pts[8][CAPTURE_TB];  // capture()'s candidate points, [k][thread]
    const uint32_t cnt = pd.scalars[CAPTURE_COUNT];
    const uint32_t* list = pd.route_list + size_t(CAPTURE_LIST) * npairs;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        capture_one(b, shapes, pairs, sp, pd, list[t], &s_pts[0][threadIdx.x], CAPTURE_TB);
    }
}

// Plane-plane pairs (route NP_NONE) detect nothing: their manifold (if any) is dropped.
__global__ void k_drop_undetectable(uint32_t npairs, PairDataDev pd) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    if (pd.status[p] == (PS_DETECT | (NP_NONE << 8))) store_meta_only(pd.entries + size_t(p) * ENTRY_F4, 0u);
}

constexpr uint32_t COLLIDE_QUERIES_TB = 64;

__global__ __launch_bounds__(COLLIDE_QUERIES_TB) void k_collide_queries(const Shape* __restrict__ shapes, const float4* __restrict__ hull, uint32_t n,
                                  const uint32_t* __restrict__ sai, const float4* __restrict__ pa4,
                                  const float4* __restrict__ qa4, const uint32_t* __restrict__ sbi,
                                  const float4* __restrict__ pb4, const float4* __restrict__ qb4,
                                  const float4* __restrict__ seeds, int force_convex, float4* out, uint32_t* counts,
                                  uint32_t* status) {
    __shared__ BoxBoxScratch s_bbs[COLLIDE_QUERIES_TB];
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    Shape sa = shapes[sai[t]], sb = shapes[sbi[t]];
    V3 pa = from4(pa4[t]), pb = from4(pb4[t]);
    Q qa = q4(qa4[t]), qb = q4(qb4[t]);
    Manifold m;
    m.n = 0;
    uint32_t route = route_of(sa.type, sb.type);
    if (force_convex && route != NP_MESH && route != NP_NONE) route = NP_CONVEX;
    if (route == NP_CONVEX || route == NP_MESH) {
        EpaScratch scratch;
        bool has_seed = seeds != nullptr;
        V3 seed = has_seed ? from4(seeds[t]) : V3{0.f, 0.f, 0.f};
        if (route == NP_MESH) collide_mesh_pair(sa, pa, qa, sb, pb, qb, has_seed, seed, hull, scratch, m, status);
        else collide_convex(sa, pa, qa, sb, pb, qb, has_seed, seed, hull, scratch, m, status);
    } else if (route != NP_NONE) {
        collide_analytic(route, sa, pa, qa, sb, pb, qb, hull, m, s_bbs[threadIdx.x]);
    }
    counts[t] = uint32_t(m.n);
    for (int k = 0; k < m.n; ++k) {
        out[(size_t(t) * 4 + k) * 2] = to4(m.pos[k], m.pen[k]);
        out[(size_t(t) * 4 + k) * 2 + 1] = to4(m.nrm[k], 0.0f);
    }
}

// Stand-alone row preparation: contacts (body_a, body_b, pos3, normal3, penetration,
// impulse) grouped by consecutive body pairs; group g owns row slots [4g, 4g + n).
__global__ void k_prepare_contacts(BodyDev b, uint32_t ngroups, const uint32_t* __restrict__ group_first,
                                   const uint32_t* __restrict__ group_n, const float* __restrict__ contacts,
                                   const uint64_t* __restrict__ group_keys, StepParams sp, float4* rows,
                                   uint32_t* row_count) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint64_t key = group_keys[g];
    uint32_t i = key_lo(key), j = key_hi(key);
    Out o;
    o.n = int(group_n[g]);
    for (int k = 0; k < o.n; ++k) {
        const float* c = contacts + size_t(group_first[g] + k) * 10;
        o.pos[k] = V3{c[2], c[3], c[4]};
        o.nrm[k] = V3{c[5], c[6], c[7]};
        o.pen[k] = c[8];
        o.imp[k] = c[9];
    }
    // The caller's impulse is already the warm-start value: undo the factor emit_rows applies.
    StepParams q = sp;
    q.info.warmstarting_factor = 1.0f;
    emit_rows(b, i, j, o, q, rows, row_count, g, nullptr, -1);
}

}  // namespace

void run_pair_pass(const WorldView& w, const uint64_t* pairs, uint32_t npairs, const Manifolds& old_cache,
                   PairData& pd, const StepParams& sp, const uint32_t* simulate_flag, uint32_t* status_dev,
                   cudaStream_t s) {
    (void)simulate_flag;
    if (npairs == 0) return;
    PairDataDev d = pd.dev();
    check_cuda(cudaMemsetAsync(pd.scalars.p, 0, 8 * sizeof(uint32_t), s), "memset scalars");
    check_cuda(cudaMemsetAsync(pd.scalars.p + ROUTE_COUNT0, 0, (CAPTURE_COUNT + 1 - ROUTE_COUNT0) * sizeof(uint32_t), s),
               "memset scalars");
    const int TB = 128;
    k_classify<<<(npairs + TB - 1) / TB, TB, 0, s>>>(w.b, w.shapes, pairs, npairs, old_cache.keys.p,
                                                     old_cache.entries.p, old_cache.count_dev, sp, d);
    k_drop_undetectable<<<(npairs + 255) / 256, 256, 0, s>>>(npairs, d);
    uint32_t grid = std::min<uint32_t>((npairs + TB - 1) / TB, 148u * 16u);
    k_narrow_analytic<<<grid, NARROW_ANALYTIC_TB, 0, s>>>(w.b, w.shapes, w.hull, pairs, npairs, d);
    uint32_t cgrid = std::min<uint32_t>((npairs + 63) / 64, 148u * 8u);
    k_narrow_convex<<<cgrid, 64, 0, s>>>(w.b, w.shapes, w.hull, pairs, npairs, d, status_dev);
    if (w.has_mesh) {
        const uint32_t mgrid = std::min<uint32_t>((npairs + MESH_WARPS - 1) / MESH_WARPS, 148u * 8u);
        k_narrow_mesh<<<mgrid, 32 * MESH_WARPS, 0, s>>>(w.b, w.shapes, w.hull, pairs, npairs, d, status_dev);
    }
    // The GJK/EPA kernels keep their polytopes in local memory (12-15 KB a thread): a launch
    // the device cannot back with local memory fails here rather than dropping detections.
    check_cuda(cudaGetLastError(), "narrow phase launch");
    k_capture<<<(npairs + CAPTURE_TB - 1) / CAPTURE_TB < 148u * 16u ? (npairs + CAPTURE_TB - 1) / CAPTURE_TB : 148u * 16u,
                CAPTURE_TB, 0, s>>>(w.b, w.shapes, pairs, npairs, sp, d);
}

void run_collide_queries(const Shape* shapes, const float4* hull, uint32_t n, const uint32_t* sa, const float4* pa,
                         const float4* qa, const uint32_t* sb, const float4* pb, const float4* qb, const float4* seeds,
                         int force_convex, float4* out, uint32_t* counts, uint32_t* status_dev, cudaStream_t s) {
    if (n == 0) return;
    k_collide_queries<<<(n + COLLIDE_QUERIES_TB - 1) / COLLIDE_QUERIES_TB, COLLIDE_QUERIES_TB, 0, s>>>(shapes, hull, n, sa, pa, qa, sb, pb, qb, seeds, force_convex, out,
                                                   counts, status_dev);
}

}  // namespace bgpu

namespace bgpu {
void run_prepare_contacts(const BodyDev& b, uint32_t ngroups, const uint32_t* group_first, const uint32_t* group_n,
                          const float* contacts, const uint64_t* group_keys, const StepParams& sp, float4* rows,
                          uint32_t* row_count, cudaStream_t s) {
    if (ngroups == 0) return;
    k_prepare_contacts<<<(ngroups + 127) / 128, 128, 0, s>>>(b, ngroups, group_first, group_n, contacts, group_keys, sp,
                                                             rows, row_count);
}
}  // namespace bgpu
