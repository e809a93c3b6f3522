// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_math.hpp).
// Persistent manifolds (bullet-collision/src/manifold.rs), rigid bodies
// (bullet-dynamics/src/body.rs), the sequential-impulse solver
// (bullet-dynamics/src/solver/{info,sequential_impulse}.rs), islands
// (bullet-dynamics/src/island.rs, world/islands.rs) and the rigid subset of
// the step pipeline (bullet-dynamics/src/world/step.rs:281-1287).
#pragma once
#include <chrono>
#include <cstring>
#include <map>
#include <unordered_map>
#include "oracle_joints.hpp"
#include "oracle_ccd.hpp"
#include "oracle_narrow.hpp"

namespace oracle {

// ------------------------------------------------------------ manifold.rs
// IEEE total order of f32/f64::total_cmp as a signed integer key.
inline int64_t total_order_key(double v) {
    int64_t b;
    std::memcpy(&b, &v, sizeof(b));
    return b ^ int64_t(uint64_t(b >> 63) >> 1);
}
inline int64_t total_order_key(float v) {
    int32_t b;
    std::memcpy(&b, &v, sizeof(b));
    return int64_t(b ^ int32_t(uint32_t(b >> 31) >> 1));
}

template <class R>
struct PersistentPoint {  // manifold.rs:124-142
    V3<R> local_a, local_b, normal;
    R penetration = 0, normal_impulse = 0;
    uint32_t lifetime = 0;
};

template <class R>
inline R rotation_angle(const Quat<R>& q) {  // manifold.rs:158-160
    return R(2) * std::acos(std::min(std::max(q.w, R(-1)), R(1)));
}

template <class R>
struct PersistentManifold {  // manifold.rs:168-386
    std::vector<PersistentPoint<R>> points;
    V3<R> detect_pos_a, detect_pos_b;
    Quat<R> detect_ori_a, detect_ori_b;
    bool initialized = false;
    R threshold = CONTACT_BREAKING_THRESHOLD<R>;
    uint32_t touched = 0;

    // manifold.rs:246-282
    void refresh(const V3<R>& pa, const Quat<R>& qa, const V3<R>& pb, const Quat<R>& qb,
                 std::vector<ContactPoint<R>>& out) {
        out.clear();
        R thr = threshold, thr_sq = thr * thr;
        std::vector<PersistentPoint<R>> kept;
        kept.reserve(points.size());
        for (auto p : points) {
            V3<R> wa = pa + qa.rotate(p.local_a);
            V3<R> wb = pb + qb.rotate(p.local_b);
            V3<R> d = wa - wb;
            R pen = d.dot(p.normal);
            if (pen < -thr) continue;
            V3<R> lat = d - p.normal * pen;
            if (lat.length_squared() > thr_sq) continue;
            p.penetration = pen;
            p.lifetime += 1;
            ContactPoint<R> cp(wb, p.normal, pen);
            cp.normal_impulse = p.normal_impulse;
            cp.lifetime = p.lifetime;
            out.push_back(cp);
            kept.push_back(p);
        }
        points.swap(kept);
    }

    // manifold.rs:287-304
    bool needs_redetect(const V3<R>& pa, const Quat<R>& qa, const V3<R>& pb, const Quat<R>& qb) const {
        if (!initialized) return true;
        V3<R> drift = (pb - detect_pos_b) - (pa - detect_pos_a);
        const R T = R(0.005);
        if (drift.length_squared() > T * T) return true;
        Quat<R> ra = qa * detect_ori_a.inverse();
        Quat<R> rb = qb * detect_ori_b.inverse();
        return rotation_angle(ra) + rotation_angle(rb) > R(0.01);
    }

    // manifold.rs:326-376
    void capture(const Manifold<R>& m, const V3<R>& pa, const Quat<R>& qa, const V3<R>& pb, const Quat<R>& qb, R thr) {
        threshold = thr;
        Quat<R> ia = qa.inverse(), ib = qb.inverse();
        R thr_sq = thr * thr;
        for (auto& cp : m.points) {
            V3<R> wb = cp.position;
            V3<R> wa = cp.position + cp.normal * cp.penetration;
            PersistentPoint<R> pt;
            pt.local_a = ia.rotate(wa - pa);
            pt.local_b = ib.rotate(wb - pb);
            pt.normal = cp.normal;
            pt.penetration = cp.penetration;
            pt.normal_impulse = 0;
            pt.lifetime = 0;
            bool matched = false;
            for (auto& o : points) {
                if ((o.local_a - pt.local_a).length_squared() < thr_sq && o.normal.dot(pt.normal) >= R(0.9)) {
                    pt.normal_impulse = o.normal_impulse;
                    o = pt;
                    matched = true;
                    break;
                }
            }
            if (!matched) points.push_back(pt);
        }
        if (points.size() > 4) {
            // Stable descending sort by penetration (Rust sort_by + total_cmp).
            std::stable_sort(points.begin(), points.end(), [](const PersistentPoint<R>& a, const PersistentPoint<R>& b) {
                return total_order_key(a.penetration) > total_order_key(b.penetration);
            });
            points.resize(4);
        }
        detect_pos_a = pa; detect_ori_a = qa; detect_pos_b = pb; detect_ori_b = qb;
        initialized = true;
    }

    // manifold.rs:380-386
    bool seed(V3<R>& s) const {
        if (points.empty()) return false;
        if (points[0].normal.length_squared() > R(0.5)) { s = points[0].normal; return true; }
        return false;
    }
};

// ------------------------------------------------------------ body.rs
enum Activation : uint32_t {  // body.rs:140-153 (numbered like Bullet's tags)
    ACT_ACTIVE = 1, ACT_ISLAND_SLEEPING = 2, ACT_WANTS_DEACTIVATION = 3,
    ACT_DISABLE_DEACTIVATION = 4, ACT_DISABLE_SIMULATION = 5,
};
enum BodyFlags : uint32_t {  // body.rs:204-252
    CF_NO_CONTACT_RESPONSE = 0x1, CF_DISABLE_WORLD_GRAVITY = 0x2, CF_KINEMATIC = 0x4,
};

template <class R>
struct Body {  // body.rs:270-384 (rigid, shape by index)
    uint32_t shape = 0;
    V3<R> position;
    Quat<R> orientation;
    V3<R> linear_velocity, angular_velocity, force, torque;
    R inv_mass = 0;
    V3<R> inv_inertia_local;
    R friction = R(0.5), restitution = 0;
    V3<R> gravity;
    uint16_t group = 1, mask = 0xFFFF;
    uint32_t flags = 0;
    R linear_damping = 0, angular_damping = 0;
    bool additional_damping = false;
    R additional_damping_factor = R(0.005), additional_lin_thr_sqr = R(0.01), additional_ang_thr_sqr = R(0.01),
      additional_ang_damping_factor = R(0.01);
    bool is_static = false;
    uint32_t activation = ACT_ACTIVE;
    R deactivation_time = 0;
    R lin_sleep = R(0.8), ang_sleep = R(1.0);
    V3<R> push_linear, push_angular;
    R ccd_threshold = 0, ccd_radius = 0;  // body.rs:365-367, 680-692 (RigidBody::ccd); 0 = off

    bool is_kinematic() const { return (flags & CF_KINEMATIC) != 0; }
    bool is_static_or_kinematic() const { return is_static || is_kinematic(); }
    // body.rs:524-532
    bool is_active() const {
        return activation == ACT_ACTIVE || activation == ACT_WANTS_DEACTIVATION || activation == ACT_DISABLE_DEACTIVATION;
    }
    bool participates_in_islands() const { return !is_static && !is_kinematic(); }  // body.rs:595-597
    bool is_island_awake() const { return activation == ACT_ACTIVE || activation == ACT_DISABLE_DEACTIVATION; }
    void island_wake() {  // body.rs:615-624
        if (is_static || activation != ACT_ISLAND_SLEEPING) return;
        activation = ACT_WANTS_DEACTIVATION;
        deactivation_time = 0;
    }
    void go_to_sleep() {  // body.rs:578-589
        if (activation == ACT_DISABLE_SIMULATION) return;
        activation = ACT_ISLAND_SLEEPING;
        linear_velocity = V3<R>();
        angular_velocity = V3<R>();
    }
    M3<R> inv_inertia_world() const { return inertia_tensor_world(inv_inertia_local, orientation); }

    // body.rs:1066-1105
    void apply_damping(R dt) {
        if (linear_damping != R(0)) linear_velocity *= std::pow(R(1) - linear_damping, dt);
        if (angular_damping != R(0)) angular_velocity *= std::pow(R(1) - angular_damping, dt);
        if (!additional_damping) return;
        if (angular_velocity.length_squared() < additional_ang_thr_sqr &&
            linear_velocity.length_squared() < additional_lin_thr_sqr) {
            angular_velocity *= additional_damping_factor;
            linear_velocity *= additional_damping_factor;
        }
        const R damp_vel = R(0.005);
        R speed = linear_velocity.length();
        if (speed < linear_damping) {
            if (speed > damp_vel) linear_velocity -= (linear_velocity / linear_velocity.length()) * damp_vel;
            else linear_velocity = V3<R>();
        }
        R aspeed = angular_velocity.length();
        if (aspeed < angular_damping) {
            if (aspeed > damp_vel) angular_velocity -= (angular_velocity / angular_velocity.length()) * damp_vel;
            else angular_velocity = V3<R>();
        }
    }

    // body.rs:1135-1148
    V3<R> gyroscopic_impulse_implicit_body(R step) const {
        V3<R> inv = inv_inertia_local;
        if (inv.x <= R(0) || inv.y <= R(0) || inv.z <= R(0)) return V3<R>();
        V3<R> inertia(R(1) / inv.x, R(1) / inv.y, R(1) / inv.z);
        M3<R> ib = M3<R>::diag(inertia);
        V3<R> ob = orientation.inverse().rotate(angular_velocity);
        V3<R> ibo = inertia * ob;
        V3<R> residual = ob.cross(ibo) * step;
        M3<R> jac = ib + (skew(ob) * ib - skew(ibo)) * step;
        V3<R> delta = jac.inverse() * residual;
        return orientation.rotate(ob - delta) - angular_velocity;
    }

    // body.rs:1113-1126
    void integrate_velocities(R dt) {
        if (is_static || is_kinematic() || !is_active()) return;
        apply_damping(dt);
        linear_velocity += (gravity + force * inv_mass) * dt;
        M3<R> iw = inv_inertia_world();
        angular_velocity += iw * (torque * dt);
        angular_velocity += gyroscopic_impulse_implicit_body(dt);
    }

    // body.rs:1175-1181
    V3<R> predicted_position(R dt) const {
        if (is_static || !is_active()) return position;
        return position + linear_velocity * dt;
    }

    // body.rs:639-657
    void update_deactivation(R dt) {
        if (!is_active() || activation == ACT_DISABLE_DEACTIVATION) return;
        bool slow = linear_velocity.length_squared() < lin_sleep * lin_sleep &&
                    angular_velocity.length_squared() < ang_sleep * ang_sleep;
        if (slow) deactivation_time += dt;
        else { deactivation_time = 0; activation = ACT_ACTIVE; }
        if (deactivation_time > R(2)) { deactivation_time = 0; activation = ACT_WANTS_DEACTIVATION; }
    }
};

// body.rs:92-137 (btTransformUtil::integrateTransform)
template <class R>
inline void interpolate_pose(const V3<R>& pos, const Quat<R>& ori, const V3<R>& lv, const V3<R>& av, R dt, V3<R>& npos,
                             Quat<R>& nori) {
    npos = pos + lv * dt;
    R angle_sqr = av.length_squared();
    R angle = 0;
    if (angle_sqr > Consts<R>::EPS) angle = std::sqrt(angle_sqr);
    if (angle * dt > Consts<R>::FRAC_PI_4) angle = Consts<R>::FRAC_PI_4 / dt;
    V3<R> axis;
    if (angle < R(0.001)) axis = av * (R(0.5) * dt - (dt * dt * dt) * Consts<R>::TAYLOR * angle * angle);
    else axis = av * (std::sin(R(0.5) * angle * dt) / angle);
    Quat<R> dorn(axis.x, axis.y, axis.z, std::cos(angle * dt * R(0.5)));
    Quat<R> pred = dorn * ori;
    R ls = pred.length_squared();
    if (ls < Consts<R>::EPS) pred = Quat<R>(0, 0, 0, 0);
    else {
        R l = std::sqrt(ls);
        pred = Quat<R>(pred.x / l, pred.y / l, pred.z / l, pred.w / l);
    }
    nori = pred.length_squared() > Consts<R>::EPS ? pred : ori;
}

// ------------------------------------------------------------ solver/info.rs:88-107
template <class R>
struct SolverInfo {
    R erp = R(0.2), erp2 = R(0.2), linear_slop = R(0.005), restitution_velocity_threshold = R(1);
    bool split_impulse = true;
    R split_impulse_penetration_threshold = R(-0.04), split_impulse_turn_erp = R(0.1);
    R warmstarting_factor = R(0.85), friction_erp = R(0.2), global_cfm = 0, sor = 1, damping = 1;
    uint32_t num_iterations = 10;
};

// ------------------------------------------------------------ sequential_impulse.rs
template <class R>
struct ContactConstraint {  // sequential_impulse.rs:18-117 (rolling/anchor/aniso/stiffness channels not built)
    uint32_t body_a = 0, body_b = 0;
    V3<R> normal, tangent1, tangent2, r_a, r_b;
    R inv_mass_a = 0, inv_mass_b = 0;
    V3<R> ang_normal_a, ang_normal_b, ang_t1_a, ang_t1_b, ang_t2_a, ang_t2_b;
    R normal_mass = 0, tangent1_mass = 0, tangent2_mass = 0;
    R penetration = 0, baumgarte_span = 0, separation = 0, restitution = 0, friction = 0;
    R normal_impulse = 0, tangent1_impulse = 0, tangent2_impulse = 0;
    uint32_t point_index = 0;
    bool split_active = false;
    R rhs_penetration = 0, push_impulse = 0;
    bool applies_a = false, applies_b = false;
    V3<R> kn, kt1, kt2;
    R erp = 0, normal_cfm = 0;
};

// sequential_impulse.rs:620-629
template <class R>
inline void tangent_basis(const V3<R>& n, V3<R>& t1, V3<R>& t2) {
    V3<R> helper = std::fabs(n.x) < R(0.9) ? V3<R>(1, 0, 0) : V3<R>(0, 1, 0);
    V3<R> c = n.cross(helper);
    t1 = c * (R(1) / c.length());
    t2 = n.cross(t1);
}

// sequential_impulse.rs:655-673
template <class R>
inline R effective_mass(R ima, R imb, const V3<R>& aa, const V3<R>& ab, const V3<R>& ra, const V3<R>& rb, const V3<R>& d) {
    R k = ima + imb + d.dot(aa.cross(ra)) + d.dot(ab.cross(rb));
    return k > R(0) ? R(1) / k : R(0);
}

// sequential_impulse.rs:339-550
template <class R>
ContactConstraint<R> prepare_contact(uint32_t ia, uint32_t ib, const ContactPoint<R>& cp, const Body<R>& a, const Body<R>& b,
                                     uint32_t point_index, R inv_dt, const SolverInfo<R>& info) {
    ContactConstraint<R> c;
    c.body_a = ia; c.body_b = ib;
    c.normal = cp.normal;
    tangent_basis(c.normal, c.tangent1, c.tangent2);
    c.r_a = cp.position - a.position;
    c.r_b = cp.position - b.position;
    M3<R> iia = a.inv_inertia_world(), iib = b.inv_inertia_world();
    c.inv_mass_a = a.inv_mass; c.inv_mass_b = b.inv_mass;
    c.ang_normal_a = iia * c.r_a.cross(c.normal);
    c.ang_normal_b = iib * c.r_b.cross(c.normal);
    c.ang_t1_a = iia * c.r_a.cross(c.tangent1);
    c.ang_t1_b = iib * c.r_b.cross(c.tangent1);
    c.ang_t2_a = iia * c.r_a.cross(c.tangent2);
    c.ang_t2_b = iib * c.r_b.cross(c.tangent2);
    c.normal_mass = effective_mass(c.inv_mass_a, c.inv_mass_b, c.ang_normal_a, c.ang_normal_b, c.r_a, c.r_b, c.normal);
    c.tangent1_mass = effective_mass(c.inv_mass_a, c.inv_mass_b, c.ang_t1_a, c.ang_t1_b, c.r_a, c.r_b, c.tangent1);
    c.tangent2_mass = effective_mass(c.inv_mass_a, c.inv_mass_b, c.ang_t2_a, c.ang_t2_b, c.r_a, c.r_b, c.tangent2);
    R ims = c.inv_mass_a + c.inv_mass_b;
    c.kn = c.normal * ims + c.ang_normal_b.cross(c.r_b) + c.ang_normal_a.cross(c.r_a);
    c.kt1 = c.tangent1 * ims + c.ang_t1_b.cross(c.r_b) + c.ang_t1_a.cross(c.r_a);
    c.kt2 = c.tangent2 * ims + c.ang_t2_b.cross(c.r_b) + c.ang_t2_a.cross(c.r_a);
    c.friction = a.friction * b.friction;
    c.restitution = a.restitution * b.restitution;
    c.erp = info.erp2;
    c.normal_cfm = 0;
    R cfm_global = info.global_cfm * inv_dt;
    if (cfm_global != R(0) || info.sor != R(1)) {  // :454-466
        R k = c.normal_mass > R(0) ? R(1) / c.normal_mass : R(0);
        c.normal_mass = k + cfm_global > R(0) ? info.sor / (k + cfm_global) : R(0);
        c.normal_cfm = cfm_global * c.normal_mass;
    }
    if (info.sor != R(1)) { c.tangent1_mass *= info.sor; c.tangent2_mass *= info.sor; }
    c.penetration = cp.penetration;
    c.baumgarte_span = std::max(cp.penetration - info.linear_slop, R(0));
    c.separation = std::min(cp.penetration, R(0));
    c.normal_impulse = cp.normal_impulse;
    c.tangent1_impulse = cp.tangent_impulse[0];
    c.tangent2_impulse = cp.tangent_impulse[1];
    c.point_index = point_index;
    c.split_active = info.split_impulse && cp.penetration > -info.split_impulse_penetration_threshold;
    c.applies_a = c.inv_mass_a > R(0);
    c.applies_b = c.inv_mass_b > R(0);
    return c;
}

template <class R>
inline void apply_impulse(Body<R>& a, Body<R>& b, const ContactConstraint<R>& c, const V3<R>& d, const V3<R>& ca,
                          const V3<R>& cb, R j) {  // sequential_impulse.rs:989-1009
    if (c.applies_a) { a.linear_velocity -= d * (j * c.inv_mass_a); a.angular_velocity -= ca * j; }
    if (c.applies_b) { b.linear_velocity += d * (j * c.inv_mass_b); b.angular_velocity += cb * j; }
}

// sequential_impulse.rs:804-930 (no rolling rows)
template <class R>
void solve_contact(std::vector<Body<R>>& bodies, ContactConstraint<R>& c, R inv_dt, const SolverInfo<R>& info) {
    Body<R>& a = bodies[c.body_a];
    Body<R>& b = bodies[c.body_b];
    bool soft = c.normal_cfm != R(0);
    V3<R> va = a.linear_velocity + a.angular_velocity.cross(c.r_a);
    V3<R> vb = b.linear_velocity + b.angular_velocity.cross(c.r_b);
    V3<R> rel = vb - va;
    R vn = rel.dot(c.normal);
    R bias = 0;
    if (vn < -info.restitution_velocity_threshold) bias = -c.restitution * vn;
    if (!c.split_active) bias += c.erp * inv_dt * c.baumgarte_span;
    if (c.separation < R(0)) bias += c.separation * inv_dt;
    R lambda = soft ? c.normal_mass * (bias - vn) - c.normal_cfm * c.normal_impulse : c.normal_mass * (bias - vn);
    R old = c.normal_impulse;
    c.normal_impulse = std::max(old + lambda, R(0));
    R jn = c.normal_impulse - old;
    apply_impulse(a, b, c, c.normal, c.ang_normal_a, c.ang_normal_b, jn);
    rel += c.kn * jn;
    R maxf = c.friction * c.normal_impulse;
    {
        R vt = rel.dot(c.tangent1);
        R lam = -c.tangent1_mass * (vt - R(0) * inv_dt);
        R o = c.tangent1_impulse;
        R nw = std::min(std::max(o + lam, -maxf), maxf);
        c.tangent1_impulse = nw;
        R j = nw - o;
        apply_impulse(a, b, c, c.tangent1, c.ang_t1_a, c.ang_t1_b, j);
        rel += c.kt1 * j;
    }
    {
        R vt = rel.dot(c.tangent2);
        R lam = -c.tangent2_mass * (vt - R(0) * inv_dt);
        R o = c.tangent2_impulse;
        R nw = std::min(std::max(o + lam, -maxf), maxf);
        c.tangent2_impulse = nw;
        R j = nw - o;
        apply_impulse(a, b, c, c.tangent2, c.ang_t2_a, c.ang_t2_b, j);
        rel += c.kt2 * j;
    }
}

// sequential_impulse.rs:692-802; each velocity sweep solves the contacts, then the joint rows
// (sequential_impulse.rs:720-735); joint rows take no warm start and no split pass.
template <class R>
void solve(std::vector<Body<R>>& bodies, std::vector<ContactConstraint<R>>& cs, R inv_dt, const SolverInfo<R>& info,
           std::vector<JointRow<R>>* joint_rows = nullptr) {
    for (auto& c : cs) {  // warm_start :710-717
        Body<R>& a = bodies[c.body_a];
        Body<R>& b = bodies[c.body_b];
        apply_impulse(a, b, c, c.normal, c.ang_normal_a, c.ang_normal_b, c.normal_impulse);
        apply_impulse(a, b, c, c.tangent1, c.ang_t1_a, c.ang_t1_b, c.tangent1_impulse);
        apply_impulse(a, b, c, c.tangent2, c.ang_t2_a, c.ang_t2_b, c.tangent2_impulse);
    }
    for (uint32_t it = 0; it < info.num_iterations; ++it) {
        for (auto& c : cs) solve_contact(bodies, c, inv_dt, info);
        if (joint_rows)
            for (auto& jr : *joint_rows) solve_joint_row(bodies, jr, info.damping);
    }
    for (auto& c : cs)
        if (c.split_active) c.rhs_penetration = c.penetration * c.erp * inv_dt * c.normal_mass;
    for (uint32_t it = 0; it < info.num_iterations; ++it) {
        for (auto& c : cs) {
            if (!c.split_active) continue;
            Body<R>& a = bodies[c.body_a];
            Body<R>& b = bodies[c.body_b];
            V3<R> pva = a.push_linear + a.push_angular.cross(c.r_a);
            V3<R> pvb = b.push_linear + b.push_angular.cross(c.r_b);
            R pvn = (pvb - pva).dot(c.normal);
            R delta = c.normal_cfm != R(0) ? c.rhs_penetration - pvn * c.normal_mass - c.normal_cfm * c.push_impulse
                                           : c.rhs_penetration - pvn * c.normal_mass;
            R old = c.push_impulse;
            c.push_impulse = std::max(old + delta, R(0));
            R j = c.push_impulse - old;
            if (j != R(0)) {  // apply_push :793-802
                if (c.applies_a) { a.push_linear -= c.normal * (j * c.inv_mass_a); a.push_angular -= c.ang_normal_a * j; }
                if (c.applies_b) { b.push_linear += c.normal * (j * c.inv_mass_b); b.push_angular += c.ang_normal_b * j; }
            }
        }
    }
}

// ------------------------------------------------------------ island.rs:17-57
struct UnionFind {
    std::vector<size_t> parent, size;
    void reset(size_t n) {
        parent.resize(n); size.assign(n, 1);
        for (size_t i = 0; i < n; ++i) parent[i] = i;
    }
    size_t find(size_t x) {
        while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
        return x;
    }
    void unite(size_t a, size_t b) {
        size_t ra = find(a), rb = find(b);
        if (ra == rb) return;
        if (size[ra] < size[rb]) { parent[ra] = rb; size[rb] += size[ra]; }
        else { parent[rb] = ra; size[ra] += size[rb]; }
    }
};

// ------------------------------------------------------------ broadphase
// brute_force.rs:54-68 — the contract: every (i<j) with closed overlap, lexicographic.
template <class R>
void brute_force_pairs(const std::vector<Aabb<R>>& aabbs, std::vector<std::pair<uint32_t, uint32_t>>& out) {
    out.clear();
    for (size_t i = 0; i < aabbs.size(); ++i)
        for (size_t j = i + 1; j < aabbs.size(); ++j)
            if (aabbs[i].overlaps(aabbs[j])) out.push_back({uint32_t(i), uint32_t(j)});
}

// Sort-and-sweep on x with an exact 3-axis filter; emits the same set as
// brute_force_pairs (the reference's SAP/DBVT contract, axis_sweep3.rs:498-508,
// dbvt.rs:768-806), sorted lexicographically.
template <class R>
void sweep_pairs(const std::vector<Aabb<R>>& aabbs, std::vector<std::pair<uint32_t, uint32_t>>& out) {
    out.clear();
    std::vector<uint32_t> order(aabbs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = uint32_t(i);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        if (aabbs[a].min.x != aabbs[b].min.x) return aabbs[a].min.x < aabbs[b].min.x;
        return a < b;
    });
    std::vector<uint64_t> keys;
    for (size_t s = 0; s < order.size(); ++s) {
        uint32_t i = order[s];
        const Aabb<R>& a = aabbs[i];
        for (size_t t = s + 1; t < order.size(); ++t) {
            uint32_t j = order[t];
            const Aabb<R>& b = aabbs[j];
            if (b.min.x > a.max.x) break;
            if (a.overlaps(b)) {
                uint32_t lo = std::min(i, j), hi = std::max(i, j);
                keys.push_back((uint64_t(lo) << 32) | hi);
            }
        }
    }
    std::sort(keys.begin(), keys.end());
    out.reserve(keys.size());
    for (uint64_t k : keys) out.push_back({uint32_t(k >> 32), uint32_t(k & 0xffffffffu)});
}

// Uniform-grid pair finder with the same output contract as brute_force_pairs:
// bounded proxies are hashed by their min corner into cells no smaller than the
// largest proxy extent, so each overlapping pair meets in adjacent cells; proxies
// larger than 1e15 (planes) are tested against everything. Exact 3-axis closed
// overlap filter, lexicographic output.
template <class R>
void grid_pairs(const std::vector<Aabb<R>>& aabbs, std::vector<std::pair<uint32_t, uint32_t>>& out,
                const std::vector<char>* force_big = nullptr) {
    out.clear();
    const size_t n = aabbs.size();
    std::vector<uint32_t> big, small;
    R cell = 0;
    V3<R> lo = V3<R>::splat(std::numeric_limits<R>::infinity());
    for (size_t i = 0; i < n; ++i) {
        const Aabb<R>& a = aabbs[i];
        R ex = std::max(std::max(a.max.x - a.min.x, a.max.y - a.min.y), a.max.z - a.min.z);
        // unbounded proxies, and the caller's large ones (static meshes), are tested against all
        if (!(ex < R(1e15)) || (force_big && (*force_big)[i])) { big.push_back(uint32_t(i)); continue; }
        small.push_back(uint32_t(i));
        cell = std::max(cell, ex);
        lo = lo.min(a.min);
    }
    std::vector<uint64_t> keys;
    if (!small.empty()) {
        if (!(cell > R(0))) cell = R(1);
        auto coord = [&](R v, R l) { return int64_t(std::floor(double(v - l) / double(cell))); };
        // cell key -> bucket (sorted vector of (cell, body))
        std::vector<std::pair<uint64_t, uint32_t>> cells;
        cells.reserve(small.size());
        auto pack = [](int64_t x, int64_t y, int64_t z) {
            return (uint64_t(x & 0x1FFFFF) << 42) | (uint64_t(y & 0x1FFFFF) << 21) | uint64_t(z & 0x1FFFFF);
        };
        for (uint32_t i : small) {
            const Aabb<R>& a = aabbs[i];
            cells.push_back({pack(coord(a.min.x, lo.x), coord(a.min.y, lo.y), coord(a.min.z, lo.z)), i});
        }
        std::sort(cells.begin(), cells.end());
        // Open-addressed table: cell key -> [first, last) run in `cells`.
        size_t cap = 16;
        int bits = 4;
        while (cap < 2 * cells.size()) { cap <<= 1; ++bits; }
        std::vector<uint64_t> tkey(cap, ~0ull);
        std::vector<uint32_t> tbeg(cap, 0), tend(cap, 0);
        auto slot_of = [&](uint64_t k) {
            uint64_t h = k * 0x9E3779B97F4A7C15ull;  // Fibonacci hashing: keep the top bits
            return size_t(h >> (64 - bits));
        };
        for (size_t r = 0; r < cells.size();) {
            size_t e = r;
            while (e < cells.size() && cells[e].first == cells[r].first) ++e;
            size_t sl = slot_of(cells[r].first);
            while (tkey[sl] != ~0ull) sl = (sl + 1) & (cap - 1);
            tkey[sl] = cells[r].first;
            tbeg[sl] = uint32_t(r);
            tend[sl] = uint32_t(e);
            r = e;
        }
        for (uint32_t i : small) {
            const Aabb<R>& a = aabbs[i];
            int64_t cx = coord(a.min.x, lo.x), cy = coord(a.min.y, lo.y), cz = coord(a.min.z, lo.z);
            for (int64_t dx = -1; dx <= 1; ++dx)
                for (int64_t dy = -1; dy <= 1; ++dy)
                    for (int64_t dz = -1; dz <= 1; ++dz) {
                        if (cx + dx < 0 || cy + dy < 0 || cz + dz < 0) continue;
                        uint64_t key = pack(cx + dx, cy + dy, cz + dz);
                        size_t sl = slot_of(key);
                        while (tkey[sl] != ~0ull && tkey[sl] != key) sl = (sl + 1) & (cap - 1);
                        if (tkey[sl] != key) continue;
                        for (uint32_t t = tbeg[sl]; t < tend[sl]; ++t) {
                            uint32_t j = cells[t].second;
                            if (j > i && a.overlaps(aabbs[j])) keys.push_back((uint64_t(i) << 32) | j);
                        }
                    }
        }
    }
    for (uint32_t h : big)
        for (size_t j = 0; j < n; ++j) {
            if (j == h) continue;
            bool other_big = std::binary_search(big.begin(), big.end(), uint32_t(j));
            if (other_big && j < h) continue;  // a big-big pair is emitted once, from the smaller index
            if (aabbs[h].overlaps(aabbs[j])) {
                uint32_t a = std::min<uint32_t>(h, uint32_t(j)), b = std::max<uint32_t>(h, uint32_t(j));
                keys.push_back((uint64_t(a) << 32) | b);
            }
        }
    std::sort(keys.begin(), keys.end());
    out.reserve(keys.size());
    for (uint64_t k : keys) out.push_back({uint32_t(k >> 32), uint32_t(k & 0xffffffffu)});
}

// ------------------------------------------------------------ world
inline uint64_t pair_key(uint32_t a, uint32_t b) {
    uint32_t lo = std::min(a, b), hi = std::max(a, b);
    return (uint64_t(lo) << 32) | hi;
}

template <class R>
struct World {
    std::vector<Shape<R>> shapes;
    std::vector<Body<R>> bodies;
    std::vector<Aabb<R>> proxy_aabbs;  // broad-phase proxies (index = body index)
    std::vector<R> last_ccd_clamps;    // CCD clamp fraction per body of the last step (1: none)
    V3<R> gravity = V3<R>(0, R(-9.81), 0);
    SolverInfo<R> info;
    std::unordered_map<uint64_t, PersistentManifold<R>> cache;
    uint32_t step_counter = 0;
    bool prev_simulate = false;
    bool brute_force_broadphase = false;

    // Optional solve order: pair keys in the order their row groups are solved.
    // Empty = the reference's pair order.
    std::vector<uint64_t> solve_order;

    // Joints (constraint.rs) and the order their rows are solved in (empty: index order).
    std::vector<Joint<R>> joints;
    std::vector<uint32_t> joint_order;
    std::vector<JointRow<R>> last_joint_rows;

    // Snapshots of the last step (for parity checks).
    std::vector<std::pair<uint32_t, uint32_t>> last_pairs;
    std::vector<ContactConstraint<R>> last_rows;     // after the solve, in solve order
    std::vector<ContactConstraint<R>> last_rows_pre; // prepared rows, in solve order, before the solve
    std::vector<V3<R>> last_predicted;
    uint32_t last_narrowphase_calls = 0;

    // timing.rs:20-47 StepTimings: cumulative seconds per stage (integrate
    // velocities, update aabbs, broadphase, islands, narrowphase, solve,
    // integrate positions).
    double stage_s[7] = {0, 0, 0, 0, 0, 0, 0};
    std::chrono::steady_clock::time_point clk_;
    void clk_start() { clk_ = std::chrono::steady_clock::now(); }
    void clk_mark(int stage) {
        auto t = std::chrono::steady_clock::now();
        stage_s[stage] += std::chrono::duration<double>(t - clk_).count();
        clk_ = t;
    }

    // world.rs:524-563 (add_body: gravity inheritance + padded proxy AABB)
    uint32_t add_body(Body<R> b) {
        if (!b.is_static_or_kinematic() && !(b.flags & CF_DISABLE_WORLD_GRAVITY)) b.gravity = gravity;
        Aabb<R> aabb = shapes[b.shape].world_aabb(b.position, b.orientation).expanded(CONTACT_BREAKING_THRESHOLD<R>);
        proxy_aabbs.push_back(aabb);
        bodies.push_back(b);
        return uint32_t(bodies.size() - 1);
    }

    // body.rs:388-439 / 455-499
    Body<R> make_dynamic(uint32_t shape, const V3<R>& pos, R mass) const {
        Body<R> b;
        b.shape = shape;
        b.position = pos;
        V3<R> in = shapes[shape].local_inertia(mass);
        b.inv_inertia_local = V3<R>(in.x != R(0) ? R(1) / in.x : R(0), in.y != R(0) ? R(1) / in.y : R(0),
                                    in.z != R(0) ? R(1) / in.z : R(0));
        b.inv_mass = R(1) / mass;
        return b;
    }
    Body<R> make_static(uint32_t shape, const V3<R>& pos) const {
        Body<R> b;
        b.shape = shape;
        b.position = pos;
        b.is_static = true;
        b.activation = ACT_ISLAND_SLEEPING;
        return b;
    }

    // world/islands.rs:31-305 (rigid bodies only; no sensors merge)
    void step_islands(const std::vector<std::pair<uint32_t, uint32_t>>& pairs) {
        size_t n = bodies.size();
        UnionFind uf;
        uf.reset(n);
        std::vector<char> island_awake(n, 0);
        for (auto& p : pairs) {
            const Body<R>& a = bodies[p.first];
            const Body<R>& b = bodies[p.second];
            if ((a.flags | b.flags) & CF_NO_CONTACT_RESPONSE) continue;
            if ((a.group & b.mask) == 0 || (b.group & a.mask) == 0) continue;
            if (a.participates_in_islands() && b.participates_in_islands()) uf.unite(p.first, p.second);
        }
        for (auto& jt : joints) {  // islands.rs:186-196: enabled joints between two dynamic bodies
            if (!jt.enabled) continue;
            if (bodies[jt.body_a].participates_in_islands() && bodies[jt.body_b].participates_in_islands())
                uf.unite(jt.body_a, jt.body_b);
        }
        for (size_t i = 0; i < n; ++i)
            if (bodies[i].participates_in_islands() && bodies[i].is_island_awake()) island_awake[uf.find(i)] = 1;
        bool any_moving_kin = false;
        for (auto& b : bodies)
            if (b.is_kinematic() && (b.linear_velocity.length_squared() != R(0) || b.angular_velocity.length_squared() != R(0)))
                any_moving_kin = true;
        if (any_moving_kin) {
            for (auto& p : pairs) {
                uint32_t ends[2] = {p.first, p.second};
                int ks = -1;
                for (int s = 0; s < 2; ++s) {
                    const Body<R>& kb = bodies[ends[s]];
                    if (kb.is_kinematic() && (kb.linear_velocity.length_squared() != R(0) ||
                                              kb.angular_velocity.length_squared() != R(0))) { ks = s; break; }
                }
                if (ks < 0) continue;
                const Body<R>& a = bodies[p.first];
                const Body<R>& b = bodies[p.second];
                if ((a.flags | b.flags) & CF_NO_CONTACT_RESPONSE) continue;
                if ((a.group & b.mask) == 0 || (b.group & a.mask) == 0) continue;
                uint32_t other = ends[1 - ks];
                if (!bodies[other].participates_in_islands()) continue;
                island_awake[uf.find(other)] = 1;
            }
        }
        std::vector<char> awake(n);
        for (size_t i = 0; i < n; ++i) awake[i] = island_awake[uf.find(i)];
        for (size_t i = 0; i < n; ++i) {
            if (awake[i]) bodies[i].island_wake();
            else if (bodies[i].participates_in_islands()) bodies[i].go_to_sleep();
        }
    }

    void emit_rows(uint32_t i, uint32_t j, const std::vector<ContactPoint<R>>& refresh_out, R inv_dt,
                   std::vector<ContactConstraint<R>>& rows) {
        for (size_t k = 0; k < refresh_out.size(); ++k) {
            ContactPoint<R> cp = refresh_out[k];
            cp.normal_impulse *= info.warmstarting_factor;
            rows.push_back(prepare_contact(i, j, cp, bodies[i], bodies[j], uint32_t(k), inv_dt, info));
        }
    }

    // world/step.rs:281-1287, rigid subset (no joints, multibodies, soft bodies,
    // events, CCD, motion states).
    void step(R dt) {
        clk_start();
        R inv_dt = R(1) / dt;
        size_t n = bodies.size();
        // 1. settled speeds, then integrate velocities (step.rs:306-314)
        std::vector<R> settled(n);
        for (size_t i = 0; i < n; ++i)
            settled[i] = bodies[i].linear_velocity.length_squared() + bodies[i].angular_velocity.length_squared();
        for (auto& b : bodies) b.integrate_velocities(dt);
        clk_mark(0);
        // 2. predicted positions (step.rs:341-343)
        std::vector<V3<R>> pred(n);
        for (size_t i = 0; i < n; ++i) pred[i] = bodies[i].predicted_position(dt);
        // 3. AABBs of active bodies (step.rs:349-363)
        for (size_t i = 0; i < n; ++i) {
            if (!bodies[i].is_active()) continue;
            proxy_aabbs[i] = shapes[bodies[i].shape].world_aabb(pred[i], bodies[i].orientation)
                                 .expanded(CONTACT_BREAKING_THRESHOLD<R>);
        }
        clk_mark(1);
        // 4. broad phase (step.rs:413-415)
        std::vector<std::pair<uint32_t, uint32_t>> pairs;
        if (brute_force_broadphase) brute_force_pairs(proxy_aabbs, pairs);
        else {
            std::vector<char> mesh_proxy(bodies.size(), 0);
            for (size_t i = 0; i < bodies.size(); ++i) mesh_proxy[i] = shapes[bodies[i].shape].type == SHAPE_MESH;
            grid_pairs(proxy_aabbs, pairs, &mesh_proxy);
        }
        clk_mark(2);
        // 4b. islands (step.rs:423)
        step_islands(pairs);
        clk_mark(3);
        // 5. pair pass (step.rs:439-854)
        step_counter += 1;
        bool simulate = false;
        for (auto& b : bodies) if (b.is_active()) { simulate = true; break; }
        uint32_t stamp = step_counter;
        bool prune = simulate && prev_simulate;
        prev_simulate = simulate;
        std::vector<ContactConstraint<R>> rows;
        std::vector<ContactPoint<R>> refresh_out;
        const R REDETECT_SPEED_SQUARED = R(0.08) * R(0.08);  // world.rs:62
        // world.rs:873-880 + step.rs:645-651: pairs linked by a joint with disable_collisions
        // (enabled or not) are skipped like group/mask rejects.
        std::vector<uint64_t> suppressed;
        for (auto& jt : joints)
            if (jt.disable_collisions) suppressed.push_back(pair_key(jt.body_a, jt.body_b));
        std::sort(suppressed.begin(), suppressed.end());
        last_narrowphase_calls = 0;
        for (auto& pr : pairs) {
            uint32_t i = pr.first, j = pr.second;
            Body<R>& a = bodies[i];
            Body<R>& b = bodies[j];
            if ((a.group & b.mask) == 0 || (b.group & a.mask) == 0) continue;
            uint64_t key = pair_key(i, j);
            if (!suppressed.empty() && std::binary_search(suppressed.begin(), suppressed.end(), key)) continue;
            auto it = cache.find(key);
            if (simulate && it != cache.end()) it->second.touched = stamp;
            if (!a.is_active() && !b.is_active()) continue;
            bool no_response = ((a.flags | b.flags) & CF_NO_CONTACT_RESPONSE) != 0;
            if (a.is_static_or_kinematic() && b.is_static_or_kinematic()) continue;
            V3<R> pa = pred[i], pb = pred[j];
            bool fast = settled[i] > REDETECT_SPEED_SQUARED || settled[j] > REDETECT_SPEED_SQUARED;
            bool served = false;
            if (it != cache.end() && !it->second.needs_redetect(pa, a.orientation, pb, b.orientation)) {
                it->second.refresh(pa, a.orientation, pb, b.orientation, refresh_out);
                bool deep = false;
                for (auto& cp : refresh_out) if (cp.penetration > info.linear_slop) deep = true;
                if (!fast || !deep) {
                    if (!no_response) emit_rows(i, j, refresh_out, inv_dt, rows);
                    served = true;
                }
            }
            if (served) continue;
            V3<R> seed;
            bool has_seed = it != cache.end() && it->second.seed(seed);
            Manifold<R> m;
            last_narrowphase_calls++;
            if (collide(shapes[a.shape], pa, a.orientation, shapes[b.shape], pb, b.orientation, has_seed, seed, m)) {
                PersistentManifold<R>& pm = cache[key];
                pm.touched = stamp;
                R thr = std::min(shapes[a.shape].contact_breaking_threshold(), shapes[b.shape].contact_breaking_threshold());
                pm.capture(m, pa, a.orientation, pb, b.orientation, thr);
                pm.refresh(pa, a.orientation, pb, b.orientation, refresh_out);
                if (!no_response) emit_rows(i, j, refresh_out, inv_dt, rows);
            } else {
                cache.erase(key);
            }
        }
        // Optional re-ordering of the row groups (same rows, different solve order).
        if (!solve_order.empty()) {
            std::unordered_map<uint64_t, size_t> rank;
            for (size_t r = 0; r < solve_order.size(); ++r) rank[solve_order[r]] = r;
            std::stable_sort(rows.begin(), rows.end(), [&](const ContactConstraint<R>& x, const ContactConstraint<R>& y) {
                auto rx = rank.find(pair_key(x.body_a, x.body_b));
                auto ry = rank.find(pair_key(y.body_a, y.body_b));
                size_t vx = rx == rank.end() ? SIZE_MAX : rx->second;
                size_t vy = ry == rank.end() ? SIZE_MAX : ry->second;
                return vx < vy;
            });
        }
        last_rows_pre = rows;
        // 5a. joint rows from the current poses (step.rs:928-949): joints of a sleeping island
        // (both bodies inactive) produce none.
        std::vector<JointRow<R>> jrows;
        for (size_t o = 0; o < joints.size(); ++o) {
            uint32_t jid = joint_order.empty() ? uint32_t(o) : joint_order[o];
            Joint<R>& jt = joints[jid];
            if (!bodies[jt.body_a].is_active() && !bodies[jt.body_b].is_active()) continue;
            prepare_joint_rows(jt, jid, bodies, inv_dt, info.erp, jrows, info.global_cfm);
        }
        clk_mark(4);
        // 6. solve (step.rs:959-972)
        solve(bodies, rows, inv_dt, info, &jrows);
        last_joint_rows = jrows;
        // 6b. impulse writeback + prune (step.rs:982-1010)
        for (auto& c : rows) {
            auto ci = cache.find(pair_key(c.body_a, c.body_b));
            if (ci == cache.end()) continue;
            if (c.point_index < ci->second.points.size()) ci->second.points[c.point_index].normal_impulse = c.normal_impulse;
        }
        if (prune) {
            for (auto ci = cache.begin(); ci != cache.end();) {
                if (ci->second.touched != stamp) ci = cache.erase(ci);
                else ++ci;
            }
        }
        clk_mark(5);
        // 6c. deactivation (step.rs:1059-1061)
        for (auto& b : bodies) b.update_deactivation(dt);
        // 7a. CCD clamp fractions (step.rs:1068-1155): a fast CCD body is swept as a sphere from its
        // position along v dt against every other body that passes the collision filters and whose
        // broad-phase proxy AABB touches the swept box; the first hit fraction is kept.
        std::vector<R> ccd_clamps(n, R(1));
        for (size_t i = 0; i < n; ++i) {
            const Body<R>& body = bodies[i];
            const R threshold = body.ccd_threshold;
            if (!body.is_active() || body.is_static_or_kinematic() || threshold <= R(0)) continue;
            const R radius = body.ccd_radius;
            if (radius <= R(0) || !shapes[body.shape].is_convex()) continue;
            const V3<R> from = body.position;
            const V3<R> to = from + body.linear_velocity * dt;
            if ((to - from).length_squared() <= threshold * threshold) continue;
            R best = R(1);
            const Aabb<R> swept = Aabb<R>(from.min(to), from.max(to)).expanded(radius);
            for (size_t j = 0; j < n; ++j) {
                if (i == j) continue;
                const Body<R>& other = bodies[j];
                if (other.flags & CF_NO_CONTACT_RESPONSE) continue;
                if (!suppressed.empty() &&
                    std::binary_search(suppressed.begin(), suppressed.end(), pair_key(uint32_t(i), uint32_t(j))))
                    continue;
                if ((body.group & other.mask) == 0 || (other.group & body.mask) == 0) continue;
                if (!proxy_aabbs[j].overlaps(swept)) continue;
                SweepHit<R> hit;
                if (swept_sphere_cast(from, to, radius, shapes[other.shape], other.position, other.orientation, hit) &&
                    hit.fraction < best)
                    best = hit.fraction;
            }
            ccd_clamps[i] = best;
        }
        last_ccd_clamps = ccd_clamps;
        // 7. integrate positions + split-impulse push (step.rs:1171-1215)
        for (size_t bi = 0; bi < n; ++bi) {
            Body<R>& b = bodies[bi];
            if (!(b.is_static || !b.is_active())) {
                V3<R> np; Quat<R> nq;
                interpolate_pose(b.position, b.orientation, b.linear_velocity, b.angular_velocity, dt, np, nq);
                b.position = np;
                b.orientation = nq;
            }
            V3<R> pl = b.push_linear, pw = b.push_angular;
            if (b.is_active() && !b.is_static_or_kinematic() && (pl.x != R(0) || pl.y != R(0) || pl.z != R(0)))
                b.position += pl * dt;
            if (b.is_active() && !b.is_static_or_kinematic() && (pw.x != R(0) || pw.y != R(0) || pw.z != R(0))) {
                V3<R> w = pw * info.split_impulse_turn_erp;
                Quat<R> dq = Quat<R>(w.x * dt * R(0.5), w.y * dt * R(0.5), w.z * dt * R(0.5), R(0)) * b.orientation;
                b.orientation = (b.orientation + dq).normalize();
            }
            b.push_linear = V3<R>();
            b.push_angular = V3<R>();
            if (ccd_clamps[bi] < R(1)) {  // step.rs:1210-1214
                V3<R> from = b.position - b.linear_velocity * dt;
                b.position = from + (b.position - from) * ccd_clamps[bi];
            }
        }
        // 8. clear forces (step.rs:1272-1274)
        for (auto& b : bodies) { b.force = V3<R>(); b.torque = V3<R>(); }
        last_pairs = pairs;
        last_rows = rows;
        last_predicted = pred;
        clk_mark(6);
    }
};

}  // namespace oracle
