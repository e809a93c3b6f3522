// CPU oracle — TEST INFRASTRUCTURE ONLY: joint rows in the PGS solve.
//
// Restates, for the point-to-point, fixed and hinge joints:
//   crates/bullet-dynamics/src/solver/sequential_impulse.rs:214-328 (ConstraintRow, prepare),
//     :931-971 (solve_joint_row), :720-735 (joint rows after the contacts in each sweep);
//   crates/bullet-dynamics/src/constraint.rs:755-842 (prepare_rows: point-to-point rows),
//     :658-752 (JointFrame, AngularLimit::test);
//   crates/bullet-dynamics/src/constraint/fixed.rs:33-90 (locked-6DOF rows);
//   crates/bullet-dynamics/src/constraint/hinge.rs:60-100 (frames from pivot/axis), :130-267 (rows);
//   crates/bullet-dynamics/src/constraint/shared.rs:6-155 (hinge angle, angle wrap, Euler XYZ,
//     relative rotation axes, motor factor);
//   crates/bullet-dynamics/src/constraint/gear.rs:33-57 (gear: one angular coupling row; the
//     axes are the frames' z columns here);
//   crates/bullet-dynamics/src/constraint/slider.rs:159-475 (slider: frame-offset rows, linear and
//     angular limits and motors), shared.rs:30-55 (adjust_angle_to_limits), :126-145
//     (mirrored_row_limits);
//   crates/bullet-dynamics/src/constraint/generic6dof.rs:159-546 (classic 6DOF: per-axis limit or
//     motor rows, the universal frames);
//   crates/bullet-dynamics/src/constraint/conetwist.rs:222-548 (cone twist: pivot rows, elliptical
//     swing limit, fixed and hinge configurations, twist limit, motor target);
//   crates/bullet-dynamics/src/constraint/generic6dof_spring2.rs:650-1383 (spring 2: per-axis
//     limit pairs, lock rows, motors, servos, clamped springs, six Euler orders, static-body
//     mass split), with the global ERP / CFM fallback of prepare_rows (constraint.rs:755-829).
// Frame construction uses glam 0.33.3's `Quat::from_rotation_arc` (not in the reference tree);
// its published algorithm is restated in rotation_arc() below.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>
#include "oracle_math.hpp"

namespace oracle {

enum : uint32_t { JOINT_POINT2POINT = 0, JOINT_FIXED = 1, JOINT_HINGE = 2, JOINT_GEAR = 3, JOINT_SLIDER = 4, JOINT_SPRING2 = 5,
                  JOINT_CONETWIST = 6, JOINT_GENERIC6DOF = 7 };
// RowLimits (sequential_impulse.rs): which clamp the accumulated impulse takes.
enum : uint32_t { LIM_UNBOUNDED = 0, LIM_BILATERAL = 1, LIM_LOWER = 2, LIM_UPPER = 3, LIM_WINDOW = 4 };

template <class R>
struct JointFrame {  // constraint.rs:658-682
    V3<R> origin;
    M3<R> basis;  // column 2 is the hinge axis
};

template <class R>
struct AngularLimit {  // constraint.rs:684-752
    R low = 0, high = 0, softness = R(0.9), bias_factor = R(0.3), relaxation = R(1);
};

// Generic6DofSpring2 per-axis parameters: RotationalLimitMotor2 (generic6dof_spring2.rs:47-128)
// for the angular axes 3-5, and one column of TranslationalLimitMotor2 (:155-232) for the linear
// axes 0-2. lower > upper frees the axis, == locks it, < limits it (two one-sided rows).
enum : uint32_t {
    S2_MOTOR = 1, S2_SERVO = 2, S2_SPRING = 4, S2_STIFFNESS_LIMITED = 8, S2_DAMPING_LIMITED = 16,
    // per-axis ERP/CFM overrides (Bullet's BT_6DOF_FLAGS_*2): without them the global values apply
    S2_STOP_ERP = 32, S2_STOP_CFM = 64, S2_MOTOR_ERP = 128, S2_MOTOR_CFM = 256
};
template <class R>
struct Spring2Axis {
    R lower = 1, upper = -1, bounce = 0, stop_erp = R(0.2), stop_cfm = 0, motor_erp = R(0.9), motor_cfm = 0;
    R target_velocity = 0, max_motor_force = R(6), servo_target = 0, stiffness = 0, damping = 0, equilibrium = 0;
    uint32_t flags = 0;
    // per-step state (testLimitValue): 0 free, 3 locked, 4 limited
    int current_limit = 0;
    R error = 0, error_hi = 0, position = 0;
};
enum : uint32_t { ORDER_XYZ = 0, ORDER_XZY = 1, ORDER_YXZ = 2, ORDER_YZX = 3, ORDER_ZXY = 4, ORDER_ZYX = 5 };

template <class R>
struct Joint {
    uint32_t kind = JOINT_POINT2POINT, body_a = 0, body_b = 0;
    bool enabled = true, disable_collisions = true;
    JointFrame<R> frame_a, frame_b;  // point-to-point: the origins are the pivots
    R impulse_clamp = 0;             // point-to-point (p2p.rs:11-17)
    bool has_erp = false;
    R erp = 0;
    bool angular_only = false, has_limit = false, has_motor = false;  // hinge (hinge.rs:20-45)
    AngularLimit<R> limit;
    R motor_target = 0, motor_max = 0;
    R gear_ratio = 1;   // gear (gear.rs:9-13): axes are the frames' basis z columns
    R hinge_angle = 0;  // per-step state (hinge.rs:37)
    // slider (slider.rs:8-60, defaults of SliderConstraint::new)
    R lower_lin = 1, upper_lin = -1, lower_ang = 0, upper_ang = 0;
    R softness_lim_lin = 1, softness_lim_ang = 1, damping_lim_lin = 1, damping_lim_ang = 1;
    R softness_ortho_lin = 1, softness_ortho_ang = 1;
    bool has_lin_motor = false, has_ang_motor = false, use_frame_a = true;
    R lin_motor_target = 0, lin_motor_max = 0, ang_motor_target = 0, ang_motor_max = 0;
    R lin_pos = 0, ang_pos = 0;  // per-step state
    // generic 6DOF spring 2 (Generic6DofSpring2Constraint::new: linear axes locked, angular free)
    uint32_t rotate_order = ORDER_XYZ;
    Spring2Axis<R> s2[6];
    V3<R> s2_diff, s2_euler;  // per-step state: pivot offset in A's frame, relative Euler angles
    R fact_a = R(0.5), fact_b = R(0.5);
    bool has_static_body = false;
    // cone twist (ConeTwistConstraint, conetwist.rs:5-116): spans, limit softness, bias and
    // relaxation; an optional motor target in constraint space with its max impulse (< 0: none)
    R ct_span1 = R(1e30), ct_span2 = R(1e30), ct_twist = R(1e30), ct_softness = 1, ct_bias = R(0.3), ct_relax = 1;
    bool ct_has_motor = false;
    Quat<R> ct_target;
    R ct_max_impulse = -1;
    R ct_twist_angle = 0;  // per-step state
    Joint() {
        for (int i = 0; i < 3; ++i) { s2[i].lower = 0; s2[i].upper = 0; s2[i].max_motor_force = 0; }
    }
};

template <class R>
struct JointRow {  // sequential_impulse.rs:214-258
    uint32_t body_a = 0, body_b = 0, joint = 0;
    V3<R> lin_a, ang_a, lin_b, ang_b;
    R inv_mass_a = 0, inv_mass_b = 0;
    M3<R> iia, iib;
    R mass = 0, bias = 0, cfm = 0;
    uint32_t lim = LIM_UNBOUNDED;
    R lo = 0, hi = 0;
    R impulse = 0;
};

// sequential_impulse.rs:260-299 (ConstraintRow::prepare)
template <class R, class B>
JointRow<R> prepare_joint_row(uint32_t ia, uint32_t ib, const V3<R>& lin_a, const V3<R>& ang_a, const V3<R>& lin_b,
                              const V3<R>& ang_b, const B& a, const B& b, R bias, uint32_t lim, R lo, R hi) {
    JointRow<R> r;
    r.body_a = ia; r.body_b = ib;
    r.lin_a = lin_a; r.ang_a = ang_a; r.lin_b = lin_b; r.ang_b = ang_b;
    r.iia = a.inv_inertia_world();
    r.iib = b.inv_inertia_world();
    r.inv_mass_a = a.inv_mass;
    r.inv_mass_b = b.inv_mass;
    R k = r.inv_mass_a * lin_a.length_squared() + r.inv_mass_b * lin_b.length_squared() + ang_a.dot(r.iia * ang_a) +
          ang_b.dot(r.iib * ang_b);
    r.mass = k > R(0) ? R(1) / k : R(0);
    r.bias = bias;
    r.lim = lim; r.lo = lo; r.hi = hi;
    return r;
}

// sequential_impulse.rs:931-971 (solve_joint_row)
template <class R, class B>
void solve_joint_row(std::vector<B>& bodies, JointRow<R>& c, R damping) {
    B& a = bodies[c.body_a];
    B& b = bodies[c.body_b];
    R row_vel = (c.lin_b.dot(b.linear_velocity) + c.ang_b.dot(b.angular_velocity)) -
                (c.lin_a.dot(a.linear_velocity) + c.ang_a.dot(a.angular_velocity));
    R old = c.impulse;
    R base = damping != R(1) ? c.mass * (c.bias - row_vel * damping) : c.mass * (c.bias - row_vel);
    R lambda = c.cfm != R(0) ? base - c.cfm * old : base;
    R nw = old + lambda;
    switch (c.lim) {
        case LIM_BILATERAL: nw = std::min(std::max(nw, -c.hi), c.hi); break;
        case LIM_LOWER: nw = std::max(nw, c.lo); break;
        case LIM_UPPER: nw = std::min(nw, c.hi); break;
        case LIM_WINDOW: nw = std::min(std::max(nw, c.lo), c.hi); break;
        default: break;
    }
    c.impulse = nw;
    R j = nw - old;
    if (j != R(0)) {
        a.linear_velocity -= c.lin_a * (j * c.inv_mass_a);
        b.linear_velocity += c.lin_b * (j * c.inv_mass_b);
        a.angular_velocity -= c.iia * (c.ang_a * j);
        b.angular_velocity += c.iib * (c.ang_b * j);
    }
}

// shared.rs:9-14 (get_hinge_angle)
template <class R>
R hinge_angle_of(const M3<R>& tr_a, const M3<R>& tr_b) {
    V3<R> swing = tr_b.c1;
    return std::atan2(swing.dot(tr_a.c0), swing.dot(tr_a.c1));
}

// shared.rs:17-27 (normalize_angle; % truncates like fmod)
template <class R>
R normalize_angle(R angle) {
    const R pi = R(3.14159265358979323846);
    const R two_pi = R(2) * pi;
    R a = std::fmod(angle, two_pi);
    if (a < -pi) a += two_pi;
    else if (a > pi) a -= two_pi;
    return a;
}

// constraint.rs:735-751 (AngularLimit::test): correction, sign, active
template <class R>
void limit_test(const AngularLimit<R>& l, R angle, R& correction, R& sign, bool& active) {
    R half_range = (l.high - l.low) / R(2);
    correction = 0; sign = 0; active = false;
    if (half_range >= R(0)) {
        R center = normalize_angle(l.low + half_range);
        R deviation = normalize_angle(angle - center);
        if (deviation < -half_range) { correction = -(deviation + half_range); sign = 1; active = true; return; }
        if (deviation > half_range) { correction = half_range - deviation; sign = -1; active = true; return; }
    }
}

// shared.rs:123-155 (get_motor_factor)
template <class R>
R motor_factor(R pos, R low_lim, R upp_lim, R vel, R time_fact) {
    if (low_lim > upp_lim) return R(1);
    if (low_lim == upp_lim) return R(0);
    R delta_max = vel / time_fact;
    if (delta_max < R(0)) {
        if (pos >= low_lim && pos < low_lim - delta_max) return (low_lim - pos) / delta_max;
        if (pos < low_lim) return R(0);
        return R(1);
    }
    if (delta_max > R(0)) {
        if (pos <= upp_lim && pos > upp_lim - delta_max) return (upp_lim - pos) / delta_max;
        if (pos > upp_lim) return R(0);
        return R(1);
    }
    return R(0);
}

// shared.rs:85-101 (euler_xyz: Bullet's matrixToEulerXYZ on column-major storage)
template <class R>
V3<R> euler_xyz(const M3<R>& m) {
    const R half_pi = R(1.57079632679489661923);
    R r20 = m.c0.z, r21 = m.c1.z, r22 = m.c2.z, r10 = m.c0.y, r11 = m.c1.y, r01 = m.c1.x, r00 = m.c0.x;
    if (r20 < R(1)) {
        if (r20 > R(-1)) return V3<R>(std::atan2(-r21, r22), std::asin(r20), std::atan2(-r10, r00));
        return V3<R>(-std::atan2(r01, r11), -half_pi, R(0));
    }
    return V3<R>(std::atan2(r01, r11), half_pi, R(0));
}

// shared.rs:108-123 (relative_rotation_info)
template <class R>
void relative_rotation_info(const M3<R>& tr_a, const M3<R>& tr_b, V3<R>& euler, V3<R> axes[3]) {
    M3<R> relative = tr_a.transpose() * tr_b;
    euler = euler_xyz(relative);
    V3<R> axis0 = tr_b.c0, axis2 = tr_a.c2;
    axes[1] = axis2.cross(axis0);
    axes[0] = axes[1].cross(axis2);
    axes[2] = axis0.cross(axes[1]);
    for (int i = 0; i < 3; ++i) axes[i] = axes[i].normalize();
}

// shared.rs:30-55 (adjust_angle_to_limits)
template <class R>
R adjust_angle_to_limits(R angle, R lo, R hi) {
    const R two_pi = R(2) * R(3.14159265358979323846);
    if (lo >= hi) return angle;
    if (angle < lo) {
        R diff_lo = std::fabs(normalize_angle(lo - angle));
        R diff_hi = std::fabs(normalize_angle(hi - angle));
        return diff_lo < diff_hi ? angle : angle + two_pi;
    }
    if (angle > hi) {
        R diff_hi = std::fabs(normalize_angle(angle - hi));
        R diff_lo = std::fabs(normalize_angle(angle - lo));
        return diff_lo < diff_hi ? angle - two_pi : angle;
    }
    return angle;
}

// shared.rs:126-145 (mirrored_row_limits): Bullet's window [lower, upper] in the row convention.
template <class R>
void mirrored_row_limits(R lower, R upper, uint32_t& lim, R& lo, R& hi) {
    const bool lower_inf = std::isinf(lower) && lower < R(0);
    const bool upper_inf = std::isinf(upper) && upper > R(0);
    lo = 0; hi = 0;
    if (lower_inf && upper_inf) lim = LIM_UNBOUNDED;
    else if (lower_inf) lim = LIM_LOWER;   // lower bound 0
    else if (upper_inf) lim = LIM_UPPER;   // upper bound 0
    else { lim = LIM_BILATERAL; hi = (upper - lower) / R(2); lo = -hi; }
}

// glam Quat::from_rotation_arc (published algorithm): identity for parallel unit vectors, a half
// turn about any orthonormal vector for opposite ones, else normalize(from x to, 1 + from . to).
template <class R>
Quat<R> rotation_arc(const V3<R>& from, const V3<R>& to) {
    const R eps = std::numeric_limits<R>::epsilon();
    const R one_minus_eps = R(1) - R(2) * eps;
    R d = from.dot(to);
    if (d > one_minus_eps) return Quat<R>::identity();
    if (d < -one_minus_eps) {
        // A half turn about a vector orthonormal to `from` (Duff et al. 2017 branchless basis).
        // Which of the two basis vectors glam picks is not pinned here: hinge frames of exactly
        // opposite axes are outside the parity cases.
        R sign = std::signbit(from.z) ? R(-1) : R(1);
        R aa = R(-1) / (sign + from.z);
        R bb = from.x * from.y * aa;
        V3<R> o(bb, sign + from.y * from.y * aa, -from.y);
        R half = R(3.14159265358979323846) * R(0.5);
        R s = std::sin(half);
        return Quat<R>(o.x * s, o.y * s, o.z * s, std::cos(half));
    }
    V3<R> c = from.cross(to);
    return Quat<R>(c.x, c.y, c.z, R(1) + d).normalize();
}

// hinge.rs:60-100 (HingeConstraint::new): frames from pivots and axes.
template <class R>
void hinge_frames(const V3<R>& pivot_a, const V3<R>& axis_a_in, const V3<R>& pivot_b, const V3<R>& axis_b_in,
                  JointFrame<R>& fa, JointFrame<R>& fb) {
    V3<R> axis_a = axis_a_in.normalize(), axis_b = axis_b_in.normalize();
    V3<R> helper = std::fabs(axis_a.x) < R(0.9) ? V3<R>(1, 0, 0) : V3<R>(0, 1, 0);
    V3<R> t1 = axis_a.cross(helper).normalize();
    V3<R> t2 = axis_a.cross(t1);
    fa.origin = pivot_a;
    fa.basis = M3<R>(t1, t2, axis_a);
    Quat<R> rot = rotation_arc(axis_a, axis_b);
    V3<R> t1b = rot.rotate(t1);
    V3<R> t2b = axis_b.cross(t1b);
    fb.origin = pivot_b;
    fb.basis = M3<R>(t1b, t2b, axis_b);
}

// glam 0.33.3 Quat::from_mat3 (not in the reference tree; used through compat.rs:52-62): the
// published branch on the diagonal (m22, then m11 -/+ m00) choosing the largest of x, y, z, w to
// divide by. mRC below is column R, row C.
template <class R>
Quat<R> quat_from_mat3(const M3<R>& m) {
    const R m00 = m.c0.x, m01 = m.c0.y, m02 = m.c0.z, m10 = m.c1.x, m11 = m.c1.y, m12 = m.c1.z;
    const R m20 = m.c2.x, m21 = m.c2.y, m22 = m.c2.z;
    if (m22 <= R(0)) {
        const R dif10 = m11 - m00, omm22 = R(1) - m22;
        if (dif10 <= R(0)) {
            const R f = omm22 - dif10, inv = R(0.5) / std::sqrt(f);
            return Quat<R>(f * inv, (m01 + m10) * inv, (m02 + m20) * inv, (m12 - m21) * inv);
        }
        const R f = omm22 + dif10, inv = R(0.5) / std::sqrt(f);
        return Quat<R>((m01 + m10) * inv, f * inv, (m12 + m21) * inv, (m20 - m02) * inv);
    }
    const R sum10 = m11 + m00, opm22 = R(1) + m22;
    if (sum10 <= R(0)) {
        const R f = opm22 - sum10, inv = R(0.5) / std::sqrt(f);
        return Quat<R>((m02 + m20) * inv, (m12 + m21) * inv, f * inv, (m01 - m10) * inv);
    }
    const R f = opm22 + sum10, inv = R(0.5) / std::sqrt(f);
    return Quat<R>((m12 - m21) * inv, (m20 - m02) * inv, (m01 - m10) * inv, f * inv);
}

// conetwist.rs:546-548
template <class R>
R quaternion_angle(const Quat<R>& q) {
    return R(2) * std::acos(std::min(std::max(q.w, R(-1)), R(1)));
}

// conetwist.rs:481-502 (compute_cone_limit_info): swing angle, axis, elliptical limit
template <class R>
void ct_cone_limit_info(const Joint<R>& jt, const Quat<R>& q, R& angle, V3<R>& axis, R& limit) {
    const R eps = std::numeric_limits<R>::epsilon();
    angle = quaternion_angle(q);
    axis = V3<R>();
    limit = jt.ct_span1;
    if (angle > eps) {
        axis = q.xyz().normalize();
        const R xe = axis.y, ye = -axis.z;
        if (std::fabs(xe) > eps) {
            const R slope2 = (ye * ye) / (xe * xe);
            R norm = R(1) / (jt.ct_span2 * jt.ct_span2);
            norm += slope2 / (jt.ct_span1 * jt.ct_span1);
            limit = std::sqrt((R(1) + slope2) / norm);
        }
    }
}

// conetwist.rs:504-519 (compute_twist_limit_info)
template <class R>
void ct_twist_limit_info(const Quat<R>& q, R& angle, V3<R>& axis) {
    Quat<R> qm = q;
    angle = quaternion_angle(q);
    if (angle > R(3.14159265358979323846)) {
        qm = Quat<R>(-q.x, -q.y, -q.z, -q.w);
        angle = quaternion_angle(qm);
    }
    axis = qm.xyz();
    if (angle > std::numeric_limits<R>::epsilon()) axis = axis.normalize();
}

// conetwist.rs:222-342 (prepare_rows) with calc_angle_info (:344-479) and
// adjust_swing_axis_to_use_ellipse_normal (:521-539).
template <class R, class B>
void prepare_conetwist_rows(Joint<R>& jt, uint32_t ia, uint32_t ib, const B& a, const B& b, R inv_dt, R erp,
                            std::vector<JointRow<R>>& out) {
    const R eps = std::numeric_limits<R>::epsilon(), fix = R(0.05);
    const R inf = std::numeric_limits<R>::infinity();
    M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
    M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
    V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
    V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
    V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
    const R k = inv_dt * erp;
    auto push = [&](const V3<R>& la, const V3<R>& aa, const V3<R>& lb, const V3<R>& ab, R bias, uint32_t lim, R lo,
                    R hi) { out.push_back(prepare_joint_row(ia, ib, la, aa, lb, ab, a, b, bias, lim, lo, hi)); };
    const V3<R> zero;
    for (int axis = 0; axis < 3; ++axis) {
        V3<R> n;
        n.at(axis) = R(1);
        push(n, r_a.cross(n), n, r_b.cross(n), k * (pivot_a - pivot_b)[axis], LIM_UNBOUNDED, 0, 0);
    }
    // calc_angle_info
    R swing_corr = 0, twist_corr = 0;
    V3<R> swing_axis, twist_axis;
    bool solve_swing = false, solve_twist = false;
    const V3<R> X(1, 0, 0);
    if (jt.ct_has_motor) {
        M3<R> r_delta = tr_b * M3<R>::from_quat(jt.ct_target) * tr_a.transpose();
        Quat<R> q_delta = quat_from_mat3(r_delta).normalize();
        V3<R> sa = q_delta.xyz();
        R l2 = sa.length_squared();
        if (l2 > eps) {
            swing_axis = sa / std::sqrt(l2);
            swing_corr = quaternion_angle(q_delta);
            if (std::fabs(swing_corr) > eps) solve_swing = true;
        }
    } else {
        Quat<R> q_a = quat_from_mat3(tr_a), q_b = quat_from_mat3(tr_b);
        Quat<R> q_ab = (q_b.inverse() * q_a).normalize();
        V3<R> v_cone = q_ab.rotate(X).normalize();
        Quat<R> q_cone = rotation_arc(X, v_cone).normalize();
        Quat<R> q_twist = (q_cone.inverse() * q_ab).normalize();
        const R s1 = jt.ct_span1, s2 = jt.ct_span2;
        if (s1 >= fix && s2 >= fix) {
            R angle, limit;
            V3<R> axis;
            ct_cone_limit_info(jt, q_cone, angle, axis, limit);
            if (angle > limit * jt.ct_softness) {
                solve_swing = true;
                swing_corr = angle - limit * jt.ct_softness;
                // adjust_swing_axis_to_use_ellipse_normal
                R y = -axis.z, z = axis.y;
                if (std::fabs(z) > eps) {
                    R grad = y / z;
                    grad *= s2 / s1;
                    y = y > R(0) ? std::fabs(grad * z) : -std::fabs(grad * z);
                    axis.z = -y;
                    axis.y = z;
                    axis = axis.normalize();
                }
                swing_axis = q_b.rotate(-axis);
            }
        } else {
            const V3<R> iv_a = tr_a.c0, jv_a = tr_a.c1, kv_a = tr_a.c2, iv_b = tr_b.c0;
            R x = iv_b.dot(iv_a), y = iv_b.dot(jv_a), z = iv_b.dot(kv_a);
            if (s1 < fix && s2 < fix) {
                if (std::fabs(y) > eps || std::fabs(z) > eps) {
                    solve_swing = true;
                    swing_axis = -iv_b.cross(iv_a);
                }
            } else {
                if (s1 < fix) {
                    if (std::fabs(x) > eps || std::fabs(z) > eps) {
                        solve_swing = true;
                        if (s2 >= fix) {
                            y = 0;
                            R span2 = std::atan2(z, x);
                            if (span2 > s2) { x = std::cos(s2); z = std::sin(s2); }
                            else if (span2 < -s2) { x = std::cos(s2); z = -std::sin(s2); }
                        }
                    }
                } else {
                    if (std::fabs(x) > eps || std::fabs(y) > eps) {
                        solve_swing = true;
                        if (s1 >= fix) {
                            z = 0;
                            R span1 = std::atan2(y, x);
                            if (span1 > s1) { x = std::cos(s1); y = std::sin(s1); }
                            else if (span1 < -s1) { x = std::cos(s1); y = -std::sin(s1); }
                        }
                    }
                }
                V3<R> target = (iv_a * x + jv_a * y + kv_a * z).normalize();
                swing_axis = -iv_b.cross(target);
                swing_corr = swing_axis.length();
                if (std::fabs(swing_corr) > eps) swing_axis = swing_axis.normalize();
            }
        }
        if (jt.ct_twist >= R(0)) {
            R angle;
            V3<R> axis;
            ct_twist_limit_info(q_twist, angle, axis);
            jt.ct_twist_angle = angle;
            if (angle > jt.ct_twist * jt.ct_softness) {
                solve_twist = true;
                twist_corr = angle - jt.ct_twist * jt.ct_softness;
                twist_axis = q_b.rotate(-axis);
            }
        } else {
            jt.ct_twist_angle = 0;
        }
    }
    const R relax = jt.ct_relax;
    if (solve_swing) {
        if (jt.ct_span1 < fix && jt.ct_span2 < fix) {
            const R fact = inv_dt * relax;
            const V3<R> dirs[2] = {tr_a.c1, tr_a.c2};
            for (const V3<R>& dir : dirs) push(zero, dir, zero, dir, -fact * swing_axis.dot(dir), LIM_UNBOUNDED, 0, 0);
        } else {
            V3<R> ax1 = swing_axis * (relax * relax);
            if (jt.ct_has_motor && jt.ct_max_impulse >= R(0))
                push(zero, ax1, zero, ax1, -inv_dt * jt.ct_bias * swing_corr, LIM_WINDOW, -jt.ct_max_impulse, R(0));
            else
                push(zero, ax1, zero, ax1, -inv_dt * jt.ct_bias * swing_corr, LIM_UPPER, R(0), R(0));
        }
    }
    if (solve_twist) {
        V3<R> ax1 = twist_axis * (relax * relax);
        uint32_t lim = jt.ct_twist > R(0) ? (twist_corr > R(0) ? LIM_UPPER : LIM_LOWER) : LIM_UNBOUNDED;
        push(zero, ax1, zero, ax1, -inv_dt * jt.ct_bias * twist_corr, lim, R(0), R(0));
    }
    (void)inf;
}

// generic6dof_spring2.rs:1236-1241 (btGetMatrixElem): row index % 3 of column index / 3.
template <class R>
R mat_elem(const M3<R>& m, int index) {
    return m.col(index / 3)[index % 3];
}

// generic6dof_spring2.rs:1243-1373 (matrixToEuler{XZY,YXZ,YZX,ZXY,ZYX}); XYZ is euler_xyz above.
// The gimbal fallback angles feed the state (the "exact" flag is ignored upstream).
template <class R>
V3<R> matrix_to_euler(const M3<R>& m, uint32_t order) {
    const R half_pi = R(1.57079632679489661923);
    auto e = [&](int i) { return mat_elem(m, i); };
    switch (order) {
        case ORDER_XZY: {
            R fi = e(1);
            if (fi < R(1)) {
                if (fi > R(-1)) return V3<R>(std::atan2(e(7), e(4)), std::atan2(e(2), e(0)), std::asin(-e(1)));
                return V3<R>(-std::atan2(-e(6), e(8)), R(0), half_pi);
            }
            return V3<R>(std::atan2(-e(6), e(8)), R(0), -half_pi);
        }
        case ORDER_YXZ: {
            R fi = e(5);
            if (fi < R(1)) {
                if (fi > R(-1)) return V3<R>(std::asin(-e(5)), std::atan2(e(2), e(8)), std::atan2(e(3), e(4)));
                return V3<R>(half_pi, -std::atan2(-e(1), e(0)), R(0));
            }
            return V3<R>(-half_pi, std::atan2(-e(1), e(0)), R(0));
        }
        case ORDER_YZX: {
            R fi = e(3);
            if (fi < R(1)) {
                if (fi > R(-1)) return V3<R>(std::atan2(-e(5), e(4)), std::atan2(-e(6), e(0)), std::asin(e(3)));
                return V3<R>(R(0), -std::atan2(e(7), e(8)), -half_pi);
            }
            return V3<R>(R(0), std::atan2(e(7), e(8)), half_pi);
        }
        case ORDER_ZXY: {
            R fi = e(7);
            if (fi < R(1)) {
                if (fi > R(-1)) return V3<R>(std::asin(e(7)), std::atan2(-e(6), e(8)), std::atan2(-e(1), e(4)));
                return V3<R>(-half_pi, R(0), -std::atan2(e(2), e(0)));
            }
            return V3<R>(half_pi, R(0), std::atan2(e(2), e(0)));
        }
        case ORDER_ZYX: {
            R fi = e(6);
            if (fi < R(1)) {
                if (fi > R(-1)) return V3<R>(std::atan2(e(7), e(8)), std::asin(-e(6)), std::atan2(e(3), e(0)));
                return V3<R>(R(0), half_pi, -std::atan2(-e(1), -e(2)));
            }
            return V3<R>(R(0), -half_pi, std::atan2(-e(1), -e(2)));
        }
        default: return euler_xyz(m);
    }
}

// generic6dof_spring2.rs:1164-1233 (calculate_angle_info): Euler angles of trA^-1 trB in the
// configured order and the three normalized world axes built from per-order cross products.
template <class R>
void spring2_angle_info(const M3<R>& tr_a, const M3<R>& tr_b, uint32_t order, V3<R>& euler, V3<R> axes[3]) {
    euler = matrix_to_euler(tr_a.transpose() * tr_b, order);
    switch (order) {
        case ORDER_XZY: {
            V3<R> axis0 = tr_b.c0, axis1 = tr_a.c1;
            axes[2] = axis0.cross(axis1); axes[0] = axis1.cross(axes[2]); axes[1] = axes[2].cross(axis0);
            break;
        }
        case ORDER_YXZ: {
            V3<R> axis1 = tr_b.c1, axis2 = tr_a.c2;
            axes[0] = axis1.cross(axis2); axes[1] = axis2.cross(axes[0]); axes[2] = axes[0].cross(axis1);
            break;
        }
        case ORDER_YZX: {
            V3<R> axis0 = tr_a.c0, axis1 = tr_b.c1;
            axes[2] = axis0.cross(axis1); axes[0] = axis1.cross(axes[2]); axes[1] = axes[2].cross(axis0);
            break;
        }
        case ORDER_ZXY: {
            V3<R> axis1 = tr_a.c1, axis2 = tr_b.c2;
            axes[0] = axis1.cross(axis2); axes[1] = axis2.cross(axes[0]); axes[2] = axes[0].cross(axis1);
            break;
        }
        case ORDER_ZYX: {
            V3<R> axis0 = tr_a.c0, axis2 = tr_b.c2;
            axes[1] = axis2.cross(axis0); axes[0] = axes[1].cross(axis2); axes[2] = axis0.cross(axes[1]);
            break;
        }
        default: {
            V3<R> axis0 = tr_b.c0, axis2 = tr_a.c2;
            axes[1] = axis2.cross(axis0); axes[0] = axes[1].cross(axis2); axes[2] = axis0.cross(axes[1]);
            break;
        }
    }
    for (int i = 0; i < 3; ++i) axes[i] = axes[i].normalize();
}

// generic6dof_spring2.rs:1375-1383 (mirrored_window): Bullet's window [lower, upper] in the row
// convention (lambda_ours = -lambda_bullet).
template <class R>
void mirrored_window(R lower, R upper, uint32_t& lim, R& lo, R& hi) {
    const bool lf = std::isfinite(lower), uf = std::isfinite(upper);
    lo = 0; hi = 0;
    if (lf && uf) {
        if (lower == -upper) { lim = LIM_BILATERAL; hi = upper; lo = -upper; }
        else { lim = LIM_WINDOW; lo = -upper; hi = -lower; }
    } else if (!lf && uf) { lim = LIM_LOWER; lo = -upper; }
    else if (lf && !uf) { lim = LIM_UPPER; hi = -lower; }
    else lim = LIM_UNBOUNDED;
}

// generic6dof_spring2.rs:135-151 and :237-256 (testLimitValue)
template <class R>
void spring2_test_limit(Spring2Axis<R>& m, R value) {
    if (m.lower > m.upper) { m.current_limit = 0; m.error = 0; }
    else if (m.lower == m.upper) { m.error = value - m.lower; m.current_limit = 3; }
    else { m.error = value - m.lower; m.error_hi = value - m.upper; m.current_limit = 4; }
}

// generic6dof_spring2.rs:1154-1162 (angular_axis_violated)
template <class R>
bool spring2_axis_violated(const Spring2Axis<R>& m) {
    const R t = R(1.0e-3);
    return (m.current_limit == 3 && (m.error < -t || m.error > t)) ||
           (m.current_limit == 4 && (m.error < -t || m.error_hi > t));
}

// generic6dof_spring2.rs:650-820 (prepare_rows), :846-1111 (push_limit_motor_rows),
// :1113-1152 (push_row): the rows of one spring-2 joint.
template <class R, class B>
void prepare_spring2_rows(Joint<R>& jt, uint32_t ia, uint32_t ib, const B& a, const B& b, R inv_dt, R erp,
                          R global_cfm, std::vector<JointRow<R>>& out) {
    const R pi = R(3.14159265358979323846);
    const R inf = std::numeric_limits<R>::infinity();
    M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
    M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
    V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
    V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
    V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
    V3<R> diff = tr_a.transpose() * (pivot_b - pivot_a);
    jt.s2_diff = diff;
    for (int i = 0; i < 3; ++i) spring2_test_limit(jt.s2[i], diff[i]);
    V3<R> euler, axes[3];
    spring2_angle_info(tr_a, tr_b, jt.rotate_order, euler, axes);
    jt.s2_euler = euler;
    for (int i = 0; i < 3; ++i) {
        Spring2Axis<R>& m = jt.s2[3 + i];
        m.position = adjust_angle_to_limits(euler[i], m.lower, m.upper);
        spring2_test_limit(m, m.position);
    }
    const R mi_a = a.inv_mass, mi_b = b.inv_mass;
    const R eps = std::numeric_limits<R>::epsilon();
    jt.has_static_body = mi_a < eps || mi_b < eps;
    const R mi_s = mi_a + mi_b;
    jt.fact_a = mi_s > R(0) ? mi_b / mi_s : R(0.5);
    jt.fact_b = R(1) - jt.fact_a;

    auto push_row = [&](const V3<R>& ax1, bool rotational, bool rot_allowed, R bullet_error, R cfm, R lower,
                        R upper) {
        V3<R> lin_a, ang_a, lin_b, ang_b;
        if (rotational) { ang_a = ax1; ang_b = ax1; }
        else {
            lin_a = ax1; lin_b = ax1;
            ang_a = r_a.cross(ax1); ang_b = r_b.cross(ax1);
            if (jt.has_static_body && !rot_allowed) { ang_a = ang_a * jt.fact_a; ang_b = ang_b * jt.fact_b; }
        }
        uint32_t lim; R lo, hi;
        mirrored_window(lower, upper, lim, lo, hi);
        out.push_back(prepare_joint_row(ia, ib, lin_a, ang_a, lin_b, ang_b, a, b, -bullet_error, lim, lo, hi));
        out.back().cfm = cfm;
    };
    // stop/motor ERP and CFM of an axis: the override when its flag is set, else the global value
    auto stop_erp = [&](const Spring2Axis<R>& m) { return (m.flags & S2_STOP_ERP) ? m.stop_erp : erp; };
    auto stop_cfm = [&](const Spring2Axis<R>& m) { return (m.flags & S2_STOP_CFM) ? m.stop_cfm : global_cfm; };
    auto motor_erp = [&](const Spring2Axis<R>& m) { return (m.flags & S2_MOTOR_ERP) ? m.motor_erp : erp; };
    auto motor_cfm = [&](const Spring2Axis<R>& m) { return (m.flags & S2_MOTOR_CFM) ? m.motor_cfm : global_cfm; };

    auto axis_rows = [&](const Spring2Axis<R>& m, R position, const V3<R>& ax1, bool rotational, bool rot_allowed) {
        const R sign = rotational ? R(-1) : R(1);
        const bool motor = (m.flags & S2_MOTOR) != 0, servo = (m.flags & S2_SERVO) != 0;
        if (m.current_limit == 4) {
            const R vel = rotational ? a.angular_velocity.dot(ax1) - b.angular_velocity.dot(ax1)
                                     : a.linear_velocity.dot(ax1) - b.linear_velocity.dot(ax1);
            const R serp = stop_erp(m);
            R row_error = inv_dt * serp * m.error * sign;
            if (rotational) {
                if (row_error - vel * serp > R(0)) {
                    R bounce_error = -m.bounce * vel;
                    if (bounce_error > row_error) row_error = bounce_error;
                }
            } else if (row_error - vel * serp < R(0)) {
                R bounce_error = -m.bounce * vel;
                if (bounce_error < row_error) row_error = bounce_error;
            }
            if (rotational) push_row(ax1, rotational, rot_allowed, row_error, stop_cfm(m), R(0), inf);
            else push_row(ax1, rotational, rot_allowed, row_error, stop_cfm(m), -inf, R(0));
            row_error = inv_dt * serp * m.error_hi * sign;
            if (rotational) {
                if (row_error - vel * serp < R(0)) {
                    R bounce_error = -m.bounce * vel;
                    if (bounce_error < row_error) row_error = bounce_error;
                }
            } else if (row_error - vel * serp > R(0)) {
                R bounce_error = -m.bounce * vel;
                if (bounce_error > row_error) row_error = bounce_error;
            }
            if (rotational) push_row(ax1, rotational, rot_allowed, row_error, stop_cfm(m), -inf, R(0));
            else push_row(ax1, rotational, rot_allowed, row_error, stop_cfm(m), R(0), inf);
        }
        if (m.current_limit == 3) {
            R row_error = inv_dt * stop_erp(m) * m.error * sign;
            push_row(ax1, rotational, rot_allowed, row_error, stop_cfm(m), -inf, inf);
        }
        if (motor && !servo) {
            R tag_vel = rotational ? m.target_velocity : -m.target_velocity;
            R mot_fact = motor_factor(position, m.lower, m.upper, tag_vel, inv_dt * motor_erp(m));
            R row_error = mot_fact * m.target_velocity;
            R f = m.max_motor_force / inv_dt;
            push_row(ax1, rotational, rot_allowed, row_error, motor_cfm(m), -f, f);
        }
        if (motor && servo) {
            R error = position - m.servo_target;
            R cur_servo_target = m.servo_target;
            if (rotational) {
                if (error > pi) { error -= R(2) * pi; cur_servo_target += R(2) * pi; }
                if (error < -pi) { error += R(2) * pi; cur_servo_target -= R(2) * pi; }
            }
            R targetvelocity = error < R(0) ? -m.target_velocity : m.target_velocity;
            R tag_vel = -targetvelocity;
            R mot_fact = R(0);
            if (error != R(0)) {
                R low_limit, hi_limit;
                if (m.lower > m.upper) {
                    low_limit = error > R(0) ? cur_servo_target : -inf;
                    hi_limit = error < R(0) ? cur_servo_target : inf;
                } else {
                    low_limit = error > R(0) && cur_servo_target > m.lower ? cur_servo_target : m.lower;
                    hi_limit = error < R(0) && cur_servo_target < m.upper ? cur_servo_target : m.upper;
                }
                mot_fact = motor_factor(position, low_limit, hi_limit, tag_vel, inv_dt * motor_erp(m));
            }
            R row_error = mot_fact * targetvelocity * sign;
            R f = m.max_motor_force / inv_dt;
            push_row(ax1, rotational, rot_allowed, row_error, motor_cfm(m), -f, f);
        }
        if (m.flags & S2_SPRING) {
            R error = position - m.equilibrium;
            R vel;
            if (rotational) vel = a.angular_velocity.dot(ax1) - b.angular_velocity.dot(ax1);
            else {
                V3<R> tan_vel_a = a.angular_velocity.cross(r_a), tan_vel_b = b.angular_velocity.cross(r_b);
                vel = (a.linear_velocity + tan_vel_a).dot(ax1) - (b.linear_velocity + tan_vel_b).dot(ax1);
            }
            R m_a = R(1) / mi_a, m_b = R(1) / mi_b;
            if (rotational) {
                if (mi_a != R(0)) {
                    R rr_a = r_a.length_squared();
                    m_a = m_a * rr_a + R(1) / (a.inv_inertia_world() * ax1).length();
                }
                if (mi_b != R(0)) {
                    R rr_b = r_b.length_squared();
                    m_b = m_b * rr_b + R(1) / (b.inv_inertia_world() * ax1).length();
                }
            }
            R mm = mi_a == R(0) ? m_b : (mi_b == R(0) ? m_a : m_a * m_b / (m_a + m_b));
            R dt = R(1) / inv_dt;
            R kd = m.damping, ks = m.stiffness;
            R angularfreq = std::sqrt(ks / mm);
            if ((m.flags & S2_STIFFNESS_LIMITED) && R(0.25) < angularfreq * dt) ks = R(1) / dt / dt / R(16) * mm;
            if ((m.flags & S2_DAMPING_LIMITED) && kd * dt > mm) kd = mm / dt;
            R fs = ks * error * dt;
            R fd = -kd * vel * sign * dt;
            R f = fs + fd;
            R row_error = vel + f / mm * sign;
            R minf = f < fd ? f : fd;
            R maxf = f < fd ? fd : f;
            R lo, hi;
            if (!rotational) { lo = minf > R(0) ? R(0) : minf; hi = maxf < R(0) ? R(0) : maxf; }
            else { lo = -maxf > R(0) ? R(0) : -maxf; hi = -minf < R(0) ? R(0) : -minf; }
            push_row(ax1, rotational, rot_allowed, row_error, R(0), lo, hi);
        }
    };
    auto produces_rows = [](const Spring2Axis<R>& m) {
        return m.current_limit != 0 || (m.flags & (S2_MOTOR | S2_SPRING)) != 0;
    };
    for (int i = 0; i < 3; ++i)
        if (produces_rows(jt.s2[3 + i])) axis_rows(jt.s2[3 + i], jt.s2[3 + i].position, axes[i], true, true);
    for (int i = 0; i < 3; ++i) {
        if (!produces_rows(jt.s2[i])) continue;
        const bool rot_allowed = !(spring2_axis_violated(jt.s2[3 + (i + 1) % 3]) &&
                                   spring2_axis_violated(jt.s2[3 + (i + 2) % 3]));
        axis_rows(jt.s2[i], diff[i], tr_a.col(i), false, rot_allowed);
    }
}

// generic6dof.rs:264-326, 328-546 (Generic6DofConstraint: test_linear_limit,
// test_angular_limit_motor, prepare_rows, push_limit_motor_row). The per-axis parameters sit in
// the spring-2 axis table: lower, upper, bounce (angular), stop_erp, target_velocity,
// max_motor_force and S2_MOTOR; the per-step state in s2_diff / s2_euler.
template <class R, class B>
void prepare_generic6dof_rows(Joint<R>& jt, uint32_t ia, uint32_t ib, const B& a, const B& b, R inv_dt,
                              std::vector<JointRow<R>>& out) {
    const R pi = R(3.14159265358979323846);
    const R inf = std::numeric_limits<R>::infinity();
    M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
    M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
    V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
    V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
    V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
    V3<R> diff = tr_a.transpose() * (pivot_b - pivot_a);
    jt.s2_diff = diff;
    int lin_limit[3];
    R lin_err[3];
    for (int i = 0; i < 3; ++i) {
        const Spring2Axis<R>& m = jt.s2[i];
        const R v = diff[i];
        if (m.lower > m.upper) { lin_limit[i] = 0; lin_err[i] = 0; }
        else if (v < m.lower) { lin_limit[i] = 2; lin_err[i] = v - m.lower; }
        else if (v > m.upper) { lin_limit[i] = 1; lin_err[i] = v - m.upper; }
        else { lin_limit[i] = 0; lin_err[i] = 0; }
    }
    V3<R> euler, axes[3];
    relative_rotation_info(tr_a, tr_b, euler, axes);
    jt.s2_euler = euler;
    auto push_row = [&](const V3<R>& ax1, bool linear, int limit, R limit_err, R lo, R hi, R stop_erp, bool powered,
                        R target_velocity, R max_motor_force, R current_pos, R bounce, R row_vel) {
        if (limit != 0 && lo == hi) powered = false;
        R row_error = 0;
        if (powered && limit == 0) {
            R tag_vel = linear ? -target_velocity : target_velocity;
            R mot_fact = motor_factor(current_pos, lo, hi, tag_vel, inv_dt * stop_erp);
            row_error += mot_fact * target_velocity;
        }
        if (limit != 0) {
            R k = inv_dt * stop_erp;
            row_error += linear ? k * limit_err : -k * limit_err;
            if (bounce > R(0)) {
                if (limit == 1) {
                    if (row_vel < R(0)) { R newc = -bounce * row_vel; if (newc > row_error) row_error = newc; }
                } else if (row_vel > R(0)) {
                    R newc = -bounce * row_vel;
                    if (newc < row_error) row_error = newc;
                }
            }
        }
        R lower = 0, upper = 0;
        if (powered && limit == 0) { lower = -max_motor_force / inv_dt; upper = max_motor_force / inv_dt; }
        else if (limit != 0) {
            if (lo == hi) { lower = -inf; upper = inf; }
            else if (limit == 1) { lower = 0; upper = inf; }
            else { lower = -inf; upper = 0; }
        }
        uint32_t lim;
        R rlo, rhi;
        mirrored_row_limits(lower, upper, lim, rlo, rhi);
        const V3<R> zero;
        if (linear)
            out.push_back(prepare_joint_row(ia, ib, ax1, r_a.cross(ax1), ax1, r_b.cross(ax1), a, b, -row_error, lim, rlo, rhi));
        else
            out.push_back(prepare_joint_row(ia, ib, zero, ax1, zero, ax1, a, b, -row_error, lim, rlo, rhi));
    };
    for (int i = 0; i < 3; ++i) {
        Spring2Axis<R>& m = jt.s2[3 + i];
        const bool motor = (m.flags & S2_MOTOR) != 0;
        const R angle = adjust_angle_to_limits(euler[i], m.lower, m.upper);
        m.position = angle;
        int limit = 0;
        R err = m.error;
        if (m.lower > m.upper) limit = 0;
        else if (angle < m.lower || angle > m.upper) {
            limit = angle < m.lower ? 1 : 2;
            err = angle - (angle < m.lower ? m.lower : m.upper);
            if (err > pi) err -= R(2) * pi;
            else if (err < -pi) err += R(2) * pi;
        }
        m.error = err;
        if (limit != 0 || motor) {
            R row_vel = a.angular_velocity.dot(axes[i]) - b.angular_velocity.dot(axes[i]);
            push_row(axes[i], false, limit, err, m.lower, m.upper, m.stop_erp, motor, m.target_velocity,
                     m.max_motor_force, angle, m.bounce, row_vel);
        }
    }
    for (int i = 0; i < 3; ++i) {
        const Spring2Axis<R>& m = jt.s2[i];
        const bool motor = (m.flags & S2_MOTOR) != 0;
        if (lin_limit[i] != 0 || motor) {
            V3<R> ax1 = tr_a.col(i);
            R row_vel = a.linear_velocity.dot(ax1) - b.linear_velocity.dot(ax1);
            push_row(ax1, true, lin_limit[i], lin_err[i], m.lower, m.upper, m.stop_erp, motor, m.target_velocity,
                     m.max_motor_force, diff[i], R(0), row_vel);
        }
    }
}

// constraint.rs:755-842 + fixed.rs:33-90 + hinge.rs:130-267: the joint's rows for this step.
template <class R, class B>
void prepare_joint_rows(Joint<R>& jt, uint32_t jid, const std::vector<B>& bodies, R inv_dt, R erp,
                        std::vector<JointRow<R>>& out, R global_cfm = R(0)) {
    if (!jt.enabled) return;
    const uint32_t ia = jt.body_a, ib = jt.body_b;
    const B& a = bodies[ia];
    const B& b = bodies[ib];
    const size_t first = out.size();
    auto push = [&](const V3<R>& la, const V3<R>& aa, const V3<R>& lb, const V3<R>& ab, R bias, uint32_t lim, R lo, R hi) {
        out.push_back(prepare_joint_row(ia, ib, la, aa, lb, ab, a, b, bias, lim, lo, hi));
    };
    const V3<R> zero;
    if (jt.kind == JOINT_POINT2POINT) {
        V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
        V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
        V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
        R k = inv_dt * (jt.has_erp ? jt.erp : erp);
        uint32_t lim = jt.impulse_clamp > R(0) ? LIM_BILATERAL : LIM_UNBOUNDED;
        for (int axis = 0; axis < 3; ++axis) {
            V3<R> n;
            n.at(axis) = R(1);
            push(n, r_a.cross(n), n, r_b.cross(n), k * (pivot_a - pivot_b)[axis], lim, -jt.impulse_clamp, jt.impulse_clamp);
        }
    } else if (jt.kind == JOINT_SPRING2) {
        prepare_spring2_rows(jt, ia, ib, a, b, inv_dt, erp, global_cfm, out);
    } else if (jt.kind == JOINT_GENERIC6DOF) {
        prepare_generic6dof_rows(jt, ia, ib, a, b, inv_dt, out);
    } else if (jt.kind == JOINT_CONETWIST) {
        prepare_conetwist_rows(jt, ia, ib, a, b, inv_dt, erp, out);
    } else if (jt.kind == JOINT_GEAR) {  // gear.rs:33-57
        V3<R> axis_a_world = a.orientation.rotate(jt.frame_a.basis.c2);
        V3<R> axis_b_world = b.orientation.rotate(jt.frame_b.basis.c2);
        push(zero, axis_a_world, zero, -(axis_b_world * jt.gear_ratio), R(0), LIM_UNBOUNDED, 0, 0);
    } else if (jt.kind == JOINT_SLIDER) {  // slider.rs:159-475
        const R eps = std::numeric_limits<R>::epsilon();
        const R inf = std::numeric_limits<R>::infinity();
        M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
        M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
        V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
        V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
        V3<R> delta = pivot_b - pivot_a;
        V3<R> ax1_a = tr_a.c0;
        R depth0 = delta.dot(tr_a.c0);
        jt.lin_pos = depth0;
        bool solve_lin_limit = false;
        if (jt.lower_lin <= jt.upper_lin) {
            if (depth0 > jt.upper_lin) { depth0 -= jt.upper_lin; solve_lin_limit = true; }
            else if (depth0 < jt.lower_lin) { depth0 -= jt.lower_lin; solve_lin_limit = true; }
            else depth0 = 0;
        } else {
            depth0 = 0;
        }
        const R lin_depth = depth0;
        bool solve_ang_limit = false;
        R ang_depth = 0;
        if (jt.lower_ang <= jt.upper_ang) {
            V3<R> axis_a0 = tr_a.c1, axis_a1 = tr_a.c2, axis_b0 = tr_b.c1;
            R rot = adjust_angle_to_limits(std::atan2(axis_b0.dot(axis_a1), axis_b0.dot(axis_a0)), jt.lower_ang,
                                           jt.upper_ang);
            jt.ang_pos = rot;
            if (rot < jt.lower_ang) { ang_depth = rot - jt.lower_ang; solve_ang_limit = true; }
            else if (rot > jt.upper_ang) { ang_depth = rot - jt.upper_ang; solve_ang_limit = true; }
        }
        const R sign_fact = jt.use_frame_a ? R(1) : R(-1);
        V3<R> ofs = pivot_b - pivot_a;
        const R ima = a.inv_mass, imb = b.inv_mass;
        const bool has_static = ima < eps || imb < eps;
        const R ims = ima + imb;
        const R fact_a = ims > R(0) ? imb / ims : R(0.5);
        const R fact_b = R(1) - fact_a;
        V3<R> ax1 = (ax1_a * fact_a + tr_b.c0 * fact_b).normalize();
        const R k = inv_dt * (jt.softness_ortho_ang * erp);
        V3<R> u = ax1_a.cross(tr_b.c0);
        V3<R> rel_pa = pivot_a - a.position, rel_pb = pivot_b - b.position;
        V3<R> ortho_a = rel_pa - ax1 * rel_pa.dot(ax1);
        V3<R> ortho_b = rel_pb - ax1 * rel_pb.dot(ax1);
        const R slider_offs = jt.lin_pos - depth0;
        V3<R> total_dist = ax1 * (ax1.dot(pivot_a - a.position) + slider_offs) - ax1 * ax1.dot(pivot_b - b.position);
        V3<R> rel_a = ortho_a + total_dist * fact_a;
        V3<R> rel_b = ortho_b - total_dist * fact_b;
        V3<R> avg = ortho_b * fact_a + ortho_a * fact_b;
        V3<R> p = avg.length_squared() > eps ? avg.normalize() : tr_a.c1;
        V3<R> q = ax1.cross(p);
        push(zero, p, zero, p, -k * u.dot(p), LIM_UNBOUNDED, 0, 0);
        push(zero, q, zero, q, -k * u.dot(q), LIM_UNBOUNDED, 0, 0);
        const R k_lin = inv_dt * (jt.softness_ortho_lin * erp);
        push(p, rel_a.cross(p), p, rel_b.cross(p), -k_lin * p.dot(ofs), LIM_UNBOUNDED, 0, 0);
        {
            V3<R> tmp_a = rel_a.cross(q), tmp_b = rel_b.cross(q);
            if (has_static && solve_ang_limit) { tmp_a *= fact_a; tmp_b *= fact_b; }
            push(q, tmp_a, q, tmp_b, -k_lin * q.dot(ofs), LIM_UNBOUNDED, 0, 0);
        }
        // linear limit / motor row
        R limit_err = 0;
        int limit = 0;
        if (solve_lin_limit) {
            limit_err = lin_depth * sign_fact;
            limit = limit_err > R(0) ? 2 : 1;
        }
        bool powered = jt.has_lin_motor;
        if (limit != 0 && jt.lower_lin == jt.upper_lin) powered = false;
        if (limit != 0 || powered) {
            const R curr_erp = erp;
            R row_error = 0, lower = 0, upper = 0;
            if (powered) {
                R mf = motor_factor(jt.lin_pos, jt.lower_lin, jt.upper_lin, jt.lin_motor_target, inv_dt * curr_erp);
                row_error -= sign_fact * mf * jt.lin_motor_target;
                lower += -jt.lin_motor_max / inv_dt;
                upper += jt.lin_motor_max / inv_dt;
            }
            if (limit != 0) {
                row_error += inv_dt * curr_erp * limit_err;
                if (jt.lower_lin == jt.upper_lin) { lower = -inf; upper = inf; }
                else if (limit == 1) { lower = -inf; upper = 0; }
                else { lower = 0; upper = inf; }
                R bounce = std::fabs(R(1) - jt.damping_lim_lin);
                if (bounce > R(0)) {
                    R vel = a.linear_velocity.dot(ax1) - b.linear_velocity.dot(ax1);
                    vel *= sign_fact;
                    if (limit == 1) {
                        if (vel < R(0)) { R newc = -bounce * vel; if (newc > row_error) row_error = newc; }
                    } else if (vel > R(0)) {
                        R newc = -bounce * vel;
                        if (newc < row_error) row_error = newc;
                    }
                }
                row_error *= jt.softness_lim_lin;
            }
            uint32_t lim; R lo, hi;
            mirrored_row_limits(lower, upper, lim, lo, hi);
            V3<R> ang_a = has_static ? zero : rel_a.cross(ax1);
            V3<R> ang_b = has_static ? zero : rel_b.cross(ax1);
            push(ax1, ang_a, ax1, ang_b, -row_error, lim, lo, hi);
        }
        // angular limit / motor row
        limit_err = 0;
        limit = 0;
        if (solve_ang_limit) {
            limit_err = ang_depth;
            limit = limit_err > R(0) ? 1 : 2;
        }
        powered = jt.has_ang_motor;
        if (limit != 0 && jt.lower_ang == jt.upper_ang) powered = false;
        if (limit != 0 || powered) {
            const R curr_erp = erp;
            R row_error = 0, lower = 0, upper = 0;
            if (powered) {
                R mf = motor_factor(jt.ang_pos, jt.lower_ang, jt.upper_ang, jt.ang_motor_target, inv_dt * curr_erp);
                row_error = mf * jt.ang_motor_target;
                lower = -jt.ang_motor_max / inv_dt;
                upper = jt.ang_motor_max / inv_dt;
            }
            if (limit != 0) {
                row_error += inv_dt * curr_erp * limit_err;
                if (jt.lower_ang == jt.upper_ang) { lower = -inf; upper = inf; }
                else if (limit == 1) { lower = 0; upper = inf; }
                else { lower = -inf; upper = 0; }
                R bounce = std::fabs(R(1) - jt.damping_lim_ang);
                if (bounce > R(0)) {
                    R vel = a.angular_velocity.dot(ax1) - b.angular_velocity.dot(ax1);
                    if (limit == 1) {
                        if (vel < R(0)) { R newc = -bounce * vel; if (newc > row_error) row_error = newc; }
                    } else if (vel > R(0)) {
                        R newc = -bounce * vel;
                        if (newc < row_error) row_error = newc;
                    }
                }
                row_error *= jt.softness_lim_ang;
            }
            uint32_t lim; R lo, hi;
            mirrored_row_limits(lower, upper, lim, lo, hi);
            push(zero, ax1, zero, ax1, -row_error, lim, lo, hi);
        }
    } else if (jt.kind == JOINT_FIXED) {
        M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
        M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
        V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
        V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
        V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
        R k = inv_dt * erp;
        for (int axis = 0; axis < 3; ++axis) {
            V3<R> n;
            n.at(axis) = R(1);
            push(n, r_a.cross(n), n, r_b.cross(n), k * (pivot_a - pivot_b)[axis], LIM_UNBOUNDED, 0, 0);
        }
        V3<R> euler, axes[3];
        relative_rotation_info(tr_a, tr_b, euler, axes);
        for (int i = 0; i < 3; ++i) push(zero, axes[i], zero, axes[i], k * euler[i], LIM_UNBOUNDED, 0, 0);
    } else {  // hinge
        M3<R> tr_a = M3<R>::from_quat(a.orientation) * jt.frame_a.basis;
        M3<R> tr_b = M3<R>::from_quat(b.orientation) * jt.frame_b.basis;
        V3<R> pivot_a = a.position + a.orientation.rotate(jt.frame_a.origin);
        V3<R> pivot_b = b.position + b.orientation.rotate(jt.frame_b.origin);
        V3<R> r_a = pivot_a - a.position, r_b = pivot_b - b.position;
        V3<R> ax1 = tr_a.c2, p = tr_a.c0, q = tr_a.c1, ax2 = tr_b.c2;
        R k = inv_dt * erp;
        if (!jt.angular_only) {
            for (int axis = 0; axis < 3; ++axis) {
                V3<R> n;
                n.at(axis) = R(1);
                push(n, r_a.cross(n), n, r_b.cross(n), k * (pivot_a - pivot_b)[axis], LIM_UNBOUNDED, 0, 0);
            }
        }
        V3<R> u = ax1.cross(ax2);
        push(zero, p, zero, p, -k * u.dot(p), LIM_UNBOUNDED, 0, 0);
        push(zero, q, zero, q, -k * u.dot(q), LIM_UNBOUNDED, 0, 0);
        jt.hinge_angle = hinge_angle_of(tr_a, tr_b);
        R correction = 0, sign = 0;
        bool solve = false;
        if (jt.has_limit) limit_test(jt.limit, jt.hinge_angle, correction, sign, solve);
        const bool powered = jt.has_motor;
        if (solve || powered) {
            R row_error = 0;
            R lostop = jt.has_limit ? jt.limit.low : R(1);
            R histop = jt.has_limit ? jt.limit.high : R(-1);
            bool motor_ineffective = solve && lostop == histop;
            if (powered && !motor_ineffective) {
                R mf = motor_factor(jt.hinge_angle, lostop, histop, jt.motor_target, inv_dt * erp);
                row_error += mf * jt.motor_target;
            }
            if (solve) {
                row_error += k * correction;
                R bounce = jt.has_limit ? jt.limit.relaxation : R(1);
                if (bounce > R(0)) {
                    R vel = a.angular_velocity.dot(ax1) - b.angular_velocity.dot(ax1);
                    if (sign > R(0)) {
                        if (vel < R(0)) {
                            R newc = -bounce * vel;
                            if (newc > row_error) row_error = newc;
                        }
                    } else if (vel > R(0)) {
                        R newc = -bounce * vel;
                        if (newc < row_error) row_error = newc;
                    }
                }
                row_error *= jt.has_limit ? jt.limit.bias_factor : R(1);
            }
            uint32_t lim;
            R lo = 0, hi = 0;
            if (solve) {
                if (lostop == histop) lim = LIM_UNBOUNDED;
                else if (sign > R(0)) { lim = LIM_UPPER; hi = 0; }
                else { lim = LIM_LOWER; lo = 0; }
            } else {
                lim = LIM_BILATERAL;
                hi = jt.has_motor ? jt.motor_max : R(0);
                lo = -hi;
            }
            push(zero, ax1, zero, ax1, -row_error, lim, lo, hi);
        }
    }
    for (size_t r = first; r < out.size(); ++r) out[r].joint = jid;
}

}  // namespace oracle
