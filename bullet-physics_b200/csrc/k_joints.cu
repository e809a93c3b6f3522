// Joint rows of one step (constraint.rs:755-842; fixed.rs:33-90; hinge.rs:130-267; gear.rs:33-57;
// slider.rs:159-475; generic6dof_spring2.rs:650-1383;
// row preparation sequential_impulse.rs:260-299), one thread per joint slot in solve
// order. Each joint of an awake island is flattened into its rows from the current
// (pre-integration) poses, with the reference's arithmetic: the three pivot rows along
// the world axes, the fixed joint's three angular rows along the relative-rotation axes,
// the hinge's two alignment rows and its limit/motor row. Rows are solved inside the PGS
// kernel after the contact rows of each sweep (solve_joint_slot).
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

constexpr float PI_F = 3.14159265358979323846f;

__device__ __forceinline__ M3 load_iw_body(const float4* __restrict__ iw, uint32_t i, float& im) {
    const float4 x = iw[3 * i], y = iw[3 * i + 1], z = iw[3 * i + 2];
    im = z.y;
    return M3{V3{x.x, x.y, x.z}, V3{x.w, y.x, y.y}, V3{y.z, y.w, z.x}};
}

// shared.rs:17-27 (normalize_angle; Rust's % truncates like fmodf)
__device__ __forceinline__ float normalize_angle(float angle) {
    const float two_pi = 2.0f * PI_F;
    float a = fmodf(angle, two_pi);
    if (a < -PI_F) a += two_pi;
    else if (a > PI_F) a -= two_pi;
    return a;
}

// shared.rs:123-155 (get_motor_factor)
__device__ __forceinline__ float motor_factor(float pos, float low_lim, float upp_lim, float vel, float time_fact) {
    if (low_lim > upp_lim) return 1.0f;
    if (low_lim == upp_lim) return 0.0f;
    const float delta_max = vel / time_fact;
    if (delta_max < 0.0f) {
        if (pos >= low_lim && pos < low_lim - delta_max) return (low_lim - pos) / delta_max;
        if (pos < low_lim) return 0.0f;
        return 1.0f;
    }
    if (delta_max > 0.0f) {
        if (pos <= upp_lim && pos > upp_lim - delta_max) return (upp_lim - pos) / delta_max;
        if (pos > upp_lim) return 0.0f;
        return 1.0f;
    }
    return 0.0f;
}

// shared.rs:30-55 (adjust_angle_to_limits)
__device__ __forceinline__ float adjust_angle_to_limits(float angle, float lo, float hi) {
    const float two_pi = 2.0f * PI_F;
    if (lo >= hi) return angle;
    if (angle < lo) {
        const float diff_lo = fabsf(normalize_angle(lo - angle)), diff_hi = fabsf(normalize_angle(hi - angle));
        return diff_lo < diff_hi ? angle : angle + two_pi;
    }
    if (angle > hi) {
        const float diff_hi = fabsf(normalize_angle(angle - hi)), diff_lo = fabsf(normalize_angle(angle - lo));
        return diff_lo < diff_hi ? angle - two_pi : angle;
    }
    return angle;
}

// shared.rs:126-145 (mirrored_row_limits): Bullet's window [lower, upper] in the row convention.
__device__ __forceinline__ void mirrored_row_limits(float lower, float upper, uint32_t& lim, float& lo, float& hi) {
    const bool lower_inf = isinf(lower) && lower < 0.0f, upper_inf = isinf(upper) && upper > 0.0f;
    lo = 0.0f;
    hi = 0.0f;
    if (lower_inf && upper_inf) lim = JL_UNBOUNDED;
    else if (lower_inf) lim = JL_LOWER;
    else if (upper_inf) lim = JL_UPPER;
    else {
        lim = JL_BILATERAL;
        hi = (upper - lower) / 2.0f;
        lo = -hi;
    }
}

// shared.rs:85-101 (euler_xyz)
__device__ __forceinline__ V3 euler_xyz(const M3& m) {
    const float half_pi = 1.57079632679489661923f;
    const float r20 = m.c0.z, r21 = m.c1.z, r22 = m.c2.z, r10 = m.c0.y, r11 = m.c1.y, r01 = m.c1.x, r00 = m.c0.x;
    if (r20 < 1.0f) {
        if (r20 > -1.0f) return V3{atan2f(-r21, r22), asinf(r20), atan2f(-r10, r00)};
        return V3{-atan2f(r01, r11), -half_pi, 0.0f};
    }
    return V3{atan2f(r01, r11), half_pi, 0.0f};
}

struct RowOut {
    float4* row;
    uint32_t n;
    float ima, imb;
    M3 iia, iib;
    // ConstraintRow::prepare (sequential_impulse.rs:260-299)
    __device__ __forceinline__ void push(V3 lin_a, V3 ang_a, V3 lin_b, V3 ang_b, float bias, uint32_t lim, float lo,
                                         float hi, float cfm = 0.0f) {
        const float k = ima * len2(lin_a) + imb * len2(lin_b) + dot(ang_a, mul(iia, ang_a)) + dot(ang_b, mul(iib, ang_b));
        const float mass = k > 0.0f ? 1.0f / k : 0.0f;
        float4* r = row + size_t(n) * JROW_F4;
        r[0] = to4(lin_a, mass);
        r[1] = to4(ang_a, bias);
        r[2] = to4(lin_b, cfm);
        r[3] = to4(ang_b, __uint_as_float(lim));
        r[4] = make_float4(lo, hi, 0.0f, 0.0f);
        ++n;
    }
};

__device__ __forceinline__ V3 axis_vec(int axis) {
    return V3{axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f};
}

__device__ __forceinline__ Q qnormalize(Q q) {
    const float l = sqrtf(qlen2(q));
    return Q{q.x / l, q.y / l, q.z / l, q.w / l};
}

// glam 0.33.3 Quat::from_mat3 (the published branch on the diagonal; mRC is column R, row C)
__device__ Q quat_from_mat3(const M3& m) {
    const float m00 = m.c0.x, m01 = m.c0.y, m02 = m.c0.z, m10 = m.c1.x, m11 = m.c1.y, m12 = m.c1.z;
    const float m20 = m.c2.x, m21 = m.c2.y, m22 = m.c2.z;
    if (m22 <= 0.0f) {
        const float dif10 = m11 - m00, omm22 = 1.0f - m22;
        if (dif10 <= 0.0f) {
            const float f = omm22 - dif10, inv = 0.5f / sqrtf(f);
            return Q{f * inv, (m01 + m10) * inv, (m02 + m20) * inv, (m12 - m21) * inv};
        }
        const float f = omm22 + dif10, inv = 0.5f / sqrtf(f);
        return Q{(m01 + m10) * inv, f * inv, (m12 + m21) * inv, (m20 - m02) * inv};
    }
    const float sum10 = m11 + m00, opm22 = 1.0f + m22;
    if (sum10 <= 0.0f) {
        const float f = opm22 - sum10, inv = 0.5f / sqrtf(f);
        return Q{(m02 + m20) * inv, (m12 + m21) * inv, f * inv, (m01 - m10) * inv};
    }
    const float f = opm22 + sum10, inv = 0.5f / sqrtf(f);
    return Q{(m12 - m21) * inv, (m20 - m02) * inv, (m01 - m10) * inv, f * inv};
}

// glam Quat::from_rotation_arc (published algorithm), as the host frames use it
__device__ Q rotation_arc(V3 from, V3 to) {
    const float eps = 1.1920929e-7f;
    const float one_minus_eps = 1.0f - 2.0f * eps;
    const float d = dot(from, to);
    if (d > one_minus_eps) return Q{0.0f, 0.0f, 0.0f, 1.0f};
    if (d < -one_minus_eps) {
        const float sign = signbit(from.z) ? -1.0f : 1.0f;
        const float aa = -1.0f / (sign + from.z);
        const float bb = from.x * from.y * aa;
        const V3 o = V3{bb, sign + from.y * from.y * aa, -from.y};
        const float half = PI_F * 0.5f;
        const float sn = sinf(half);
        return Q{o.x * sn, o.y * sn, o.z * sn, cosf(half)};
    }
    const V3 c = cross(from, to);
    return qnormalize(Q{c.x, c.y, c.z, 1.0f + d});
}

// conetwist.rs:546-548
__device__ __forceinline__ float quaternion_angle(Q q) { return 2.0f * acosf(fminf(fmaxf(q.w, -1.0f), 1.0f)); }

// conetwist.rs:222-342 (prepare_rows) with calc_angle_info (:344-479), compute_cone_limit_info
// (:481-502), compute_twist_limit_info (:504-519) and the ellipse-normal swing axis (:521-539).
__device__ __noinline__ void conetwist_rows(RowOut& out, const BodyDev& b, const JointsDev& jd, uint32_t jid,
                                            const float4* d, uint32_t flags, Q qa, Q qb, V3 r_a, V3 r_b, V3 pivot_a,
                                            V3 pivot_b, float inv_dt, float erp) {
    const float eps = 1.1920929e-7f, fix = 0.05f;
    const V3 zero = V3{0.0f, 0.0f, 0.0f}, X = V3{1.0f, 0.0f, 0.0f};
    const float4 p12 = d[12], p13 = d[13], p14 = d[14];
    const float s1 = p12.x, s2 = p12.y, twist_span = p12.z, softness = p12.w;
    const float bias = p13.x, relax = p13.y, max_impulse = p13.z;
    const bool has_motor = (flags & JF_CONE_MOTOR) != 0;
    const M3 tr_a = mul(from_quat(qa), M3{from4(d[2]), from4(d[3]), from4(d[4])});
    const M3 tr_b = mul(from_quat(qb), M3{from4(d[6]), from4(d[7]), from4(d[8])});
    const float k = inv_dt * erp;
    const V3 dp = pivot_a - pivot_b;
    for (int axis = 0; axis < 3; ++axis) {
        const V3 nrm = axis_vec(axis);
        out.push(nrm, cross(r_a, nrm), nrm, cross(r_b, nrm), k * comp(dp, axis), JL_UNBOUNDED, 0.0f, 0.0f);
    }
    float swing_corr = 0.0f, twist_corr = 0.0f;
    V3 swing_axis = zero, twist_axis = zero;
    bool solve_swing = false, solve_twist = false;
    if (has_motor) {
        const M3 r_delta = mul(mul(tr_b, from_quat(Q{p14.x, p14.y, p14.z, p14.w})), transpose(tr_a));
        const Q q_delta = qnormalize(quat_from_mat3(r_delta));
        const V3 sa = V3{q_delta.x, q_delta.y, q_delta.z};
        const float l2 = len2(sa);
        if (l2 > eps) {
            swing_axis = sa / sqrtf(l2);
            swing_corr = quaternion_angle(q_delta);
            if (fabsf(swing_corr) > eps) solve_swing = true;
        }
    } else {
        const Q q_a = quat_from_mat3(tr_a), q_b = quat_from_mat3(tr_b);
        const Q q_ab = qnormalize(qmul(qinv(q_b), q_a));
        const V3 v_cone = normalize(rotate(q_ab, X));
        const Q q_cone = qnormalize(rotation_arc(X, v_cone));
        const Q q_twist = qnormalize(qmul(qinv(q_cone), q_ab));
        if (s1 >= fix && s2 >= fix) {
            const float angle = quaternion_angle(q_cone);
            V3 axis = zero;
            float limit = s1;
            if (angle > eps) {
                axis = normalize(V3{q_cone.x, q_cone.y, q_cone.z});
                const float xe = axis.y, ye = -axis.z;
                if (fabsf(xe) > eps) {
                    const float slope2 = (ye * ye) / (xe * xe);
                    float norm = 1.0f / (s2 * s2);
                    norm += slope2 / (s1 * s1);
                    limit = sqrtf((1.0f + slope2) / norm);
                }
            }
            if (angle > limit * softness) {
                solve_swing = true;
                swing_corr = angle - limit * softness;
                float y = -axis.z;
                const float z = axis.y;
                if (fabsf(z) > eps) {
                    float grad = y / z;
                    grad *= s2 / s1;
                    y = y > 0.0f ? fabsf(grad * z) : -fabsf(grad * z);
                    axis.z = -y;
                    axis.y = z;
                    axis = normalize(axis);
                }
                swing_axis = rotate(q_b, -axis);
            }
        } else {
            const V3 iv_a = tr_a.c0, jv_a = tr_a.c1, kv_a = tr_a.c2, iv_b = tr_b.c0;
            float x = dot(iv_b, iv_a), y = dot(iv_b, jv_a), z = dot(iv_b, kv_a);
            if (s1 < fix && s2 < fix) {
                if (fabsf(y) > eps || fabsf(z) > eps) {
                    solve_swing = true;
                    swing_axis = -cross(iv_b, iv_a);
                }
            } else {
                if (s1 < fix) {
                    if (fabsf(x) > eps || fabsf(z) > eps) {
                        solve_swing = true;
                        if (s2 >= fix) {
                            y = 0.0f;
                            const float span2 = atan2f(z, x);
                            if (span2 > s2) { x = cosf(s2); z = sinf(s2); }
                            else if (span2 < -s2) { x = cosf(s2); z = -sinf(s2); }
                        }
                    }
                } else {
                    if (fabsf(x) > eps || fabsf(y) > eps) {
                        solve_swing = true;
                        if (s1 >= fix) {
                            z = 0.0f;
                            const float span1 = atan2f(y, x);
                            if (span1 > s1) { x = cosf(s1); y = sinf(s1); }
                            else if (span1 < -s1) { x = cosf(s1); y = -sinf(s1); }
                        }
                    }
                }
                const V3 target = normalize(iv_a * x + jv_a * y + kv_a * z);
                swing_axis = -cross(iv_b, target);
                swing_corr = len(swing_axis);
                if (fabsf(swing_corr) > eps) swing_axis = normalize(swing_axis);
            }
        }
        float twist_angle = 0.0f;
        if (twist_span >= 0.0f) {
            Q qm = q_twist;
            twist_angle = quaternion_angle(q_twist);
            if (twist_angle > PI_F) {
                qm = Q{-q_twist.x, -q_twist.y, -q_twist.z, -q_twist.w};
                twist_angle = quaternion_angle(qm);
            }
            V3 axis = V3{qm.x, qm.y, qm.z};
            if (twist_angle > eps) axis = normalize(axis);
            if (twist_angle > twist_span * softness) {
                solve_twist = true;
                twist_corr = twist_angle - twist_span * softness;
                twist_axis = rotate(q_b, -axis);
            }
        }
        jd.angle[jid] = twist_angle;
    }
    if (solve_swing) {
        if (s1 < fix && s2 < fix) {
            const float fact = inv_dt * relax;
            out.push(zero, tr_a.c1, zero, tr_a.c1, -fact * dot(swing_axis, tr_a.c1), JL_UNBOUNDED, 0.0f, 0.0f);
            out.push(zero, tr_a.c2, zero, tr_a.c2, -fact * dot(swing_axis, tr_a.c2), JL_UNBOUNDED, 0.0f, 0.0f);
        } else {
            const V3 ax1 = swing_axis * (relax * relax);
            if (has_motor && max_impulse >= 0.0f)
                out.push(zero, ax1, zero, ax1, -inv_dt * bias * swing_corr, JL_WINDOW, -max_impulse, 0.0f);
            else
                out.push(zero, ax1, zero, ax1, -inv_dt * bias * swing_corr, JL_UPPER, 0.0f, 0.0f);
        }
    }
    if (solve_twist) {
        const V3 ax1 = twist_axis * (relax * relax);
        const uint32_t lim = twist_span > 0.0f ? (twist_corr > 0.0f ? JL_UPPER : JL_LOWER) : JL_UNBOUNDED;
        out.push(zero, ax1, zero, ax1, -inv_dt * bias * twist_corr, lim, 0.0f, 0.0f);
    }
}

// generic6dof.rs:264-546 (classic 6DOF rows): per axis one limit-or-motor row, angular axes
// first; the parameters come from the spring-2 axis table (lower, upper, bounce, stop erp,
// target velocity, max motor force, S2_MOTOR).
__device__ __noinline__ void generic6dof_rows(RowOut& out, const BodyDev& b, const JointsDev& jd, uint32_t jid,
                                              const float4* d, uint32_t ia, uint32_t ib, Q qa, Q qb, V3 r_a, V3 r_b,
                                              V3 pivot_a, V3 pivot_b, float inv_dt) {
    const float inf = INFINITY;
    const V3 zero = V3{0.0f, 0.0f, 0.0f};
    const float4* aux = jd.aux + __float_as_uint(d[9].x);
    const M3 tr_a = mul(from_quat(qa), M3{from4(d[2]), from4(d[3]), from4(d[4])});
    const M3 tr_b = mul(from_quat(qb), M3{from4(d[6]), from4(d[7]), from4(d[8])});
    const V3 diff = mul(transpose(tr_a), pivot_b - pivot_a);
    // shared.rs:108-123 (relative_rotation_info)
    const V3 euler = euler_xyz(mul(transpose(tr_a), tr_b));
    const V3 axis0 = tr_b.c0, axis2 = tr_a.c2;
    V3 axes[3];
    axes[1] = cross(axis2, axis0);
    axes[0] = cross(axes[1], axis2);
    axes[2] = cross(axis0, axes[1]);
    for (int i = 0; i < 3; ++i) axes[i] = normalize(axes[i]);
    jd.s2_state[2 * size_t(jid)] = to4(euler, diff.x);
    jd.s2_state[2 * size_t(jid) + 1] = make_float4(diff.y, diff.z, 0.5f, 0.0f);  // no static-body split here
    const V3 va = from4(b.linvel[ia]), vb = from4(b.linvel[ib]), wa = from4(b.angvel[ia]), wb = from4(b.angvel[ib]);
    auto push_row = [&](V3 ax1, bool linear, int limit, float limit_err, float lo, float hi, float stop_erp, bool powered,
                        float target_velocity, float max_motor_force, float current_pos, float bounce, float row_vel) {
        if (limit != 0 && lo == hi) powered = false;
        float row_error = 0.0f;
        if (powered && limit == 0) {
            const float tag_vel = linear ? -target_velocity : target_velocity;
            row_error += motor_factor(current_pos, lo, hi, tag_vel, inv_dt * stop_erp) * target_velocity;
        }
        if (limit != 0) {
            const float k = inv_dt * stop_erp;
            row_error += linear ? k * limit_err : -k * limit_err;
            if (bounce > 0.0f) {
                if (limit == 1) {
                    if (row_vel < 0.0f) { const float newc = -bounce * row_vel; if (newc > row_error) row_error = newc; }
                } else if (row_vel > 0.0f) {
                    const float newc = -bounce * row_vel;
                    if (newc < row_error) row_error = newc;
                }
            }
        }
        float lower = 0.0f, upper = 0.0f;
        if (powered && limit == 0) { lower = -max_motor_force / inv_dt; upper = max_motor_force / inv_dt; }
        else if (limit != 0) {
            if (lo == hi) { lower = -inf; upper = inf; }
            else if (limit == 1) { lower = 0.0f; upper = inf; }
            else { lower = -inf; upper = 0.0f; }
        }
        uint32_t lim;
        float rlo, rhi;
        mirrored_row_limits(lower, upper, lim, rlo, rhi);
        if (linear) out.push(ax1, cross(r_a, ax1), ax1, cross(r_b, ax1), -row_error, lim, rlo, rhi);
        else out.push(zero, ax1, zero, ax1, -row_error, lim, rlo, rhi);
    };
    for (int i = 0; i < 3; ++i) {
        const float4 x = aux[(3 + i) * S2_AXIS_F4], y = aux[(3 + i) * S2_AXIS_F4 + 1], z = aux[(3 + i) * S2_AXIS_F4 + 2];
        const bool motor = (__float_as_uint(aux[(3 + i) * S2_AXIS_F4 + 3].y) & S2_MOTOR) != 0;
        const float lo = x.x, hi = x.y;
        const float angle = adjust_angle_to_limits(comp(euler, i), lo, hi);
        int limit = 0;
        float err = 0.0f;
        if (!(lo > hi) && (angle < lo || angle > hi)) {
            limit = angle < lo ? 1 : 2;
            err = angle - (angle < lo ? lo : hi);
            if (err > PI_F) err -= 2.0f * PI_F;
            else if (err < -PI_F) err += 2.0f * PI_F;
        }
        if (limit != 0 || motor)
            push_row(axes[i], false, limit, err, lo, hi, x.w, motor, y.w, z.x, angle, x.z,
                     dot(wa, axes[i]) - dot(wb, axes[i]));
    }
    for (int i = 0; i < 3; ++i) {
        const float4 x = aux[i * S2_AXIS_F4], y = aux[i * S2_AXIS_F4 + 1], z = aux[i * S2_AXIS_F4 + 2];
        const bool motor = (__float_as_uint(aux[i * S2_AXIS_F4 + 3].y) & S2_MOTOR) != 0;
        const float lo = x.x, hi = x.y, v = comp(diff, i);
        int limit = 0;
        float err = 0.0f;
        if (!(lo > hi)) {
            if (v < lo) { limit = 2; err = v - lo; }
            else if (v > hi) { limit = 1; err = v - hi; }
        }
        if (limit != 0 || motor) {
            const V3 ax1 = i == 0 ? tr_a.c0 : (i == 1 ? tr_a.c1 : tr_a.c2);
            push_row(ax1, true, limit, err, lo, hi, x.w, motor, y.w, z.x, v, 0.0f, dot(va, ax1) - dot(vb, ax1));
        }
    }
}

// generic6dof_spring2.rs:1236-1241 (btGetMatrixElem): row index % 3 of column index / 3.
__device__ __forceinline__ float mat_elem(const M3& m, int index) {
    const V3& c = index < 3 ? m.c0 : (index < 6 ? m.c1 : m.c2);
    return comp(c, index % 3);
}

// generic6dof_spring2.rs:1243-1373 (matrixToEuler* for the five orders other than XYZ)
__device__ V3 matrix_to_euler(const M3& m, uint32_t order) {
    const float half_pi = 1.57079632679489661923f;
    auto e = [&](int i) { return mat_elem(m, i); };
    switch (order) {
        case 1: {  // XZY
            const float fi = e(1);
            if (fi < 1.0f) {
                if (fi > -1.0f) return V3{atan2f(e(7), e(4)), atan2f(e(2), e(0)), asinf(-e(1))};
                return V3{-atan2f(-e(6), e(8)), 0.0f, half_pi};
            }
            return V3{atan2f(-e(6), e(8)), 0.0f, -half_pi};
        }
        case 2: {  // YXZ
            const float fi = e(5);
            if (fi < 1.0f) {
                if (fi > -1.0f) return V3{asinf(-e(5)), atan2f(e(2), e(8)), atan2f(e(3), e(4))};
                return V3{half_pi, -atan2f(-e(1), e(0)), 0.0f};
            }
            return V3{-half_pi, atan2f(-e(1), e(0)), 0.0f};
        }
        case 3: {  // YZX
            const float fi = e(3);
            if (fi < 1.0f) {
                if (fi > -1.0f) return V3{atan2f(-e(5), e(4)), atan2f(-e(6), e(0)), asinf(e(3))};
                return V3{0.0f, -atan2f(e(7), e(8)), -half_pi};
            }
            return V3{0.0f, atan2f(e(7), e(8)), half_pi};
        }
        case 4: {  // ZXY
            const float fi = e(7);
            if (fi < 1.0f) {
                if (fi > -1.0f) return V3{asinf(e(7)), atan2f(-e(6), e(8)), atan2f(-e(1), e(4))};
                return V3{-half_pi, 0.0f, -atan2f(e(2), e(0))};
            }
            return V3{half_pi, 0.0f, atan2f(e(2), e(0))};
        }
        case 5: {  // ZYX
            const float fi = e(6);
            if (fi < 1.0f) {
                if (fi > -1.0f) return V3{atan2f(e(7), e(8)), asinf(-e(6)), atan2f(e(3), e(0))};
                return V3{0.0f, half_pi, -atan2f(-e(1), -e(2))};
            }
            return V3{0.0f, -half_pi, atan2f(-e(1), -e(2))};
        }
        default: return euler_xyz(m);
    }
}

// generic6dof_spring2.rs:1375-1383 (mirrored_window)
__device__ __forceinline__ void mirrored_window(float lower, float upper, uint32_t& lim, float& lo, float& hi) {
    const bool lf = isfinite(lower), uf = isfinite(upper);
    lo = 0.0f;
    hi = 0.0f;
    if (lf && uf) {
        if (lower == -upper) { lim = JL_BILATERAL; hi = upper; lo = -upper; }
        else { lim = JL_WINDOW; lo = -upper; hi = -lower; }
    } else if (!lf && uf) { lim = JL_LOWER; lo = -upper; }
    else if (lf && !uf) { lim = JL_UPPER; hi = -lower; }
    else lim = JL_UNBOUNDED;
}

// One axis of a spring-2 joint, with its step state (testLimitValue: 0 free, 3 locked, 4 limited).
struct S2Axis {
    float lower, upper, bounce, stop_erp, stop_cfm, motor_erp, motor_cfm, target_velocity, max_motor_force,
        servo_target, stiffness, damping, equilibrium;
    uint32_t flags;
    int current_limit;
    float error, error_hi;
};

__device__ __forceinline__ S2Axis load_s2_axis(const float4* a, float erp, float global_cfm) {
    const float4 x = a[0], y = a[1], z = a[2], w = a[3];
    S2Axis m;
    m.lower = x.x; m.upper = x.y; m.bounce = x.z;
    m.flags = __float_as_uint(w.y);
    // generic6dof_spring2.rs:690-709, :736-760: without its override flag an axis takes the
    // global ERP / CFM
    m.stop_erp = (m.flags & S2_STOP_ERP) ? x.w : erp;
    m.stop_cfm = (m.flags & S2_STOP_CFM) ? y.x : global_cfm;
    m.motor_erp = (m.flags & S2_MOTOR_ERP) ? y.y : erp;
    m.motor_cfm = (m.flags & S2_MOTOR_CFM) ? y.z : global_cfm;
    m.target_velocity = y.w; m.max_motor_force = z.x; m.servo_target = z.y; m.stiffness = z.z; m.damping = z.w;
    m.equilibrium = w.x;
    m.current_limit = 0; m.error = 0.0f; m.error_hi = 0.0f;
    return m;
}

// generic6dof_spring2.rs:135-151, :237-256 (testLimitValue)
__device__ __forceinline__ void s2_test_limit(S2Axis& m, float value) {
    if (m.lower > m.upper) { m.current_limit = 0; m.error = 0.0f; }
    else if (m.lower == m.upper) { m.error = value - m.lower; m.current_limit = 3; }
    else { m.error = value - m.lower; m.error_hi = value - m.upper; m.current_limit = 4; }
}

// generic6dof_spring2.rs:1154-1162 (angular_axis_violated)
__device__ __forceinline__ bool s2_violated(const S2Axis& m) {
    const float t = 1.0e-3f;
    return (m.current_limit == 3 && (m.error < -t || m.error > t)) ||
           (m.current_limit == 4 && (m.error < -t || m.error_hi > t));
}

struct S2Ctx {
    V3 r_a, r_b, va, vb, wa, wb;
    M3 iia, iib;
    float ima, imb, inv_dt, fact_a, fact_b;
    bool has_static;
};

// generic6dof_spring2.rs:1113-1152 (push_row)
__device__ __forceinline__ void s2_push(RowOut& out, const S2Ctx& c, V3 ax1, bool rotational, bool rot_allowed,
                                        float bullet_error, float cfm, float lower, float upper) {
    const V3 zero = V3{0.0f, 0.0f, 0.0f};
    V3 lin_a = zero, lin_b = zero, ang_a = ax1, ang_b = ax1;
    if (!rotational) {
        lin_a = ax1;
        lin_b = ax1;
        ang_a = cross(c.r_a, ax1);
        ang_b = cross(c.r_b, ax1);
        if (c.has_static && !rot_allowed) { ang_a = ang_a * c.fact_a; ang_b = ang_b * c.fact_b; }
    }
    uint32_t lim;
    float lo, hi;
    mirrored_window(lower, upper, lim, lo, hi);
    out.push(lin_a, ang_a, lin_b, ang_b, -bullet_error, lim, lo, hi, cfm);
}

// generic6dof_spring2.rs:846-1111 (push_limit_motor_rows): the limit pair or lock row, the
// motor or servo row and the spring row of one axis, in that order.
__device__ __noinline__ void s2_axis_rows(RowOut& out, const S2Ctx& c, const S2Axis& m, float position, V3 ax1,
                                          bool rotational, bool rot_allowed) {
    const float inf = INFINITY;
    const float sign = rotational ? -1.0f : 1.0f;
    const bool motor = (m.flags & S2_MOTOR) != 0, servo = (m.flags & S2_SERVO) != 0;
    const float inv_dt = c.inv_dt;
    if (m.current_limit == 4) {
        const float vel = rotational ? dot(c.wa, ax1) - dot(c.wb, ax1) : dot(c.va, ax1) - dot(c.vb, ax1);
        float row_error = inv_dt * m.stop_erp * m.error * sign;
        if (rotational) {
            if (row_error - vel * m.stop_erp > 0.0f) {
                const float bounce_error = -m.bounce * vel;
                if (bounce_error > row_error) row_error = bounce_error;
            }
        } else if (row_error - vel * m.stop_erp < 0.0f) {
            const float bounce_error = -m.bounce * vel;
            if (bounce_error < row_error) row_error = bounce_error;
        }
        if (rotational) s2_push(out, c, ax1, true, rot_allowed, row_error, m.stop_cfm, 0.0f, inf);
        else s2_push(out, c, ax1, false, rot_allowed, row_error, m.stop_cfm, -inf, 0.0f);
        row_error = inv_dt * m.stop_erp * m.error_hi * sign;
        if (rotational) {
            if (row_error - vel * m.stop_erp < 0.0f) {
                const float bounce_error = -m.bounce * vel;
                if (bounce_error < row_error) row_error = bounce_error;
            }
        } else if (row_error - vel * m.stop_erp > 0.0f) {
            const float bounce_error = -m.bounce * vel;
            if (bounce_error > row_error) row_error = bounce_error;
        }
        if (rotational) s2_push(out, c, ax1, true, rot_allowed, row_error, m.stop_cfm, -inf, 0.0f);
        else s2_push(out, c, ax1, false, rot_allowed, row_error, m.stop_cfm, 0.0f, inf);
    }
    if (m.current_limit == 3) {
        const float row_error = inv_dt * m.stop_erp * m.error * sign;
        s2_push(out, c, ax1, rotational, rot_allowed, row_error, m.stop_cfm, -inf, inf);
    }
    if (motor && !servo) {
        const float tag_vel = rotational ? m.target_velocity : -m.target_velocity;
        const float mot_fact = motor_factor(position, m.lower, m.upper, tag_vel, inv_dt * m.motor_erp);
        const float row_error = mot_fact * m.target_velocity;
        const float f = m.max_motor_force / inv_dt;
        s2_push(out, c, ax1, rotational, rot_allowed, row_error, m.motor_cfm, -f, f);
    }
    if (motor && servo) {
        float error = position - m.servo_target;
        float cur_servo_target = m.servo_target;
        if (rotational) {
            if (error > PI_F) { error -= 2.0f * PI_F; cur_servo_target += 2.0f * PI_F; }
            if (error < -PI_F) { error += 2.0f * PI_F; cur_servo_target -= 2.0f * PI_F; }
        }
        const float targetvelocity = error < 0.0f ? -m.target_velocity : m.target_velocity;
        const float tag_vel = -targetvelocity;
        float mot_fact = 0.0f;
        if (error != 0.0f) {
            float low_limit, hi_limit;
            if (m.lower > m.upper) {
                low_limit = error > 0.0f ? cur_servo_target : -inf;
                hi_limit = error < 0.0f ? cur_servo_target : inf;
            } else {
                low_limit = error > 0.0f && cur_servo_target > m.lower ? cur_servo_target : m.lower;
                hi_limit = error < 0.0f && cur_servo_target < m.upper ? cur_servo_target : m.upper;
            }
            mot_fact = motor_factor(position, low_limit, hi_limit, tag_vel, inv_dt * m.motor_erp);
        }
        const float row_error = mot_fact * targetvelocity * sign;
        const float f = m.max_motor_force / inv_dt;
        s2_push(out, c, ax1, rotational, rot_allowed, row_error, m.motor_cfm, -f, f);
    }
    if (m.flags & S2_SPRING) {
        const float error = position - m.equilibrium;
        float vel;
        if (rotational) vel = dot(c.wa, ax1) - dot(c.wb, ax1);
        else vel = dot(c.va + cross(c.wa, c.r_a), ax1) - dot(c.vb + cross(c.wb, c.r_b), ax1);
        float m_a = 1.0f / c.ima, m_b = 1.0f / c.imb;
        if (rotational) {
            if (c.ima != 0.0f) m_a = m_a * len2(c.r_a) + 1.0f / len(mul(c.iia, ax1));
            if (c.imb != 0.0f) m_b = m_b * len2(c.r_b) + 1.0f / len(mul(c.iib, ax1));
        }
        const float mm = c.ima == 0.0f ? m_b : (c.imb == 0.0f ? m_a : m_a * m_b / (m_a + m_b));
        const float dt = 1.0f / inv_dt;
        float kd = m.damping, ks = m.stiffness;
        const float angularfreq = sqrtf(ks / mm);
        if ((m.flags & S2_STIFFNESS_LIMITED) && 0.25f < angularfreq * dt) ks = 1.0f / dt / dt / 16.0f * mm;
        if ((m.flags & S2_DAMPING_LIMITED) && kd * dt > mm) kd = mm / dt;
        const float fs = ks * error * dt;
        const float fd = -kd * vel * sign * dt;
        const float f = fs + fd;
        const float row_error = vel + f / mm * sign;
        const float minf = f < fd ? f : fd, maxf = f < fd ? fd : f;
        float lo, hi;
        if (!rotational) { lo = minf > 0.0f ? 0.0f : minf; hi = maxf < 0.0f ? 0.0f : maxf; }
        else { lo = -maxf > 0.0f ? 0.0f : -maxf; hi = -minf < 0.0f ? 0.0f : -minf; }
        s2_push(out, c, ax1, rotational, rot_allowed, row_error, 0.0f, lo, hi);
    }
}

// generic6dof_spring2.rs:650-820 (prepare_rows) with calculate_angle_info (:1164-1233)
__device__ __noinline__ void spring2_rows(RowOut& out, const BodyDev& b, const JointsDev& jd, uint32_t jid,
                                          const float4* d, uint32_t ia, uint32_t ib, V3 pa, V3 pb, Q qa, Q qb,
                                          V3 pivot_a, V3 pivot_b, float inv_dt, float erp) {
    const uint32_t aux0 = __float_as_uint(d[9].x), order = __float_as_uint(d[9].y);
    const float4* aux = jd.aux + aux0;
    const M3 tr_a = mul(from_quat(qa), M3{from4(d[2]), from4(d[3]), from4(d[4])});
    const M3 tr_b = mul(from_quat(qb), M3{from4(d[6]), from4(d[7]), from4(d[8])});
    S2Ctx c;
    c.r_a = pivot_a - pa;
    c.r_b = pivot_b - pb;
    c.va = from4(b.linvel[ia]); c.vb = from4(b.linvel[ib]);
    c.wa = from4(b.angvel[ia]); c.wb = from4(b.angvel[ib]);
    c.iia = out.iia; c.iib = out.iib; c.ima = out.ima; c.imb = out.imb;
    c.inv_dt = inv_dt;
    const V3 diff = mul(transpose(tr_a), pivot_b - pivot_a);
    const V3 euler = matrix_to_euler(mul(transpose(tr_a), tr_b), order);
    V3 axes[3];
    switch (order) {
        case 1: { const V3 axis0 = tr_b.c0, axis1 = tr_a.c1;
                  axes[2] = cross(axis0, axis1); axes[0] = cross(axis1, axes[2]); axes[1] = cross(axes[2], axis0); break; }
        case 2: { const V3 axis1 = tr_b.c1, axis2 = tr_a.c2;
                  axes[0] = cross(axis1, axis2); axes[1] = cross(axis2, axes[0]); axes[2] = cross(axes[0], axis1); break; }
        case 3: { const V3 axis0 = tr_a.c0, axis1 = tr_b.c1;
                  axes[2] = cross(axis0, axis1); axes[0] = cross(axis1, axes[2]); axes[1] = cross(axes[2], axis0); break; }
        case 4: { const V3 axis1 = tr_a.c1, axis2 = tr_b.c2;
                  axes[0] = cross(axis1, axis2); axes[1] = cross(axis2, axes[0]); axes[2] = cross(axes[0], axis1); break; }
        case 5: { const V3 axis0 = tr_a.c0, axis2 = tr_b.c2;
                  axes[1] = cross(axis2, axis0); axes[0] = cross(axes[1], axis2); axes[2] = cross(axis0, axes[1]); break; }
        default: { const V3 axis0 = tr_b.c0, axis2 = tr_a.c2;
                   axes[1] = cross(axis2, axis0); axes[0] = cross(axes[1], axis2); axes[2] = cross(axis0, axes[1]); break; }
    }
    for (int i = 0; i < 3; ++i) axes[i] = normalize(axes[i]);
    const float eps = 1.1920929e-7f;  // f32::EPSILON
    c.has_static = c.ima < eps || c.imb < eps;
    const float ims = c.ima + c.imb;
    c.fact_a = ims > 0.0f ? c.imb / ims : 0.5f;
    c.fact_b = 1.0f - c.fact_a;
    jd.s2_state[2 * size_t(jid)] = to4(euler, diff.x);
    jd.s2_state[2 * size_t(jid) + 1] = make_float4(diff.y, diff.z, c.fact_a, c.has_static ? 1.0f : 0.0f);
    // the angular axes first (their limit states gate the linear rows' rot_allowed)
    S2Axis ang[3];
    float ang_pos[3];
    for (int i = 0; i < 3; ++i) {
        ang[i] = load_s2_axis(aux + (3 + i) * S2_AXIS_F4, erp, jd.global_cfm);
        ang_pos[i] = adjust_angle_to_limits(comp(euler, i), ang[i].lower, ang[i].upper);
        s2_test_limit(ang[i], ang_pos[i]);
    }
    for (int i = 0; i < 3; ++i)
        if (ang[i].current_limit != 0 || (ang[i].flags & (S2_MOTOR | S2_SPRING)))
            s2_axis_rows(out, c, ang[i], ang_pos[i], axes[i], true, true);
    for (int i = 0; i < 3; ++i) {
        S2Axis lin = load_s2_axis(aux + i * S2_AXIS_F4, erp, jd.global_cfm);
        const float pos = comp(diff, i);
        s2_test_limit(lin, pos);
        if (lin.current_limit == 0 && !(lin.flags & (S2_MOTOR | S2_SPRING))) continue;
        const bool rot_allowed = !(s2_violated(ang[(i + 1) % 3]) && s2_violated(ang[(i + 2) % 3]));
        s2_axis_rows(out, c, lin, pos, i == 0 ? tr_a.c0 : (i == 1 ? tr_a.c1 : tr_a.c2), false, rot_allowed);
    }
}

__global__ void k_joint_rows(BodyDev b, JointsDev jd, float inv_dt, float erp) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= jd.n) return;
    const uint32_t jid = jd.order[t];
    const float4* d = jd.desc + size_t(jid) * JOINT_F4;
    const float4 h = d[0];
    const uint32_t kind = __float_as_uint(h.x), ia = __float_as_uint(h.y), ib = __float_as_uint(h.z);
    const uint32_t flags = __float_as_uint(h.w);
    const uint32_t act_a = b.info[ia].z, act_b = b.info[ib].z;
    auto active = [](uint32_t z) { return z == ACT_ACTIVE || z == ACT_WANTS_DEACTIVATION || z == ACT_DISABLE_DEACTIVATION; };
    // step.rs:928-949: a disabled joint, or one whose bodies both sleep, has no rows.
    if ((flags & JF_DISABLED) || (!active(act_a) && !active(act_b))) {
        jd.count[t] = 0;
        return;
    }
    RowOut out;
    out.row = jd.rows + size_t(jd.row_off[t]) * JROW_F4;
    out.n = 0;
    out.iia = load_iw_body(b.iw, ia, out.ima);
    out.iib = load_iw_body(b.iw, ib, out.imb);
    const V3 pa = from4(b.pos[ia]), pb = from4(b.pos[ib]);
    const Q qa = q4(b.quat[ia]), qb = q4(b.quat[ib]);
    const V3 origin_a = from4(d[1]), origin_b = from4(d[5]);
    const V3 pivot_a = pa + rotate(qa, origin_a), pivot_b = pb + rotate(qb, origin_b);
    const V3 r_a = pivot_a - pa, r_b = pivot_b - pb;
    const V3 zero = V3{0.0f, 0.0f, 0.0f};
    const float4 p9 = d[9], p10 = d[10], p11 = d[11];
    if (kind == JK_POINT2POINT) {
        const float k = inv_dt * ((flags & JF_ERP) ? p9.x : erp);
        const float clamp = p9.y;
        const uint32_t lim = clamp > 0.0f ? JL_BILATERAL : JL_UNBOUNDED;
        const V3 dp = pivot_a - pivot_b;
        for (int axis = 0; axis < 3; ++axis) {
            const V3 nrm = axis_vec(axis);
            out.push(nrm, cross(r_a, nrm), nrm, cross(r_b, nrm), k * comp(dp, axis), lim, -clamp, clamp);
        }
    } else if (kind == JK_SLIDER) {  // slider.rs:159-475
        const float eps = 1.1920929e-7f;  // f32::EPSILON
        const float inf = INFINITY;
        const float4 p12 = d[12], p13 = d[13], p14 = d[14], p15 = d[15];
        const float lower_lin = p12.x, upper_lin = p12.y, lower_ang = p12.z, upper_ang = p12.w;
        const float softness_lim_lin = p13.x, softness_lim_ang = p13.y, damping_lim_lin = p13.z, damping_lim_ang = p13.w;
        const float softness_ortho_lin = p14.x, softness_ortho_ang = p14.y;
        const M3 tr_a = mul(from_quat(qa), M3{from4(d[2]), from4(d[3]), from4(d[4])});
        const M3 tr_b = mul(from_quat(qb), M3{from4(d[6]), from4(d[7]), from4(d[8])});
        const V3 delta = pivot_b - pivot_a;
        const V3 ax1_a = tr_a.c0;
        float depth0 = dot(delta, tr_a.c0);
        const float lin_pos = depth0;
        jd.position[jid] = lin_pos;
        bool solve_lin_limit = false;
        if (lower_lin <= upper_lin) {
            if (depth0 > upper_lin) { depth0 -= upper_lin; solve_lin_limit = true; }
            else if (depth0 < lower_lin) { depth0 -= lower_lin; solve_lin_limit = true; }
            else depth0 = 0.0f;
        } else {
            depth0 = 0.0f;
        }
        const float lin_depth = depth0;
        bool solve_ang_limit = false;
        float ang_depth = 0.0f, ang_pos = 0.0f;
        if (lower_ang <= upper_ang) {
            const V3 axis_a0 = tr_a.c1, axis_a1 = tr_a.c2, axis_b0 = tr_b.c1;
            const float rot = adjust_angle_to_limits(atan2f(dot(axis_b0, axis_a1), dot(axis_b0, axis_a0)), lower_ang, upper_ang);
            ang_pos = rot;
            jd.angle[jid] = rot;
            if (rot < lower_ang) { ang_depth = rot - lower_ang; solve_ang_limit = true; }
            else if (rot > upper_ang) { ang_depth = rot - upper_ang; solve_ang_limit = true; }
        }
        const float sign_fact = (flags & JF_FRAME_B) ? -1.0f : 1.0f;
        const V3 ofs = pivot_b - pivot_a;
        const bool has_static = out.ima < eps || out.imb < eps;
        const float ims = out.ima + out.imb;
        const float fact_a = ims > 0.0f ? out.imb / ims : 0.5f;
        const float fact_b = 1.0f - fact_a;
        const V3 ax1 = normalize(ax1_a * fact_a + tr_b.c0 * fact_b);
        const float k = inv_dt * (softness_ortho_ang * erp);
        const V3 u = cross(ax1_a, tr_b.c0);
        const V3 rel_pa = pivot_a - pa, rel_pb = pivot_b - pb;
        const V3 ortho_a = rel_pa - ax1 * dot(rel_pa, ax1);
        const V3 ortho_b = rel_pb - ax1 * dot(rel_pb, ax1);
        const float slider_offs = lin_pos - depth0;
        const V3 total_dist = ax1 * (dot(ax1, pivot_a - pa) + slider_offs) - ax1 * dot(ax1, pivot_b - pb);
        const V3 rel_a = ortho_a + total_dist * fact_a;
        const V3 rel_b = ortho_b - total_dist * fact_b;
        const V3 avg = ortho_b * fact_a + ortho_a * fact_b;
        const V3 p = len2(avg) > eps ? normalize(avg) : tr_a.c1;
        const V3 q = cross(ax1, p);
        out.push(zero, p, zero, p, -k * dot(u, p), JL_UNBOUNDED, 0.0f, 0.0f);
        out.push(zero, q, zero, q, -k * dot(u, q), JL_UNBOUNDED, 0.0f, 0.0f);
        const float k_lin = inv_dt * (softness_ortho_lin * erp);
        out.push(p, cross(rel_a, p), p, cross(rel_b, p), -k_lin * dot(p, ofs), JL_UNBOUNDED, 0.0f, 0.0f);
        {
            V3 tmp_a = cross(rel_a, q), tmp_b = cross(rel_b, q);
            if (has_static && solve_ang_limit) { tmp_a = tmp_a * fact_a; tmp_b = tmp_b * fact_b; }
            out.push(q, tmp_a, q, tmp_b, -k_lin * dot(q, ofs), JL_UNBOUNDED, 0.0f, 0.0f);
        }
        // linear limit / motor row
        float limit_err = 0.0f;
        int limit = 0;
        if (solve_lin_limit) {
            limit_err = lin_depth * sign_fact;
            limit = limit_err > 0.0f ? 2 : 1;
        }
        bool powered = (flags & JF_LIN_MOTOR) != 0;
        if (limit != 0 && lower_lin == upper_lin) powered = false;
        if (limit != 0 || powered) {
            const float curr_erp = erp;
            float row_error = 0.0f, lower = 0.0f, upper = 0.0f;
            if (powered) {
                const float target = p14.z, max_force = p14.w;
                const float mf = motor_factor(lin_pos, lower_lin, upper_lin, target, inv_dt * curr_erp);
                row_error -= sign_fact * mf * target;
                lower += -max_force / inv_dt;
                upper += max_force / inv_dt;
            }
            if (limit != 0) {
                row_error += inv_dt * curr_erp * limit_err;
                if (lower_lin == upper_lin) { lower = -inf; upper = inf; }
                else if (limit == 1) { lower = -inf; upper = 0.0f; }
                else { lower = 0.0f; upper = inf; }
                const float bounce = fabsf(1.0f - damping_lim_lin);
                if (bounce > 0.0f) {
                    float vel = dot(from4(b.linvel[ia]), ax1) - dot(from4(b.linvel[ib]), ax1);
                    vel *= sign_fact;
                    if (limit == 1) {
                        if (vel < 0.0f) { const float newc = -bounce * vel; if (newc > row_error) row_error = newc; }
                    } else if (vel > 0.0f) {
                        const float newc = -bounce * vel;
                        if (newc < row_error) row_error = newc;
                    }
                }
                row_error *= softness_lim_lin;
            }
            uint32_t lim;
            float lo, hi;
            mirrored_row_limits(lower, upper, lim, lo, hi);
            const V3 ang_a = has_static ? zero : cross(rel_a, ax1);
            const V3 ang_b = has_static ? zero : cross(rel_b, ax1);
            out.push(ax1, ang_a, ax1, ang_b, -row_error, lim, lo, hi);
        }
        // angular limit / motor row
        limit_err = 0.0f;
        limit = 0;
        if (solve_ang_limit) {
            limit_err = ang_depth;
            limit = limit_err > 0.0f ? 1 : 2;
        }
        powered = (flags & JF_ANG_MOTOR) != 0;
        if (limit != 0 && lower_ang == upper_ang) powered = false;
        if (limit != 0 || powered) {
            const float curr_erp = erp;
            float row_error = 0.0f, lower = 0.0f, upper = 0.0f;
            if (powered) {
                const float target = p15.x, max_force = p15.y;
                const float mf = motor_factor(ang_pos, lower_ang, upper_ang, target, inv_dt * curr_erp);
                row_error = mf * target;
                lower = -max_force / inv_dt;
                upper = max_force / inv_dt;
            }
            if (limit != 0) {
                row_error += inv_dt * curr_erp * limit_err;
                if (lower_ang == upper_ang) { lower = -inf; upper = inf; }
                else if (limit == 1) { lower = 0.0f; upper = inf; }
                else { lower = -inf; upper = 0.0f; }
                const float bounce = fabsf(1.0f - damping_lim_ang);
                if (bounce > 0.0f) {
                    const float vel = dot(from4(b.angvel[ia]), ax1) - dot(from4(b.angvel[ib]), ax1);
                    if (limit == 1) {
                        if (vel < 0.0f) { const float newc = -bounce * vel; if (newc > row_error) row_error = newc; }
                    } else if (vel > 0.0f) {
                        const float newc = -bounce * vel;
                        if (newc < row_error) row_error = newc;
                    }
                }
                row_error *= softness_lim_ang;
            }
            uint32_t lim;
            float lo, hi;
            mirrored_row_limits(lower, upper, lim, lo, hi);
            out.push(zero, ax1, zero, ax1, -row_error, lim, lo, hi);
        }
    } else if (kind == JK_SPRING2) {
        spring2_rows(out, b, jd, jid, d, ia, ib, pa, pb, qa, qb, pivot_a, pivot_b, inv_dt, erp);
    } else if (kind == JK_GENERIC6DOF) {
        generic6dof_rows(out, b, jd, jid, d, ia, ib, qa, qb, r_a, r_b, pivot_a, pivot_b, inv_dt);
    } else if (kind == JK_CONETWIST) {
        conetwist_rows(out, b, jd, jid, d, flags, qa, qb, r_a, r_b, pivot_a, pivot_b, inv_dt, erp);
    } else if (kind == JK_GEAR) {  // gear.rs:33-57: the spins about the frames' z columns, coupled
        const V3 axis_a_world = rotate(qa, from4(d[4])), axis_b_world = rotate(qb, from4(d[8]));
        out.push(zero, axis_a_world, zero, -(axis_b_world * p11.y), 0.0f, JL_UNBOUNDED, 0.0f, 0.0f);
    } else {
        const M3 basis_a = M3{from4(d[2]), from4(d[3]), from4(d[4])};
        const M3 basis_b = M3{from4(d[6]), from4(d[7]), from4(d[8])};
        const M3 tr_a = mul(from_quat(qa), basis_a), tr_b = mul(from_quat(qb), basis_b);
        const float k = inv_dt * erp;
        const V3 dp = pivot_a - pivot_b;
        if (kind == JK_FIXED) {
            for (int axis = 0; axis < 3; ++axis) {
                const V3 nrm = axis_vec(axis);
                out.push(nrm, cross(r_a, nrm), nrm, cross(r_b, nrm), k * comp(dp, axis), JL_UNBOUNDED, 0.0f, 0.0f);
            }
            // shared.rs:108-123 (relative_rotation_info)
            const V3 euler = euler_xyz(mul(transpose(tr_a), tr_b));
            const V3 axis0 = tr_b.c0, axis2 = tr_a.c2;
            V3 ax1 = cross(axis2, axis0);
            V3 ax0 = cross(ax1, axis2);
            V3 ax2 = cross(axis0, ax1);
            ax0 = normalize(ax0);
            ax1 = normalize(ax1);
            ax2 = normalize(ax2);
            out.push(zero, ax0, zero, ax0, k * euler.x, JL_UNBOUNDED, 0.0f, 0.0f);
            out.push(zero, ax1, zero, ax1, k * euler.y, JL_UNBOUNDED, 0.0f, 0.0f);
            out.push(zero, ax2, zero, ax2, k * euler.z, JL_UNBOUNDED, 0.0f, 0.0f);
        } else {  // hinge
            const V3 ax1 = tr_a.c2, p = tr_a.c0, q = tr_a.c1, ax2 = tr_b.c2;
            if (!(flags & JF_ANGULAR_ONLY)) {
                for (int axis = 0; axis < 3; ++axis) {
                    const V3 nrm = axis_vec(axis);
                    out.push(nrm, cross(r_a, nrm), nrm, cross(r_b, nrm), k * comp(dp, axis), JL_UNBOUNDED, 0.0f, 0.0f);
                }
            }
            const V3 u = cross(ax1, ax2);
            out.push(zero, p, zero, p, -k * dot(u, p), JL_UNBOUNDED, 0.0f, 0.0f);
            out.push(zero, q, zero, q, -k * dot(u, q), JL_UNBOUNDED, 0.0f, 0.0f);
            // shared.rs:9-14 (get_hinge_angle)
            const V3 swing = tr_b.c1;
            const float angle = atan2f(dot(swing, tr_a.c0), dot(swing, tr_a.c1));
            jd.angle[jid] = angle;
            const bool has_limit = (flags & JF_LIMIT) != 0, powered = (flags & JF_MOTOR) != 0;
            const float low = p9.z, high = p9.w, bias_factor = p10.y, relaxation = p10.z;
            const float motor_target = p10.w, motor_max = p11.x;
            // constraint.rs:735-751 (AngularLimit::test)
            float correction = 0.0f, sign = 0.0f;
            bool solve = false;
            if (has_limit) {
                const float half_range = (high - low) / 2.0f;
                if (half_range >= 0.0f) {
                    const float center = normalize_angle(low + half_range);
                    const float deviation = normalize_angle(angle - center);
                    if (deviation < -half_range) {
                        correction = -(deviation + half_range);
                        sign = 1.0f;
                        solve = true;
                    } else if (deviation > half_range) {
                        correction = half_range - deviation;
                        sign = -1.0f;
                        solve = true;
                    }
                }
            }
            if (solve || powered) {
                float row_error = 0.0f;
                const float lostop = has_limit ? low : 1.0f, histop = has_limit ? high : -1.0f;
                const bool motor_ineffective = solve && lostop == histop;
                if (powered && !motor_ineffective) {
                    const float mf = motor_factor(angle, lostop, histop, motor_target, inv_dt * erp);
                    row_error += mf * motor_target;
                }
                if (solve) {
                    row_error += k * correction;
                    const float bounce = has_limit ? relaxation : 1.0f;
                    if (bounce > 0.0f) {
                        const float vel = dot(from4(b.angvel[ia]), ax1) - dot(from4(b.angvel[ib]), ax1);
                        if (sign > 0.0f) {
                            if (vel < 0.0f) {
                                const float newc = -bounce * vel;
                                if (newc > row_error) row_error = newc;
                            }
                        } else if (vel > 0.0f) {
                            const float newc = -bounce * vel;
                            if (newc < row_error) row_error = newc;
                        }
                    }
                    row_error *= has_limit ? bias_factor : 1.0f;
                }
                uint32_t lim;
                float lo = 0.0f, hi = 0.0f;
                if (solve) {
                    lim = lostop == histop ? JL_UNBOUNDED : (sign > 0.0f ? JL_UPPER : JL_LOWER);
                } else {
                    lim = JL_BILATERAL;
                    hi = powered ? motor_max : 0.0f;
                    lo = -hi;
                }
                out.push(zero, ax1, zero, ax1, -row_error, lim, lo, hi);
            }
        }
    }
    jd.count[t] = out.n;
}

}  // namespace

void launch_joint_rows(const BodyDev& b, const JointsDev& j, float inv_dt, float erp, cudaStream_t s) {
    if (j.n == 0) return;
    k_joint_rows<<<(j.n + 127) / 128, 128, 0, s>>>(b, j, inv_dt, erp);
}

}  // namespace bgpu
