// Joint rows of one step (constraint.rs:755-842; fixed.rs:33-90; hinge.rs:130-267;
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
                                         float hi) {
        const float k = ima * len2(lin_a) + imb * len2(lin_b) + dot(ang_a, mul(iia, ang_a)) + dot(ang_b, mul(iib, ang_b));
        const float mass = k > 0.0f ? 1.0f / k : 0.0f;
        float4* r = row + size_t(n) * JROW_F4;
        r[0] = to4(lin_a, mass);
        r[1] = to4(ang_a, bias);
        r[2] = to4(lin_b, 0.0f);
        r[3] = to4(ang_b, __uint_as_float(lim));
        r[4] = make_float4(lo, hi, 0.0f, 0.0f);
        ++n;
    }
};

__device__ __forceinline__ V3 axis_vec(int axis) {
    return V3{axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f};
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
    out.row = jd.rows + size_t(t) * JOINT_MAX_ROWS * JROW_F4;
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
