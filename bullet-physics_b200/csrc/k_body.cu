// Per-body kernels of the step: velocity integration fused with the
// predicted detection pose, the padded broad-phase AABB and the world inverse
// inertia (one pass over the body arrays), and the end-of-step pass that
// fuses deactivation, exp-map pose integration and the split-impulse push.
#include "bgpu_kernels.cuh"

namespace bgpu {

__device__ __forceinline__ bool is_active(uint32_t act) {
    return act == ACT_ACTIVE || act == ACT_WANTS_DEACTIVATION || act == ACT_DISABLE_DEACTIVATION;
}

// body.rs:1066-1105
__device__ __forceinline__ void apply_damping(V3& v, V3& w, float ld, float ad, bool additional, float dt) {
    if (ld != 0.0f) v = v * powf(1.0f - ld, dt);
    if (ad != 0.0f) w = w * powf(1.0f - ad, dt);
    if (!additional) return;
    if (len2(w) < 0.01f && len2(v) < 0.01f) {
        w = w * 0.005f;
        v = v * 0.005f;
    }
    const float damp_vel = 0.005f;
    float speed = len(v);
    if (speed < ld) {
        if (speed > damp_vel) v -= (v / len(v)) * damp_vel;
        else v = V3{0.f, 0.f, 0.f};
    }
    float aspeed = len(w);
    if (aspeed < ad) {
        if (aspeed > damp_vel) w -= (w / len(w)) * damp_vel;
        else w = V3{0.f, 0.f, 0.f};
    }
}

// body.rs:1135-1148 — one Newton step of the implicit gyroscopic term.
__device__ __forceinline__ V3 gyroscopic_implicit(V3 inv, Q q, V3 w, float step) {
    if (inv.x <= 0.0f || inv.y <= 0.0f || inv.z <= 0.0f) return V3{0.f, 0.f, 0.f};
    V3 inertia = V3{1.0f / inv.x, 1.0f / inv.y, 1.0f / inv.z};
    M3 ib = diag(inertia);
    V3 ob = rotate(qinv(q), w);
    V3 ibo = inertia * ob;
    V3 residual = cross(ob, ibo) * step;
    M3 jac = madd(ib, mscale(msub(mul(skew(ob), ib), skew(ibo)), step));
    V3 delta = mul(inverse(jac), residual);
    return rotate(q, ob - delta) - w;
}

// step.rs:306-363 + body.rs:1113-1126, 1175-1181, shapes/mod.rs:350, util.rs:52-55.
__global__ void k_integrate_velocities(BodyDev b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                       uint32_t n, float dt, float aabb_margin) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 info = b.info[i];
    float4 p4 = b.pos[i];
    float4 q4v = b.quat[i];
    float4 lv4 = b.linvel[i];
    float4 av4 = b.angvel[i];
    float4 ii4 = b.inv_inertia[i];
    V3 v = from4(lv4), w = from4(av4);
    b.settled[i] = len2(v) + len2(w);
    Q q = q4(q4v);
    bool stat = (info.y & BF_STATIC) != 0;
    bool kin = (info.y & BF_KINEMATIC) != 0;
    bool active = is_active(info.z);
    V3 inv_local = from4(ii4);
    M3 iw = inertia_world(inv_local, q);
    if (!stat && !kin && active) {
        float4 mat = b.material[i];
        apply_damping(v, w, mat.z, mat.w, (info.y & BF_ADDITIONAL_DAMPING) != 0, dt);
        V3 g = from4(b.gravity[i]);
        V3 f = from4(b.force[i]);
        V3 t = from4(b.torque[i]);
        v += (g + f * ii4.w) * dt;
        w += mul(iw, t * dt);
        w += gyroscopic_implicit(inv_local, q, w, dt);
        b.linvel[i] = to4(v, 0.0f);
        b.angvel[i] = to4(w, 0.0f);
        if (b.rec_flags) b.rec_flags[i] |= RF_INTEGRATED;
    }
    V3 p = from4(p4);
    V3 pred = (stat || !active) ? p : p + v * dt;
    b.pred[i] = to4(pred, 0.0f);
    if (active) {
        Shape s = shapes[info.x];
        V3 mn, mx;
        world_aabb(s, pred, q, hull, mn, mx);
        mn = mn - splat(aabb_margin);
        mx = mx + splat(aabb_margin);
        b.aabb_min[i] = to4(mn, 0.0f);
        b.aabb_max[i] = to4(mx, 0.0f);
    }
    b.iw[3 * i + 0] = make_float4(iw.c0.x, iw.c0.y, iw.c0.z, iw.c1.x);
    b.iw[3 * i + 1] = make_float4(iw.c1.y, iw.c1.z, iw.c2.x, iw.c2.y);
    b.iw[3 * i + 2] = make_float4(iw.c2.z, ii4.w, 0.0f, 0.0f);
    b.push_lin[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    b.push_ang[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Static body AABBs at insertion (world.rs:548-552): pose, not predicted pose.
__global__ void k_initial_aabbs(BodyDev b, const Shape* __restrict__ shapes, const float4* __restrict__ hull,
                                uint32_t first, uint32_t n, float aabb_margin) {
    uint32_t i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= first + n) return;
    uint4 info = b.info[i];
    Shape s = shapes[info.x];
    V3 mn, mx;
    world_aabb(s, from4(b.pos[i]), q4(b.quat[i]), hull, mn, mx);
    b.aabb_min[i] = to4(mn - splat(aabb_margin), 0.0f);
    b.aabb_max[i] = to4(mx + splat(aabb_margin), 0.0f);
}

// body.rs:92-137 (btTransformUtil::integrateTransform)
__device__ __forceinline__ void interpolate_pose(V3& p, Q& q, V3 lv, V3 av, float dt) {
    const float EPS = 1.1920929e-7f;
    const float FRAC_PI_4 = 0.785398163397448309615f;
    p = p + lv * dt;
    float angle_sqr = len2(av);
    float angle = 0.0f;
    if (angle_sqr > EPS) angle = sqrtf(angle_sqr);
    if (angle * dt > FRAC_PI_4) angle = FRAC_PI_4 / dt;
    V3 axis;
    if (angle < 0.001f) axis = av * (0.5f * dt - (dt * dt * dt) * 0.020833333f * angle * angle);
    else axis = av * (sinf(0.5f * angle * dt) / angle);
    Q dorn = Q{axis.x, axis.y, axis.z, cosf(angle * dt * 0.5f)};
    Q pr = qmul(dorn, q);
    float ls = qlen2(pr);
    if (ls < EPS) pr = Q{0.f, 0.f, 0.f, 0.f};
    else {
        float l = sqrtf(ls);
        pr = Q{pr.x / l, pr.y / l, pr.z / l, pr.w / l};
    }
    if (qlen2(pr) > EPS) q = pr;
}

// step.rs:1059-1061 (update_deactivation, body.rs:639-657) fused with
// step.rs:1171-1215 (integrate_position + split-impulse push) and step.rs:1272 (clear forces).
__global__ void k_integrate_positions(BodyDev b, uint32_t n, float dt, float turn_erp) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 info = b.info[i];
    bool stat = (info.y & BF_STATIC) != 0;
    bool kin = (info.y & BF_KINEMATIC) != 0;
    uint32_t act = info.z;
    V3 v = from4(b.linvel[i]), w = from4(b.angvel[i]);
    // update_deactivation
    if (is_active(act) && act != ACT_DISABLE_DEACTIVATION) {
        float4 sl = b.sleep[i];
        float dtime = sl.x;
        bool slow = len2(v) < sl.y * sl.y && len2(w) < sl.z * sl.z;
        if (slow) dtime += dt;
        else { dtime = 0.0f; act = ACT_ACTIVE; }
        if (dtime > 2.0f) { dtime = 0.0f; act = ACT_WANTS_DEACTIVATION; }
        sl.x = dtime;
        b.sleep[i] = sl;
        info.z = act;
        b.info[i] = info;
    }
    bool active = is_active(act);
    V3 p = from4(b.pos[i]);
    Q q = q4(b.quat[i]);
    bool moved = false;
    if (!stat && active) {
        interpolate_pose(p, q, v, w, dt);
        moved = true;
        if (b.rec_flags) b.rec_flags[i] |= RF_MOVED;
    }
    V3 pl = from4(b.push_lin[i]), pw = from4(b.push_ang[i]);
    if (active && !stat && !kin && (pl.x != 0.0f || pl.y != 0.0f || pl.z != 0.0f)) {
        p = p + pl * dt;
        moved = true;
    }
    if (active && !stat && !kin && (pw.x != 0.0f || pw.y != 0.0f || pw.z != 0.0f)) {
        V3 tw = pw * turn_erp;
        Q dq = qmul(Q{tw.x * dt * 0.5f, tw.y * dt * 0.5f, tw.z * dt * 0.5f, 0.0f}, q);
        Q s = Q{q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w};
        float l = sqrtf(qlen2(s));
        q = Q{s.x / l, s.y / l, s.z / l, s.w / l};
        moved = true;
    }
    if (moved) {
        b.pos[i] = to4(p, 0.0f);
        b.quat[i] = to4(q);
    }
    b.push_lin[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    b.push_ang[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    b.force[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    b.torque[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_compute_iw(BodyDev b, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 ii4 = b.inv_inertia[i];
    M3 iw = inertia_world(from4(ii4), q4(b.quat[i]));
    b.iw[3 * i + 0] = make_float4(iw.c0.x, iw.c0.y, iw.c0.z, iw.c1.x);
    b.iw[3 * i + 1] = make_float4(iw.c1.y, iw.c1.z, iw.c2.x, iw.c2.y);
    b.iw[3 * i + 2] = make_float4(iw.c2.z, ii4.w, 0.0f, 0.0f);
}

void launch_compute_iw(const BodyDev& b, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    k_compute_iw<<<(n + 255) / 256, 256, 0, s>>>(b, n);
}

void launch_integrate_velocities(const BodyDev& b, const Shape* shapes, const float4* hull, uint32_t n, float dt,
                                 cudaStream_t s) {
    if (n == 0) return;
    k_integrate_velocities<<<(n + 255) / 256, 256, 0, s>>>(b, shapes, hull, n, dt, 0.02f);
}

void launch_initial_aabbs(const BodyDev& b, const Shape* shapes, const float4* hull, uint32_t first, uint32_t n,
                          cudaStream_t s) {
    if (n == 0) return;
    k_initial_aabbs<<<(n + 255) / 256, 256, 0, s>>>(b, shapes, hull, first, n, 0.02f);
}

void launch_integrate_positions(const BodyDev& b, uint32_t n, float dt, float turn_erp, cudaStream_t s) {
    if (n == 0) return;
    k_integrate_positions<<<(n + 255) / 256, 256, 0, s>>>(b, n, dt, turn_erp);
}

namespace {

// n x 3 floats (the caller's layout) -> float4 lanes.
__global__ void k_unpack3(uint32_t n, const float* __restrict__ src, float4* dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0f);
}

// position + orientation -> n x 7 floats (x y z qx qy qz qw).
__global__ void k_pack_poses(uint32_t n, const float4* __restrict__ pos, const float4* __restrict__ quat, float* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i], q = quat[i];
    float* o = out + size_t(i) * 7;
    o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = q.x; o[4] = q.y; o[5] = q.z; o[6] = q.w;
}

}  // namespace

void launch_unpack3(uint32_t n, const float* src, float4* dst, cudaStream_t s) {
    if (n) k_unpack3<<<(n + 255) / 256, 256, 0, s>>>(n, src, dst);
}

void launch_pack_poses(uint32_t n, const float4* pos, const float4* quat, float* out, cudaStream_t s) {
    if (n) k_pack_poses<<<(n + 255) / 256, 256, 0, s>>>(n, pos, quat, out);
}

}  // namespace bgpu
