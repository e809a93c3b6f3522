// CPU oracle C interface — TEST INFRASTRUCTURE ONLY.
// Loaded by tests/ (ctypes) and by bench.py's CPU baseline leg; the shipped
// library never links it. All values cross the boundary as double; the world
// computes in float (precision 0, the reference's default f32 build) or in
// double (precision 1, the reference's `--features f64` build).
#include <cstring>
#include <memory>
#include "oracle_world.hpp"

using namespace oracle;

namespace {

struct Handle {
    int f64 = 0;
    double accumulator = 0.0;  // step_simulation_fixed's accumulator (a value of the world's precision)
    std::unique_ptr<World<float>> wf;
    std::unique_ptr<World<double>> wd;
};

template <class R>
Shape<R> make_shape(uint32_t type, const double* p, const double* pts, uint32_t npts) {
    switch (type) {
        case SHAPE_SPHERE: return Shape<R>::sphere(static_cast<R>(p[0]));
        case SHAPE_BOX: return Shape<R>::box(V3<R>(static_cast<R>(p[0]), static_cast<R>(p[1]), static_cast<R>(p[2])));
        case SHAPE_CAPSULE: return Shape<R>::capsule(static_cast<R>(p[0]), static_cast<R>(p[1]));
        case SHAPE_PLANE: return Shape<R>::plane(V3<R>(static_cast<R>(p[0]), static_cast<R>(p[1]), static_cast<R>(p[2])), static_cast<R>(p[3]));
        default: {
            std::vector<V3<R>> v;
            for (uint32_t i = 0; i < npts; ++i) v.push_back(V3<R>(static_cast<R>(pts[3 * i]), static_cast<R>(pts[3 * i + 1]), static_cast<R>(pts[3 * i + 2])));
            return Shape<R>::hull(v);
        }
    }
}

// Body descriptor layout (doubles), shared with tests/oracle_api.py:
//  0 shape, 1-3 pos, 4-7 quat xyzw, 8-10 linvel, 11-13 angvel, 14 mass (0 = static),
//  15 friction, 16 restitution, 17 flags (| 0x10: additional damping), 18 group, 19 mask, 20 lin damping,
//  21 ang damping, 22 activation override (0 = default), 23 kinematic (0/1)
constexpr int DESC = 24;

template <class R>
uint32_t add_body(World<R>& w, const double* d) {
    uint32_t shape = uint32_t(d[0]);
    V3<R> pos(static_cast<R>(d[1]), static_cast<R>(d[2]), static_cast<R>(d[3]));
    Body<R> b = d[14] > 0 ? w.make_dynamic(shape, pos, static_cast<R>(d[14])) : w.make_static(shape, pos);
    b.orientation = Quat<R>(static_cast<R>(d[4]), static_cast<R>(d[5]), static_cast<R>(d[6]), static_cast<R>(d[7]));
    b.linear_velocity = V3<R>(static_cast<R>(d[8]), static_cast<R>(d[9]), static_cast<R>(d[10]));
    b.angular_velocity = V3<R>(static_cast<R>(d[11]), static_cast<R>(d[12]), static_cast<R>(d[13]));
    b.friction = static_cast<R>(d[15]);
    b.restitution = static_cast<R>(d[16]);
    b.flags = uint32_t(d[17]);
    b.group = uint16_t(d[18]);
    b.mask = uint16_t(d[19]);
    b.linear_damping = static_cast<R>(d[20]);
    b.angular_damping = static_cast<R>(d[21]);
    if (d[23] != 0) {  // body.rs:440-449 new_kinematic: a static body turned kinematic
        b = w.make_static(shape, pos);
        b.orientation = Quat<R>(static_cast<R>(d[4]), static_cast<R>(d[5]), static_cast<R>(d[6]), static_cast<R>(d[7]));
        b.linear_velocity = V3<R>(static_cast<R>(d[8]), static_cast<R>(d[9]), static_cast<R>(d[10]));
        b.angular_velocity = V3<R>(static_cast<R>(d[11]), static_cast<R>(d[12]), static_cast<R>(d[13]));
        b.friction = static_cast<R>(d[15]);
        b.restitution = static_cast<R>(d[16]);
        b.is_static = false;
        b.flags = uint32_t(d[17]) | CF_KINEMATIC;
        b.activation = ACT_DISABLE_DEACTIVATION;
        // The filter and damping a caller sets on the built body (collision_filter, set_damping).
        b.group = uint16_t(d[18]);
        b.mask = uint16_t(d[19]);
        b.linear_damping = static_cast<R>(d[20]);
        b.angular_damping = static_cast<R>(d[21]);
    }
    // Flag bit 0x10 (not a collision flag): the additional_damping(true) builder (body.rs:1066-1105).
    b.additional_damping = (b.flags & 0x10u) != 0;
    b.flags &= ~0x10u;
    if (d[22] != 0) b.activation = uint32_t(d[22]);
    return w.add_body(b);
}

// Body state layout (doubles): pos3, quat4, linvel3, angvel3, activation, deactivation_time = 15
constexpr int STATE = 15;

template <class R>
void get_state(const World<R>& w, double* out) {
    for (size_t i = 0; i < w.bodies.size(); ++i) {
        const Body<R>& b = w.bodies[i];
        double* o = out + i * STATE;
        o[0] = b.position.x; o[1] = b.position.y; o[2] = b.position.z;
        o[3] = b.orientation.x; o[4] = b.orientation.y; o[5] = b.orientation.z; o[6] = b.orientation.w;
        o[7] = b.linear_velocity.x; o[8] = b.linear_velocity.y; o[9] = b.linear_velocity.z;
        o[10] = b.angular_velocity.x; o[11] = b.angular_velocity.y; o[12] = b.angular_velocity.z;
        o[13] = b.activation; o[14] = b.deactivation_time;
    }
}

template <class R>
void set_state(World<R>& w, const double* in) {
    for (size_t i = 0; i < w.bodies.size(); ++i) {
        Body<R>& b = w.bodies[i];
        const double* o = in + i * STATE;
        b.position = V3<R>(static_cast<R>(o[0]), static_cast<R>(o[1]), static_cast<R>(o[2]));
        b.orientation = Quat<R>(static_cast<R>(o[3]), static_cast<R>(o[4]), static_cast<R>(o[5]), static_cast<R>(o[6]));
        b.linear_velocity = V3<R>(static_cast<R>(o[7]), static_cast<R>(o[8]), static_cast<R>(o[9]));
        b.angular_velocity = V3<R>(static_cast<R>(o[10]), static_cast<R>(o[11]), static_cast<R>(o[12]));
        b.activation = uint32_t(o[13]);
        b.deactivation_time = static_cast<R>(o[14]);
    }
}

// Row layout (doubles): body_a, body_b, point_index, normal3, r_a3, r_b3,
// penetration, normal_impulse, tangent1_impulse, tangent2_impulse, push_impulse,
// split_active, friction, restitution, normal_mass, tangent1_mass, tangent2_mass,
// baumgarte_span, normal_cfm, erp = 26
constexpr int ROW = 26;

template <class R>
void get_rows(const std::vector<ContactConstraint<R>>& rows, double* out) {
    for (size_t i = 0; i < rows.size(); ++i) {
        const ContactConstraint<R>& c = rows[i];
        double* o = out + i * ROW;
        o[0] = c.body_a; o[1] = c.body_b; o[2] = c.point_index;
        o[3] = c.normal.x; o[4] = c.normal.y; o[5] = c.normal.z;
        o[6] = c.r_a.x; o[7] = c.r_a.y; o[8] = c.r_a.z;
        o[9] = c.r_b.x; o[10] = c.r_b.y; o[11] = c.r_b.z;
        o[12] = c.penetration; o[13] = c.normal_impulse; o[14] = c.tangent1_impulse; o[15] = c.tangent2_impulse;
        o[16] = c.push_impulse; o[17] = c.split_active ? 1 : 0; o[18] = c.friction; o[19] = c.restitution;
        o[20] = c.normal_mass; o[21] = c.tangent1_mass; o[22] = c.tangent2_mass;
        o[23] = c.baumgarte_span; o[24] = c.normal_cfm; o[25] = c.erp;
    }
}

template <class R>
Quat<R> q_of(const double* p) { return Quat<R>(static_cast<R>(p[3]), static_cast<R>(p[4]), static_cast<R>(p[5]), static_cast<R>(p[6])); }
template <class R>
V3<R> v_of(const double* p) { return V3<R>(static_cast<R>(p[0]), static_cast<R>(p[1]), static_cast<R>(p[2])); }

template <class R>
int collide_impl(World<R>& w, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b, const double* seed,
                 double* out) {
    Manifold<R> m;
    V3<R> s;
    bool has_seed = seed != nullptr;
    if (has_seed) s = V3<R>(static_cast<R>(seed[0]), static_cast<R>(seed[1]), static_cast<R>(seed[2]));
    if (!collide(w.shapes[sa], v_of<R>(pose_a), q_of<R>(pose_a), w.shapes[sb], v_of<R>(pose_b), q_of<R>(pose_b), has_seed, s, m))
        return 0;
    int n = 0;
    for (auto& cp : m.points) {
        double* o = out + n * 7;
        o[0] = cp.position.x; o[1] = cp.position.y; o[2] = cp.position.z;
        o[3] = cp.normal.x; o[4] = cp.normal.y; o[5] = cp.normal.z;
        o[6] = cp.penetration;
        if (++n == 8) break;
    }
    return n;
}

template <class R>
int convex_impl(World<R>& w, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b, double* out) {
    Manifold<R> m;
    R thr = pair_threshold(w.shapes[sa], w.shapes[sb]);
    if (!convex_convex(w.shapes[sa], v_of<R>(pose_a), q_of<R>(pose_a), w.shapes[sb], v_of<R>(pose_b), q_of<R>(pose_b),
                       false, V3<R>(), thr, m))
        return 0;
    const ContactPoint<R>& cp = m.points[0];
    out[0] = cp.position.x; out[1] = cp.position.y; out[2] = cp.position.z;
    out[3] = cp.normal.x; out[4] = cp.normal.y; out[5] = cp.normal.z;
    out[6] = cp.penetration;
    return 1;
}

template <class R>
int gjk_kind_impl(World<R>& w, uint32_t sa, const double* pa, uint32_t sb, const double* pb) {
    R thr = pair_threshold(w.shapes[sa], w.shapes[sb]);
    GjkOutcome<R> g = gjk_contact(w.shapes[sa], v_of<R>(pa), q_of<R>(pa), w.shapes[sb], v_of<R>(pb), q_of<R>(pb), false,
                                  V3<R>(), thr);
    return g.kind;
}

// gjk.rs:171-288 gjk_contact with the caller's threshold and optional seed; out: distance,
// normal3, point_on_b3 (the band outcome's fields), the overlap simplex's point count. Returns
// the outcome kind.
template <class R>
int gjk_contact_impl(World<R>& w, uint32_t sa, const double* pa, uint32_t sb, const double* pb, const double* seed,
                     double threshold, double* out) {
    const V3<R> sd = seed ? V3<R>(static_cast<R>(seed[0]), static_cast<R>(seed[1]), static_cast<R>(seed[2])) : V3<R>();
    GjkOutcome<R> g = gjk_contact(w.shapes[sa], v_of<R>(pa), q_of<R>(pa), w.shapes[sb], v_of<R>(pb), q_of<R>(pb),
                                  seed != nullptr, sd, static_cast<R>(threshold));
    out[0] = g.distance;
    out[1] = g.normal.x; out[2] = g.normal.y; out[3] = g.normal.z;
    out[4] = g.point_on_b.x; out[5] = g.point_on_b.y; out[6] = g.point_on_b.z;
    out[7] = g.simplex_len;
    return g.kind;
}

// step.rs:136-199 (step_simulation_fixed, the default latency mode, motion states left out): the
// accumulator, at most max_sub_steps substeps of fixed_dt, the unclamped demand returned; the
// forces applied before the call act in each substep and are cleared once after the last, and a
// call without a substep drops them.
template <class R>
uint32_t step_fixed_impl(World<R>& w, double& accumulator, double dt, uint32_t max_sub_steps, double fixed_dt) {
    auto drop = [&]() {
        for (auto& b : w.bodies) {
            b.force = V3<R>();
            b.torque = V3<R>();
        }
    };
    uint32_t num = 0;
    R step_dt = static_cast<R>(fixed_dt);
    if (max_sub_steps != 0) {
        R acc = static_cast<R>(accumulator) + static_cast<R>(dt), fx = static_cast<R>(fixed_dt);
        if (acc >= fx) {
            num = uint32_t(acc / fx);
            acc -= static_cast<R>(num) * fx;
        }
        accumulator = acc;
    } else {
        step_dt = static_cast<R>(dt);
        accumulator = 0.0;
        if (std::fabs(static_cast<R>(dt)) > std::numeric_limits<R>::epsilon()) num = 1;
    }
    if (num == 0) {
        drop();
        return 0;
    }
    const uint32_t clamped = max_sub_steps ? std::min(num, max_sub_steps) : num;
    std::vector<V3<R>> keep_f, keep_t;
    for (auto& b : w.bodies) {
        keep_f.push_back(b.force);
        keep_t.push_back(b.torque);
    }
    for (uint32_t k = 0; k < clamped; ++k) {
        if (k > 0)
            for (size_t i = 0; i < w.bodies.size(); ++i) {
                w.bodies[i].force = keep_f[i];
                w.bodies[i].torque = keep_t[i];
            }
        w.step(step_dt);
    }
    return num;
}

template <class R>
void pairs_impl(const double* aabbs, uint32_t n, int method, std::vector<std::pair<uint32_t, uint32_t>>& out) {
    std::vector<Aabb<R>> a(n);
    for (uint32_t i = 0; i < n; ++i) {
        const double* p = aabbs + 6 * i;
        a[i] = Aabb<R>(V3<R>(static_cast<R>(p[0]), static_cast<R>(p[1]), static_cast<R>(p[2])), V3<R>(static_cast<R>(p[3]), static_cast<R>(p[4]), static_cast<R>(p[5])));
    }
    if (method == 0) brute_force_pairs(a, out);
    else if (method == 1) sweep_pairs(a, out);
    else grid_pairs(a, out);
}

// Contacts layout for a standalone solve (doubles): body_a, body_b, pos3, normal3,
// penetration, normal_impulse = 10
template <class R>
void solve_impl(World<R>& w, const double* contacts, uint32_t n, double inv_dt, double* out_rows) {
    std::vector<ContactConstraint<R>> rows;
    for (uint32_t i = 0; i < n; ++i) {
        const double* c = contacts + 10 * i;
        uint32_t ia = uint32_t(c[0]), ib = uint32_t(c[1]);
        ContactPoint<R> cp(V3<R>(static_cast<R>(c[2]), static_cast<R>(c[3]), static_cast<R>(c[4])), V3<R>(static_cast<R>(c[5]), static_cast<R>(c[6]), static_cast<R>(c[7])), static_cast<R>(c[8]));
        cp.normal_impulse = static_cast<R>(c[9]);
        rows.push_back(prepare_contact(ia, ib, cp, w.bodies[ia], w.bodies[ib], i, static_cast<R>(inv_dt), w.info));
    }
    solve(w.bodies, rows, static_cast<R>(inv_dt), w.info);
    if (out_rows) get_rows(rows, out_rows);
}

template <class R>
void push_impl(const World<R>& w, double* out) {
    for (size_t i = 0; i < w.bodies.size(); ++i) {
        const Body<R>& b = w.bodies[i];
        out[6 * i + 0] = b.push_linear.x; out[6 * i + 1] = b.push_linear.y; out[6 * i + 2] = b.push_linear.z;
        out[6 * i + 3] = b.push_angular.x; out[6 * i + 4] = b.push_angular.y; out[6 * i + 5] = b.push_angular.z;
    }
}

#define DISPATCH(h, expr)                  \
    do {                                   \
        if ((h)->f64) { auto& w = *(h)->wd; expr; } \
        else { auto& w = *(h)->wf; expr; } \
    } while (0)

}  // namespace

extern "C" {

void* orc_world_new(int f64) {
    Handle* h = new Handle();
    h->f64 = f64;
    if (f64) h->wd.reset(new World<double>());
    else h->wf.reset(new World<float>());
    return h;
}

void orc_world_free(void* p) { delete static_cast<Handle*>(p); }

void orc_world_set_gravity(void* p, double gx, double gy, double gz) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { using R = std::remove_reference_t<decltype(w.gravity.x)>; w.gravity = V3<R>(static_cast<R>(gx), static_cast<R>(gy), static_cast<R>(gz)); });
}

// params: erp2, linear_slop, restitution_threshold, split_impulse, split_threshold,
// split_turn_erp, warmstarting_factor, global_cfm, sor, num_iterations, erp (joints), damping (joints)
void orc_world_set_solver(void* p, const double* s) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        w.info.erp2 = static_cast<R>(s[0]); w.info.linear_slop = static_cast<R>(s[1]); w.info.restitution_velocity_threshold = static_cast<R>(s[2]);
        w.info.split_impulse = s[3] != 0; w.info.split_impulse_penetration_threshold = static_cast<R>(s[4]);
        w.info.split_impulse_turn_erp = static_cast<R>(s[5]); w.info.warmstarting_factor = static_cast<R>(s[6]); w.info.global_cfm = static_cast<R>(s[7]);
        w.info.sor = static_cast<R>(s[8]); w.info.num_iterations = uint32_t(s[9]);
        w.info.erp = static_cast<R>(s[10]); w.info.damping = static_cast<R>(s[11]);
    });
}

void orc_world_set_brute_force(void* p, int on) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { w.brute_force_broadphase = on != 0; });
}

using Tri3 = std::array<uint32_t, 3>;  // (a typedef: the dispatch macro splits on template commas)

// Static triangle mesh: nv vertices (xyz) and nt triangles (3 vertex indices each).
uint32_t orc_world_add_mesh(void* p, const double* v, uint32_t nv, const uint32_t* idx, uint32_t nt) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        std::vector<V3<R>> verts;
        for (uint32_t i = 0; i < nv; ++i)
            verts.push_back(V3<R>(static_cast<R>(v[3 * i]), static_cast<R>(v[3 * i + 1]), static_cast<R>(v[3 * i + 2])));
        std::vector<Tri3> tris(nt);
        for (uint32_t t = 0; t < nt; ++t)
            for (int k = 0; k < 3; ++k) tris[t][k] = idx[3 * t + k];
        w.shapes.push_back(Shape<R>::triangle_mesh(verts, tris));
        r = uint32_t(w.shapes.size() - 1);
    });
    return r;
}

// Heightfield (heightfield.rs:84-140): width x depth heights, cell size xyz, option bits.
uint32_t orc_world_add_heightfield(void* p, const double* heights, uint32_t width, uint32_t depth, const double* cell,
                                   uint32_t options) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        std::vector<R> hv(size_t(width) * depth);
        for (size_t i = 0; i < hv.size(); ++i) hv[i] = static_cast<R>(heights[i]);
        V3<R> c(static_cast<R>(cell[0]), static_cast<R>(cell[1]), static_cast<R>(cell[2]));
        w.shapes.push_back(Shape<R>::heightfield(hv, width, depth, c, options));
        r = uint32_t(w.shapes.size() - 1);
    });
    return r;
}

// The triangles of a mesh shape (after any heightfield construction): vertices and indices.
uint32_t orc_mesh_counts(void* p, uint32_t s, uint32_t* nv) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t nt = 0;
    DISPATCH(h, {
        const auto& m = *w.shapes[s].mesh;
        *nv = uint32_t(m.vertices.size());
        nt = uint32_t(m.indices.size());
    });
    return nt;
}

void orc_mesh_data(void* p, uint32_t s, double* v, uint32_t* idx) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        const auto& m = *w.shapes[s].mesh;
        for (size_t i = 0; i < m.vertices.size(); ++i) {
            v[3 * i] = m.vertices[i].x; v[3 * i + 1] = m.vertices[i].y; v[3 * i + 2] = m.vertices[i].z;
        }
        for (size_t t = 0; t < m.indices.size(); ++t)
            for (int k = 0; k < 3; ++k) idx[3 * t + k] = m.indices[t][k];
    });
}

// BVH query of a mesh shape (bvh.rs:45-66): candidate triangles in walk order; returns the count.
uint32_t orc_mesh_query(void* p, uint32_t s, const double* box6, uint32_t* out, uint32_t cap) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t n = 0;
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        Aabb<R> q(V3<R>(static_cast<R>(box6[0]), static_cast<R>(box6[1]), static_cast<R>(box6[2])),
                  V3<R>(static_cast<R>(box6[3]), static_cast<R>(box6[4]), static_cast<R>(box6[5])));
        std::vector<uint32_t> c;
        w.shapes[s].mesh->triangles_in_aabb(q, c);
        n = uint32_t(c.size());
        for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = c[i];
    });
    return n;
}

uint32_t orc_world_add_shape(void* p, uint32_t type, const double* params, const double* pts, uint32_t npts) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        w.shapes.push_back(make_shape<R>(type, params, pts, npts));
        r = uint32_t(w.shapes.size() - 1);
    });
    return r;
}

double orc_shape_threshold(void* p, uint32_t s) {
    Handle* h = static_cast<Handle*>(p);
    double r = 0;
    DISPATCH(h, { r = double(w.shapes[s].contact_breaking_threshold()); });
    return r;
}

void orc_shape_world_aabb(void* p, uint32_t s, const double* pose, double* out6) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        Aabb<R> a = w.shapes[s].world_aabb(v_of<R>(pose), q_of<R>(pose));
        out6[0] = a.min.x; out6[1] = a.min.y; out6[2] = a.min.z; out6[3] = a.max.x; out6[4] = a.max.y; out6[5] = a.max.z;
    });
}

void orc_shape_inertia(void* p, uint32_t s, double mass, double* out3) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        V3<R> in = w.shapes[s].local_inertia(static_cast<R>(mass));
        out3[0] = in.x; out3[1] = in.y; out3[2] = in.z;
    });
}

uint32_t orc_world_add_body(void* p, const double* desc) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = add_body(w, desc); });
    return r;
}

uint32_t orc_world_num_bodies(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = uint32_t(w.bodies.size()); });
    return r;
}

void orc_world_step(void* p, double dt) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        w.step(static_cast<R>(dt));
    });
}

uint32_t orc_world_step_fixed(void* p, double dt, uint32_t max_sub_steps, double fixed_dt) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t num = 0;
    DISPATCH(h, { num = step_fixed_impl(w, h->accumulator, dt, max_sub_steps, fixed_dt); });
    return num;
}

void orc_world_get_state(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { get_state(w, out); });
}

void orc_world_set_state(void* p, const double* in) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { set_state(w, in); });
}

// body.rs:883-886 apply_force (wakes the body, as activate() at body.rs:562-574) and the
// torque accumulator beside it; the step clears both (world/step.rs:206, clear_forces).
void orc_world_apply_force(void* p, uint32_t i, const double* f, const double* t) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        auto& b = w.bodies.at(i);
        if (!b.is_static && b.activation != ACT_DISABLE_SIMULATION && b.activation != ACT_DISABLE_DEACTIVATION) {
            b.activation = ACT_ACTIVE;
            b.deactivation_time = R(0);
        }
        b.force += V3<R>(static_cast<R>(f[0]), static_cast<R>(f[1]), static_cast<R>(f[2]));
        b.torque += V3<R>(static_cast<R>(t[0]), static_cast<R>(t[1]), static_cast<R>(t[2]));
    });
}

// The body's public collision_group / collision_mask fields (body.rs:325-328), written
// between steps; the broad phase's pair test reads them every step.
void orc_world_set_filter(void* p, uint32_t i, uint32_t group, uint32_t mask) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        auto& b = w.bodies.at(i);
        b.group = uint16_t(group);
        b.mask = uint16_t(mask);
    });
}

void orc_world_get_push(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { push_impl(w, out); });
}

uint32_t orc_world_num_pairs(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = uint32_t(w.last_pairs.size()); });
    return r;
}

void orc_world_get_pairs(void* p, uint32_t* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        for (size_t i = 0; i < w.last_pairs.size(); ++i) { out[2 * i] = w.last_pairs[i].first; out[2 * i + 1] = w.last_pairs[i].second; }
    });
}

uint32_t orc_world_num_rows(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = uint32_t(w.last_rows.size()); });
    return r;
}

// which: 0 = after the solve, 1 = as prepared (before the solve)
void orc_world_get_rows(void* p, int which, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { get_rows(which ? w.last_rows_pre : w.last_rows, out); });
}

uint32_t orc_world_narrowphase_calls(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = w.last_narrowphase_calls; });
    return r;
}

uint32_t orc_world_num_manifolds(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = uint32_t(w.cache.size()); });
    return r;
}

// RigidBody::ccd (body.rs:680-692): motion threshold and swept-sphere radius of body i.
void orc_world_set_ccd(void* p, uint32_t i, double threshold, double radius) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        w.bodies[i].ccd_threshold = static_cast<R>(threshold);
        w.bodies[i].ccd_radius = static_cast<R>(radius);
    });
}

// CCD clamp fraction per body of the last step (1: not clamped).
void orc_world_ccd_clamps(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { for (size_t k = 0; k < w.last_ccd_clamps.size(); ++k) out[k] = w.last_ccd_clamps[k]; });
}

void orc_world_set_solve_order(void* p, const uint64_t* keys, uint32_t n) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { w.solve_order.assign(keys, keys + n); });
}

// Joint descriptor layout (doubles), shared with tests/oracle_api.py and the GPU's
// bgpu_joint_desc: 0 kind, 1 body_a, 2 body_b, 3 flags (1 disable collisions, 2 disabled,
// 4 angular only, 8 limit, 16 motor, 32 ERP override), 4-15 frame A (origin, basis columns
// x y z), 16-27 frame B, 28 erp, 29 impulse clamp, 30 limit low, 31 limit high,
// 32 softness, 33 bias factor, 34 relaxation, 35 motor target velocity, 36 motor max impulse,
// 37 gear ratio; slider: 38 lower / 39 upper linear limit, 40 lower / 41 upper angular limit,
// 42 softness lim lin, 43 softness lim ang, 44 damping lim lin, 45 damping lim ang, 46 softness
// ortho lin, 47 softness ortho ang, 48 / 49 linear motor target velocity / max force, 50 / 51
// angular motor (flags 64 linear motor, 128 angular motor, 256 linear reference frame B);
// spring 2: 52 rotate order, then per axis (0-2 linear, 3-5 angular) 14 values from 53 + 14 i:
// lower, upper, bounce, stop erp, stop cfm, motor erp, motor cfm, target velocity, max motor
// force, servo target, stiffness, damping, equilibrium point, axis flags (S2_*);
// cone twist: 137 swing span 1, 138 swing span 2, 139 twist span, 140 limit softness, 141 bias
// factor, 142 relaxation factor, 143-146 motor target (x y z w, constraint space), 147 motor max
// impulse (flag 512: motor on).
constexpr int JDESC = 148;

uint32_t orc_world_add_joint(void* p, const double* d) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, {
        using R = std::remove_reference_t<decltype(w.gravity.x)>;
        Joint<R> jt;
        auto v3 = [&](int o) { return V3<R>(static_cast<R>(d[o]), static_cast<R>(d[o + 1]), static_cast<R>(d[o + 2])); };
        jt.kind = uint32_t(d[0]);
        jt.body_a = uint32_t(d[1]);
        jt.body_b = uint32_t(d[2]);
        uint32_t f = uint32_t(d[3]);
        jt.disable_collisions = (f & 1u) != 0;
        jt.enabled = (f & 2u) == 0;
        jt.angular_only = (f & 4u) != 0;
        jt.has_limit = (f & 8u) != 0;
        jt.has_motor = (f & 16u) != 0;
        jt.has_erp = (f & 32u) != 0;
        jt.frame_a.origin = v3(4);
        jt.frame_a.basis = M3<R>(v3(7), v3(10), v3(13));
        jt.frame_b.origin = v3(16);
        jt.frame_b.basis = M3<R>(v3(19), v3(22), v3(25));
        jt.erp = static_cast<R>(d[28]);
        jt.impulse_clamp = static_cast<R>(d[29]);
        jt.limit.low = static_cast<R>(d[30]);
        jt.limit.high = static_cast<R>(d[31]);
        jt.limit.softness = static_cast<R>(d[32]);
        jt.limit.bias_factor = static_cast<R>(d[33]);
        jt.limit.relaxation = static_cast<R>(d[34]);
        jt.motor_target = static_cast<R>(d[35]);
        jt.motor_max = static_cast<R>(d[36]);
        jt.gear_ratio = static_cast<R>(d[37]);
        jt.lower_lin = static_cast<R>(d[38]); jt.upper_lin = static_cast<R>(d[39]);
        jt.lower_ang = static_cast<R>(d[40]); jt.upper_ang = static_cast<R>(d[41]);
        jt.softness_lim_lin = static_cast<R>(d[42]); jt.softness_lim_ang = static_cast<R>(d[43]);
        jt.damping_lim_lin = static_cast<R>(d[44]); jt.damping_lim_ang = static_cast<R>(d[45]);
        jt.softness_ortho_lin = static_cast<R>(d[46]); jt.softness_ortho_ang = static_cast<R>(d[47]);
        jt.lin_motor_target = static_cast<R>(d[48]); jt.lin_motor_max = static_cast<R>(d[49]);
        jt.ang_motor_target = static_cast<R>(d[50]); jt.ang_motor_max = static_cast<R>(d[51]);
        jt.has_lin_motor = (f & 64u) != 0;
        jt.has_ang_motor = (f & 128u) != 0;
        jt.use_frame_a = (f & 256u) == 0;
        jt.rotate_order = uint32_t(d[52]);
        jt.ct_span1 = static_cast<R>(d[137]); jt.ct_span2 = static_cast<R>(d[138]); jt.ct_twist = static_cast<R>(d[139]);
        jt.ct_softness = static_cast<R>(d[140]); jt.ct_bias = static_cast<R>(d[141]); jt.ct_relax = static_cast<R>(d[142]);
        jt.ct_target = Quat<R>(static_cast<R>(d[143]), static_cast<R>(d[144]), static_cast<R>(d[145]), static_cast<R>(d[146]));
        jt.ct_max_impulse = static_cast<R>(d[147]);
        jt.ct_has_motor = (f & 512u) != 0;
        for (int i = 0; i < 6; ++i) {
            const double* x = d + 53 + 14 * i;
            Spring2Axis<R>& m = jt.s2[i];
            m.lower = static_cast<R>(x[0]); m.upper = static_cast<R>(x[1]); m.bounce = static_cast<R>(x[2]);
            m.stop_erp = static_cast<R>(x[3]); m.stop_cfm = static_cast<R>(x[4]);
            m.motor_erp = static_cast<R>(x[5]); m.motor_cfm = static_cast<R>(x[6]);
            m.target_velocity = static_cast<R>(x[7]); m.max_motor_force = static_cast<R>(x[8]);
            m.servo_target = static_cast<R>(x[9]); m.stiffness = static_cast<R>(x[10]);
            m.damping = static_cast<R>(x[11]); m.equilibrium = static_cast<R>(x[12]);
            m.flags = uint32_t(x[13]);
        }
        w.joints.push_back(jt);
        r = uint32_t(w.joints.size() - 1);
    });
    return r;
}

// Constraint::set_enabled / set_disable_collisions between steps (constraint.rs:637-652): flag bit 1
// suppresses the pair's collisions, bit 2 disables the joint's rows.
void orc_world_set_joint_flags(void* p, uint32_t j, uint32_t flags) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        auto& jt = w.joints.at(j);
        jt.disable_collisions = (flags & 1u) != 0;
        jt.enabled = (flags & 2u) == 0;
    });
}

void orc_world_set_joint_order(void* p, const uint32_t* ids, uint32_t n) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { w.joint_order.assign(ids, ids + n); });
}

// Per joint: the hinge angle (hinge) or the angular position (slider); 0 for other kinds.
void orc_world_joint_angles(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        for (size_t k = 0; k < w.joints.size(); ++k)
            out[k] = w.joints[k].kind == JOINT_SLIDER      ? w.joints[k].ang_pos
                     : w.joints[k].kind == JOINT_CONETWIST ? w.joints[k].ct_twist_angle
                                                           : w.joints[k].hinge_angle;
    });
}

// Per joint: the slider's linear position (0 for other kinds).
void orc_world_joint_positions(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { for (size_t k = 0; k < w.joints.size(); ++k) out[k] = w.joints[k].lin_pos; });
}

// Per joint, 8 doubles of the spring-2 step state: Euler angles (3), pivot offset in A's frame
// (3), fact_a, has_static_body.
void orc_world_joint_spring2_state(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        for (size_t k = 0; k < w.joints.size(); ++k) {
            const auto& jt = w.joints[k];
            double* o = out + 8 * k;
            for (int i = 0; i < 3; ++i) { o[i] = jt.s2_euler[i]; o[3 + i] = jt.s2_diff[i]; }
            o[6] = jt.fact_a; o[7] = jt.has_static_body ? 1.0 : 0.0;
        }
    });
}

// generic6dof_spring2.rs:1164-1233 on two frames: Euler angles (3) then the three axes (9).
void orc_spring2_angle_info(int f64, const double* tr_a, const double* tr_b, uint32_t order, double* out) {
    auto run = [&](auto tag) {
        using R = decltype(tag);
        auto m3 = [](const double* c) {
            return M3<R>(V3<R>(R(c[0]), R(c[1]), R(c[2])), V3<R>(R(c[3]), R(c[4]), R(c[5])),
                         V3<R>(R(c[6]), R(c[7]), R(c[8])));
        };
        V3<R> euler, axes[3];
        spring2_angle_info(m3(tr_a), m3(tr_b), order, euler, axes);
        for (int i = 0; i < 3; ++i) out[i] = euler[i];
        for (int a = 0; a < 3; ++a)
            for (int i = 0; i < 3; ++i) out[3 + 3 * a + i] = axes[a][i];
    };
    if (f64) run(double(0)); else run(float(0));
}

uint32_t orc_world_num_joint_rows(void* p) {
    Handle* h = static_cast<Handle*>(p);
    uint32_t r = 0;
    DISPATCH(h, { r = uint32_t(w.last_joint_rows.size()); });
    return r;
}

// Joint rows of the last step in solve order, 8 doubles each: joint, body_a, body_b, mass,
// bias, limit kind, accumulated impulse, cfm.
void orc_world_joint_rows(void* p, double* out) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, {
        for (size_t k = 0; k < w.last_joint_rows.size(); ++k) {
            const auto& jr = w.last_joint_rows[k];
            double* o = out + 8 * k;
            o[0] = jr.joint; o[1] = jr.body_a; o[2] = jr.body_b; o[3] = jr.mass; o[4] = jr.bias;
            o[5] = jr.lim; o[6] = jr.impulse; o[7] = jr.cfm;
        }
    });
}

// hinge.rs:60-100: frames (24 doubles: origin + basis columns, for A then B) from pivots and axes.
void orc_hinge_frames(int f64, const double* pa, const double* axa, const double* pb, const double* axb, double* out) {
    auto run = [&](auto tag) {
        using R = decltype(tag);
        JointFrame<R> fa, fb;
        auto v3 = [](const double* x) { return V3<R>(static_cast<R>(x[0]), static_cast<R>(x[1]), static_cast<R>(x[2])); };
        hinge_frames(v3(pa), v3(axa), v3(pb), v3(axb), fa, fb);
        const JointFrame<R>* fr[2] = {&fa, &fb};
        for (int f = 0; f < 2; ++f) {
            const V3<R> cols[4] = {fr[f]->origin, fr[f]->basis.c0, fr[f]->basis.c1, fr[f]->basis.c2};
            for (int c = 0; c < 4; ++c) {
                out[12 * f + 3 * c] = cols[c].x; out[12 * f + 3 * c + 1] = cols[c].y; out[12 * f + 3 * c + 2] = cols[c].z;
            }
        }
    };
    if (f64) run(double(0));
    else run(float(0));
}

void orc_world_stage_seconds(void* p, double* out7) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { for (int k = 0; k < 7; ++k) out7[k] = w.stage_s[k]; });
}

int orc_collide(void* p, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b, const double* seed,
                double* out) {
    Handle* h = static_cast<Handle*>(p);
    int r = 0;
    DISPATCH(h, { r = collide_impl(w, sa, pose_a, sb, pose_b, seed, out); });
    return r;
}

// The generic GJK/EPA path (convex_convex.rs:30) regardless of the shape pair.
int orc_convex_convex(void* p, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b, double* out) {
    Handle* h = static_cast<Handle*>(p);
    int r = 0;
    DISPATCH(h, { r = convex_impl(w, sa, pose_a, sb, pose_b, out); });
    return r;
}

// convex_mesh.rs:160-232 on its own: out = point3, normal3 (toward the centre), penetration.
int orc_sphere_triangle(int f64, const double* center, double radius, double threshold, const double* tri9,
                        double* out7) {
    auto run = [&](auto zero) -> int {
        using R = decltype(zero);
        auto v = [&](const double* d) { return V3<R>(static_cast<R>(d[0]), static_cast<R>(d[1]), static_cast<R>(d[2])); };
        V3<R> pt, n;
        R pen;
        if (!sphere_triangle_contact(v(center), static_cast<R>(radius), static_cast<R>(threshold), v(tri9), v(tri9 + 3),
                                     v(tri9 + 6), pt, n, pen))
            return 0;
        out7[0] = pt.x; out7[1] = pt.y; out7[2] = pt.z;
        out7[3] = n.x; out7[4] = n.y; out7[5] = n.z;
        out7[6] = pen;
        return 1;
    };
    return f64 ? run(0.0) : run(0.0f);
}

int orc_gjk_kind(void* p, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b) {
    Handle* h = static_cast<Handle*>(p);
    int r = 0;
    DISPATCH(h, { r = gjk_kind_impl(w, sa, pose_a, sb, pose_b); });
    return r;
}

int orc_gjk_contact(void* p, uint32_t sa, const double* pose_a, uint32_t sb, const double* pose_b, const double* seed,
                    double threshold, double* out) {
    Handle* h = static_cast<Handle*>(p);
    int r = 0;
    DISPATCH(h, { r = gjk_contact_impl(w, sa, pose_a, sb, pose_b, seed, threshold, out); });
    return r;
}

void orc_solve_contacts(void* p, const double* contacts, uint32_t n, double inv_dt, double* out_rows) {
    Handle* h = static_cast<Handle*>(p);
    DISPATCH(h, { solve_impl(w, contacts, n, inv_dt, out_rows); });
}

// Pairs of an AABB set (n x [min3, max3]); method 0 = brute force, 1 = sweep, 2 = grid.
// Returns the pair count; writes up to cap pairs.
uint64_t orc_pairs(int f64, const double* aabbs, uint32_t n, int method, uint32_t* out, uint64_t cap) {
    std::vector<std::pair<uint32_t, uint32_t>> pr;
    if (f64) pairs_impl<double>(aabbs, n, method, pr);
    else pairs_impl<float>(aabbs, n, method, pr);
    for (size_t i = 0; i < pr.size() && i < cap; ++i) { out[2 * i] = pr[i].first; out[2 * i + 1] = pr[i].second; }
    return pr.size();
}

// ContactManifold::reduce (manifold.rs:80-108) on n points (pos3, normal3, penetration); writes
// the kept points in the same layout and returns their count.
uint32_t orc_manifold_reduce(int f64, const double* pts, uint32_t n, uint32_t keep, double* out) {
    uint32_t k = 0;
    auto run = [&](auto zero) {
        using R = decltype(zero);
        Manifold<R> m;
        for (uint32_t i = 0; i < n; ++i) {
            const double* c = pts + 7 * i;
            m.points.push_back(ContactPoint<R>(V3<R>(static_cast<R>(c[0]), static_cast<R>(c[1]), static_cast<R>(c[2])),
                                               V3<R>(static_cast<R>(c[3]), static_cast<R>(c[4]), static_cast<R>(c[5])),
                                               static_cast<R>(c[6])));
        }
        reduce_manifold(m, keep);
        for (auto& cp : m.points) {
            double* d = out + 7 * k;
            d[0] = cp.position.x; d[1] = cp.position.y; d[2] = cp.position.z;
            d[3] = cp.normal.x; d[4] = cp.normal.y; d[5] = cp.normal.z;
            d[6] = cp.penetration;
            ++k;
        }
    };
    if (f64) run(0.0); else run(0.0f);
    return k;
}

// Persistent manifold handle (float or double).
struct PmHandle { int f64; PersistentManifold<float> f; PersistentManifold<double> d; };

void* orc_pm_new(int f64) { PmHandle* h = new PmHandle(); h->f64 = f64; return h; }
void orc_pm_free(void* p) { delete static_cast<PmHandle*>(p); }

// points: n x (pos3, normal3, penetration)
void orc_pm_capture(void* p, const double* pts, uint32_t n, const double* pose_a, const double* pose_b, double thr) {
    PmHandle* h = static_cast<PmHandle*>(p);
    auto run = [&](auto& pm, auto zero) {
        using R = decltype(zero);
        Manifold<R> m;
        for (uint32_t i = 0; i < n; ++i) {
            const double* c = pts + 7 * i;
            m.points.push_back(ContactPoint<R>(V3<R>(static_cast<R>(c[0]), static_cast<R>(c[1]), static_cast<R>(c[2])), V3<R>(static_cast<R>(c[3]), static_cast<R>(c[4]), static_cast<R>(c[5])), static_cast<R>(c[6])));
        }
        pm.capture(m, v_of<R>(pose_a), q_of<R>(pose_a), v_of<R>(pose_b), q_of<R>(pose_b), static_cast<R>(thr));
    };
    if (h->f64) run(h->d, 0.0); else run(h->f, 0.0f);
}

// out: n x (pos3, normal3, penetration, normal_impulse, lifetime); returns n
uint32_t orc_pm_refresh(void* p, const double* pose_a, const double* pose_b, double* out) {
    PmHandle* h = static_cast<PmHandle*>(p);
    uint32_t n = 0;
    auto run = [&](auto& pm, auto zero) {
        using R = decltype(zero);
        std::vector<ContactPoint<R>> o;
        pm.refresh(v_of<R>(pose_a), q_of<R>(pose_a), v_of<R>(pose_b), q_of<R>(pose_b), o);
        for (auto& cp : o) {
            double* d = out + 9 * n;
            d[0] = cp.position.x; d[1] = cp.position.y; d[2] = cp.position.z;
            d[3] = cp.normal.x; d[4] = cp.normal.y; d[5] = cp.normal.z;
            d[6] = cp.penetration; d[7] = cp.normal_impulse; d[8] = cp.lifetime;
            ++n;
        }
    };
    if (h->f64) run(h->d, 0.0); else run(h->f, 0.0f);
    return n;
}

int orc_pm_needs_redetect(void* p, const double* pose_a, const double* pose_b) {
    PmHandle* h = static_cast<PmHandle*>(p);
    if (h->f64) return h->d.needs_redetect(v_of<double>(pose_a), q_of<double>(pose_a), v_of<double>(pose_b), q_of<double>(pose_b));
    return h->f.needs_redetect(v_of<float>(pose_a), q_of<float>(pose_a), v_of<float>(pose_b), q_of<float>(pose_b));
}

void orc_pm_set_impulse(void* p, uint32_t k, double imp) {
    PmHandle* h = static_cast<PmHandle*>(p);
    if (h->f64) h->d.points[k].normal_impulse = imp; else h->f.points[k].normal_impulse = float(imp);
}

// out: n x (local_a3, local_b3, normal3, penetration, impulse, lifetime)
uint32_t orc_pm_points(void* p, double* out) {
    PmHandle* h = static_cast<PmHandle*>(p);
    uint32_t n = 0;
    auto run = [&](auto& pm) {
        for (auto& q : pm.points) {
            double* d = out + 12 * n;
            d[0] = q.local_a.x; d[1] = q.local_a.y; d[2] = q.local_a.z;
            d[3] = q.local_b.x; d[4] = q.local_b.y; d[5] = q.local_b.z;
            d[6] = q.normal.x; d[7] = q.normal.y; d[8] = q.normal.z;
            d[9] = q.penetration; d[10] = q.normal_impulse; d[11] = q.lifetime;
            ++n;
        }
    };
    if (h->f64) run(h->d); else run(h->f);
    return n;
}

// Pose integration (body.rs:92-137): in = pos3, quat4, linvel3, angvel3; out = pos3, quat4
void orc_interpolate_pose(int f64, const double* in, double dt, double* out) {
    auto run = [&](auto zero) {
        using R = decltype(zero);
        V3<R> np; Quat<R> nq;
        interpolate_pose(V3<R>(static_cast<R>(in[0]), static_cast<R>(in[1]), static_cast<R>(in[2])), Quat<R>(static_cast<R>(in[3]), static_cast<R>(in[4]), static_cast<R>(in[5]), static_cast<R>(in[6])),
                         V3<R>(static_cast<R>(in[7]), static_cast<R>(in[8]), static_cast<R>(in[9])), V3<R>(static_cast<R>(in[10]), static_cast<R>(in[11]), static_cast<R>(in[12])), static_cast<R>(dt), np, nq);
        out[0] = np.x; out[1] = np.y; out[2] = np.z; out[3] = nq.x; out[4] = nq.y; out[5] = nq.z; out[6] = nq.w;
    };
    if (f64) run(0.0); else run(0.0f);
}

}  // extern "C"
