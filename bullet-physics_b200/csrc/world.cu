// Host side of the rigid-body world: device memory ownership, the step
// orchestration (step.rs:281-1287 order: integrate velocities + AABBs, broad
// phase, islands, pair pass, solve, manifold writeback/prune, integrate
// positions), and the C ABI declared in include/bgpu.h.
#include <algorithm>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "../../include/bgpu.h"
#include "bgpu_kernels.cuh"

namespace bgpu {

void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw CudaError{e, std::string(where) + ": " + cudaGetErrorString(e)};
}

namespace {

thread_local std::string g_last_error;

struct InvalidArg {
    std::string what;
};

}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {

const float CONTACT_BREAKING_THRESHOLD = 0.02f;  // manifold.rs:8

// shapes/mod.rs:388-392 (float arithmetic, host)
float contact_breaking_threshold(const float lmin[3], const float lmax[3]) {
    float dx = lmax[0] - lmin[0], dy = lmax[1] - lmin[1], dz = lmax[2] - lmin[2];
    float len = std::sqrt(dx * dx + dy * dy + dz * dz);
    float cx = (lmin[0] + lmax[0]) * 0.5f, cy = (lmin[1] + lmax[1]) * 0.5f, cz = (lmin[2] + lmax[2]) * 0.5f;
    float clen = std::sqrt(cx * cx + cy * cy + cz * cz);
    float disc = len * 0.5f + clen;
    return disc * CONTACT_BREAKING_THRESHOLD;
}

// Diagonal local inertia (shapes/mod.rs:396-412), float host arithmetic.
void local_inertia(const Shape& s, float mass, float out[3]) {
    switch (s.type) {
        case SHAPE_SPHERE: {
            float v = 0.4f * mass * s.p0 * s.p0;
            out[0] = out[1] = out[2] = v;
            return;
        }
        case SHAPE_BOX: {
            float m = mass / 3.0f;
            out[0] = m * (s.p1 * s.p1 + s.p2 * s.p2);
            out[1] = m * (s.p0 * s.p0 + s.p2 * s.p2);
            out[2] = m * (s.p0 * s.p0 + s.p1 * s.p1);
            return;
        }
        case SHAPE_CAPSULE: {
            const float PI = 3.14159265358979323846f;
            float h = 2.0f * s.p1;
            float r2 = s.p0 * s.p0;
            float h2 = h * h;
            float v_cyl = PI * r2 * h;
            float v_sph = 4.0f / 3.0f * PI * r2 * s.p0;
            float v = v_cyl + v_sph;
            float m_cyl = mass * v_cyl / v;
            float m_sph = mass * v_sph / v;
            float ixx = m_cyl * (3.0f * r2 + h2) / 12.0f + m_sph * (0.4f * r2 + 0.25f * h2);
            float iyy = m_cyl * r2 / 2.0f + m_sph * 0.4f * r2;
            out[0] = ixx; out[1] = iyy; out[2] = ixx;
            return;
        }
        case SHAPE_HULL: {
            float hx = (s.lmax[0] - s.lmin[0]) * 0.5f, hy = (s.lmax[1] - s.lmin[1]) * 0.5f,
                  hz = (s.lmax[2] - s.lmin[2]) * 0.5f;
            float m = mass / 3.0f;
            out[0] = m * (hy * hy + hz * hz);
            out[1] = m * (hx * hx + hz * hz);
            out[2] = m * (hx * hx + hy * hy);
            return;
        }
        default:
            out[0] = out[1] = out[2] = 0.0f;
    }
}

struct HostStats {  // pinned, written by async copies at the end of a step
    uint32_t scalars[16];
    uint32_t status;
    uint32_t cache_count;
    uint32_t simulate;
};

}  // namespace

// One forward step recorded for the adjoint (the reverse solve's inputs).
struct StepRecord {
    uint32_t ncol = 0, iters = 0, slots = 0, npairs = 0, nold = 0;
    DevBuf<uint4> recs;                  // batch slot records (colour order)
    DevBuf<float4> tab, sweeps;          // velocity contact table, per-sweep records
    DevBuf<uint32_t> row_src, merge_pos; // warm-start sources, merged cache positions
    DevBuf<uint32_t> off, end;           // colour batch starts / ends (per-world solver: its world records)
    DevBuf<uint8_t> flags;               // RF_* per body
    bool per_world = false;              // recorded from the per-world solver
    AdjStep view() const {
        return AdjStep{recs.p, off.p, end.p, ncol, iters, tab.p, sweeps.p, merge_pos.p, row_src.p};
    }
};

inline float __uint_as_float_host(uint32_t u) {
    float f;
    std::memcpy(&f, &u, sizeof(f));
    return f;
}

struct World {
    cudaStream_t stream = nullptr;
    SolverParams info{};
    float gravity[3] = {0.0f, -9.81f, 0.0f};
    // shapes
    std::vector<Shape> shapes_h;
    std::vector<float4> hull_h;
    DevBuf<Shape> shapes_d;
    DevBuf<float4> hull_d;
    bool shapes_dirty = false;
    // bodies
    uint32_t n = 0, cap = 0;
    DevBuf<float4> pos, quat, linvel, angvel, inv_inertia, grav, force, torque, material, sleep, aabb_min, aabb_max,
        pred, iw, push_lin, push_ang;
    DevBuf<uint4> info_d;
    DevBuf<float> settled;
    std::vector<uint32_t> unbounded;  // plane and mesh bodies (kept out of the BVH)
    // batched worlds: world k owns bodies [world_off_h[k], world_off_h[k + 1])
    bool batch = false;
    std::vector<uint32_t> world_off_h{0u};
    DevBuf<uint32_t> world_off_d, world_of_d;
    DevBuf<uint32_t> world_sim;  // [0, W) simulate, [W, 2W) prev_simulate, per world
    // per-world solver of a batch (k_solver.cu): its launch plan, chosen by bgpu_batch_autotune
    // (threads per CTA, largest world solved by one warp), and the per-world batch records
    WorldPlan wplan;
    uint32_t wplan_block = 128, wplan_tau = 64;  // 0 threads: the global (all-worlds) solver
    DevBuf<uint32_t> wcol;
    DevBuf<uint32_t> plain_off_d;    // a plain world's {0, n}, for the per-world solver
    static constexpr uint32_t PLAIN_WORLD_SOLVER_MAX_BODIES = 1024;
    static constexpr uint32_t PLAIN_WORLD_SOLVER_THREADS = 512;
    bool last_world_solver = false;  // the last step ran the per-world solver
    float tuned_ms = 0.0f, tuned_global_ms = 0.0f;
    uint32_t tuned_candidates = 0;
    // step machinery
    Broadphase bp;
    Islands islands;
    PairData pd;
    Manifolds cache[2];
    int cur = 0;
    DevBuf<uint64_t> pairs;
    uint32_t npairs = 0;
    DevBuf<uint32_t> flags;  // [0] status
    HostStats* hs = nullptr;
    bool timing = false;
    cudaEvent_t ev[2][10] = {};  // two event sets: the step being enqueued and the previous one
    int ev_cur = 0;
    bool ev_pending[2] = {false, false};
    bgpu_step_stats last{};
    bool stats_pending = false;
    float accumulator = 0.0f;  // step_simulation_fixed's m_localTime
    DevBuf<float4> force_keep;   // a fixed-step call's applied forces, kept for its later substeps
    int solved_standalone = 0;  // 1 after bgpu_solve_contacts (read_contacts reports its groups)
    uint32_t standalone_groups = 0;
    DevBuf<uint64_t> standalone_keys;
    uint64_t step_count = 0;  // steps taken (seeded vs full colouring)
    static constexpr uint64_t RECOLOUR_PERIOD = 64;
    // adjoint recording: the step being recorded (null otherwise) and the pair pass's scratch
    StepRecord* rec_step = nullptr;
    DevBuf<float> host_io;  // device staging for the caller-layout force / pose buffers
    DevBuf<uint8_t> rec_pt_src;
    DevBuf<uint32_t> rec_pair_old;
    // joints: descriptors by id, solve order (joint colour by colour), per-step rows
    std::vector<bgpu_joint_desc> joints_h;
    std::vector<uint32_t> joint_order_h, joint_coff_h;
    DevBuf<float4> joint_desc_d, joint_rows_d;
    DevBuf<uint32_t> joint_order_d, joint_coff_d, joint_count_d;
    DevBuf<float> joint_angle_d, joint_pos_d;
    // spring-2 joints: descriptors by spring-2 index, the index of each joint id (-1: other
    // kinds), axis tables and step state on the device; every slot's first row (slot order)
    std::vector<bgpu_spring2_desc> s2_h;
    std::vector<int32_t> joint_s2_h;
    std::vector<uint32_t> joint_row_off_h;
    DevBuf<float4> joint_aux_d, joint_s2_state_d;
    DevBuf<uint32_t> joint_row_off_d;
    // CCD (RigidBody::ccd): per-body motion threshold and swept-sphere radius; the bodies with both
    // positive form the list the clamp kernels walk, with one clamp fraction per entry
    std::vector<float> ccd_thr_h, ccd_rad_h;
    std::vector<uint32_t> ccd_ids_h;
    DevBuf<uint32_t> ccd_ids_d;
    DevBuf<float2> ccd_par_d;
    DevBuf<float> ccd_clamp_d;
    uint32_t nccd = 0;
    DevBuf<uint64_t> suppressed_d;  // sorted keys of the pairs a joint keeps from colliding
    uint32_t nsuppressed = 0;

    World() {
        check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check_cuda(cudaMallocHost(&hs, sizeof(HostStats)), "cudaMallocHost");
        std::memset(hs, 0, sizeof(HostStats));
        flags.reserve(4);
        check_cuda(cudaMemsetAsync(flags.p, 0, 4 * sizeof(uint32_t), stream), "memset");
        world_sim.reserve(2);
        check_cuda(cudaMemsetAsync(world_sim.p, 0, 2 * sizeof(uint32_t), stream), "memset");
        cache[0].init();
        cache[1].init();
        check_cuda(cudaMemsetAsync(cache[0].count_dev, 0, sizeof(uint32_t), stream), "memset");
        check_cuda(cudaMemsetAsync(cache[1].count_dev, 0, sizeof(uint32_t), stream), "memset");
        pd.scalars.reserve(16);
        for (auto& set : ev)
            for (auto& e : set) check_cuda(cudaEventCreate(&e), "event");
    }
    ~World() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& set : ev)
            for (auto& e : set) if (e) cudaEventDestroy(e);
        if (hs) cudaFreeHost(hs);
        if (stream) cudaStreamDestroy(stream);
    }

    BodyDev body_dev() {
        return BodyDev{pos.p, quat.p, linvel.p, angvel.p, inv_inertia.p, grav.p, force.p, torque.p, material.p,
                       sleep.p, info_d.p, aabb_min.p, aabb_max.p, pred.p, settled.p, iw.p, push_lin.p, push_ang.p,
                       rec_step ? rec_step->flags.p : nullptr};
    }
    bool has_mesh = false;  // some shape is a triangle mesh
    WorldView view() { return WorldView{body_dev(), shapes_d.p, hull_d.p, n, has_mesh}; }

    void sync_shapes() {
        if (!shapes_dirty) return;
        shapes_d.reserve(shapes_h.size() + 1);
        check_cuda(cudaMemcpyAsync(shapes_d.p, shapes_h.data(), shapes_h.size() * sizeof(Shape), cudaMemcpyHostToDevice,
                                   stream), "upload shapes");
        hull_d.reserve(hull_h.size() + 1);
        if (!hull_h.empty())
            check_cuda(cudaMemcpyAsync(hull_d.p, hull_h.data(), hull_h.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                       stream), "upload hull");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        shapes_dirty = false;
    }

    uint32_t add_shape(uint32_t type, const float* params, const float* pts, uint32_t npts) {
        Shape s;
        std::memset(&s, 0, sizeof(s));
        s.type = type;
        switch (type) {
            case SHAPE_SPHERE:
                if (!params || !(params[0] > 0.0f)) throw InvalidArg{"sphere radius must be > 0"};
                s.p0 = params[0];
                s.margin = s.p0;
                for (int k = 0; k < 3; ++k) { s.lmin[k] = -s.p0; s.lmax[k] = s.p0; }
                break;
            case SHAPE_BOX:
                if (!params || !(params[0] > 0.0f) || !(params[1] > 0.0f) || !(params[2] > 0.0f))
                    throw InvalidArg{"box half extents must be > 0"};
                s.p0 = params[0]; s.p1 = params[1]; s.p2 = params[2];
                s.margin = 0.04f;
                s.lmin[0] = -s.p0; s.lmin[1] = -s.p1; s.lmin[2] = -s.p2;
                s.lmax[0] = s.p0; s.lmax[1] = s.p1; s.lmax[2] = s.p2;
                break;
            case SHAPE_CAPSULE:
                if (!params || !(params[0] > 0.0f) || !(params[1] >= 0.0f))
                    throw InvalidArg{"capsule radius must be > 0 and half height >= 0"};
                s.p0 = params[0]; s.p1 = params[1];
                s.margin = s.p0;
                s.lmin[0] = -s.p0; s.lmin[1] = -(s.p1 + s.p0); s.lmin[2] = -s.p0;
                s.lmax[0] = s.p0; s.lmax[1] = s.p1 + s.p0; s.lmax[2] = s.p0;
                break;
            case SHAPE_HULL: {
                if (!pts || npts == 0) throw InvalidArg{"hull needs at least one point"};
                s.hull_off = uint32_t(hull_h.size());
                s.hull_cnt = npts;
                s.margin = 0.0f;
                for (int k = 0; k < 3; ++k) { s.lmin[k] = INFINITY; s.lmax[k] = -INFINITY; }
                for (uint32_t i = 0; i < npts; ++i) {
                    hull_h.push_back(make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], 0.0f));
                    for (int k = 0; k < 3; ++k) {
                        s.lmin[k] = std::min(s.lmin[k], pts[3 * i + k]);
                        s.lmax[k] = std::max(s.lmax[k], pts[3 * i + k]);
                    }
                }
                break;
            }
            case SHAPE_PLANE: {
                if (!params) throw InvalidArg{"plane needs a normal and a constant"};
                float nx = params[0], ny = params[1], nz = params[2];
                float l = std::sqrt(nx * nx + ny * ny + nz * nz);
                if (!(l > 0.0f)) throw InvalidArg{"plane normal must be nonzero"};
                s.p0 = nx / l; s.p1 = ny / l; s.p2 = nz / l; s.p3 = params[3];
                s.margin = 0.0f;
                for (int k = 0; k < 3; ++k) { s.lmin[k] = -1e30f; s.lmax[k] = 1e30f; }
                break;
            }
            default:
                throw InvalidArg{"unknown shape type"};
        }
        s.cbt = contact_breaking_threshold(s.lmin, s.lmax);
        shapes_h.push_back(s);
        shapes_dirty = true;
        return uint32_t(shapes_h.size() - 1);
    }

    // A static triangle mesh (triangle_mesh.rs:59-123) with the BVH of bvh.rs:36-206: nodes in
    // pre-order, longest-axis median split of the triangle centres (a stable sort on the
    // centre coordinate), at most four triangles per leaf. Nodes and triangles go to the hull
    // array in the layout bgpu_shapes.cuh describes.
    uint32_t add_mesh(const float* v, uint32_t nv, const uint32_t* idx, uint32_t nt) {
        if (!v || !idx || nv == 0 || nt == 0) throw InvalidArg{"a triangle mesh needs vertices and triangles"};
        for (uint64_t k = 0; k < uint64_t(nt) * 3; ++k)
            if (idx[k] >= nv) throw InvalidArg{"triangle index out of range"};
        struct F3 { float x, y, z; };
        auto vert = [&](uint32_t t, int c) { const float* p = v + 3 * size_t(idx[3 * size_t(t) + c]); return F3{p[0], p[1], p[2]}; };
        std::vector<uint32_t> order(nt);
        for (uint32_t t = 0; t < nt; ++t) order[t] = t;
        struct Node { float mn[3], mx[3]; uint32_t a, b; };
        std::vector<Node> nodes;
        auto center = [&](uint32_t t, int axis) {  // bvh.rs:248-251: (a + b + c) * (1 / 3)
            F3 a = vert(t, 0), b = vert(t, 1), c = vert(t, 2);
            const float third = 1.0f / 3.0f;
            float s3[3] = {(a.x + b.x + c.x) * third, (a.y + b.y + c.y) * third, (a.z + b.z + c.z) * third};
            return s3[axis];
        };
        std::function<uint32_t(uint32_t, uint32_t)> build = [&](uint32_t start, uint32_t count) -> uint32_t {
            Node nd;
            bool have = false;
            for (uint32_t k = start; k < start + count; ++k)  // bvh.rs:210-225
                for (int c = 0; c < 3; ++c) {
                    F3 p = vert(order[k], c);
                    float q[3] = {p.x, p.y, p.z};
                    for (int d = 0; d < 3; ++d) {
                        nd.mn[d] = have ? std::min(nd.mn[d], q[d]) : q[d];
                        nd.mx[d] = have ? std::max(nd.mx[d], q[d]) : q[d];
                    }
                    have = true;
                }
            nd.a = start | MESH_LEAF;
            nd.b = count;
            const uint32_t index = uint32_t(nodes.size());
            nodes.push_back(nd);
            if (count <= 4) return index;
            float e[3];
            for (int d = 0; d < 3; ++d) e[d] = (nd.mx[d] - nd.mn[d]) * 0.5f;
            int axis = 0;  // bvh.rs:255-268: first strict maximum
            float m = e[0];
            if (e[1] > m) { axis = 1; m = e[1]; }
            if (e[2] > m) axis = 2;
            std::stable_sort(order.begin() + start, order.begin() + start + count,
                             [&](uint32_t x, uint32_t y) { return center(x, axis) < center(y, axis); });
            const uint32_t mid = count / 2;
            const uint32_t left = build(start, mid);
            const uint32_t right = build(start + mid, count - mid);
            nodes[index].a = left;
            nodes[index].b = right;
            return index;
        };
        build(0, nt);
        if (nodes.size() >= MESH_LEAF || nt >= MESH_LEAF) throw InvalidArg{"mesh too large"};
        Shape s;
        std::memset(&s, 0, sizeof(s));
        s.type = SHAPE_MESH;
        s.hull_off = uint32_t(hull_h.size());
        s.hull_cnt = uint32_t(nodes.size());
        for (const Node& nd : nodes) {
            float fa, fb;
            std::memcpy(&fa, &nd.a, 4);
            std::memcpy(&fb, &nd.b, 4);
            hull_h.push_back(make_float4(nd.mn[0], nd.mn[1], nd.mn[2], fa));
            hull_h.push_back(make_float4(nd.mx[0], nd.mx[1], nd.mx[2], fb));
        }
        const uint32_t tri_base = uint32_t(hull_h.size());
        for (uint32_t k = 0; k < nt; ++k) {
            const uint32_t t = order[k];
            float ft;
            std::memcpy(&ft, &t, 4);
            for (int c = 0; c < 3; ++c) {
                F3 p = vert(t, c);
                hull_h.push_back(make_float4(p.x, p.y, p.z, c == 0 ? ft : 0.0f));
            }
        }
        std::memcpy(&s.p0, &tri_base, 4);
        std::memcpy(&s.p1, &nt, 4);
        s.margin = 0.0f;
        for (int d = 0; d < 3; ++d) {  // triangle_mesh.rs:98-112 local bounds (the root box)
            s.lmin[d] = nodes[0].mn[d];
            s.lmax[d] = nodes[0].mx[d];
        }
        s.cbt = contact_breaking_threshold(s.lmin, s.lmax);
        shapes_h.push_back(s);
        shapes_dirty = true;
        has_mesh = true;
        return uint32_t(shapes_h.size() - 1);
    }

    // heightfield.rs:84-140: a width x depth row-major grid centred on the origin, heights offset
    // by the min/max midpoint, two triangles per cell (diagonal and winding by the option bits:
    // 1 flip quad edges, 2 diamond, 4 zigzag, 8 flip winding; up axis in bits 4-5: 0 Y, 1 X, 2 Z).
    uint32_t add_heightfield(const float* h, uint32_t width, uint32_t depth, const float* cell, uint32_t options) {
        if (!h || !cell || width < 2 || depth < 2) throw InvalidArg{"a heightfield needs at least 2 x 2 heights"};
        if (uint64_t(width) * depth > (1ull << 26)) throw InvalidArg{"heightfield too large"};
        float mn = INFINITY, mx = -INFINITY;
        for (size_t i = 0; i < size_t(width) * depth; ++i) { mn = std::min(mn, h[i]); mx = std::max(mx, h[i]); }
        const float mid = (mn + mx) * 0.5f;
        const uint32_t up = (options >> 4) & 3u;
        if (up == 3) throw InvalidArg{"heightfield up axis must be 0 (Y), 1 (X) or 2 (Z)"};
        std::vector<float> v;
        v.reserve(size_t(width) * depth * 3);
        for (uint32_t y = 0; y < depth; ++y)
            for (uint32_t x = 0; x < width; ++x) {
                const float hh = h[size_t(y) * width + x] - mid;
                const float u = (float(x) - float(width - 1) * 0.5f) * cell[0];
                const float w = (float(y) - float(depth - 1) * 0.5f) * cell[2];
                const float p[3] = {up == 1 ? hh : u, up == 1 ? u : (up == 2 ? w : hh), up == 2 ? hh : w};
                v.insert(v.end(), p, p + 3);
            }
        const bool flip_edges = options & 1u, diamond = options & 2u, zigzag = options & 4u, flip_wind = options & 8u;
        std::vector<uint32_t> idx;
        auto tri = [&](uint32_t a, uint32_t b, uint32_t c) {
            if (flip_wind) std::swap(a, c);
            idx.push_back(a); idx.push_back(b); idx.push_back(c);
        };
        for (uint32_t y = 0; y + 1 < depth; ++y)
            for (uint32_t x = 0; x + 1 < width; ++x) {
                const uint32_t v00 = y * width + x, v10 = v00 + 1, v01 = v00 + width, v11 = v01 + 1;
                const bool flipped = flip_edges || (diamond && ((y + x) & 1u) == 0) || (zigzag && (y & 1u) == 0);
                if (flipped) { tri(v00, v01, v11); tri(v00, v11, v10); }
                else { tri(v00, v01, v10); tri(v10, v01, v11); }
            }
        return add_mesh(v.data(), width * depth, idx.data(), uint32_t(idx.size() / 3));
    }

    void grow_bodies(uint32_t need) {
        if (need <= cap) return;
        uint32_t c = std::max<uint32_t>(need, cap * 2);
        c = std::max<uint32_t>(c, 64);
        auto g4 = [&](DevBuf<float4>& b) { b.grow_keep(c, n, stream); };
        g4(pos); g4(quat); g4(linvel); g4(angvel); g4(inv_inertia); g4(grav); g4(force); g4(torque); g4(material);
        g4(sleep); g4(aabb_min); g4(aabb_max); g4(pred); g4(push_lin); g4(push_ang);
        iw.grow_keep(size_t(c) * 3, size_t(n) * 3, stream);
        info_d.grow_keep(c, n, stream);
        settled.grow_keep(c, n, stream);
        cap = c;
    }

    uint32_t add_bodies(uint32_t cnt, const bgpu_body_desc* d) {
        if (batch) throw InvalidArg{"a batched world takes bodies through bgpu_batch_add_worlds"};
        const uint32_t first = add_bodies_impl(cnt, d);
        rebuild_world_plan();
        return first;
    }

    uint32_t add_bodies_impl(uint32_t cnt, const bgpu_body_desc* d) {
        for (uint32_t k = 0; k < cnt; ++k) {
            if (d[k].shape >= shapes_h.size()) throw InvalidArg{"body shape id out of range"};
            if (shapes_h[d[k].shape].type == SHAPE_PLANE && d[k].mass != 0.0f)
                throw InvalidArg{"a plane body must be static (mass 0)"};
            if (shapes_h[d[k].shape].type == SHAPE_MESH && (d[k].mass != 0.0f || (d[k].flags & BGPU_BODY_KINEMATIC)))
                throw InvalidArg{"a triangle mesh or heightfield body must be static (mass 0, not kinematic)"};
            if (!(d[k].mass >= 0.0f)) throw InvalidArg{"mass must be >= 0"};
        }
        sync_shapes();
        uint32_t first = n;
        grow_bodies(n + cnt);
        std::vector<float4> hp(cnt), hq(cnt), hlv(cnt), hav(cnt), hinv(cnt), hg(cnt), hz(cnt), hmat(cnt), hsl(cnt);
        std::vector<uint4> hinfo(cnt);
        for (uint32_t k = 0; k < cnt; ++k) {
            const bgpu_body_desc& b = d[k];
            const Shape& s = shapes_h[b.shape];
            bool kin = (b.flags & BGPU_BODY_KINEMATIC) != 0;
            bool stat = b.mass == 0.0f && !kin;
            uint32_t fl = 0;
            if (stat) fl |= BF_STATIC;
            if (kin) fl |= BF_KINEMATIC;
            if (b.flags & BGPU_BODY_NO_CONTACT_RESPONSE) fl |= BF_NO_RESPONSE;
            if (b.flags & BGPU_BODY_DISABLE_WORLD_GRAVITY) fl |= BF_DISABLE_GRAVITY;
            if (b.flags & BGPU_BODY_ADDITIONAL_DAMPING) fl |= BF_ADDITIONAL_DAMPING;
            float inv_mass = 0.0f, inv[3] = {0.0f, 0.0f, 0.0f};
            if (!stat && !kin) {  // body.rs:388-399 new_dynamic
                float in[3];
                local_inertia(s, b.mass, in);
                for (int a = 0; a < 3; ++a) inv[a] = in[a] != 0.0f ? 1.0f / in[a] : 0.0f;
                inv_mass = 1.0f / b.mass;
            }
            uint32_t act = stat ? ACT_ISLAND_SLEEPING : (kin ? ACT_DISABLE_DEACTIVATION : ACT_ACTIVE);
            if (b.activation) act = b.activation;
            hp[k] = make_float4(b.position[0], b.position[1], b.position[2], 0.0f);
            hq[k] = make_float4(b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]);
            hlv[k] = make_float4(b.linear_velocity[0], b.linear_velocity[1], b.linear_velocity[2], 0.0f);
            hav[k] = make_float4(b.angular_velocity[0], b.angular_velocity[1], b.angular_velocity[2], 0.0f);
            hinv[k] = make_float4(inv[0], inv[1], inv[2], inv_mass);
            // world.rs:528-535: dynamic bodies inherit the world gravity.
            bool inherit = !stat && !kin && !(b.flags & BGPU_BODY_DISABLE_WORLD_GRAVITY);
            hg[k] = inherit ? make_float4(gravity[0], gravity[1], gravity[2], 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
            hz[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            hmat[k] = make_float4(b.friction, b.restitution, b.linear_damping, b.angular_damping);
            float lt = b.linear_sleeping_threshold > 0.0f ? b.linear_sleeping_threshold : 0.8f;
            float at = b.angular_sleeping_threshold > 0.0f ? b.angular_sleeping_threshold : 1.0f;
            hsl[k] = make_float4(0.0f, lt, at, 0.0f);
            uint32_t group = b.group, mask = b.mask;
            hinfo[k] = make_uint4(b.shape, fl, act, group | (mask << 16));
            // Planes, and static meshes (a terrain's box overlaps most bodies, and a tree walk
            // from it would list them one by one), go through the broad phase's all-bodies pass.
            if (s.type == SHAPE_PLANE || s.type == SHAPE_MESH) unbounded.push_back(first + k);
        }
        auto up = [&](DevBuf<float4>& dst, const std::vector<float4>& src) {
            check_cuda(cudaMemcpyAsync(dst.p + first, src.data(), cnt * sizeof(float4), cudaMemcpyHostToDevice, stream),
                       "upload bodies");
        };
        up(pos, hp); up(quat, hq); up(linvel, hlv); up(angvel, hav); up(inv_inertia, hinv); up(grav, hg);
        up(force, hz); up(torque, hz); up(material, hmat); up(sleep, hsl); up(push_lin, hz); up(push_ang, hz);
        check_cuda(cudaMemcpyAsync(info_d.p + first, hinfo.data(), cnt * sizeof(uint4), cudaMemcpyHostToDevice, stream),
                   "upload info");
        n += cnt;
        launch_initial_aabbs(body_dev(), shapes_d.p, hull_d.p, first, cnt, stream);
        check_cuda(cudaGetLastError(), "initial aabbs");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        std::sort(unbounded.begin(), unbounded.end());
        return first;
    }

    uint32_t num_worlds() const { return batch ? uint32_t(world_off_h.size() - 1) : 1u; }

    // Batched worlds: append worlds whose bodies are given back to back.
    uint32_t add_worlds(uint32_t nw, const uint32_t* bodies_per_world, const bgpu_body_desc* d) {
        if (!batch) throw InvalidArg{"bgpu_batch_add_worlds needs a world made by bgpu_batch_create"};
        uint64_t total = 0;
        for (uint32_t k = 0; k < nw; ++k) total += bodies_per_world[k];
        if (uint64_t(n) + total > 0xfffffff0ull) throw InvalidArg{"too many bodies"};
        const uint32_t first_world = num_worlds();
        const uint32_t first_body = n;
        if (total) add_bodies_impl(uint32_t(total), d);
        uint32_t acc = first_body;
        for (uint32_t k = 0; k < nw; ++k) {
            acc += bodies_per_world[k];
            world_off_h.push_back(acc);
        }
        const uint32_t W = num_worlds();
        // world offsets and per-body world ids (kept in step with the body arrays)
        world_off_d.grow_keep(W + 1, 0, stream);
        check_cuda(cudaMemcpyAsync(world_off_d.p, world_off_h.data(), (W + 1) * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, stream), "upload world offsets");
        std::vector<uint32_t> wof(total);
        for (uint32_t k = 0, i = 0; k < nw; ++k)
            for (uint32_t j = 0; j < bodies_per_world[k]; ++j) wof[i++] = first_world + k;
        world_of_d.grow_keep(std::max<uint32_t>(cap, 1), first_body, stream);
        if (total)
            check_cuda(cudaMemcpyAsync(world_of_d.p + first_body, wof.data(), total * sizeof(uint32_t),
                                       cudaMemcpyHostToDevice, stream), "upload world ids");
        // per-world simulate flags: new worlds start with prev_simulate = 0
        DevBuf<uint32_t> fresh;
        fresh.reserve(2 * size_t(W));
        check_cuda(cudaMemsetAsync(fresh.p, 0, 2 * size_t(W) * sizeof(uint32_t), stream), "memset");
        const uint32_t W0 = first_world;
        if (W0) check_cuda(cudaMemcpyAsync(fresh.p + W, world_sim.p + W0, W0 * sizeof(uint32_t),
                                           cudaMemcpyDeviceToDevice, stream), "copy flags");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        std::swap(world_sim.p, fresh.p);
        std::swap(world_sim.cap, fresh.cap);
        rebuild_world_plan();
        return first_world;
    }

    // The per-world solver's plan for the current worlds (an invalid plan, or a world with
    // joints, falls back to the global solver).
    void rebuild_world_plan() {
        wplan.valid = false;
        if (!batch) {
            // A plain world small enough for one CTA's shared memory is solved as a batch of one
            // world (one CTA of PLAIN_WORLD_SOLVER_THREADS threads, velocities in shared memory,
            // block-local syncs).
            if (n == 0 || n > PLAIN_WORLD_SOLVER_MAX_BODIES) return;
            const std::vector<uint32_t> off{0u, n};
            plain_off_d.reserve(2);
            check_cuda(cudaMemcpyAsync(plain_off_d.p, off.data(), 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, stream),
                       "h2d");
            wcol.reserve(WS_STRIDE + 1);
            build_world_plan(off, PLAIN_WORLD_SOLVER_THREADS, 0u, wplan, stream);
            return;
        }
        if (wplan_block == 0) return;
        wcol.reserve(size_t(num_worlds()) * WS_STRIDE + 1);
        build_world_plan(world_off_h, wplan_block, wplan_tau, wplan, stream);
    }

    bool use_world_solver() const { return wplan.valid && (joints_h.empty() || !batch); }
    const uint32_t* world_offsets_dev() const { return batch ? world_off_d.p : plain_off_d.p; }

    JointsDev joints_dev() {
        JointsDev j;
        j.desc = joint_desc_d.p;
        j.order = joint_order_d.p;
        j.coff = joint_coff_d.p;
        j.n = uint32_t(joints_h.size());
        j.ncol = joint_coff_h.empty() ? 0u : uint32_t(joint_coff_h.size() - 1);
        j.rows = joint_rows_d.p;
        j.count = joint_count_d.p;
        j.angle = joint_angle_d.p;
        j.position = joint_pos_d.p;
        j.row_off = joint_row_off_d.p;
        j.aux = joint_aux_d.p;
        j.s2_state = joint_s2_state_d.p;
        j.global_cfm = info.global_cfm;
        return j;
    }

    // RigidBody::ccd for bodies [first, first + cnt): the list holds the bodies whose threshold
    // and radius are both positive (the others are never swept, step.rs:1072-1079).
    void set_ccd(uint32_t first, uint32_t cnt, const float* thr, const float* rad) {
        if (uint64_t(first) + cnt > n) throw InvalidArg{"CCD body range out of bounds"};
        ccd_thr_h.resize(n, 0.0f);
        ccd_rad_h.resize(n, 0.0f);
        for (uint32_t k = 0; k < cnt; ++k) {
            if (std::isnan(thr[k]) || std::isnan(rad[k])) throw InvalidArg{"NaN CCD setting"};
            ccd_thr_h[first + k] = thr[k];
            ccd_rad_h[first + k] = rad[k];
        }
        ccd_ids_h.clear();
        std::vector<float2> par;
        for (uint32_t i = 0; i < uint32_t(ccd_thr_h.size()); ++i)
            if (ccd_thr_h[i] > 0.0f && ccd_rad_h[i] > 0.0f) {
                ccd_ids_h.push_back(i);
                par.push_back(make_float2(ccd_thr_h[i], ccd_rad_h[i]));
            }
        nccd = uint32_t(ccd_ids_h.size());
        if (!nccd) return;
        ccd_ids_d.reserve(nccd);
        ccd_par_d.reserve(nccd);
        ccd_clamp_d.reserve(nccd);
        check_cuda(cudaMemcpyAsync(ccd_ids_d.p, ccd_ids_h.data(), nccd * sizeof(uint32_t), cudaMemcpyHostToDevice, stream),
                   "upload CCD ids");
        check_cuda(cudaMemcpyAsync(ccd_par_d.p, par.data(), nccd * sizeof(float2), cudaMemcpyHostToDevice, stream),
                   "upload CCD settings");
        std::vector<float> ones(nccd, 1.0f);
        check_cuda(cudaMemcpyAsync(ccd_clamp_d.p, ones.data(), nccd * sizeof(float), cudaMemcpyHostToDevice, stream),
                   "reset CCD clamps");
        check_cuda(cudaStreamSynchronize(stream), "sync");
    }

    // Row capacity of joint j: JOINT_MAX_ROWS, or for a spring-2 joint its exact row count
    // (generic6dof_spring2.rs:846-1111): per axis 2 limit rows (lower < upper) or 1 lock row
    // (lower == upper), plus 1 for a motor or servo and 1 for a spring.
    uint32_t joint_row_capacity(uint32_t j) const {
        if (joint_s2_h[j] < 0 || joints_h[j].kind == BGPU_JOINT_GENERIC6DOF) return JOINT_MAX_ROWS;
        uint32_t r = 0;
        for (const bgpu_spring2_axis& a : s2_h[size_t(joint_s2_h[j])].axis) {
            r += a.lower_limit < a.upper_limit ? 2u : (a.lower_limit == a.upper_limit ? 1u : 0u);
            r += (a.flags & BGPU_S2_MOTOR) ? 1u : 0u;
            r += (a.flags & BGPU_S2_SPRING) ? 1u : 0u;
        }
        return r;
    }

    // Constraint::generic_6dof_spring2: validated, then added as joints of kind SPRING2 whose axis
    // tables live beside the descriptors.
    uint32_t add_spring2_joints(uint32_t cnt, const bgpu_spring2_desc* d, uint32_t kind = BGPU_JOINT_SPRING2) {
        std::vector<bgpu_joint_desc> base(cnt);
        for (uint32_t k = 0; k < cnt; ++k) {
            if (d[k].rotate_order > BGPU_ROTATE_ZYX) throw InvalidArg{"unknown rotate order"};
            for (const bgpu_spring2_axis& a : d[k].axis)
                if (std::isnan(a.lower_limit) || std::isnan(a.upper_limit)) throw InvalidArg{"NaN axis limit"};
            bgpu_joint_desc_default(&base[k]);
            base[k].kind = kind;
            base[k].body_a = d[k].body_a;
            base[k].body_b = d[k].body_b;
            base[k].flags = d[k].flags & (BGPU_JOINT_DISABLE_COLLISIONS | BGPU_JOINT_DISABLED);
            std::memcpy(base[k].frame_a, d[k].frame_a, sizeof(base[k].frame_a));
            std::memcpy(base[k].frame_b, d[k].frame_b, sizeof(base[k].frame_b));
        }
        return add_joints(cnt, base.data(), d);
    }

    // PhysicsWorld::add_constraint. The joint graph is coloured here, once per change:
    // first fit in joint id order, with only dynamic bodies in conflict (static and
    // kinematic bodies take no impulse), so a joint colour never holds a dynamic body twice.
    uint32_t add_joints(uint32_t cnt, const bgpu_joint_desc* d, const bgpu_spring2_desc* s2 = nullptr) {
        for (uint32_t k = 0; k < cnt; ++k) {
            if (s2 ? (d[k].kind != BGPU_JOINT_SPRING2 && d[k].kind != BGPU_JOINT_GENERIC6DOF)
                   : (d[k].kind > BGPU_JOINT_CONETWIST || d[k].kind == BGPU_JOINT_SPRING2))
                throw InvalidArg{"unknown joint kind (spring-2 joints go through bgpu_add_spring2_joints)"};
            if (d[k].body_a >= n || d[k].body_b >= n || d[k].body_a == d[k].body_b)
                throw InvalidArg{"joint bodies out of range or equal"};
        }
        const uint32_t first = uint32_t(joints_h.size());
        joints_h.insert(joints_h.end(), d, d + cnt);
        for (uint32_t k = 0; k < cnt; ++k) {
            joint_s2_h.push_back(s2 ? int32_t(s2_h.size()) : -1);
            if (s2) s2_h.push_back(s2[k]);
        }
        const uint32_t nj = uint32_t(joints_h.size());
        std::vector<uint4> hinfo(n);
        check_cuda(cudaMemcpyAsync(hinfo.data(), info_d.p, n * sizeof(uint4), cudaMemcpyDeviceToHost, stream), "d2h");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        auto dynamic = [&](uint32_t i) { return (hinfo[i].y & (BF_STATIC | BF_KINEMATIC)) == 0; };
        std::unordered_map<uint32_t, std::vector<uint64_t>> used;  // body -> colour bits
        std::vector<uint32_t> colour(nj);
        uint32_t ncol = 0;
        for (uint32_t j = 0; j < nj; ++j) {
            uint64_t m[2] = {0, 0};
            const uint32_t ends[2] = {joints_h[j].body_a, joints_h[j].body_b};
            for (uint32_t e : ends) {
                if (!dynamic(e)) continue;
                auto it = used.find(e);
                if (it != used.end()) { m[0] |= it->second[0]; m[1] |= it->second[1]; }
            }
            uint32_t c = 0;
            while (c < 128 && ((m[c >> 6] >> (c & 63)) & 1ull)) ++c;
            if (c >= uint32_t(MAX_COLOURS)) throw InvalidArg{"a body is linked by more than 127 joints"};
            colour[j] = c;
            ncol = std::max(ncol, c + 1);
            for (uint32_t e : ends) {
                if (!dynamic(e)) continue;
                auto& v = used[e];
                if (v.empty()) v.assign(2, 0ull);
                v[c >> 6] |= 1ull << (c & 63);
            }
        }
        joint_coff_h.assign(ncol + 1, 0u);
        for (uint32_t j = 0; j < nj; ++j) joint_coff_h[colour[j] + 1] += 1;
        for (uint32_t c = 0; c < ncol; ++c) joint_coff_h[c + 1] += joint_coff_h[c];
        joint_order_h.assign(nj, 0u);
        std::vector<uint32_t> fill(joint_coff_h.begin(), joint_coff_h.end() - 1);
        for (uint32_t j = 0; j < nj; ++j) joint_order_h[fill[colour[j]]++] = j;
        // device descriptors (JOINT_F4 float4 per joint id)
        std::vector<float4> hd(size_t(nj) * JOINT_F4);
        for (uint32_t j = 0; j < nj; ++j) {
            const bgpu_joint_desc& x = joints_h[j];
            float4* o = &hd[size_t(j) * JOINT_F4];
            o[0] = make_float4(__uint_as_float_host(x.kind), __uint_as_float_host(x.body_a),
                               __uint_as_float_host(x.body_b), __uint_as_float_host(x.flags));
            for (int f = 0; f < 2; ++f) {
                const float* fr = f ? x.frame_b : x.frame_a;
                for (int c = 0; c < 4; ++c) o[1 + 4 * f + c] = make_float4(fr[3 * c], fr[3 * c + 1], fr[3 * c + 2], 0.0f);
            }
            o[9] = make_float4(x.erp, x.impulse_clamp, x.limit_low, x.limit_high);
            o[10] = make_float4(x.limit_softness, x.limit_bias_factor, x.limit_relaxation, x.motor_target_velocity);
            o[11] = make_float4(x.motor_max_impulse, x.gear_ratio, 0.0f, 0.0f);
            o[12] = make_float4(x.lin_limit_low, x.lin_limit_high, x.ang_limit_low, x.ang_limit_high);
            o[13] = make_float4(x.softness_lim_lin, x.softness_lim_ang, x.damping_lim_lin, x.damping_lim_ang);
            o[14] = make_float4(x.softness_ortho_lin, x.softness_ortho_ang, x.lin_motor_target_velocity,
                                x.lin_motor_max_force);
            o[15] = make_float4(x.ang_motor_target_velocity, x.ang_motor_max_force, 0.0f, 0.0f);
            if (x.kind == BGPU_JOINT_CONETWIST) {  // kind-specific slots [12..14]
                o[12] = make_float4(x.swing_span1, x.swing_span2, x.twist_span, x.cone_softness);
                o[13] = make_float4(x.cone_bias_factor, x.cone_relaxation, x.cone_motor_max_impulse, 0.0f);
                o[14] = make_float4(x.cone_motor_target[0], x.cone_motor_target[1], x.cone_motor_target[2],
                                    x.cone_motor_target[3]);
            }
            if (joint_s2_h[j] >= 0) {
                const uint32_t aux0 = uint32_t(joint_s2_h[j]) * 6u * S2_AXIS_F4;
                o[9] = make_float4(__uint_as_float_host(aux0), __uint_as_float_host(s2_h[size_t(joint_s2_h[j])].rotate_order),
                                   0.0f, 0.0f);
            }
        }
        // spring-2 axis tables (S2_AXIS_F4 per axis)
        std::vector<float4> aux(std::max<size_t>(s2_h.size(), 1) * 6 * S2_AXIS_F4, make_float4(0, 0, 0, 0));
        for (size_t k = 0; k < s2_h.size(); ++k)
            for (int i = 0; i < 6; ++i) {
                const bgpu_spring2_axis& a = s2_h[k].axis[i];
                float4* o = &aux[(k * 6 + i) * S2_AXIS_F4];
                o[0] = make_float4(a.lower_limit, a.upper_limit, a.bounce, a.stop_erp);
                o[1] = make_float4(a.stop_cfm, a.motor_erp, a.motor_cfm, a.target_velocity);
                o[2] = make_float4(a.max_motor_force, a.servo_target, a.stiffness, a.damping);
                o[3] = make_float4(a.equilibrium_point, __uint_as_float_host(a.flags), 0.0f, 0.0f);
            }
        // every slot's first row, slot by slot in solve order
        joint_row_off_h.assign(nj + 1, 0u);
        for (uint32_t t = 0; t < nj; ++t) joint_row_off_h[t + 1] = joint_row_off_h[t] + joint_row_capacity(joint_order_h[t]);
        joint_desc_d.reserve(hd.size());
        joint_order_d.reserve(nj);
        joint_coff_d.reserve(ncol + 1);
        joint_count_d.reserve(nj);
        joint_rows_d.reserve(std::max<size_t>(joint_row_off_h[nj], 1) * JROW_F4);
        joint_row_off_d.reserve(nj + 1);
        joint_aux_d.reserve(aux.size());
        joint_s2_state_d.grow_keep(2 * size_t(nj), 2 * size_t(first), stream);
        check_cuda(cudaMemsetAsync(joint_s2_state_d.p + 2 * size_t(first), 0, 2 * size_t(cnt) * sizeof(float4), stream),
                   "memset");
        check_cuda(cudaMemcpyAsync(joint_row_off_d.p, joint_row_off_h.data(), (nj + 1) * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, stream), "upload joint row offsets");
        check_cuda(cudaMemcpyAsync(joint_aux_d.p, aux.data(), aux.size() * sizeof(float4), cudaMemcpyHostToDevice, stream),
                   "upload spring-2 axes");
        joint_angle_d.grow_keep(nj, first, stream);
        check_cuda(cudaMemsetAsync(joint_angle_d.p + first, 0, cnt * sizeof(float), stream), "memset");
        joint_pos_d.grow_keep(nj, first, stream);
        check_cuda(cudaMemsetAsync(joint_pos_d.p + first, 0, cnt * sizeof(float), stream), "memset");
        check_cuda(cudaMemsetAsync(joint_count_d.p, 0, nj * sizeof(uint32_t), stream), "memset");
        check_cuda(cudaMemcpyAsync(joint_desc_d.p, hd.data(), hd.size() * sizeof(float4), cudaMemcpyHostToDevice, stream),
                   "upload joints");
        check_cuda(cudaMemcpyAsync(joint_order_d.p, joint_order_h.data(), nj * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   stream), "upload joint order");
        check_cuda(cudaMemcpyAsync(joint_coff_d.p, joint_coff_h.data(), (ncol + 1) * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, stream), "upload joint colours");
        upload_suppressed();
        return first;
    }

    // world.rs:873-880: the pairs a joint keeps from colliding (independent of enabled), sorted.
    // Synchronises the stream (the keys are pageable host memory).
    void upload_suppressed() {
        std::vector<uint64_t> keys;
        for (const auto& x : joints_h)
            if (x.flags & BGPU_JOINT_DISABLE_COLLISIONS) {
                const uint32_t lo = std::min(x.body_a, x.body_b), hi = std::max(x.body_a, x.body_b);
                keys.push_back((uint64_t(lo) << 32) | hi);
            }
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        nsuppressed = uint32_t(keys.size());
        if (nsuppressed) {
            suppressed_d.reserve(nsuppressed);
            check_cuda(cudaMemcpyAsync(suppressed_d.p, keys.data(), nsuppressed * sizeof(uint64_t),
                                       cudaMemcpyHostToDevice, stream), "upload suppressed pairs");
        }
        check_cuda(cudaStreamSynchronize(stream), "sync");
    }

    // Constraint::set_enabled / set_disable_collisions between steps (constraint.rs:637-652): the
    // two bits change in the joint's device descriptor (read by every step's joint rows and island
    // links) and in the suppressed pair list (read by every step's pair pass and CCD sweep).
    void set_joint_flags(uint32_t id, uint32_t flags) {
        if (id >= joints_h.size()) throw InvalidArg{"bgpu_set_joint_flags: no joint with that id"};
        const uint32_t bits = BGPU_JOINT_DISABLE_COLLISIONS | BGPU_JOINT_DISABLED;
        if (flags & ~bits) throw InvalidArg{"bgpu_set_joint_flags: only DISABLE_COLLISIONS and DISABLED change"};
        joints_h[id].flags = (joints_h[id].flags & ~bits) | flags;
        const float word = __uint_as_float_host(joints_h[id].flags);
        check_cuda(cudaMemcpyAsync(&joint_desc_d.p[size_t(id) * JOINT_F4].w, &word, sizeof(float),
                                   cudaMemcpyHostToDevice, stream), "upload joint flags");
        upload_suppressed();  // synchronises, so `word` outlives the copy
    }

    void set_gravity(const float* g) {
        gravity[0] = g[0]; gravity[1] = g[1]; gravity[2] = g[2];
        // world.rs:467-481: active bodies that did not opt out take the new gravity.
        if (n == 0) return;
        std::vector<uint4> hinfo(n);
        std::vector<float4> hg(n);
        check_cuda(cudaMemcpyAsync(hinfo.data(), info_d.p, n * sizeof(uint4), cudaMemcpyDeviceToHost, stream), "d2h");
        check_cuda(cudaMemcpyAsync(hg.data(), grav.p, n * sizeof(float4), cudaMemcpyDeviceToHost, stream), "d2h");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t a = hinfo[i].z;
            bool active = a == ACT_ACTIVE || a == ACT_WANTS_DEACTIVATION || a == ACT_DISABLE_DEACTIVATION;
            if (active && !(hinfo[i].y & BF_DISABLE_GRAVITY)) hg[i] = make_float4(g[0], g[1], g[2], 0.0f);
        }
        check_cuda(cudaMemcpyAsync(grav.p, hg.data(), n * sizeof(float4), cudaMemcpyHostToDevice, stream), "h2d");
        check_cuda(cudaStreamSynchronize(stream), "sync");
    }

    void mark(int k) {
        if (timing) check_cuda(cudaEventRecord(ev[ev_cur][k], stream), "event");
    }

    // Adds a completed event set to the timing sums. Marks: 0 start, 1 velocities+AABBs,
    // 2 broad phase, 3 islands, 4 pair pass, 5 colouring, 6 PGS kernel, 7 writeback, 8 positions.
    void fold(int set) {
        if (!ev_pending[set]) return;
        ev_pending[set] = false;
        float ms[9] = {};
        for (int k = 0; k < 8; ++k) check_cuda(cudaEventElapsedTime(&ms[k], ev[set][k], ev[set][k + 1]), "elapsed");
        last.stage_ms[0] += ms[0];
        last.stage_ms[1] += 0.0f;  // AABBs are fused into the velocity pass
        last.stage_ms[2] += ms[1];
        last.stage_ms[3] += ms[2];
        last.stage_ms[4] += ms[3];
        last.stage_ms[5] += ms[4] + ms[5] + ms[6];
        last.stage_ms[6] += ms[7];
        last.solve_kernel_ms += ms[5];
        float total = 0.0f;
        check_cuda(cudaEventElapsedTime(&total, ev[set][0], ev[set][8]), "elapsed");
        last.step_ms += total;
        last.timed_steps += 1;
    }

    void reset_timing() {
        for (int k = 0; k < 7; ++k) last.stage_ms[k] = 0.0f;
        last.solve_kernel_ms = 0.0f;
        last.step_ms = 0.0f;
        last.timed_steps = 0;
        ev_pending[0] = ev_pending[1] = false;
    }

    // One step_simulation(dt) (step.rs:100-108 -> internal_step).
    void step_once(float dt) {
        sync_shapes();
        solved_standalone = 0;
        StepParams sp;
        sp.dt = dt;
        sp.inv_dt = 1.0f / dt;
        sp.info = info;
        sp.suppressed = nsuppressed ? suppressed_d.p : nullptr;
        sp.nsuppressed = nsuppressed;
        JointsDev jd = joints_dev();
        if (rec_step) {
            rec_step->flags.reserve(std::max<uint32_t>(n, 1));
            check_cuda(cudaMemsetAsync(rec_step->flags.p, 0, std::max<uint32_t>(n, 1), stream), "memset");
        }
        BodyDev b = body_dev();
        WorldView wv = view();
        uint32_t* status = flags.p;
        const uint32_t nw = num_worlds();
        uint32_t* simulate = world_sim.p;
        uint32_t* prev_simulate = world_sim.p + nw;
        const uint32_t* world_of = batch ? world_of_d.p : nullptr;
        check_cuda(cudaMemsetAsync(flags.p, 0, sizeof(uint32_t), stream), "memset flags");
        check_cuda(cudaMemsetAsync(simulate, 0, nw * sizeof(uint32_t), stream), "memset flags");
        mark(0);
        // 1-3: velocities, predicted poses, AABBs (fused).
        launch_integrate_velocities(b, shapes_d.p, hull_d.p, n, dt, stream);
        mark(1);
        // 4: broad phase (syncs once to size the pair arrays; the previous step's
        //    manifold count and timing events are read at the same point).
        uint64_t np = batch ? bp.run_worlds(aabb_min.p, aabb_max.p, n, world_off_d.p, nw, pairs, stream)
                            : bp.run(aabb_min.p, aabb_max.p, n, unbounded, pairs, status, stream);
        npairs = uint32_t(np);
        if (timing) fold(ev_cur ^ 1);
        Manifolds& old_cache = cache[cur];
        Manifolds& next = cache[cur ^ 1];
        old_cache.count_host = hs->cache_count;
        if (rec_step) prepare_record(old_cache.count_host);
        mark(2);
        // 4b: islands
        islands.run(b, n, pairs.p, npairs, world_of, simulate, status, stream, jd.desc, jd.n);
        mark(3);
        // 5: pair pass
        pd.reserve(std::max<uint32_t>(npairs, 1), n, old_cache.count_host);
        if (old_cache.count_host)
            check_cuda(cudaMemsetAsync(pd.old_owned.p, 0, old_cache.count_host * sizeof(uint32_t), stream), "memset");
        run_pair_pass(wv, pairs.p, npairs, old_cache, pd, sp, simulate, status, stream);
        // 5a: joint rows from the current poses (step.rs:928-949)
        launch_joint_rows(b, jd, sp.inv_dt, info.erp, stream);
        mark(4);
        // 6: solve (colouring, then the PGS kernel)
        // The colouring starts from last step's colours, except every RECOLOUR_PERIOD-th step.
        last_world_solver = use_world_solver();
        if (last_world_solver)
            run_world_solver(wv, pairs.p, npairs, pd, sp, status, stream, [&](int k) { mark(k); },
                             world_offsets_dev(), nw, wplan, wcol.p, batch ? nullptr : &jd,
                             step_count % RECOLOUR_PERIOD != 0);
        else
            run_solver(wv, pairs.p, npairs, pd, sp, status, stream, [&](int k) { mark(k); },
                       step_count % RECOLOUR_PERIOD != 0, &jd, batch ? nullptr : bp.leaf_body.p,
                       batch ? 0u : uint32_t(bp.tree_m));
        ++step_count;
        // 6b: impulse writeback + prune
        run_cache_update(pairs.p, npairs, old_cache, pd, next, world_of, simulate, prev_simulate, stream);
        check_cuda(cudaMemcpyAsync(prev_simulate, simulate, nw * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream),
                   "flag");
        mark(7);
        // 7a: CCD clamp fractions, from the solved velocities and the pre-integration poses
        launch_ccd_sweep(b, shapes_d.p, hull_d.p, ccd_ids_d.p, ccd_par_d.p, nccd, n, batch ? world_off_d.p : nullptr,
                         world_of, sp.suppressed, sp.nsuppressed, dt, ccd_clamp_d.p, status,
                         batch ? nullptr : bp.node_rec.p, bp.leaf_body.p, batch ? 0 : bp.tree_m, bp.unbounded.p,
                         batch ? 0u : bp.nunb, stream);
        // 6c + 7 + 8: deactivation, pose integration with the split push, force clear.
        launch_integrate_positions(b, n, dt, info.split_impulse_turn_erp, stream);
        launch_ccd_apply(b, ccd_ids_d.p, ccd_clamp_d.p, nccd, dt, stream);
        mark(8);
        if (timing) {
            ev_pending[ev_cur] = true;
            ev_cur ^= 1;
        }
        check_cuda(cudaGetLastError(), "step launch");
        cur ^= 1;
        check_cuda(cudaMemcpyAsync(hs->scalars, pd.scalars.p, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "d2h");
        check_cuda(cudaMemcpyAsync(&hs->status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "d2h");
        check_cuda(cudaMemcpyAsync(&hs->cache_count, next.count_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
                   "d2h");
        stats_pending = true;
        if (rec_step) finish_record();
    }

    // Adjoint recording: point the pair pass, the solver and the merge at the record's arrays.
    void prepare_record(uint32_t nold) {
        StepRecord& R = *rec_step;
        R.npairs = npairs;
        R.nold = nold;
        R.iters = info.num_iterations;
        const size_t np = std::max<uint32_t>(npairs, 1);
        rec_pt_src.reserve(np * 4);
        rec_pair_old.reserve(np);
        R.row_src.reserve(np * 4);
        R.merge_pos.reserve(np);
        check_cuda(cudaMemsetAsync(R.merge_pos.p, 0xff, np * sizeof(uint32_t), stream), "memset");
        const size_t slots_cap = (size_t(npairs) + 32u * 130u + 31u) & ~size_t(31);
        if (R.iters) R.sweeps.reserve(size_t(R.iters) * 4 * slots_cap);
        pd.rec = RecordDev{rec_pt_src.p, rec_pair_old.p, R.row_src.p, R.merge_pos.p, R.iters ? R.sweeps.p : nullptr};
    }

    // Keep the step's batch records, colour offsets and contact table (they are overwritten next step).
    void finish_record() {
        StepRecord& R = *rec_step;
        pd.rec = RecordDev{};
        check_cuda(cudaStreamSynchronize(stream), "sync");
        R.ncol = hs->scalars[4];
        R.slots = 0;
        R.per_world = last_world_solver;
        if (npairs == 0 || R.ncol == 0) {
            R.ncol = 0;
            return;
        }
        if (R.per_world) {  // slots are the contact pairs, world by world; the world records say where
            const uint32_t words = num_worlds() * WS_STRIDE;
            R.slots = (hs->scalars[2] + 31u) & ~31u;
            R.off.reserve(words);
            R.recs.reserve(R.slots);
            R.tab.reserve(size_t(R.slots) * VT_PLANES * 4);
            check_cuda(cudaMemcpyAsync(R.off.p, wcol.p, words * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream),
                       "record copy");
            check_cuda(cudaMemcpyAsync(R.recs.p, pd.batch_rec.p, size_t(R.slots) * sizeof(uint4),
                                       cudaMemcpyDeviceToDevice, stream), "record copy");
            check_cuda(cudaMemcpyAsync(R.tab.p, pd.vtab.p, size_t(R.slots) * VT_PLANES * 4 * sizeof(float4),
                                       cudaMemcpyDeviceToDevice, stream), "record copy");
            check_cuda(cudaStreamSynchronize(stream), "sync");
            return;
        }
        std::vector<uint32_t> off(R.ncol + 1);
        check_cuda(cudaMemcpy(off.data(), pd.colour_offset.p, (R.ncol + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost),
                   "d2h");
        R.slots = (off[R.ncol] + 31u) & ~31u;
        R.off.reserve(R.ncol);
        R.end.reserve(R.ncol);
        R.recs.reserve(R.slots);
        R.tab.reserve(size_t(R.slots) * VT_PLANES * 4);
        auto d2d = [&](void* dst, const void* src, size_t bytes) {
            check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream), "record copy");
        };
        d2d(R.off.p, pd.colour_offset.p, R.ncol * sizeof(uint32_t));
        d2d(R.end.p, pd.colour_cursor.p, R.ncol * sizeof(uint32_t));
        d2d(R.recs.p, pd.batch_rec.p, size_t(R.slots) * sizeof(uint4));
        d2d(R.tab.p, pd.vtab.p, size_t(R.slots) * VT_PLANES * 4 * sizeof(float4));
        check_cuda(cudaStreamSynchronize(stream), "sync");
    }

    void finish_stats() {
        if (!stats_pending) return;
        check_cuda(cudaStreamSynchronize(stream), "sync");
        stats_pending = false;
        last.num_bodies = n;
        last.num_pairs = npairs;
        last.num_contact_pairs = hs->scalars[2];
        last.num_contacts = hs->scalars[3];
        last.num_colours = hs->scalars[4];
        last.num_split_pairs = hs->scalars[5];
        last.num_split_contacts = hs->scalars[10];
        last.num_detect = hs->scalars[0] + hs->scalars[1];
        last.num_manifolds = hs->cache_count;
        last.device_status = hs->status;
        if (timing) {
            fold(ev_cur ^ 1);
            fold(ev_cur);
        }
    }
};

// ---------------------------------------------------------------- adjoint tape
// World state a replay starts from: the body arrays a step reads, the current
// manifold cache, the per-world simulate flags.
struct Snapshot {
    uint32_t n = 0, count = 0, nsim = 0;
    int cur = 0;
    uint64_t step_count = 0;
    DevBuf<float4> f4[10];
    DevBuf<uint4> info;
    DevBuf<uint64_t> keys;
    DevBuf<float4> entries;
    DevBuf<uint32_t> sim;
};

static float4* body_array(World& W, int k) {
    float4* a[10] = {W.pos.p,    W.quat.p,   W.linvel.p,   W.angvel.p,   W.sleep.p,
                     W.force.p,  W.torque.p, W.aabb_min.p, W.aabb_max.p, W.grav.p};
    return a[k];
}

static void save_snapshot(World& W, Snapshot& S) {
    check_cuda(cudaStreamSynchronize(W.stream), "sync");  // the cache's entry count is read on the host
    S.n = W.n;
    S.cur = W.cur;
    S.step_count = W.step_count;
    S.count = W.hs->cache_count;  // entries of cache[cur], written back at the end of every step
    S.nsim = 2 * W.num_worlds();
    auto d2d = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, W.stream), "snapshot copy");
    };
    for (int k = 0; k < 10; ++k) {
        S.f4[k].reserve(std::max<uint32_t>(S.n, 1));
        d2d(S.f4[k].p, body_array(W, k), S.n * sizeof(float4));
    }
    S.info.reserve(std::max<uint32_t>(S.n, 1));
    d2d(S.info.p, W.info_d.p, S.n * sizeof(uint4));
    const Manifolds& c = W.cache[W.cur];
    S.keys.reserve(S.count + 1);
    S.entries.reserve((size_t(S.count) + 1) * ENTRY_F4);
    d2d(S.keys.p, c.keys.p, S.count * sizeof(uint64_t));
    d2d(S.entries.p, c.entries.p, size_t(S.count) * ENTRY_F4 * sizeof(float4));
    S.sim.reserve(S.nsim);
    d2d(S.sim.p, W.world_sim.p, S.nsim * sizeof(uint32_t));
    // No wait here: the copies are ordered before the next step on the same stream.
}

static void restore_snapshot(World& W, const Snapshot& S) {
    if (S.n != W.n || S.nsim != 2 * W.num_worlds()) throw InvalidArg{"bodies or worlds were added after the tape's forward pass"};
    auto d2d = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, W.stream), "restore copy");
    };
    for (int k = 0; k < 10; ++k) d2d(body_array(W, k), S.f4[k].p, S.n * sizeof(float4));
    d2d(W.info_d.p, S.info.p, S.n * sizeof(uint4));
    W.cur = S.cur;
    W.step_count = S.step_count;
    Manifolds& c = W.cache[W.cur];
    c.keys.reserve(S.count + 1);
    c.entries.reserve((size_t(S.count) + 1) * ENTRY_F4);
    d2d(c.keys.p, S.keys.p, S.count * sizeof(uint64_t));
    d2d(c.entries.p, S.entries.p, size_t(S.count) * ENTRY_F4 * sizeof(float4));
    check_cuda(cudaMemcpyAsync(c.count_dev, &S.count, sizeof(uint32_t), cudaMemcpyHostToDevice, W.stream), "h2d");
    d2d(W.world_sim.p, S.sim.p, S.nsim * sizeof(uint32_t));
    check_cuda(cudaStreamSynchronize(W.stream), "sync");
    c.count_host = S.count;
    W.hs->cache_count = S.count;
    W.stats_pending = false;
}

// Autotuner of a batch's solver launch shape: every candidate steps the batch from the same
// checkpoint for `steps` timed steps (after one untimed step); the fastest is kept and the
// batch goes back to the checkpoint.
static void autotune_batch(World& W, float dt, uint32_t steps) {
    if (!W.batch) throw InvalidArg{"bgpu_batch_autotune needs a batched world"};
    if (steps == 0 || steps > 1000) throw InvalidArg{"steps_per_candidate must lie in 1..1000"};
    W.finish_stats();
    Snapshot start;
    save_snapshot(W, start);
    struct Cand {
        uint32_t block, tau;
    };
    std::vector<Cand> cands{{0u, 0u}};
    for (uint32_t block : {32u, 64u, 128u, 256u})
        for (uint32_t tau : {0u, 32u, 64u, 128u, 0x7fffffffu}) cands.push_back({block, tau});
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Release {
        cudaEvent_t &a, &b;
        ~Release() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } release{e0, e1};
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    Cand best{W.wplan_block, W.wplan_tau};
    float best_ms = 0.0f, global_ms = 0.0f;
    uint32_t timed = 0;
    for (const Cand& c : cands) {
        W.wplan_block = c.block;
        W.wplan_tau = c.tau;
        W.rebuild_world_plan();
        if (c.block && !W.wplan.valid) continue;
        restore_snapshot(W, start);
        W.step_once(dt);
        W.finish_stats();
        check_cuda(cudaEventRecord(e0, W.stream), "event");
        for (uint32_t k = 0; k < steps; ++k) W.step_once(dt);
        check_cuda(cudaEventRecord(e1, W.stream), "event");
        W.finish_stats();
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        if (W.last.device_status) continue;  // e.g. a world needing more colours than one mask holds
        ++timed;
        if (c.block == 0) global_ms = ms;
        if (best_ms == 0.0f || ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    restore_snapshot(W, start);
    W.wplan_block = best.block;
    W.wplan_tau = best.tau;
    W.rebuild_world_plan();
    W.tuned_ms = best_ms / float(steps);
    W.tuned_global_ms = global_ms / float(steps);
    W.tuned_candidates = timed;
}

// Tape::backward of the rigid-body step: a forward pass that keeps a
// checkpoint every `every` steps, and a backward pass that replays each
// segment from its checkpoint with recording on, then runs the segment's
// steps in reverse (k_adjoint.cu).
struct Tape {
    World* W;
    uint32_t every;
    float dt = 0.0f;
    uint32_t nsteps = 0;
    std::vector<std::unique_ptr<Snapshot>> cps;  // checkpoints; the first ncps belong to the last forward pass
    uint32_t ncps = 0;
    Snapshot final_state;
    std::vector<std::unique_ptr<StepRecord>> recs;
    DevBuf<float4> xbar, vbar, wbar, lbar;
    DevBuf<float> mubar, ebar, carry[2];
    DevBuf<unsigned int> bar;
    DevBuf<uint32_t> status;
    cudaEvent_t ev[4] = {};
    float forward_ms = 0.0f, backward_ms = 0.0f;

    Tape(World* w, uint32_t k) : W(w), every(k) {
        for (auto& e : ev) check_cuda(cudaEventCreate(&e), "event");
    }
    ~Tape() {
        for (auto& e : ev) if (e) cudaEventDestroy(e);
    }

    void forward(float step_dt, uint32_t steps) {
        W->finish_stats();
        dt = step_dt;
        nsteps = steps;
        // The checkpoints of an earlier pass are reused: their device buffers only grow, so a
        // repeated forward pass allocates (and frees) nothing.
        ncps = (steps + every - 1) / every;
        while (cps.size() < ncps) cps.emplace_back(new Snapshot);
        check_cuda(cudaEventRecord(ev[0], W->stream), "event");
        for (uint32_t s = 0; s < steps; ++s) {
            if (s % every == 0) save_snapshot(*W, *cps[s / every]);
            W->step_once(dt);
        }
        save_snapshot(*W, final_state);
        check_cuda(cudaEventRecord(ev[1], W->stream), "event");
        check_cuda(cudaEventSynchronize(ev[1]), "sync");
        check_cuda(cudaEventElapsedTime(&forward_ms, ev[0], ev[1]), "elapsed");
    }

    // Back to the state at the start of the last forward pass (its first checkpoint).
    void rewind() {
        if (!ncps) throw InvalidArg{"the tape has no forward pass"};
        restore_snapshot(*W, *cps[0]);
    }

    // grad_state: n x 9 floats (dL/dx, dL/dv, dL/dw of the final state). Outputs may be null.
    void backward(const float* grad_state, float* gv0, float* gw0, float* gmu, float* ge) {
        if (!ncps) throw InvalidArg{"the tape has no forward pass"};
        const uint32_t n = W->n;
        cudaStream_t s = W->stream;
        std::vector<float4> hx(n), hv(n), hw(n);
        for (uint32_t i = 0; i < n; ++i) {
            const float* g = grad_state + size_t(i) * 9;
            hx[i] = make_float4(g[0], g[1], g[2], 0.0f);
            hv[i] = make_float4(g[3], g[4], g[5], 0.0f);
            hw[i] = make_float4(g[6], g[7], g[8], 0.0f);
        }
        const size_t nn = std::max<uint32_t>(n, 1);
        xbar.reserve(nn); vbar.reserve(nn); wbar.reserve(nn); mubar.reserve(nn); ebar.reserve(nn);
        bar.reserve(4);
        status.reserve(4);
        check_cuda(cudaMemcpyAsync(xbar.p, hx.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        check_cuda(cudaMemcpyAsync(vbar.p, hv.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        check_cuda(cudaMemcpyAsync(wbar.p, hw.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        check_cuda(cudaMemsetAsync(mubar.p, 0, nn * sizeof(float), s), "memset");
        check_cuda(cudaMemsetAsync(ebar.p, 0, nn * sizeof(float), s), "memset");
        check_cuda(cudaMemsetAsync(status.p, 0, sizeof(uint32_t), s), "memset");
        check_cuda(cudaEventRecord(ev[2], s), "event");
        while (recs.size() < every) recs.emplace_back(new StepRecord);
        const float* carry_in = nullptr;
        int o = 0;
        for (size_t seg = ncps; seg-- > 0;) {
            const uint32_t s0 = uint32_t(seg) * every, s1 = std::min(s0 + every, nsteps);
            restore_snapshot(*W, *cps[seg]);
            for (uint32_t st = s0; st < s1; ++st) {
                W->rec_step = recs[st - s0].get();
                try {
                    W->step_once(dt);
                } catch (...) {
                    W->rec_step = nullptr;
                    throw;
                }
                W->rec_step = nullptr;
            }
            if (W->hs->status) throw InvalidArg{"device status set while replaying a segment"};
            for (uint32_t st = s1; st-- > s0;) {
                const StepRecord& R = *recs[st - s0];
                launch_adj_positions(n, dt, R.flags.p, xbar.p, vbar.p, s);
                float* cout = nullptr;
                if (R.nold) {
                    carry[o].reserve(size_t(R.nold) * 4);
                    check_cuda(cudaMemsetAsync(carry[o].p, 0, size_t(R.nold) * 4 * sizeof(float), s), "memset");
                    cout = carry[o].p;
                }
                if (R.ncol) {
                    lbar.reserve(size_t(R.slots) * 4);
                    if (R.per_world)
                        run_adj_solve_worlds(R.view(), W->wplan, lbar.p, vbar.p, wbar.p, mubar.p, ebar.p,
                                             W->material.p, carry_in, cout, W->info.restitution_velocity_threshold,
                                             W->info.warmstarting_factor, status.p, s);
                    else
                        run_adj_solve(R.view(), lbar.p, vbar.p, wbar.p, mubar.p, ebar.p, W->material.p, carry_in,
                                      cout, W->info.restitution_velocity_threshold, W->info.warmstarting_factor, bar.p,
                                      status.p, s);
                }
                launch_adj_velocities(n, dt, R.flags.p, W->material.p, vbar.p, wbar.p, s);
                check_cuda(cudaGetLastError(), "adjoint launch");
                carry_in = cout;
                o ^= 1;
            }
        }
        check_cuda(cudaEventRecord(ev[3], s), "event");
        restore_snapshot(*W, final_state);
        check_cuda(cudaEventElapsedTime(&backward_ms, ev[2], ev[3]), "elapsed");
        uint32_t st = 0;
        check_cuda(cudaMemcpy(&st, status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost), "d2h");
        if (st) throw InvalidArg{"device status set in the adjoint solve (barrier timeout)"};
        std::vector<float> hm(n), he(n);
        check_cuda(cudaMemcpy(hv.data(), vbar.p, n * sizeof(float4), cudaMemcpyDeviceToHost), "d2h");
        check_cuda(cudaMemcpy(hw.data(), wbar.p, n * sizeof(float4), cudaMemcpyDeviceToHost), "d2h");
        check_cuda(cudaMemcpy(hm.data(), mubar.p, n * sizeof(float), cudaMemcpyDeviceToHost), "d2h");
        check_cuda(cudaMemcpy(he.data(), ebar.p, n * sizeof(float), cudaMemcpyDeviceToHost), "d2h");
        for (uint32_t i = 0; i < n; ++i) {
            if (gv0) { gv0[3 * i] = hv[i].x; gv0[3 * i + 1] = hv[i].y; gv0[3 * i + 2] = hv[i].z; }
            if (gw0) { gw0[3 * i] = hw[i].x; gw0[3 * i + 1] = hw[i].y; gw0[3 * i + 2] = hw[i].z; }
            if (gmu) gmu[i] = hm[i];
            if (ge) ge[i] = he[i];
        }
    }
};

}  // namespace bgpu

using bgpu::World;

struct bgpu_world {
    World impl;
};

namespace {

template <class F>
bgpu_status guarded(F&& f) {
    try {
        return f();
    } catch (const bgpu::CudaError& e) {
        bgpu::g_last_error = e.where;
        return BGPU_ERR_CUDA;
    } catch (const bgpu::InvalidArg& e) {
        bgpu::g_last_error = e.what;
        return BGPU_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        bgpu::g_last_error = "host allocation failed";
        return BGPU_ERR_CAPACITY;
    } catch (const std::exception& e) {
        bgpu::g_last_error = e.what();
        return BGPU_ERR_INVALID_ARGUMENT;
    }
}

// A rejected argument (NULL where data is required, or out of range): the status, with the
// message bgpu_last_error reports.
bgpu_status bad_args(const char* fn) {
    bgpu::g_last_error = std::string(fn) + ": a required argument is NULL or out of range";
    return BGPU_ERR_INVALID_ARGUMENT;
}

bgpu_status check_device_status(World& w) {
    w.finish_stats();
    if (w.last.device_status) {
        char buf[128];
        std::snprintf(buf, sizeof(buf), "device status bits 0x%x", w.last.device_status);
        bgpu::g_last_error = buf;
        return BGPU_ERR_DEVICE_STATUS;
    }
    return BGPU_OK;
}

}  // namespace

extern "C" {

const char* bgpu_version(void) { return "bgpu 0.1 (sm_100a)"; }

bgpu_status bgpu_selftest_wait_timeout(uint32_t limit_ms, uint32_t* device_status, float* waited_ms) {
    if (limit_ms < 1 || limit_ms > 2000) {
        bgpu::g_last_error = "bgpu_selftest_wait_timeout: limit_ms must lie in 1..2000";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        bgpu::DevBuf<uint32_t> words;
        words.reserve(2);
        cudaStream_t s = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        struct Release {  // the stream and events go on every exit, a failed CUDA call included
            cudaStream_t& s;
            cudaEvent_t &e0, &e1;
            ~Release() {
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
                if (s) cudaStreamDestroy(s);
            }
        } release{s, e0, e1};
        bgpu::check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        bgpu::check_cuda(cudaEventCreate(&e0), "event");
        bgpu::check_cuda(cudaEventCreate(&e1), "event");
        bgpu::check_cuda(cudaMemsetAsync(words.p, 0, 2 * sizeof(uint32_t), s), "memset");
        bgpu::check_cuda(cudaEventRecord(e0, s), "event");
        bgpu::run_wait_selftest(uint64_t(limit_ms) * 1000000ull, reinterpret_cast<unsigned int*>(words.p), words.p + 1, s);
        bgpu::check_cuda(cudaGetLastError(), "selftest launch");
        bgpu::check_cuda(cudaEventRecord(e1, s), "event");
        uint32_t st = 0;
        bgpu::check_cuda(cudaMemcpyAsync(&st, words.p + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        float ms = 0.0f;
        bgpu::check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        if (device_status) *device_status = st;
        if (waited_ms) *waited_ms = ms;
        return BGPU_OK;
    });
}

int bgpu_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return c;
}

bgpu_status bgpu_set_device(int device) {
    const int n = bgpu_device_count();
    if (n == 0) {
        bgpu::g_last_error = "no CUDA device";
        return BGPU_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        bgpu::g_last_error = "bgpu_set_device: no device with that ordinal";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        bgpu::check_cuda(cudaSetDevice(device), "cudaSetDevice");
        return BGPU_OK;
    });
}

size_t bgpu_last_error(char* buf, size_t len) {
    const std::string& e = bgpu::g_last_error;
    if (buf && len) {
        size_t k = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return e.size();
}

void bgpu_solver_info_default(bgpu_solver_info* o) {
    if (!o) return;
    o->erp2 = 0.2f;
    o->linear_slop = 0.005f;
    o->restitution_velocity_threshold = 1.0f;
    o->split_impulse = 1;
    o->split_impulse_penetration_threshold = -0.04f;
    o->split_impulse_turn_erp = 0.1f;
    o->warmstarting_factor = 0.85f;
    o->global_cfm = 0.0f;
    o->sor = 1.0f;
    o->num_iterations = 10;
    o->erp = 0.2f;
    o->damping = 1.0f;
}

void bgpu_joint_desc_default(bgpu_joint_desc* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->flags = BGPU_JOINT_DISABLE_COLLISIONS;
    const float ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int k = 0; k < 9; ++k) o->frame_a[3 + k] = o->frame_b[3 + k] = ident[k];
    o->limit_low = 1.0f;
    o->limit_high = -1.0f;
    o->limit_softness = 0.9f;
    o->limit_bias_factor = 0.3f;
    o->limit_relaxation = 1.0f;
    o->gear_ratio = 1.0f;
    o->swing_span1 = o->swing_span2 = o->twist_span = 1e30f;
    o->cone_softness = 1.0f;
    o->cone_bias_factor = 0.3f;
    o->cone_relaxation = 1.0f;
    o->cone_motor_target[3] = 1.0f;
    o->cone_motor_max_impulse = -1.0f;
    o->lin_limit_low = 1.0f;
    o->lin_limit_high = -1.0f;
    o->ang_limit_low = 0.0f;
    o->ang_limit_high = 0.0f;
    o->softness_lim_lin = o->softness_lim_ang = o->damping_lim_lin = o->damping_lim_ang = 1.0f;
    o->softness_ortho_lin = o->softness_ortho_ang = 1.0f;
}

void bgpu_body_desc_default(bgpu_body_desc* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->orientation[3] = 1.0f;
    o->mass = 1.0f;
    o->friction = 0.5f;
    o->group = 1;
    o->mask = 0xFFFF;
}

static void copy_info(bgpu::SolverParams& d, const bgpu_solver_info& s) {
    d.erp2 = s.erp2;
    d.linear_slop = s.linear_slop;
    d.restitution_velocity_threshold = s.restitution_velocity_threshold;
    d.split_impulse = s.split_impulse;
    d.split_impulse_penetration_threshold = s.split_impulse_penetration_threshold;
    d.split_impulse_turn_erp = s.split_impulse_turn_erp;
    d.warmstarting_factor = s.warmstarting_factor;
    d.global_cfm = s.global_cfm;
    d.sor = s.sor;
    d.num_iterations = s.num_iterations;
    d.erp = s.erp;
    d.damping = s.damping;
}

bgpu_status bgpu_world_create(const bgpu_solver_info* info, const float* gravity, bgpu_world** out) {
    if (!out) {
        bgpu::g_last_error = "out is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (bgpu_device_count() == 0) {
        bgpu::g_last_error = "no CUDA device";
        return BGPU_ERR_NO_DEVICE;
    }
    return guarded([&]() -> bgpu_status {
        std::unique_ptr<bgpu_world> w(new bgpu_world());
        bgpu_solver_info d;
        bgpu_solver_info_default(&d);
        copy_info(w->impl.info, info ? *info : d);
        if (gravity) std::memcpy(w->impl.gravity, gravity, 3 * sizeof(float));
        *out = w.release();
        return BGPU_OK;
    });
}

void bgpu_world_destroy(bgpu_world* w) { delete w; }

bgpu_status bgpu_world_set_gravity(bgpu_world* w, const float* g) {
    if (!w || !g) return bad_args("bgpu_world_set_gravity");
    return guarded([&]() -> bgpu_status {
        w->impl.set_gravity(g);
        return BGPU_OK;
    });
}

bgpu_status bgpu_world_set_solver_info(bgpu_world* w, const bgpu_solver_info* info) {
    if (!w || !info) return bad_args("bgpu_world_set_solver_info");
    copy_info(w->impl.info, *info);
    return BGPU_OK;
}

bgpu_status bgpu_add_shape(bgpu_world* w, uint32_t type, const float* params, const float* pts, uint32_t npts,
                           uint32_t* out) {
    if (!w) return bad_args("bgpu_add_shape");
    return guarded([&]() -> bgpu_status {
        uint32_t id = w->impl.add_shape(type, params, pts, npts);
        if (out) *out = id;
        return BGPU_OK;
    });
}

bgpu_status bgpu_add_mesh_shape(bgpu_world* w, const float* vertices, uint32_t nverts, const uint32_t* indices,
                                uint32_t ntris, uint32_t* out) {
    if (!w) return bad_args("bgpu_add_mesh_shape");
    return guarded([&]() -> bgpu_status {
        uint32_t id = w->impl.add_mesh(vertices, nverts, indices, ntris);
        if (out) *out = id;
        return BGPU_OK;
    });
}

bgpu_status bgpu_add_heightfield_shape(bgpu_world* w, const float* heights, uint32_t width, uint32_t depth,
                                       const float* cell_size, uint32_t options, uint32_t* out) {
    if (!w) return bad_args("bgpu_add_heightfield_shape");
    return guarded([&]() -> bgpu_status {
        uint32_t id = w->impl.add_heightfield(heights, width, depth, cell_size, options);
        if (out) *out = id;
        return BGPU_OK;
    });
}

bgpu_status bgpu_add_bodies(bgpu_world* w, uint32_t n, const bgpu_body_desc* d, uint32_t* out_first) {
    if (!w || (n && !d)) return bad_args("bgpu_add_bodies");
    return guarded([&]() -> bgpu_status {
        w->impl.finish_stats();
        uint32_t f = w->impl.add_bodies(n, d);
        if (out_first) *out_first = f;
        return BGPU_OK;
    });
}

uint32_t bgpu_num_bodies(const bgpu_world* w) { return w ? w->impl.n : 0; }

bgpu_status bgpu_batch_create(const bgpu_solver_info* info, const float* gravity, bgpu_world** out) {
    bgpu_status st = bgpu_world_create(info, gravity, out);
    if (st != BGPU_OK) return st;
    (*out)->impl.batch = true;
    return BGPU_OK;
}

bgpu_status bgpu_batch_add_worlds(bgpu_world* w, uint32_t n_worlds, const uint32_t* bodies_per_world,
                                  const bgpu_body_desc* descs, uint32_t* out_first_world) {
    if (!w || (n_worlds && !bodies_per_world)) {
        bgpu::g_last_error = "world is NULL or bodies_per_world is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    uint64_t total = 0;
    for (uint32_t k = 0; k < n_worlds; ++k) total += bodies_per_world[k];
    if (total && !descs) {
        bgpu::g_last_error = "descs is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        w->impl.finish_stats();
        uint32_t f = w->impl.add_worlds(n_worlds, bodies_per_world, descs);
        if (out_first_world) *out_first_world = f;
        return BGPU_OK;
    });
}

bgpu_status bgpu_batch_step(bgpu_world* w, float dt, uint32_t nsteps) {
    if (!w || !w->impl.batch) {
        bgpu::g_last_error = "world is NULL or not batched";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return bgpu_step(w, dt, nsteps);
}

struct bgpu_tape {
    std::unique_ptr<bgpu::Tape> impl;
};

bgpu_status bgpu_tape_create(bgpu_world* w, uint32_t checkpoint_every, bgpu_tape** out) {
    if (!w || !out || checkpoint_every == 0) {
        bgpu::g_last_error = "world or out is NULL, or checkpoint_every is 0";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return guarded([&]() -> bgpu_status {
        if (!w->impl.joints_h.empty()) throw bgpu::InvalidArg{"the adjoint tape does not cover joints"};
        if (w->impl.nccd) throw bgpu::InvalidArg{"the adjoint tape does not cover the CCD clamp"};
        std::unique_ptr<bgpu_tape> t(new bgpu_tape());
        t->impl.reset(new bgpu::Tape(&w->impl, checkpoint_every));
        *out = t.release();
        return BGPU_OK;
    });
}

void bgpu_tape_destroy(bgpu_tape* t) { delete t; }

bgpu_status bgpu_tape_forward(bgpu_tape* t, float dt, uint32_t nsteps) {
    if (!t || !(dt > 0.0f)) {
        bgpu::g_last_error = "tape is NULL or dt <= 0";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        t->impl->forward(dt, nsteps);
        return check_device_status(*t->impl->W);
    });
}

bgpu_status bgpu_tape_backward(bgpu_tape* t, const float* grad_state, float* grad_v0, float* grad_w0,
                               float* grad_friction, float* grad_restitution) {
    if (!t || !grad_state) {
        bgpu::g_last_error = "tape or grad_state is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        t->impl->backward(grad_state, grad_v0, grad_w0, grad_friction, grad_restitution);
        return BGPU_OK;
    });
}

bgpu_status bgpu_tape_rewind(bgpu_tape* t) {
    if (!t) {
        bgpu::g_last_error = "tape is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        t->impl->rewind();
        return BGPU_OK;
    });
}

bgpu_status bgpu_tape_timing(const bgpu_tape* t, float* forward_ms, float* backward_ms) {
    if (!t) return bad_args("bgpu_tape_timing");
    if (forward_ms) *forward_ms = t->impl->forward_ms;
    if (backward_ms) *backward_ms = t->impl->backward_ms;
    return BGPU_OK;
}

uint32_t bgpu_batch_num_worlds(const bgpu_world* w) { return (w && w->impl.batch) ? w->impl.num_worlds() : 0u; }

bgpu_status bgpu_batch_autotune(bgpu_world* w, float dt, uint32_t steps_per_candidate, bgpu_batch_tuning* out) {
    if (!w || !(dt > 0.0f)) return bad_args("bgpu_batch_autotune");
    bgpu_status st = guarded([&]() -> bgpu_status {
        bgpu::autotune_batch(w->impl, dt, steps_per_candidate);
        return BGPU_OK;
    });
    if (st == BGPU_OK && out) st = bgpu_batch_get_tuning(w, out);
    return st;
}

bgpu_status bgpu_batch_set_tuning(bgpu_world* w, uint32_t threads_per_cta, uint32_t warp_world_max_bodies) {
    if (!w) return bad_args("bgpu_batch_set_tuning");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        if (!W.batch) throw bgpu::InvalidArg{"bgpu_batch_set_tuning needs a batched world"};
        if (threads_per_cta && (threads_per_cta < 32 || threads_per_cta > 256 || threads_per_cta % 32))
            throw bgpu::InvalidArg{"threads_per_cta must be 0 or a multiple of 32 in 32..256"};
        W.finish_stats();
        W.wplan_block = threads_per_cta;
        W.wplan_tau = warp_world_max_bodies;
        W.rebuild_world_plan();
        return BGPU_OK;
    });
}

bgpu_status bgpu_batch_get_tuning(bgpu_world* w, bgpu_batch_tuning* out) {
    if (!w || !out) return bad_args("bgpu_batch_get_tuning");
    World& W = w->impl;
    out->threads_per_cta = W.wplan_block;
    out->warp_world_max_bodies = W.wplan_tau;
    out->ctas = W.use_world_solver() ? W.wplan.ncta : 0u;
    out->candidates = W.tuned_candidates;
    out->ms_per_step = W.tuned_ms;
    out->global_ms_per_step = W.tuned_global_ms;
    return BGPU_OK;
}

bgpu_status bgpu_batch_world_offsets(bgpu_world* w, uint32_t* offsets) {
    if (!w || !offsets || !w->impl.batch) {
        bgpu::g_last_error = "world is NULL, not batched, or offsets is NULL";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    std::memcpy(offsets, w->impl.world_off_h.data(), w->impl.world_off_h.size() * sizeof(uint32_t));
    return BGPU_OK;
}

bgpu_status bgpu_step(bgpu_world* w, float dt, uint32_t nsteps) {
    if (!w || !(dt > 0.0f)) {
        bgpu::g_last_error = "world is NULL or dt <= 0";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        w->impl.accumulator = 0.0f;  // step_simulation resets the fixed-step accumulator (step.rs:105)
        for (uint32_t k = 0; k < nsteps; ++k) w->impl.step_once(dt);
        return check_device_status(w->impl);
    });
}

bgpu_status bgpu_step_timed(bgpu_world* w, float dt, uint32_t nsteps, float* device_ms) {
    if (!w || !(dt > 0.0f)) {
        bgpu::g_last_error = "world is NULL or dt <= 0";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        cudaEvent_t a, b;
        bgpu::check_cuda(cudaEventCreate(&a), "event");
        bgpu::check_cuda(cudaEventCreate(&b), "event");
        bgpu::check_cuda(cudaEventRecord(a, W.stream), "event");
        for (uint32_t k = 0; k < nsteps; ++k) W.step_once(dt);
        bgpu::check_cuda(cudaEventRecord(b, W.stream), "event");
        bgpu::check_cuda(cudaEventSynchronize(b), "event sync");
        float ms = 0.0f;
        bgpu::check_cuda(cudaEventElapsedTime(&ms, a, b), "elapsed");
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (device_ms) *device_ms = ms;
        return check_device_status(W);
    });
}

// step.rs:136-199 (fixed-timestep accumulator; motion-state interpolation is not modelled, and the
// accumulator follows the reference's default latency mode). The forces applied before a call
// act in every substep of it and are cleared once, after the last one; a call that runs no
// substep drops them (step.rs:117-121, 160-177).
bgpu_status bgpu_step_simulation_fixed(bgpu_world* w, float dt, uint32_t max_sub_steps, float fixed_dt,
                                       uint32_t* out_substeps) {
    if (!w || (max_sub_steps != 0 && !(fixed_dt > 0.0f))) {
        bgpu::g_last_error = "bgpu_step_simulation_fixed: world is NULL or fixed_dt <= 0 with substeps";
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        const size_t fbytes = size_t(W.n) * sizeof(float4);
        auto drop_forces = [&]() {
            if (!fbytes) return;
            bgpu::check_cuda(cudaMemsetAsync(W.force.p, 0, fbytes, W.stream), "memset forces");
            bgpu::check_cuda(cudaMemsetAsync(W.torque.p, 0, fbytes, W.stream), "memset torques");
        };
        uint32_t num = 0;
        float step_dt = fixed_dt;
        if (max_sub_steps != 0) {
            float& acc = W.accumulator;
            acc += dt;
            if (acc >= fixed_dt) {
                num = uint32_t(acc / fixed_dt);
                acc -= float(num) * fixed_dt;
            }
        } else {
            step_dt = dt;
            W.accumulator = 0.0f;  // step.rs:156
            if (std::fabs(dt) <= 1.1920929e-7f) {
                drop_forces();
                if (out_substeps) *out_substeps = 0;
                return BGPU_OK;
            }
            num = 1;
        }
        if (num == 0) {  // a frame without a substep: the applied forces expire
            drop_forces();
            if (out_substeps) *out_substeps = 0;
            return BGPU_OK;
        }
        const uint32_t clamped = max_sub_steps ? std::min(num, max_sub_steps) : num;
        // Each substep's position pass clears the forces, so the call's forces are kept aside
        // and put back before every later substep.
        const bool keep = clamped > 1 && fbytes;
        if (keep) {
            W.force_keep.reserve(2 * size_t(W.n));
            bgpu::check_cuda(cudaMemcpyAsync(W.force_keep.p, W.force.p, fbytes, cudaMemcpyDeviceToDevice, W.stream),
                             "keep forces");
            bgpu::check_cuda(cudaMemcpyAsync(W.force_keep.p + W.n, W.torque.p, fbytes, cudaMemcpyDeviceToDevice,
                                             W.stream), "keep torques");
        }
        for (uint32_t k = 0; k < clamped; ++k) {
            if (keep && k > 0) {
                bgpu::check_cuda(cudaMemcpyAsync(W.force.p, W.force_keep.p, fbytes, cudaMemcpyDeviceToDevice,
                                                 W.stream), "restore forces");
                bgpu::check_cuda(cudaMemcpyAsync(W.torque.p, W.force_keep.p + W.n, fbytes, cudaMemcpyDeviceToDevice,
                                                 W.stream), "restore torques");
            }
            W.step_once(step_dt);
        }
        if (out_substeps) *out_substeps = num;
        return check_device_status(W);
    });
}

bgpu_status bgpu_read_state(bgpu_world* w, float* state) {
    if (!w || !state) return bad_args("bgpu_read_state");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        uint32_t n = W.n;
        std::vector<float4> p(n), q(n), lv(n), av(n), sl(n);
        std::vector<uint4> in(n);
        cudaStream_t s = W.stream;
        bgpu::check_cuda(cudaMemcpyAsync(p.data(), W.pos.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(q.data(), W.quat.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(lv.data(), W.linvel.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(av.data(), W.angvel.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(sl.data(), W.sleep.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(in.data(), W.info_d.p, n * sizeof(uint4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        for (uint32_t i = 0; i < n; ++i) {
            float* o = state + size_t(i) * 15;
            o[0] = p[i].x; o[1] = p[i].y; o[2] = p[i].z;
            o[3] = q[i].x; o[4] = q[i].y; o[5] = q[i].z; o[6] = q[i].w;
            o[7] = lv[i].x; o[8] = lv[i].y; o[9] = lv[i].z;
            o[10] = av[i].x; o[11] = av[i].y; o[12] = av[i].z;
            o[13] = float(in[i].z);
            o[14] = sl[i].x;
        }
        return BGPU_OK;
    });
}

bgpu_status bgpu_write_state(bgpu_world* w, const float* state) {
    if (!w || !state) return bad_args("bgpu_write_state");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        uint32_t n = W.n;
        std::vector<float4> p(n), q(n), lv(n), av(n), sl(n);
        std::vector<uint4> in(n);
        cudaStream_t s = W.stream;
        bgpu::check_cuda(cudaMemcpyAsync(sl.data(), W.sleep.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(in.data(), W.info_d.p, n * sizeof(uint4), cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        for (uint32_t i = 0; i < n; ++i) {
            const float* o = state + size_t(i) * 15;
            p[i] = make_float4(o[0], o[1], o[2], 0.0f);
            q[i] = make_float4(o[3], o[4], o[5], o[6]);
            lv[i] = make_float4(o[7], o[8], o[9], 0.0f);
            av[i] = make_float4(o[10], o[11], o[12], 0.0f);
            in[i].z = uint32_t(o[13]);
            sl[i].x = o[14];
        }
        bgpu::check_cuda(cudaMemcpyAsync(W.pos.p, p.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaMemcpyAsync(W.quat.p, q.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaMemcpyAsync(W.linvel.p, lv.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaMemcpyAsync(W.angvel.p, av.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaMemcpyAsync(W.sleep.p, sl.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaMemcpyAsync(W.info_d.p, in.data(), n * sizeof(uint4), cudaMemcpyHostToDevice, s), "h2d");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_poses(bgpu_world* w, float* poses) {
    if (!w || !poses) return bad_args("bgpu_read_poses");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        uint32_t n = W.n;
        if (!n) return BGPU_OK;
        cudaStream_t s = W.stream;
        // Packed on the device, one copy into the caller's buffer (direct DMA when it is pinned).
        W.host_io.reserve(size_t(n) * 7);
        bgpu::launch_pack_poses(n, W.pos.p, W.quat.p, W.host_io.p, s);
        bgpu::check_cuda(cudaMemcpyAsync(poses, W.host_io.p, size_t(n) * 7 * sizeof(float), cudaMemcpyDeviceToHost, s),
                         "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_apply_forces(bgpu_world* w, const float* force, const float* torque) {
    if (!w) return bad_args("bgpu_apply_forces");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        uint32_t n = W.n;
        if (!n) return BGPU_OK;
        cudaStream_t s = W.stream;
        // One copy of the caller's n x 3 floats each, widened on the device; the sync at the
        // end returns the caller's buffers (the copies may read them asynchronously when pinned).
        W.host_io.reserve(size_t(n) * 6);
        for (int which = 0; which < 2; ++which) {
            const float* src = which ? torque : force;
            if (!src) continue;
            float* stage = W.host_io.p + size_t(which) * 3 * n;
            bgpu::check_cuda(cudaMemcpyAsync(stage, src, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, s),
                             "h2d");
            bgpu::launch_unpack3(n, stage, which ? W.torque.p : W.force.p, s);
        }
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_pairs(bgpu_world* w, uint32_t* out, uint64_t cap, uint64_t* out_n) {
    if (!w) return bad_args("bgpu_read_pairs");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        if (out_n) *out_n = W.npairs;
        uint64_t k = std::min<uint64_t>(cap, W.npairs);
        if (!out || !k) return BGPU_OK;
        std::vector<uint64_t> keys(k);
        bgpu::check_cuda(cudaMemcpyAsync(keys.data(), W.pairs.p, k * sizeof(uint64_t), cudaMemcpyDeviceToHost, W.stream),
                         "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        for (uint64_t i = 0; i < k; ++i) {
            out[2 * i] = bgpu::key_lo(keys[i]);
            out[2 * i + 1] = bgpu::key_hi(keys[i]);
        }
        return BGPU_OK;
    });
}

// Gather the solved rows in (colour, pair key) order.
static void gather_solve_order(World& W, uint32_t ngroups, const uint64_t* keys_dev, std::vector<uint64_t>& order_keys,
                               std::vector<float>& rows_out) {
    bgpu::PairData& pd = W.pd;
    cudaStream_t s = W.stream;
    uint32_t sc[16];
    bgpu::check_cuda(cudaMemcpyAsync(sc, pd.scalars.p, sizeof(sc), cudaMemcpyDeviceToHost, s), "d2h");
    bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
    uint32_t K = sc[2], ncol = sc[4];
    std::vector<uint32_t> cp(K), col(K), cnt(ngroups);
    std::vector<uint64_t> keys(ngroups);
    std::vector<float4> rows(size_t(ngroups) * 4 * bgpu::ROW_F4);
    if (K) {
        bgpu::check_cuda(cudaMemcpyAsync(cp.data(), pd.contact_pairs.p, K * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(col.data(), pd.colour.p, K * 4, cudaMemcpyDeviceToHost, s), "d2h");
    }
    if (ngroups) {
        bgpu::check_cuda(cudaMemcpyAsync(cnt.data(), pd.row_count.p, ngroups * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(keys.data(), keys_dev, ngroups * 8, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(rows.data(), pd.rows.p, rows.size() * sizeof(float4), cudaMemcpyDeviceToHost, s),
                         "d2h");
    }
    bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
    (void)ncol;
    std::vector<uint32_t> idx(K);
    for (uint32_t k = 0; k < K; ++k) idx[k] = k;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        if (col[a] != col[b]) return col[a] < col[b];
        return cp[a] < cp[b];
    });
    order_keys.clear();
    rows_out.clear();
    for (uint32_t t : idx) {
        uint32_t p = cp[t];
        order_keys.push_back(keys[p]);
        for (uint32_t k = 0; k < cnt[p]; ++k) {
            const float4* r = &rows[(size_t(p) * 4 + k) * bgpu::ROW_F4];
            float rec[16] = {float(bgpu::key_lo(keys[p])), float(bgpu::key_hi(keys[p])), float(k),
                             r[0].x, r[0].y, r[0].z, r[1].x, r[1].y, r[1].z, r[2].x, r[2].y, r[2].z,
                             r[5].w, r[3].x, r[3].y, r[3].z};
            rows_out.insert(rows_out.end(), rec, rec + 16);
            rows_out.push_back(r[5].y);
            rows_out.push_back(r[5].z);
        }
    }
}

bgpu_status bgpu_read_contacts(bgpu_world* w, float* out, uint64_t cap, uint64_t* out_n) {
    if (!w) return bad_args("bgpu_read_contacts");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        std::vector<uint64_t> keys;
        std::vector<float> rows;
        if (W.solved_standalone) gather_solve_order(W, W.standalone_groups, W.standalone_keys.p, keys, rows);
        else gather_solve_order(W, W.npairs, W.pairs.p, keys, rows);
        uint64_t n = rows.size() / 18;
        if (out_n) *out_n = n;
        uint64_t k = std::min<uint64_t>(cap, n);
        for (uint64_t i = 0; i < k; ++i) std::memcpy(out + 18 * i, rows.data() + 18 * i, 18 * sizeof(float));
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_solve_order(bgpu_world* w, uint64_t* out, uint64_t cap, uint64_t* out_n) {
    if (!w) return bad_args("bgpu_read_solve_order");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        std::vector<uint64_t> keys;
        std::vector<float> rows;
        if (W.solved_standalone) gather_solve_order(W, W.standalone_groups, W.standalone_keys.p, keys, rows);
        else gather_solve_order(W, W.npairs, W.pairs.p, keys, rows);
        if (out_n) *out_n = keys.size();
        uint64_t k = std::min<uint64_t>(cap, keys.size());
        if (out && k) std::memcpy(out, keys.data(), k * sizeof(uint64_t));
        return BGPU_OK;
    });
}

void bgpu_spring2_desc_default(bgpu_spring2_desc* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->flags = BGPU_JOINT_DISABLE_COLLISIONS;
    o->rotate_order = BGPU_ROTATE_XYZ;
    const float ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int k = 0; k < 9; ++k) o->frame_a[3 + k] = o->frame_b[3 + k] = ident[k];
    for (int i = 0; i < 6; ++i) {
        bgpu_spring2_axis& a = o->axis[i];
        const bool angular = i >= 3;
        a.lower_limit = angular ? 1.0f : 0.0f;
        a.upper_limit = angular ? -1.0f : 0.0f;
        a.stop_erp = 0.2f;
        a.motor_erp = 0.9f;
        a.max_motor_force = angular ? 6.0f : 0.0f;
    }
}

namespace {
// shared.rs:17-27 (normalize_angle) on the host
float normalize_angle_host(float angle) {
    const float pi = 3.14159265358979323846f, two_pi = 2.0f * pi;
    float a = std::fmod(angle, two_pi);
    if (a < -pi) a += two_pi;
    else if (a > pi) a -= two_pi;
    return a;
}
// shared.rs:85-101 (euler_xyz) on the host
bgpu::V3 euler_xyz_host(const bgpu::M3& m) {
    const float half_pi = 1.57079632679489661923f;
    const float r20 = m.c0.z, r21 = m.c1.z, r22 = m.c2.z, r10 = m.c0.y, r11 = m.c1.y, r01 = m.c1.x, r00 = m.c0.x;
    if (r20 < 1.0f) {
        if (r20 > -1.0f) return bgpu::V3{std::atan2(-r21, r22), std::asin(r20), std::atan2(-r10, r00)};
        return bgpu::V3{-std::atan2(r01, r11), -half_pi, 0.0f};
    }
    return bgpu::V3{std::atan2(r01, r11), half_pi, 0.0f};
}
}  // namespace

bgpu_status bgpu_spring2_hinge2(const float* pos_a, const float* quat_a, const float* pos_b, const float* quat_b,
                                const float* anchor, const float* axis1, const float* axis2, uint32_t body_a,
                                uint32_t body_b, bgpu_spring2_desc* out) {
    if (!pos_a || !quat_a || !pos_b || !quat_b || !anchor || !axis1 || !axis2 || !out) return bad_args("bgpu_spring2_hinge2");
    using bgpu::V3;
    using bgpu::M3;
    const V3 pa{pos_a[0], pos_a[1], pos_a[2]}, pb{pos_b[0], pos_b[1], pos_b[2]}, an{anchor[0], anchor[1], anchor[2]};
    const bgpu::Q qa{quat_a[0], quat_a[1], quat_a[2], quat_a[3]}, qb{quat_b[0], quat_b[1], quat_b[2], quat_b[3]};
    // generic6dof_spring2.rs:338-350: axis1 is the frame z, axis2 the frame x, y = z x x
    const V3 z_axis = bgpu::normalize(V3{axis1[0], axis1[1], axis1[2]});
    const V3 x_axis = bgpu::normalize(V3{axis2[0], axis2[1], axis2[2]});
    const V3 y_axis = bgpu::cross(z_axis, x_axis);
    const M3 basis{x_axis, y_axis, z_axis};
    const M3 rot_a = bgpu::from_quat(qa), rot_b = bgpu::from_quat(qb);
    const M3 ba = bgpu::mul(bgpu::transpose(rot_a), basis), bb = bgpu::mul(bgpu::transpose(rot_b), basis);
    const V3 oa = bgpu::mul(bgpu::transpose(rot_a), an - pa), ob = bgpu::mul(bgpu::transpose(rot_b), an - pb);
    bgpu_spring2_desc_default(out);
    out->body_a = body_a;
    out->body_b = body_b;
    auto put = [](float* f, const V3& o, const M3& m) {
        const V3 c[4] = {o, m.c0, m.c1, m.c2};
        for (int k = 0; k < 4; ++k) { f[3 * k] = c[k].x; f[3 * k + 1] = c[k].y; f[3 * k + 2] = c[k].z; }
    };
    put(out->frame_a, oa, ba);
    put(out->frame_b, ob, bb);
    // :352-362: linear x/y locked, z over [-1, 1]; angular x free, y locked, z +-pi/4
    out->axis[2].lower_limit = -1.0f;
    out->axis[2].upper_limit = 1.0f;
    const float steer = 1.57079632679489661923f * 0.5f;
    const float lo[3] = {1.0f, 0.0f, -steer}, hi[3] = {-1.0f, 0.0f, steer};
    for (int i = 0; i < 3; ++i) {
        out->axis[3 + i].lower_limit = normalize_angle_host(lo[i]);
        out->axis[3 + i].upper_limit = normalize_angle_host(hi[i]);
    }
    // :363-367: the suspension spring on linear z
    const float pi = 3.14159265358979323846f;
    out->axis[2].flags |= BGPU_S2_SPRING | BGPU_S2_STIFFNESS_LIMITED | BGPU_S2_DAMPING_LIMITED;
    out->axis[2].stiffness = pi * pi * 4.0f;
    out->axis[2].damping = 0.01f;
    // :368-376: the equilibrium is the construction pose (pivot offset and XYZ Euler angles)
    const M3 tr_a = bgpu::mul(rot_a, ba), tr_b = bgpu::mul(rot_b, bb);
    const V3 pivot_a = pa + bgpu::rotate(qa, oa), pivot_b = pb + bgpu::rotate(qb, ob);
    const V3 diff = bgpu::mul(bgpu::transpose(tr_a), pivot_b - pivot_a);
    const V3 euler = euler_xyz_host(bgpu::mul(bgpu::transpose(tr_a), tr_b));
    for (int i = 0; i < 3; ++i) {
        out->axis[i].equilibrium_point = bgpu::comp(diff, i);
        out->axis[3 + i].equilibrium_point = bgpu::comp(euler, i);
    }
    return BGPU_OK;
}

bgpu_status bgpu_add_spring2_joints(bgpu_world* w, uint32_t n, const bgpu_spring2_desc* d, uint32_t* first_id) {
    if (!w || (n && !d)) return bad_args("bgpu_add_spring2_joints");
    return guarded([&]() -> bgpu_status {
        uint32_t f = w->impl.add_spring2_joints(n, d);
        if (first_id) *first_id = f;
        return BGPU_OK;
    });
}

bgpu_status bgpu_add_generic6dof_joints(bgpu_world* w, uint32_t n, const bgpu_spring2_desc* d, uint32_t* first_id) {
    if (!w || (n && !d)) return bad_args("bgpu_add_generic6dof_joints");
    return guarded([&]() -> bgpu_status {
        uint32_t f = w->impl.add_spring2_joints(n, d, BGPU_JOINT_GENERIC6DOF);
        if (first_id) *first_id = f;
        return BGPU_OK;
    });
}

bgpu_status bgpu_generic6dof_universal(const float* pos_a, const float* quat_a, const float* pos_b, const float* quat_b,
                                       const float* anchor, const float* axis1, const float* axis2, uint32_t body_a,
                                       uint32_t body_b, bgpu_spring2_desc* out) {
    if (!pos_a || !quat_a || !pos_b || !quat_b || !anchor || !axis1 || !axis2 || !out) return bad_args("bgpu_generic6dof_universal");
    using bgpu::V3;
    using bgpu::M3;
    const V3 pa{pos_a[0], pos_a[1], pos_a[2]}, pb{pos_b[0], pos_b[1], pos_b[2]}, an{anchor[0], anchor[1], anchor[2]};
    const bgpu::Q qa{quat_a[0], quat_a[1], quat_a[2], quat_a[3]}, qb{quat_b[0], quat_b[1], quat_b[2], quat_b[3]};
    // generic6dof.rs:168-176: axis1 is the frame z, axis2 the frame y, x = y x z
    const V3 z_axis = bgpu::normalize(V3{axis1[0], axis1[1], axis1[2]});
    const V3 y_axis = bgpu::normalize(V3{axis2[0], axis2[1], axis2[2]});
    const V3 x_axis = bgpu::cross(y_axis, z_axis);
    const M3 basis{x_axis, y_axis, z_axis};
    const M3 rot_a = bgpu::from_quat(qa), rot_b = bgpu::from_quat(qb);
    const M3 ba = bgpu::mul(bgpu::transpose(rot_a), basis), bb = bgpu::mul(bgpu::transpose(rot_b), basis);
    const V3 oa = bgpu::mul(bgpu::transpose(rot_a), an - pa), ob = bgpu::mul(bgpu::transpose(rot_b), an - pb);
    bgpu_spring2_desc_default(out);
    out->body_a = body_a;
    out->body_b = body_b;
    auto put = [](float* f, const V3& o, const M3& m) {
        const V3 c[4] = {o, m.c0, m.c1, m.c2};
        for (int k = 0; k < 4; ++k) { f[3 * k] = c[k].x; f[3 * k + 1] = c[k].y; f[3 * k + 2] = c[k].z; }
    };
    put(out->frame_a, oa, ba);
    put(out->frame_b, ob, bb);
    // :181-188: linear locked; angular x locked, y within +-(pi/2 - 0.01), z within +-(pi - 0.01)
    const float half_pi = 1.57079632679489661923f, pi = 3.14159265358979323846f;
    const float lo[3] = {0.0f, -half_pi + 0.01f, -pi + 0.01f}, hi[3] = {0.0f, half_pi - 0.01f, pi - 0.01f};
    for (int i = 0; i < 3; ++i) {
        out->axis[i].lower_limit = 0.0f;
        out->axis[i].upper_limit = 0.0f;
        out->axis[3 + i].lower_limit = normalize_angle_host(lo[i]);
        out->axis[3 + i].upper_limit = normalize_angle_host(hi[i]);
    }
    return BGPU_OK;
}

bgpu_status bgpu_read_joint_spring2_state(bgpu_world* w, float* state) {
    if (!w || !state) return bad_args("bgpu_read_joint_spring2_state");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        const size_t nj = W.joints_h.size();
        if (!nj) return BGPU_OK;
        bgpu::check_cuda(cudaMemcpyAsync(state, W.joint_s2_state_d.p, 2 * nj * sizeof(float4), cudaMemcpyDeviceToHost,
                                         W.stream), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_set_ccd(bgpu_world* w, uint32_t first, uint32_t n, const float* motion_threshold,
                         const float* swept_sphere_radius) {
    if (!w || (n && (!motion_threshold || !swept_sphere_radius))) return bad_args("bgpu_set_ccd");
    return guarded([&]() -> bgpu_status {
        w->impl.set_ccd(first, n, motion_threshold, swept_sphere_radius);
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_ccd_clamps(bgpu_world* w, float* clamps) {
    if (!w || !clamps) return bad_args("bgpu_read_ccd_clamps");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        for (uint32_t i = 0; i < W.n; ++i) clamps[i] = 1.0f;
        if (!W.nccd) return BGPU_OK;
        std::vector<float> c(W.nccd);
        bgpu::check_cuda(cudaMemcpyAsync(c.data(), W.ccd_clamp_d.p, W.nccd * sizeof(float), cudaMemcpyDeviceToHost,
                                         W.stream), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        for (uint32_t k = 0; k < W.nccd; ++k) clamps[W.ccd_ids_h[k]] = c[k];
        return BGPU_OK;
    });
}

bgpu_status bgpu_add_joints(bgpu_world* w, uint32_t n, const bgpu_joint_desc* d, uint32_t* first_id) {
    if (!w || (n && !d)) return bad_args("bgpu_add_joints");
    return guarded([&]() -> bgpu_status {
        uint32_t f = w->impl.add_joints(n, d);
        if (first_id) *first_id = f;
        return BGPU_OK;
    });
}

uint32_t bgpu_num_joints(bgpu_world* w) { return w ? uint32_t(w->impl.joints_h.size()) : 0u; }

bgpu_status bgpu_set_joint_flags(bgpu_world* w, uint32_t id, uint32_t flags) {
    if (!w) return bad_args("bgpu_set_joint_flags");
    return guarded([&]() -> bgpu_status {
        w->impl.set_joint_flags(id, flags);
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_joint_angles(bgpu_world* w, float* angles) {
    if (!w || !angles) return bad_args("bgpu_read_joint_angles");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        const size_t nj = W.joints_h.size();
        if (!nj) return BGPU_OK;
        bgpu::check_cuda(cudaMemcpyAsync(angles, W.joint_angle_d.p, nj * sizeof(float), cudaMemcpyDeviceToHost, W.stream),
                         "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_joint_positions(bgpu_world* w, float* positions) {
    if (!w || !positions) return bad_args("bgpu_read_joint_positions");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        const size_t nj = W.joints_h.size();
        if (!nj) return BGPU_OK;
        bgpu::check_cuda(cudaMemcpyAsync(positions, W.joint_pos_d.p, nj * sizeof(float), cudaMemcpyDeviceToHost,
                                         W.stream), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_joint_order(bgpu_world* w, uint32_t* ids, uint32_t cap, uint32_t* out_n) {
    if (!w) return bad_args("bgpu_read_joint_order");
    const auto& o = w->impl.joint_order_h;
    if (out_n) *out_n = uint32_t(o.size());
    const uint32_t k = std::min<uint32_t>(cap, uint32_t(o.size()));
    if (ids && k) std::memcpy(ids, o.data(), k * sizeof(uint32_t));
    return BGPU_OK;
}

bgpu_status bgpu_read_joint_rows(bgpu_world* w, float* rows, uint32_t cap, uint32_t* out_n) {
    if (!w) return bad_args("bgpu_read_joint_rows");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        const uint32_t nj = uint32_t(W.joints_h.size());
        std::vector<uint32_t> cnt(nj);
        std::vector<float4> r(size_t(nj ? W.joint_row_off_h[nj] : 0) * bgpu::JROW_F4);
        if (nj) {
            bgpu::check_cuda(cudaMemcpyAsync(cnt.data(), W.joint_count_d.p, nj * 4, cudaMemcpyDeviceToHost, W.stream), "d2h");
            bgpu::check_cuda(cudaMemcpyAsync(r.data(), W.joint_rows_d.p, r.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                                             W.stream), "d2h");
            bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        }
        uint32_t total = 0;
        for (uint32_t t = 0; t < nj; ++t) {
            const bgpu_joint_desc& jd = W.joints_h[W.joint_order_h[t]];
            for (uint32_t k = 0; k < cnt[t]; ++k, ++total) {
                if (!rows || total >= cap) continue;
                const float4* x = &r[(size_t(W.joint_row_off_h[t]) + k) * bgpu::JROW_F4];
                float* o = rows + 8 * size_t(total);
                uint32_t lim;
                std::memcpy(&lim, &x[3].w, 4);
                o[0] = float(W.joint_order_h[t]); o[1] = float(jd.body_a); o[2] = float(jd.body_b);
                o[3] = x[0].w; o[4] = x[1].w; o[5] = float(lim); o[6] = x[4].z; o[7] = x[2].w;
            }
        }
        if (out_n) *out_n = total;
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_colour_batches(bgpu_world* w, uint32_t* groups, uint32_t* split_groups, uint32_t cap,
                                     uint32_t* out_n) {
    if (!w) return bad_args("bgpu_read_colour_batches");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        bgpu::PairData& pd = W.pd;
        cudaStream_t s = W.stream;
        uint32_t ncol = 0;
        if (W.npairs && pd.scalars.p && pd.colour_offset.p) {
            uint32_t sc[16];
            bgpu::check_cuda(cudaMemcpyAsync(sc, pd.scalars.p, sizeof(sc), cudaMemcpyDeviceToHost, s), "d2h");
            bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
            ncol = std::min<uint32_t>(sc[4], uint32_t(bgpu::MAX_COLOURS));
        }
        if (out_n) *out_n = ncol;
        const uint32_t k = std::min(cap, ncol);
        if (!k) return BGPU_OK;
        std::vector<uint32_t> off(k), end(k), soff(k), send(k);
        if (W.last_world_solver) {  // per-world solver: groups per colour summed over the worlds
            bgpu::check_cuda(cudaMemcpyAsync(end.data(), pd.colour_count.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
            bgpu::check_cuda(cudaMemcpyAsync(send.data(), pd.split_count.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
            bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
            for (uint32_t c = 0; c < k; ++c) {
                if (groups) groups[c] = end[c];
                if (split_groups) split_groups[c] = send[c];
            }
            return BGPU_OK;
        }
        bgpu::check_cuda(cudaMemcpyAsync(off.data(), pd.colour_offset.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(end.data(), pd.colour_cursor.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(soff.data(), pd.split_offset.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(send.data(), pd.split_cursor.p, k * 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        for (uint32_t c = 0; c < k; ++c) {
            if (groups) groups[c] = end[c] - off[c];
            if (split_groups) split_groups[c] = send[c] - soff[c];
        }
        return BGPU_OK;
    });
}

bgpu_status bgpu_get_stats(bgpu_world* w, bgpu_step_stats* out) {
    if (!w || !out) return bad_args("bgpu_get_stats");
    return guarded([&]() -> bgpu_status {
        w->impl.finish_stats();
        *out = w->impl.last;
        return BGPU_OK;
    });
}

bgpu_status bgpu_enable_step_timing(bgpu_world* w, int on) {
    if (!w) return bad_args("bgpu_enable_step_timing");
    return guarded([&]() -> bgpu_status {
        w->impl.finish_stats();
        w->impl.timing = on != 0;
        w->impl.reset_timing();
        return BGPU_OK;
    });
}

bgpu_status bgpu_broadphase_pairs(const float* aabbs, uint32_t n, uint32_t* out, uint64_t cap, uint64_t* out_n) {
    if (!aabbs && n) return bad_args("bgpu_broadphase_pairs");
    if (bgpu_device_count() == 0) {
        bgpu::g_last_error = "no CUDA device";
        return BGPU_ERR_NO_DEVICE;
    }
    return guarded([&]() -> bgpu_status {
        cudaStream_t s;
        bgpu::check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        } guard{s};
        std::vector<float4> mn(n), mx(n);
        std::vector<uint32_t> unb;
        for (uint32_t i = 0; i < n; ++i) {
            const float* a = aabbs + 6 * size_t(i);
            mn[i] = make_float4(a[0], a[1], a[2], 0.0f);
            mx[i] = make_float4(a[3], a[4], a[5], 0.0f);
            bool huge = false;
            for (int k = 0; k < 3; ++k) {
                float e = a[3 + k] - a[k];
                if (!(e < 1e15f)) huge = true;
            }
            if (huge) unb.push_back(i);
        }
        bgpu::DevBuf<float4> dmn, dmx;
        bgpu::DevBuf<uint64_t> pairs;
        bgpu::DevBuf<uint32_t> status;
        dmn.reserve(n + 1);
        dmx.reserve(n + 1);
        status.reserve(1);
        bgpu::check_cuda(cudaMemsetAsync(status.p, 0, 4, s), "memset");
        if (n) {
            bgpu::check_cuda(cudaMemcpyAsync(dmn.p, mn.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
            bgpu::check_cuda(cudaMemcpyAsync(dmx.p, mx.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s), "h2d");
        }
        bgpu::Broadphase bp;
        uint64_t np = bp.run(dmn.p, dmx.p, n, unb, pairs, status.p, s);
        uint32_t st = 0;
        bgpu::check_cuda(cudaMemcpyAsync(&st, status.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
        std::vector<uint64_t> keys(np);
        if (np)
            bgpu::check_cuda(cudaMemcpyAsync(keys.data(), pairs.p, np * 8, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        if (out_n) *out_n = np;
        uint64_t k = std::min<uint64_t>(cap, np);
        for (uint64_t i = 0; i < k && out; ++i) {
            out[2 * i] = bgpu::key_lo(keys[i]);
            out[2 * i + 1] = bgpu::key_hi(keys[i]);
        }
        if (st) {
            bgpu::g_last_error = "broad-phase traversal stack overflow";
            return BGPU_ERR_DEVICE_STATUS;
        }
        return BGPU_OK;
    });
}

bgpu_status bgpu_collide(bgpu_world* w, uint32_t n, const uint32_t* sa, const float* pa, const uint32_t* sb,
                         const float* pb, const float* seeds, int force_convex, float* out, uint32_t* counts) {
    if (!w || (n && (!sa || !pa || !sb || !pb || !out || !counts))) return bad_args("bgpu_collide");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        for (uint32_t i = 0; i < n; ++i)
            if (sa[i] >= W.shapes_h.size() || sb[i] >= W.shapes_h.size()) throw bgpu::InvalidArg{"shape id out of range"};
        W.sync_shapes();
        cudaStream_t s = W.stream;
        std::vector<float4> hpa(n), hqa(n), hpb(n), hqb(n), hs(n);
        for (uint32_t i = 0; i < n; ++i) {
            const float* a = pa + 7 * size_t(i);
            const float* b = pb + 7 * size_t(i);
            hpa[i] = make_float4(a[0], a[1], a[2], 0.0f);
            hqa[i] = make_float4(a[3], a[4], a[5], a[6]);
            hpb[i] = make_float4(b[0], b[1], b[2], 0.0f);
            hqb[i] = make_float4(b[3], b[4], b[5], b[6]);
            if (seeds) hs[i] = make_float4(seeds[3 * i], seeds[3 * i + 1], seeds[3 * i + 2], 0.0f);
        }
        bgpu::DevBuf<float4> d_pa, d_qa, d_pb, d_qb, d_seed, d_out;
        bgpu::DevBuf<uint32_t> d_sa, d_sb, d_cnt, d_status;
        size_t m = size_t(n) + 1;
        d_pa.reserve(m); d_qa.reserve(m); d_pb.reserve(m); d_qb.reserve(m); d_seed.reserve(m);
        d_out.reserve(m * 8); d_sa.reserve(m); d_sb.reserve(m); d_cnt.reserve(m); d_status.reserve(1);
        auto h2d = [&](void* dst, const void* src, size_t bytes) {
            if (bytes) bgpu::check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "h2d");
        };
        h2d(d_pa.p, hpa.data(), n * sizeof(float4));
        h2d(d_qa.p, hqa.data(), n * sizeof(float4));
        h2d(d_pb.p, hpb.data(), n * sizeof(float4));
        h2d(d_qb.p, hqb.data(), n * sizeof(float4));
        h2d(d_seed.p, hs.data(), n * sizeof(float4));
        h2d(d_sa.p, sa, n * 4);
        h2d(d_sb.p, sb, n * 4);
        bgpu::check_cuda(cudaMemsetAsync(d_status.p, 0, 4, s), "memset");
        bgpu::run_collide_queries(W.shapes_d.p, W.hull_d.p, n, d_sa.p, d_pa.p, d_qa.p, d_sb.p, d_pb.p, d_qb.p,
                                  seeds ? d_seed.p : nullptr, force_convex, d_out.p, d_cnt.p, d_status.p, s);
        bgpu::check_cuda(cudaGetLastError(), "collide launch");
        std::vector<float4> hout(size_t(n) * 8);
        uint32_t st = 0;
        if (n) {
            bgpu::check_cuda(cudaMemcpyAsync(hout.data(), d_out.p, hout.size() * sizeof(float4), cudaMemcpyDeviceToHost, s),
                             "d2h");
            bgpu::check_cuda(cudaMemcpyAsync(counts, d_cnt.p, n * 4, cudaMemcpyDeviceToHost, s), "d2h");
        }
        bgpu::check_cuda(cudaMemcpyAsync(&st, d_status.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        for (uint32_t i = 0; i < n; ++i) {
            for (uint32_t k = 0; k < counts[i] && k < 4; ++k) {
                float4 a = hout[(size_t(i) * 4 + k) * 2], b = hout[(size_t(i) * 4 + k) * 2 + 1];
                float* o = out + (size_t(i) * 4 + k) * 7;
                o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = b.x; o[4] = b.y; o[5] = b.z; o[6] = a.w;
            }
        }
        if (st) {
            bgpu::g_last_error = "narrow phase status bits set";
            return BGPU_ERR_DEVICE_STATUS;
        }
        return BGPU_OK;
    });
}

bgpu_status bgpu_solve_contacts(bgpu_world* w, uint32_t n, const float* contacts, float inv_dt, float* rows_out,
                                uint64_t* order_keys_out) {
    if (!w || (n && !contacts) || !(inv_dt > 0.0f)) return bad_args("bgpu_solve_contacts");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        W.finish_stats();
        W.sync_shapes();
        cudaStream_t s = W.stream;
        // Row groups: consecutive contacts of the same (body_a, body_b), at most four.
        std::vector<uint32_t> first, cnt;
        std::vector<uint64_t> keys;
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t a = uint32_t(contacts[10 * size_t(i)]), b = uint32_t(contacts[10 * size_t(i) + 1]);
            if (a >= W.n || b >= W.n || a == b) throw bgpu::InvalidArg{"contact body index out of range"};
            uint64_t key = (uint64_t(a) << 32) | b;
            if (!keys.empty() && keys.back() == key && cnt.back() < 4) {
                cnt.back()++;
            } else {
                first.push_back(i);
                cnt.push_back(1);
                keys.push_back(key);
            }
        }
        uint32_t G = uint32_t(keys.size());
        W.pd.reserve(std::max<uint32_t>(G, 1), W.n, 1);
        bgpu::DevBuf<uint32_t> d_first, d_cnt;
        bgpu::DevBuf<float> d_c;
        d_first.reserve(G + 1);
        d_cnt.reserve(G + 1);
        d_c.reserve(size_t(n) * 10 + 1);
        W.standalone_keys.reserve(G + 1);
        if (G) {
            bgpu::check_cuda(cudaMemcpyAsync(d_first.p, first.data(), G * 4, cudaMemcpyHostToDevice, s), "h2d");
            bgpu::check_cuda(cudaMemcpyAsync(d_cnt.p, cnt.data(), G * 4, cudaMemcpyHostToDevice, s), "h2d");
            bgpu::check_cuda(cudaMemcpyAsync(W.standalone_keys.p, keys.data(), G * 8, cudaMemcpyHostToDevice, s), "h2d");
            bgpu::check_cuda(cudaMemcpyAsync(d_c.p, contacts, size_t(n) * 10 * 4, cudaMemcpyHostToDevice, s), "h2d");
        }
        bgpu::check_cuda(cudaMemsetAsync(W.pd.row_count.p, 0, std::max<uint32_t>(G, 1) * 4, s), "memset");
        bgpu::check_cuda(cudaMemsetAsync(W.push_lin.p, 0, W.n * sizeof(float4), s), "memset");
        bgpu::check_cuda(cudaMemsetAsync(W.push_ang.p, 0, W.n * sizeof(float4), s), "memset");
        bgpu::check_cuda(cudaMemsetAsync(W.flags.p, 0, 4, s), "memset");
        bgpu::launch_compute_iw(W.body_dev(), W.n, s);
        bgpu::StepParams sp;
        sp.inv_dt = inv_dt;
        sp.dt = 1.0f / inv_dt;
        sp.info = W.info;
        bgpu::run_prepare_contacts(W.body_dev(), G, d_first.p, d_cnt.p, d_c.p, W.standalone_keys.p, sp, W.pd.rows.p,
                                   W.pd.row_count.p, s);
        bgpu::run_solver(W.view(), W.standalone_keys.p, G, W.pd, sp, W.flags.p, s, [](int) {}, false);
        bgpu::check_cuda(cudaGetLastError(), "solve launch");
        uint32_t st = 0;
        bgpu::check_cuda(cudaMemcpyAsync(&st, W.flags.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(s), "sync");
        W.solved_standalone = 1;
        W.standalone_groups = G;
        std::vector<uint64_t> okeys;
        std::vector<float> rows;
        gather_solve_order(W, G, W.standalone_keys.p, okeys, rows);
        if (rows_out) std::memcpy(rows_out, rows.data(), rows.size() * sizeof(float));
        if (order_keys_out) std::memcpy(order_keys_out, okeys.data(), okeys.size() * sizeof(uint64_t));
        if (st) {
            char buf[96];
            std::snprintf(buf, sizeof(buf), "device status bits 0x%x", st);
            bgpu::g_last_error = buf;
            return BGPU_ERR_DEVICE_STATUS;
        }
        return BGPU_OK;
    });
}

bgpu_status bgpu_read_push(bgpu_world* w, float* out) {
    if (!w || !out) return bad_args("bgpu_read_push");
    return guarded([&]() -> bgpu_status {
        World& W = w->impl;
        uint32_t n = W.n;
        std::vector<float4> pl(n), pa(n);
        bgpu::check_cuda(cudaMemcpyAsync(pl.data(), W.push_lin.p, n * sizeof(float4), cudaMemcpyDeviceToHost, W.stream), "d2h");
        bgpu::check_cuda(cudaMemcpyAsync(pa.data(), W.push_ang.p, n * sizeof(float4), cudaMemcpyDeviceToHost, W.stream), "d2h");
        bgpu::check_cuda(cudaStreamSynchronize(W.stream), "sync");
        for (uint32_t i = 0; i < n; ++i) {
            float* o = out + 6 * size_t(i);
            o[0] = pl[i].x; o[1] = pl[i].y; o[2] = pl[i].z; o[3] = pa[i].x; o[4] = pa[i].y; o[5] = pa[i].z;
        }
        return BGPU_OK;
    });
}

}  // extern "C"
