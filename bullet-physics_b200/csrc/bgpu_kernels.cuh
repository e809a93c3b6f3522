// Host-side declarations shared by the kernel translation units and the world.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>
#include "bgpu_world.cuh"

namespace bgpu {

// ---------------------------------------------------------------- device buffers
struct CudaError {
    cudaError_t code;
    std::string where;
};

void check_cuda(cudaError_t e, const char* where);  // throws CudaError
void set_last_error(const std::string& msg);         // text returned by bgpu_last_error

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    size_t cap_hint = 0;  // capacity before the last growth
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cap_hint = 0;
    }
    void release_keep_cap() {
        cap_hint = cap;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    // Grow to at least n elements (contents are not preserved). Growth is
    // geometric, so a scene whose pair or contact counts creep up step by step
    // reallocates (and synchronises in cudaFree) only a few times.
    void reserve(size_t n) {
        if (n <= cap) return;
        release_keep_cap();
        size_t c = n < 16 ? 16 : n;
        if (c < cap_hint + cap_hint / 2) c = cap_hint + cap_hint / 2;
        check_cuda(cudaMalloc(&p, c * sizeof(T)), "cudaMalloc");
        cap = c;
    }
    // Grow to at least n elements, preserving the first `keep` elements.
    void grow_keep(size_t n, size_t keep, cudaStream_t s) {
        if (n <= cap) return;
        size_t c = n < 16 ? 16 : n;
        T* q = nullptr;
        check_cuda(cudaMalloc(&q, c * sizeof(T)), "cudaMalloc");
        if (p && keep) check_cuda(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s), "copy");
        if (p) {
            check_cuda(cudaStreamSynchronize(s), "sync");
            cudaFree(p);
        }
        p = q;
        cap = c;
    }
};

// ---------------------------------------------------------------- device helpers shared by the solver and its adjoint
constexpr unsigned int BARRIER_SPIN_LIMIT = 1u << 26;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;  // 2 s: phases take microseconds

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Barrier of a team of co-resident blocks (a cooperative launch) on a counter
// that only grows during the launch: the k-th barrier (k from 1) of a team of
// n blocks completes when the counter reaches k * n. One atomic per block,
// then a tight spin. The spin is bounded in time (limit_ns, measured from the
// 64th poll on the global timer, with a poll count as a second bound): when it
// gives up the status word records ST_BARRIER_TIMEOUT, and every block's spin
// also gives up within 64 polls once the word shows it, so no launch can hang
// the device and the host reads the error. The status word is not read before
// the arrival: that read would put an L2 round trip in front of every barrier.
// (Spinning on relaxed loads with one acquire fence at the end measured slower.)
__device__ __forceinline__ void team_barrier(unsigned int* ctr, unsigned int target, uint32_t* status,
                                             unsigned long long limit_ns = BARRIER_TIMEOUT_NS) {
    __syncthreads();
    if (threadIdx.x == 0) {
        // The release add publishes the block's writes (ordered before it by the
        // bar.sync above); the acquire load makes the other blocks' writes visible.
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(ctr) : "memory");
        unsigned int v, spins = 0;
        unsigned long long t0 = 0;
        for (;;) {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
            if (v >= target) break;
            if ((++spins & 63u) == 0u) {
                const unsigned long long now = globaltimer_ns();
                if (t0 == 0) t0 = now;
                if ((*(volatile uint32_t*)status & ST_BARRIER_TIMEOUT) || now - t0 > limit_ns ||
                    spins > BARRIER_SPIN_LIMIT) {
                    atomicOr(status, ST_BARRIER_TIMEOUT);
                    break;
                }
            }
        }
    }
    __syncthreads();
}

// PGS colours per step (a colouring that needs more records ST_COLOUR_OVERFLOW).
constexpr int MAX_COLOURS = 128;

// Per-step contact tables in batch-slot order. Slots are grouped 32 at a time
// (colour batches start on a multiple of 32, so a warp's lanes hold exactly one
// such group), and each group stores field ("plane") by field and contact by
// contact, 32 float4 per (plane, contact): element (plane, k, t) sits at
// ((t / 32 * PLANES + plane) * 4 + k) * 32 + t % 32. A warp's loads are
// coalesced and everything one warp reads in a sweep lies in one contiguous
// span of at most 30 KB, so scattered page (TLB) lookups stay few. The first
// sweep of each team fills its table from the rows and the bodies' inverse
// inertia; the later sweeps read only the table and the velocities. A slot's
// table entries are written and read by the same thread only (the slot-to-thread
// deal is fixed for the launch), so plain L1-cached loads see them; they are
// never read through the read-only (non-coherent) path, since this kernel
// writes them.
//
// Velocity table planes: 0 n|friction 1 r_a|bias 2 r_b|bias 3 t1|1/m_a
// 4 Iw_a(r_a x n)|normal mass 5 Iw_b(r_b x n)|t1 mass 6 Iw_a(r_a x t1)|t2 mass
// 7 Iw_b(r_b x t1)|cfm 8 Iw_a(r_a x t2)|restitution 9 Iw_b(r_b x t2)|1/m_b
// 10 accumulated impulses (row 3). The second tangent t2 = n x t1 and the velocity couplings
// kn / kt1 / kt2 are recomputed by each sweep with the same operations that first made them
// (so their values are the same), which keeps a large pile's table (176 B per contact) inside L2.
// Split table planes: 0 n|normal mass 1 r_a|cfm 2 r_b 3 Iw_a(r_a x n)|1/m_a
// 4 Iw_b(r_b x n)|1/m_b 5 row 5 (rhs, push impulse, active, penetration).
constexpr uint32_t VT_PLANES = 11;
enum : uint32_t { VT_N = 0, VT_RA = 1, VT_RB = 2, VT_T1 = 3, VT_ANA = 4, VT_ANB = 5, VT_A1A = 6, VT_A1B = 7,
                  VT_A2A = 8, VT_A2B = 9, VT_IMP = 10 };
constexpr uint32_t ST_PLANES = 6;

// Adjoint sweep record of (sweep >= 1, contact k, slot t), in 32-slot blocks like the tables.
__device__ __forceinline__ size_t sweep_index(uint32_t sweep, uint32_t k, uint32_t t, uint32_t iters) {
    return ((size_t(t >> 5) * iters + (sweep - 1)) * 4 + k) * 32 + (t & 31u);
}

template <uint32_t PLANES>
__device__ __forceinline__ size_t tix(uint32_t plane, uint32_t k, uint32_t t) {
    return ((size_t(t >> 5) * PLANES + plane) * 4 + k) * 32 + (t & 31u);
}

// float4 between consecutive planes of one (contact, slot): plane p of (k, t) is
// tab[tix<PLANES>(0, k, t) + p * PLANE_STRIDE], a constant offset the loads fold in.
constexpr uint32_t PLANE_STRIDE = 4 * 32;

// ---------------------------------------------------------------- body kernels (k_body.cu)
void launch_integrate_velocities(const BodyDev& b, const Shape* shapes, const float4* hull, uint32_t n, float dt,
                                 cudaStream_t s);
void launch_initial_aabbs(const BodyDev& b, const Shape* shapes, const float4* hull, uint32_t first, uint32_t n,
                          cudaStream_t s);
void launch_integrate_positions(const BodyDev& b, uint32_t n, float dt, float turn_erp, cudaStream_t s);
// CCD swept-sphere clamp (step.rs:1068-1155): clamp[k] for the bodies ids[0..m) (par: motion
// threshold, swept-sphere radius), scanning the bodies of each one's world (all n when world_of is
// null); then, after the position integration, the clamp applied (step.rs:1210-1214).
void launch_ccd_sweep(const BodyDev& b, const Shape* shapes, const float4* hull, const uint32_t* ids, const float2* par,
                      uint32_t m, uint32_t n, const uint32_t* world_off, const uint32_t* world_of,
                      const uint64_t* suppressed, uint32_t nsuppressed, float dt, float* clamp, uint32_t* status,
                      const float4* tree_rec, const uint32_t* tree_leaf, int tree_m, const uint32_t* unb,
                      uint32_t nunb, cudaStream_t s);
void launch_ccd_apply(const BodyDev& b, const uint32_t* ids, const float* clamp, uint32_t m, float dt, cudaStream_t s);
// Host-facing layouts: n x 3 floats -> float4 lanes, and poses -> n x 7 floats.
void launch_unpack3(uint32_t n, const float* src, float4* dst, cudaStream_t s);
void launch_pack_poses(uint32_t n, const float4* pos, const float4* quat, float* out, cudaStream_t s);

// ---------------------------------------------------------------- broad phase (k_broadphase.cu)
// Sorted closed-overlap pairs of n AABBs. `unbounded` lists (ascending) the
// proxies kept out of the tree (planes, +-1e30 boxes); they are tested
// against every proxy by an ordered compaction.
struct Broadphase {
    DevBuf<uint64_t> keys, keys_alt;
    DevBuf<uint32_t> leaf_body, parent, left, right, counts, offsets, refit_flag, flags, scan_out, unbounded;
    DevBuf<uint32_t> stash, overflow;  // partners of proxies with few of them; proxies with many
    DevBuf<float4> node_min, node_max;
    DevBuf<uint32_t> node_maxid;       // largest body index below each node
    DevBuf<float4> node_rec;           // per internal node: both children's boxes and references
    DevBuf<unsigned char> cub_tmp;
    DevBuf<int> bounds;          // 6 ordered ints: scene min/max of leaf centres
    DevBuf<uint32_t> scalars;    // [0] total pairs, [1] proxies with more partners than the stash holds
    uint32_t* host_scalars = nullptr;  // pinned
    int tree_m = 0;                    // bounded proxies in the last run's tree (0: no tree)
    uint32_t nunb = 0;                 // proxies of the last run kept out of the tree (device list `unbounded`)
    Broadphase();
    ~Broadphase();
    // Returns the pair count; pairs are written to `out` (grown as needed).
    uint64_t run(const float4* aabb_min, const float4* aabb_max, uint32_t n, const std::vector<uint32_t>& unbounded_host,
                 DevBuf<uint64_t>& out, uint32_t* status_dev, cudaStream_t s);
    // Batched worlds: pairs only inside each world [world_off[k], world_off[k + 1]) (device array).
    uint64_t run_worlds(const float4* aabb_min, const float4* aabb_max, uint32_t n, const uint32_t* world_off,
                        uint32_t n_worlds, DevBuf<uint64_t>& out, cudaStream_t s);
};

// ---------------------------------------------------------------- islands (k_islands.cu)
// ---------------------------------------------------------------- joints (k_joints.cu)
// Joint descriptor on the device, JOINT_F4 float4 per joint id: [0] kind, body a, body b,
// flags (as bits); [1] frame A origin; [2..4] frame A basis columns; [5] frame B origin;
// [6..8] frame B basis columns; [9] erp, impulse clamp, limit low, limit high;
// [10] softness, bias factor, relaxation, motor target velocity; [11] motor max impulse, gear ratio;
// slider: [12] linear limits low/high, angular limits low/high; [13] softness lim lin/ang, damping
// lim lin/ang; [14] softness ortho lin/ang, linear motor target/max force; [15] angular motor;
// cone twist: [12] swing spans 1 and 2, twist span, softness; [13] bias, relaxation, motor max
// impulse; [14] motor target quaternion;
// spring 2: [9].x first float4 of the joint's axis table in JointsDev::aux, [9].y rotate order.
constexpr uint32_t JOINT_F4 = 16;
// Row capacity of a joint of every kind but spring 2, whose capacity follows its axis settings.
constexpr uint32_t JOINT_MAX_ROWS = 6;
// Spring-2 axis table (generic6dof_spring2.rs:47-232), S2_AXIS_F4 float4 per axis, axes 0-2
// linear and 3-5 angular: [0] lower, upper, bounce, stop erp; [1] stop cfm, motor erp, motor cfm,
// target velocity; [2] max motor force, servo target, stiffness, damping; [3] equilibrium point,
// axis flags (S2_*), 0, 0.
constexpr uint32_t S2_AXIS_F4 = 4;
enum : uint32_t { S2_MOTOR = 1u, S2_SERVO = 2u, S2_SPRING = 4u, S2_STIFFNESS_LIMITED = 8u, S2_DAMPING_LIMITED = 16u,
                  S2_STOP_ERP = 32u, S2_STOP_CFM = 64u, S2_MOTOR_ERP = 128u, S2_MOTOR_CFM = 256u };
// Joint row, JROW_F4 float4: [0] lin_a | effective mass, [1] ang_a | bias, [2] lin_b | cfm,
// [3] ang_b | limit kind (bits), [4] lower, upper, accumulated impulse, 0.
constexpr uint32_t JROW_F4 = 5;
enum : uint32_t { JK_POINT2POINT = 0, JK_FIXED = 1, JK_HINGE = 2, JK_GEAR = 3, JK_SLIDER = 4, JK_SPRING2 = 5, JK_CONETWIST = 6,
                  JK_GENERIC6DOF = 7 };
enum : uint32_t { JF_DISABLE_COLLISIONS = 1u, JF_DISABLED = 2u, JF_ANGULAR_ONLY = 4u, JF_LIMIT = 8u, JF_MOTOR = 16u, JF_ERP = 32u,
                  JF_LIN_MOTOR = 64u, JF_ANG_MOTOR = 128u, JF_FRAME_B = 256u,
                  JF_CONE_MOTOR = 512u };
enum : uint32_t { JL_UNBOUNDED = 0, JL_BILATERAL = 1, JL_LOWER = 2, JL_UPPER = 3, JL_WINDOW = 4 };

struct JointsDev {
    const float4* desc = nullptr;    // JOINT_F4 per joint id
    const uint32_t* order = nullptr; // solve slot -> joint id (joint colour by colour)
    const uint32_t* coff = nullptr;  // joint colour c owns slots [coff[c], coff[c + 1])
    uint32_t n = 0, ncol = 0;
    float4* rows = nullptr;          // JROW_F4 per row; slot t's rows start at row row_off[t]
    const uint32_t* row_off = nullptr;  // first row of each slot (its capacity ends at row_off[t + 1])
    uint32_t* count = nullptr;       // rows per slot this step
    float* angle = nullptr;          // hinge angle / slider angular position per joint id
    float* position = nullptr;       // slider linear position per joint id
    const float4* aux = nullptr;     // spring-2 axis tables (S2_AXIS_F4 per axis, 6 axes per joint)
    float4* s2_state = nullptr;      // spring 2, 8 floats per joint id: Euler angles, pivot offset, fact_a, static
    float global_cfm = 0.0f;         // SolverInfo::global_cfm, the spring-2 rows' default compliance
};

// Rows of every joint for this step, from the current poses (constraint.rs:755-842).
void launch_joint_rows(const BodyDev& b, const JointsDev& j, float inv_dt, float erp, cudaStream_t s);

// solve_joint_row (sequential_impulse.rs:931-971) over the rows of one joint slot; the
// two bodies' velocities come from and go back to L2 (dynamic bodies only).
// SHARED: linvel / angvel point into shared memory (the per-world solver), not global memory.
template <bool SHARED = false>
__device__ __forceinline__ void solve_joint_slot(const JointsDev& jd, uint32_t t, float4* linvel, float4* angvel,
                                                 const float4* __restrict__ iw, float damping) {
    const uint32_t cnt = jd.count[t];
    if (!cnt) return;
    const uint32_t jid = jd.order[t];
    const float4 h = jd.desc[size_t(jid) * JOINT_F4];
    const uint32_t ia = __float_as_uint(h.y), ib = __float_as_uint(h.z);
    auto load_iw_j = [&](uint32_t i, float& im) {
        const float4 x = iw[3 * i], y = iw[3 * i + 1], z = iw[3 * i + 2];
        im = z.y;
        return M3{V3{x.x, x.y, x.z}, V3{x.w, y.x, y.y}, V3{y.z, y.w, z.x}};
    };
    float ima, imb;
    const M3 iia = load_iw_j(ia, ima), iib = load_iw_j(ib, imb);
    V3 la, wa, lb, wb;
    if (SHARED) {
        la = from4(linvel[ia]); wa = from4(angvel[ia]);
        lb = from4(linvel[ib]); wb = from4(angvel[ib]);
    } else {
        la = from4(__ldcg(&linvel[ia])); wa = from4(__ldcg(&angvel[ia]));
        lb = from4(__ldcg(&linvel[ib])); wb = from4(__ldcg(&angvel[ib]));
    }
    float4* row = jd.rows + size_t(jd.row_off[t]) * JROW_F4;
    for (uint32_t r = 0; r < cnt; ++r, row += JROW_F4) {
        const float4 r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3], r4 = row[4];
        const V3 lin_a = from4(r0), ang_a = from4(r1), lin_b = from4(r2), ang_b = from4(r3);
        const float mass = r0.w, bias = r1.w, cfm = r2.w;
        const uint32_t lim = __float_as_uint(r3.w);
        const float row_vel = (dot(lin_b, lb) + dot(ang_b, wb)) - (dot(lin_a, la) + dot(ang_a, wa));
        const float old = r4.z;
        const float base = damping != 1.0f ? mass * (bias - row_vel * damping) : mass * (bias - row_vel);
        const float lambda = cfm != 0.0f ? base - cfm * old : base;
        float nw = old + lambda;
        if (lim == JL_BILATERAL) nw = fminf(fmaxf(nw, -r4.y), r4.y);
        else if (lim == JL_LOWER) nw = fmaxf(nw, r4.x);
        else if (lim == JL_UPPER) nw = fminf(nw, r4.y);
        else if (lim == JL_WINDOW) nw = fminf(fmaxf(nw, r4.x), r4.y);
        row[4] = make_float4(r4.x, r4.y, nw, 0.0f);
        const float j = nw - old;
        if (j != 0.0f) {
            la -= lin_a * (j * ima);
            lb += lin_b * (j * imb);
            wa -= mul(iia, ang_a * j);
            wb += mul(iib, ang_b * j);
        }
    }
    if (SHARED) {
        if (ima > 0.0f) { linvel[ia] = to4(la, 0.0f); angvel[ia] = to4(wa, 0.0f); }
        if (imb > 0.0f) { linvel[ib] = to4(lb, 0.0f); angvel[ib] = to4(wb, 0.0f); }
    } else {
        if (ima > 0.0f) { __stcg(&linvel[ia], to4(la, 0.0f)); __stcg(&angvel[ia], to4(wa, 0.0f)); }
        if (imb > 0.0f) { __stcg(&linvel[ib], to4(lb, 0.0f)); __stcg(&angvel[ib], to4(wb, 0.0f)); }
    }
}

struct Islands {
    DevBuf<uint32_t> parent, awake, need;
    // simulate_flag[world] is raised when the world has an active body; world_of
    // (per body) is null for a single world. Enabled joints between two dynamic bodies
    // link their islands (islands.rs:186-196).
    void run(const BodyDev& b, uint32_t n, const uint64_t* pairs, uint32_t npairs, const uint32_t* world_of,
             uint32_t* simulate_flag, uint32_t* status_dev, cudaStream_t s, const float4* joint_desc = nullptr,
             uint32_t njoints = 0);
};

// ---------------------------------------------------------------- pair pass + solver (k_pairs.cu, k_solver.cu)
struct StepParams {
    float dt, inv_dt;
    SolverParams info;
    const uint64_t* suppressed = nullptr;  // sorted keys of pairs whose collisions a joint disables
    uint32_t nsuppressed = 0;
};

constexpr uint32_t REC_NONE = 0xffffffffu;

// Records of one forward step for the adjoint (every pointer null when not recording).
struct RecordDev {
    uint8_t* pt_src = nullptr;    // per pair x 4: index, in the old cache entry, of each point the pair pass
                                  // stored before the narrow phase (0xff: none)
    uint32_t* pair_old = nullptr;  // per pair: position of its manifold in the old cache, or REC_NONE
    uint32_t* row_src = nullptr;   // per pair x 4: old cache position * 4 + point whose impulse warm-started
                                   // the row, or REC_NONE
    uint32_t* merge_pos = nullptr;  // per pair: position of its manifold in the merged cache, or REC_NONE
    float4* sweeps = nullptr;       // per (sweep, slot, contact): normal velocity, normal impulse, clamp bits
};

// Raw device pointers of PairData, passed to kernels by value.
struct PairDataDev {
    uint32_t* status;
    float4* entries;
    float4* detect;
    uint32_t* detect_n;
    uint32_t* row_count;
    float4* rows;
    uint32_t* route_list;
    uint32_t* old_owned;
    uint32_t* scalars;
    RecordDev rec;
};

constexpr uint32_t ROUTE_COUNT0 = 16;  // first per-route counter in PairData::scalars
constexpr uint32_t CAPTURE_COUNT = ROUTE_COUNT0 + NP_MESH + 1;  // detections with points (capture list length)
constexpr uint32_t CAPTURE_LIST = NP_MESH;  // the capture list is route_list region [8 P, 9 P)

struct PairData {
    // Per pair (indexed like the sorted pair array).
    DevBuf<uint32_t> status;       // PS_* | route << 8
    DevBuf<float4> entries;        // new manifolds (ENTRY_F4 per pair)
    DevBuf<float4> detect;         // fresh detections: 2 float4 per point (pos,pen | normal,-), 4 points
    DevBuf<uint32_t> detect_n;     // points per fresh detection
    DevBuf<uint32_t> row_count;    // solver rows per pair (0..4)
    DevBuf<float4> rows;           // ROW_F4 per contact slot, 4 slots per pair
    DevBuf<uint32_t> route_list;   // pairs needing detection, one list per route r: [(r - 1) P, r P);
                                   // then [7 P, 8 P): the detections that found points
    DevBuf<uint32_t> old_owned;    // per old manifold: 1 when a current pair took it over
    DevBuf<uint32_t> scalars;      // [0] analytic count [1] convex count [2] contact pairs [3] contacts
                                   // [4] colours [5] split pairs [6] detect total [7] manifolds
                                   // [8] [9] cache compaction counts [10] split contacts [11] largest split batch
                                   // [ROUTE_COUNT0 + r] pairs on narrow-phase route r [CAPTURE_COUNT]
    // Solver batches
    DevBuf<uint32_t> contact_pairs;  // pair ids with rows (ascending)
    DevBuf<uint32_t> colour;         // per contact pair
    DevBuf<unsigned long long> body_prio;
    DevBuf<unsigned long long> body_mask;  // 2 words per body: colours taken at the body
    DevBuf<unsigned long long> body_dup;   // 2 words per body: colours seeded twice at the body
    DevBuf<uint32_t> colour_remap;         // colour -> dense colour (empty colours dropped)
    DevBuf<uint32_t> colour_work;          // two lists of uncoloured groups (Jones-Plassmann rounds)
    DevBuf<uint32_t> colour_sub;           // groups per (colour, row count), then the scatter's cursors
    DevBuf<uint32_t> colour_count, colour_offset, colour_cursor;
    DevBuf<uint32_t> split_count, split_offset, split_cursor;
    DevBuf<uint4> batch_rec;         // contact pairs in colour order: body a, body b, pair | rows << 29, 0
    DevBuf<uint4> split_rec;         // the same for the pairs with split-active rows
    DevBuf<float4> vtab, stab;       // solver contact tables in batch-slot order (k_solver.cu)
    // Chunked PGS (k_solver.cu): per body its chunk and the foreign chunks whose groups touch it;
    // per (colour, chunk) the group counts / cursors and bin offsets; the chunk adjacency
    // bit matrix and the per-chunk progress counters.
    DevBuf<uint32_t> chunk_of, chunk_touch, chunk_hist, chunk_off, chunk_adj;
    DevBuf<unsigned int> chunk_ctr;
    DevBuf<uint32_t> flags;          // selection flags
    DevBuf<uint32_t> sel_a, sel_b;   // cache compaction lists
    DevBuf<unsigned char> cub_tmp;
    DevBuf<unsigned int> barrier;    // grid barrier words + round counters
    RecordDev rec;                   // set by an adjoint tape while it records a step
    void reserve(size_t npairs, size_t nbodies, size_t old_manifolds) {
        status.reserve(npairs);
        entries.reserve(npairs * ENTRY_F4);
        detect.reserve(npairs * 8);
        detect_n.reserve(npairs);
        row_count.reserve(npairs);
        rows.reserve(npairs * 4 * ROW_F4);
        route_list.reserve(size_t(CAPTURE_LIST + 1) * npairs);
        old_owned.reserve(old_manifolds + 1);
        scalars.reserve(CAPTURE_COUNT + 1);
        contact_pairs.reserve(npairs);
        colour.reserve(npairs);
        body_prio.reserve(nbodies);
        body_mask.reserve(2 * nbodies);
        body_dup.reserve(2 * nbodies);
        colour_remap.reserve(132);
        colour_count.reserve(132);
        colour_offset.reserve(132);
        colour_cursor.reserve(132);
        split_count.reserve(132);
        split_offset.reserve(132);
        split_cursor.reserve(132);
        batch_rec.reserve(npairs + 32 * 130);  // batches start on multiples of 32
        split_rec.reserve(npairs + 32 * 130);
        flags.reserve(npairs + old_manifolds + 1);
        sel_a.reserve(npairs);
        sel_b.reserve(old_manifolds + 1);
        barrier.reserve(16);
    }
    PairDataDev dev() {
        return PairDataDev{status.p, entries.p, detect.p, detect_n.p, row_count.p, rows.p, route_list.p, old_owned.p,
                           scalars.p, rec};
    }
};

struct Manifolds {  // the persistent cache: sorted keys + entries
    DevBuf<uint64_t> keys;
    DevBuf<float4> entries;
    DevBuf<uint32_t> count;     // device count
    uint32_t* count_dev = nullptr;
    uint32_t count_host = 0;    // last known count (upper bound for capacity planning)
    void init() {
        count.reserve(4);
        count_dev = count.p;
    }
};

struct WorldView {
    BodyDev b;
    const Shape* shapes;
    const float4* hull;
    uint32_t nbodies;
    bool has_mesh = false;  // some shape is a triangle mesh (the mesh narrow-phase launch runs)
};

// Pair pass: classify + refresh, narrow phase, capture. Fills PairData for `npairs`.
void run_pair_pass(const WorldView& w, const uint64_t* pairs, uint32_t npairs, const Manifolds& old_cache,
                   PairData& pd, const StepParams& sp, const uint32_t* simulate_flag, uint32_t* status_dev,
                   cudaStream_t s);
// Narrow phase on explicit queries (parity harness).
void run_collide_queries(const Shape* shapes, const float4* hull, uint32_t n, const uint32_t* sa, const float4* pa,
                         const float4* qa, const uint32_t* sb, const float4* pb, const float4* qb, const float4* seeds,
                         int force_convex, float4* out, uint32_t* counts, uint32_t* status_dev, cudaStream_t s);
// Row preparation for caller-supplied contacts (parity harness).
void run_prepare_contacts(const BodyDev& b, uint32_t ngroups, const uint32_t* group_first, const uint32_t* group_n,
                          const float* contacts, const uint64_t* group_keys, const StepParams& sp, float4* rows,
                          uint32_t* row_count, cudaStream_t s);
// World inverse inertia of every body (the solver's per-body input).
void launch_compute_iw(const BodyDev& b, uint32_t n, cudaStream_t s);
// Colouring + PGS over the pairs with rows (counts stay on the device).
// `mark(5)` is called after the colouring and `mark(6)` after the PGS kernel (timing hooks).
// seed_colours: start the colouring from the colours the pairs' manifolds carry from last step.
// morton_leaf / tree_m: the broad phase's tree leaves (bodies in Morton order), which the
// chunked PGS cuts into its chunks (null: chunks are runs of body indices).
void run_solver(const WorldView& w, const uint64_t* pairs, uint32_t npairs, PairData& pd, const StepParams& sp,
                uint32_t* status_dev, cudaStream_t s, const std::function<void(int)>& mark, bool seed_colours,
                const JointsDev* joints = nullptr, const uint32_t* morton_leaf = nullptr, uint32_t tree_m = 0);
// Which PGS kernel the last run_solver launched: 0 none, 1 team barriers, 2 chunked.
int last_solver_kind();
// Batched worlds: the per-world PGS (k_solver.cu). A launch plan deals the worlds to CTAs:
// a CTA either solves one world with all its threads (block mode: __syncthreads between
// phases) or one world per warp (warp mode: __syncwarp between phases). Worlds are listed
// largest first, so the longest solves start in the first wave.
constexpr uint32_t WS_MAX_COLOURS = 64;              // colours per world (one 64-bit mask per body)
constexpr uint32_t WS_STRIDE = WS_MAX_COLOURS + 3;   // per-world record: g0, ncol, offsets[ncol + 1]
constexpr uint32_t WS_SMEM_PER_BODY = 64;            // velocities + push velocities (4 float4 per body)
constexpr uint32_t WS_MAX_WARPS = 8;                 // block size <= 256
struct WorldPlanDev {
    const uint2* cta;        // per CTA: first list index, count | 1 << 31 in block mode
    const uint32_t* list;    // world ids, largest first
    uint32_t ncta, block;    // CTAs, threads per CTA
    size_t smem;             // dynamic shared memory per CTA
};
struct WorldPlan {
    DevBuf<uint2> cta;
    DevBuf<uint32_t> list;
    uint32_t ncta = 0, block = 0, tau = 0;  // tau: worlds of at most tau bodies run one per warp
    size_t smem = 0;
    bool valid = false;
    WorldPlanDev dev() const { return WorldPlanDev{cta.p, list.p, ncta, block, smem}; }
};
// Builds the plan on the host from the world offsets (world k owns bodies [off[k], off[k + 1])).
// Returns false when some world cannot be held in one CTA's shared memory.
bool build_world_plan(const std::vector<uint32_t>& world_off, uint32_t block, uint32_t tau, WorldPlan& plan,
                      cudaStream_t s);
// The PGS of every world of a batch (no joints): world-local colouring, batches and solve.
// Writes pd.colour (world-local colours), pd.batch_rec (slots grouped per world, then colour),
// the per-world records `wcol` (WS_STRIDE words per world) and the step's counts in pd.scalars.
// joints (a plain world only, whose bodies start at index 0): joint rows solved after each
// velocity sweep's contacts, joint colour by joint colour, as the global solver does.
void run_world_solver(const WorldView& w, const uint64_t* pairs, uint32_t npairs, PairData& pd, const StepParams& sp,
                      uint32_t* status_dev, cudaStream_t s, const std::function<void(int)>& mark,
                      const uint32_t* world_off, uint32_t nworlds, const WorldPlan& plan, uint32_t* wcol,
                      const JointsDev* joints = nullptr, bool seed_colours = false);
// One team barrier that nothing completes (2 blocks): the wait gives up after limit_ns and
// leaves ST_BARRIER_TIMEOUT in *status. ctr and status are device words the caller zeroes.
void run_wait_selftest(unsigned long long limit_ns, unsigned int* ctr, uint32_t* status, cudaStream_t s);
// Impulse writeback, then compaction of the surviving manifolds into `next`.
// simulate / prev_simulate hold one flag per world, indexed through world_of (null: one world).
void run_cache_update(const uint64_t* pairs, uint32_t npairs, const Manifolds& old_cache, PairData& pd,
                      Manifolds& next, const uint32_t* world_of, const uint32_t* simulate_flag,
                      const uint32_t* prev_simulate, cudaStream_t s);

// ---------------------------------------------------------------- adjoint (k_adjoint.cu)
// One recorded step as the reverse solve reads it (device pointers).
struct AdjStep {
    const uint4* recs;          // batch slot records
    const uint32_t* off;        // colour batch starts (ncol)
    const uint32_t* end;        // colour batch ends (ncol)
    uint32_t ncol;
    uint32_t iters;
    const float4* tab;          // velocity contact table
    const float4* sweeps;       // per-sweep records
    const uint32_t* merge_pos;  // pair -> merged cache position
    const uint32_t* row_src;    // row -> old cache position * 4 + point
};
void launch_adj_positions(uint32_t n, float dt, const uint8_t* flags, const float4* xbar, float4* vbar, cudaStream_t s);
void launch_adj_velocities(uint32_t n, float dt, const uint8_t* flags, const float4* material, float4* vbar,
                           float4* wbar, cudaStream_t s);
void run_adj_solve(const AdjStep& st, float4* lbar, float4* vbar, float4* wbar, float* mubar, float* ebar,
                   const float4* material, const float* carry_in, float* carry_out, float restitution_threshold,
                   float warm_factor, unsigned int* bar, uint32_t* status_dev, cudaStream_t s);
// The same for a step the per-world solver ran: st.off holds its per-world records (WS_STRIDE
// words per world); each world's phases run in reverse inside its CTA or warp.
void run_adj_solve_worlds(const AdjStep& st, const WorldPlan& plan, float4* lbar, float4* vbar, float4* wbar,
                          float* mubar, float* ebar, const float4* material, const float* carry_in, float* carry_out,
                          float restitution_threshold, float warm_factor, uint32_t* status_dev, cudaStream_t s);

}  // namespace bgpu
