// Internal device-side layout of one simulated world (not part of the C ABI).
//
// Bodies live in structure-of-arrays form (16-byte float4 lanes, coalesced
// per-body loads). Broad-phase pairs are a sorted array of 64-bit keys
// (lo << 32 | hi). Every per-pair quantity — persistent manifold, fresh
// detection, contact rows — is indexed by the pair's position in that sorted
// array, so the stages of one step hand data to each other without
// permutation; the previous step's manifolds are found by binary search on
// the previous step's key array.
#pragma once
#include <cstdint>
#include "bgpu_narrow.cuh"

namespace bgpu {

// Body flags (bit set in BodyDev::info.y).
enum : uint32_t {
    BF_STATIC = 1u,
    BF_KINEMATIC = 2u,
    BF_NO_RESPONSE = 4u,
    BF_DISABLE_GRAVITY = 8u,
    BF_ADDITIONAL_DAMPING = 16u,
};
// Activation states (body.rs:140-153, numbered like Bullet's tags).
enum : uint32_t { ACT_ACTIVE = 1, ACT_ISLAND_SLEEPING = 2, ACT_WANTS_DEACTIVATION = 3, ACT_DISABLE_DEACTIVATION = 4, ACT_DISABLE_SIMULATION = 5 };

// Device status bits (or-ed into the world's status word).
enum : uint32_t {
    ST_PAIR_OVERFLOW = 1u << 0,
    ST_UNION_FIND_LIMIT = 1u << 1,
    ST_BARRIER_TIMEOUT = 1u << 2,
    ST_COLOUR_OVERFLOW = 1u << 3,
    ST_EPA_CAPACITY = 1u << 4,
    ST_NONFINITE = 1u << 5,
    ST_TRAVERSAL_STACK = 1u << 6,
    ST_COLOUR_ROUNDS = 1u << 7,
    ST_MESH_CANDIDATES = 1u << 8,  // a convex-vs-mesh pair found more candidate points than it keeps
};

// Pair status codes written by the classify pass.
enum : uint32_t {
    PS_NONE = 0,        // filtered: no manifold carried
    PS_KEEP = 1,        // manifold carried verbatim (sleeping island / immovable pair)
    PS_SERVED = 2,      // refreshed from the cache, rows emitted
    PS_DETECT = 3,      // needs the narrow phase
};

// Narrow-phase routes (narrowphase/mod.rs:103-285).
enum : uint32_t { NP_NONE = 0, NP_PLANE_A = 1, NP_PLANE_B = 2, NP_SPHERE_SPHERE = 3, NP_SPHERE_BOX = 4, NP_BOX_SPHERE = 5,
                  NP_BOX_BOX = 6, NP_CONVEX = 7, NP_MESH = 8 };

struct SolverParams {  // solver/info.rs:24-86 (the contact subset)
    float erp2, linear_slop, restitution_velocity_threshold;
    uint32_t split_impulse;
    float split_impulse_penetration_threshold, split_impulse_turn_erp, warmstarting_factor, global_cfm, sor;
    uint32_t num_iterations;
    float erp, damping;  // joint rows
};

struct BodyDev {
    float4* pos;          // xyz
    float4* quat;         // xyzw
    float4* linvel;       // xyz
    float4* angvel;       // xyz
    float4* inv_inertia;  // xyz local inverse inertia, w inverse mass
    float4* gravity;      // xyz
    float4* force;        // xyz
    float4* torque;       // xyz
    float4* material;     // friction, restitution, linear damping, angular damping
    float4* sleep;        // deactivation time, linear threshold, angular threshold, -
    uint4* info;          // shape, flags, activation, group | mask << 16
    float4* aabb_min;     // persistent broad-phase proxy (sleeping bodies keep theirs)
    float4* aabb_max;
    float4* pred;         // predicted position of this step
    float* settled;       // |v|^2 + |w|^2 at the end of the previous step
    float4* iw;           // world inverse inertia: 3 float4 per body (9 entries column-major + inv mass)
    float4* push_lin;
    float4* push_ang;
    uint8_t* rec_flags = nullptr;  // adjoint recording only: RF_* bits per body for the step
};

// Per-body bits of a recorded step (the adjoint's frozen sleep / integration decisions).
enum : uint8_t {
    RF_INTEGRATED = 1,  // integrate_velocities ran (dynamic and active)
    RF_ZEROED = 2,      // the island went to sleep: velocities were zeroed before the solve
    RF_MOVED = 4,       // the pose was integrated with the solved velocities
};

// Persistent manifold entry: 16 float4 (manifold.rs:168-186 + 4 points of manifold.rs:124-142).
//  e[0] detect_pos_a.xyz, threshold      e[1] detect_ori_a
//  e[2] detect_pos_b.xyz, meta bits      e[3] detect_ori_b
//  point k: e[4+3k] local_a.xyz, penetration; e[5+3k] local_b.xyz, normal impulse;
//           e[6+3k] normal.xyz, lifetime (uint bits)
// meta bits: [0..2] point count, [8] initialized, [9] valid
constexpr int ENTRY_F4 = 16;
constexpr uint32_t META_INIT = 1u << 8;
constexpr uint32_t META_VALID = 1u << 9;
constexpr uint32_t META_COLOUR_SHIFT = 16;  // bits 16-23: last PGS colour + 1 (0: none)

// Contact row slot: 6 float4 per contact, 4 slots per pair.
//  r[0] normal.xyz, friction                 r[1] r_a.xyz, Baumgarte bias
//  r[2] r_b.xyz, separation bias             r[3] normal / t1 / t2 impulse, restitution
//  r[4] normal / t1 / t2 effective mass, normal cfm
//  r[5] split rhs, push impulse, split flag, penetration
constexpr int ROW_F4 = 6;

// Contact tangent basis (sequential_impulse.rs:620-629): helper X unless |n.x| >= 0.9,
// normalised by multiplying with the reciprocal length.
__device__ __forceinline__ void tangent_basis_dev(V3 n, V3& t1, V3& t2) {
    V3 helper = fabsf(n.x) < 0.9f ? V3{1.f, 0.f, 0.f} : V3{0.f, 1.f, 0.f};
    V3 c = cross(n, helper);
    t1 = c * (1.0f / len(c));
    t2 = cross(n, t1);
}

__host__ __device__ __forceinline__ uint32_t key_lo(uint64_t k) { return uint32_t(k >> 32); }
__host__ __device__ __forceinline__ uint32_t key_hi(uint64_t k) { return uint32_t(k & 0xffffffffu); }

}  // namespace bgpu
