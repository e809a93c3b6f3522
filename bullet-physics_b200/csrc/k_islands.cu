// Simulation islands and the sleep/wake decision
// (crates/bullet-dynamics/src/world/islands.rs:31-305, island.rs:17-57).
//
// Dynamic bodies are union-find nodes; every collision-eligible broad-phase
// pair between two dynamic bodies merges their sets (sensors and group/mask
// rejects never merge). The partition is order-independent, so the parallel
// lock-free union (link the larger root under the smaller with atomicCAS,
// bounded retries) yields the same islands as the reference's sequential
// union-by-size. An island with any Active / DisableDeactivation member —
// or touching a moving kinematic body — wakes its sleepers; an island with
// none sleeps as a unit.
//
// When no dynamic body is asleep or wants deactivation, every island that has
// a dynamic body is awake and the decision changes nothing, so the union-find
// is skipped (k_island_need raises the flag that the other kernels test).
//
// Pairs whose two bodies are both awake (Active / DisableDeactivation) are not
// linked. That cannot change any body's decision: a set of the thinner
// partition that has no awake member loses no pair (each dropped pair has
// awake ends), so it is a whole island of the full partition; and a set cut
// out of an island with an awake member was cut along a dropped pair, one of
// whose awake ends it holds. So every body lands in a set with an awake member
// exactly when its island has one, and a set with none (touched by a moving
// kinematic or not) is the whole island.
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

constexpr int UF_LIMIT = 1 << 16;

__device__ __forceinline__ bool participates(uint32_t flags) { return (flags & (BF_STATIC | BF_KINEMATIC)) == 0; }

// body.rs:602-608 (is_island_awake): Active or DisableDeactivation.
__device__ __forceinline__ bool awake_member(uint4 in) {
    return participates(in.y) && (in.z == ACT_ACTIVE || in.z == ACT_DISABLE_DEACTIVATION);
}

__device__ __forceinline__ bool eligible(uint4 a, uint4 b) {
    if ((a.y | b.y) & BF_NO_RESPONSE) return false;
    uint32_t ga = a.w & 0xffffu, ma = a.w >> 16, gb = b.w & 0xffffu, mb = b.w >> 16;
    return (ga & mb) != 0 && (gb & ma) != 0;
}

__device__ __forceinline__ uint32_t find_root(const uint32_t* parent, uint32_t x, uint32_t* status) {
    for (int g = 0; g < UF_LIMIT; ++g) {
        uint32_t p = __ldcg(&parent[x]);
        if (p == x) return x;
        x = p;
    }
    atomicOr(status, ST_UNION_FIND_LIMIT);
    return x;
}

// need = 1 when some dynamic body is island-sleeping or wants deactivation.
// find with path halving: every visited node is pointed at its grandparent.
// Only roots are ever linked (atomicCAS) and a node that stopped being a root
// never becomes one again, so the grandparent is always an ancestor and the
// plain store keeps every path leading to the current root.
__device__ __forceinline__ uint32_t find_halving(uint32_t* parent, uint32_t x, uint32_t* status) {
    for (int g = 0; g < UF_LIMIT; ++g) {
        uint32_t p = __ldcg(&parent[x]);
        if (p == x) return x;
        uint32_t gp = __ldcg(&parent[p]);
        if (gp != p) __stcg(&parent[x], gp);
        x = gp;
    }
    atomicOr(status, ST_UNION_FIND_LIMIT);
    return x;
}

__global__ void k_island_need(const uint4* __restrict__ info, uint32_t n, uint32_t* need) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool c = false;
    if (i < n) {
        uint4 in = info[i];
        c = participates(in.y) && (in.z == ACT_ISLAND_SLEEPING || in.z == ACT_WANTS_DEACTIVATION);
    }
    if (__ballot_sync(0xffffffffu, c) && (threadIdx.x & 31u) == 0u && *(volatile uint32_t*)need == 0u) atomicOr(need, 1u);
}

__global__ void k_uf_init(uint32_t n, uint32_t* parent, uint32_t* awake) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    parent[i] = i;
    awake[i] = 0;
}

__device__ __forceinline__ void link(uint32_t* parent, uint32_t a, uint32_t b, uint32_t* status) {
    for (int g = 0; g < UF_LIMIT; ++g) {
        uint32_t ra = find_halving(parent, a, status), rb = find_halving(parent, b, status);
        if (ra == rb) return;
        if (ra > rb) { uint32_t t = ra; ra = rb; rb = t; }
        if (atomicCAS(&parent[rb], rb, ra) == rb) return;
    }
    atomicOr(status, ST_UNION_FIND_LIMIT);
}

__global__ void k_uf_link(const uint4* __restrict__ info, const uint64_t* __restrict__ pairs, uint32_t npairs,
                          uint32_t* parent, uint32_t* status, const uint32_t* __restrict__ need) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs || !*need) return;
    uint64_t k = pairs[p];
    uint32_t a = key_lo(k), b = key_hi(k);
    uint4 ia = info[a], ib = info[b];
    if (!eligible(ia, ib) || !participates(ia.y) || !participates(ib.y)) return;
    if (awake_member(ia) && awake_member(ib)) return;
    link(parent, a, b, status);
}

// islands.rs:186-196: an enabled joint between two dynamic bodies links their islands
// (whatever its collision suppression).
__global__ void k_uf_link_joints(const uint4* __restrict__ info, const float4* __restrict__ desc, uint32_t nj,
                                 uint32_t* parent, uint32_t* status, const uint32_t* __restrict__ need) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj || !*need) return;
    const float4 h = desc[size_t(j) * JOINT_F4];
    if (__float_as_uint(h.w) & JF_DISABLED) return;
    const uint32_t a = __float_as_uint(h.y), b = __float_as_uint(h.z);
    const uint4 ia = info[a], ib = info[b];
    if (!participates(ia.y) || !participates(ib.y)) return;
    if (awake_member(ia) && awake_member(ib)) return;
    link(parent, a, b, status);
}

__global__ void k_uf_flatten_awake(const uint4* __restrict__ info, uint32_t n, uint32_t* parent, uint32_t* awake,
                                   uint32_t* status, const uint32_t* __restrict__ need) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !*need) return;
    uint32_t r = find_root(parent, i, status);
    uint4 in = info[i];
    if (awake_member(in)) awake[r] = 1u;
}

__global__ void k_uf_store_roots(uint32_t n, uint32_t* parent, uint32_t* status, const uint32_t* __restrict__ need) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !*need) return;
    // Writing the root is safe while other threads still walk: every pointer still leads to it.
    parent[i] = find_root(parent, i, status);
}

// islands.rs:232-279 — a moving kinematic wakes every eligible island it pairs with.
__global__ void k_kinematic_wake(const uint4* __restrict__ info, const float4* __restrict__ lv, const float4* __restrict__ av,
                                 const uint64_t* __restrict__ pairs, uint32_t npairs, const uint32_t* __restrict__ root,
                                 uint32_t* awake, const uint32_t* __restrict__ need) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs || !*need) return;
    uint64_t k = pairs[p];
    uint32_t ends[2] = {key_lo(k), key_hi(k)};
    int ks = -1;
    for (int s = 0; s < 2; ++s) {
        uint4 in = info[ends[s]];
        if (in.y & BF_KINEMATIC) {
            V3 v = from4(lv[ends[s]]), w = from4(av[ends[s]]);
            if (len2(v) != 0.0f || len2(w) != 0.0f) { ks = s; break; }
        }
    }
    if (ks < 0) return;
    uint4 ia = info[ends[0]], ib = info[ends[1]];
    if (!eligible(ia, ib)) return;
    uint32_t other = ends[1 - ks];
    if (!participates(info[other].y)) return;
    awake[root[other]] = 1u;
}

// islands.rs:281-294 + body.rs:578-624; also raises the `simulate` flag (step.rs:440) of the
// body's world (world_of is null for a single world).
__global__ void k_uf_apply(uint4* info, float4* lv, float4* av, float4* sleep, uint32_t n, const uint32_t* __restrict__ root,
                           const uint32_t* __restrict__ awake, const uint32_t* __restrict__ world_of, uint32_t* simulate,
                           uint8_t* rec_flags, const uint32_t* __restrict__ need) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 in = info[i];
    bool aw = !*need || awake[root[i]] != 0;
    bool part = participates(in.y);
    if (aw) {
        if (!(in.y & BF_STATIC) && in.z == ACT_ISLAND_SLEEPING) {  // island_wake
            in.z = ACT_WANTS_DEACTIVATION;
            float4 s = sleep[i];
            s.x = 0.0f;
            sleep[i] = s;
            info[i] = in;
        }
    } else if (part && in.z != ACT_DISABLE_SIMULATION) {  // go_to_sleep
        if (in.z != ACT_ISLAND_SLEEPING) {
            in.z = ACT_ISLAND_SLEEPING;
            info[i] = in;
        }
        lv[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        av[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (rec_flags) rec_flags[i] |= RF_ZEROED;
    }
    bool active = in.z == ACT_ACTIVE || in.z == ACT_WANTS_DEACTIVATION || in.z == ACT_DISABLE_DEACTIVATION;
    if (active) {
        // One lane per world among the warp's active bodies raises the flag, and only while
        // it reads as 0 (the flag only goes from 0 to 1): a word shared by every body of a
        // world would otherwise take one atomic per body.
        const uint32_t w = world_of ? world_of[i] : 0u;
        const uint32_t peers = __match_any_sync(__activemask(), w);
        uint32_t* f = &simulate[w];
        if ((threadIdx.x & 31u) == uint32_t(__ffs(int(peers)) - 1) && *f == 0u) atomicOr(f, 1u);
    }
}

}  // namespace

void Islands::run(const BodyDev& b, uint32_t n, const uint64_t* pairs, uint32_t npairs, const uint32_t* world_of,
                  uint32_t* simulate_flag, uint32_t* status_dev, cudaStream_t s, const float4* joint_desc,
                  uint32_t njoints) {
    if (n == 0) return;
    parent.reserve(n);
    awake.reserve(n);
    need.reserve(1);
    check_cuda(cudaMemsetAsync(need.p, 0, sizeof(uint32_t), s), "memset");
    const int TB = 256;
    k_island_need<<<(n + TB - 1) / TB, TB, 0, s>>>(b.info, n, need.p);
    k_uf_init<<<(n + TB - 1) / TB, TB, 0, s>>>(n, parent.p, awake.p);
    if (npairs) k_uf_link<<<(npairs + TB - 1) / TB, TB, 0, s>>>(b.info, pairs, npairs, parent.p, status_dev, need.p);
    if (njoints)
        k_uf_link_joints<<<(njoints + TB - 1) / TB, TB, 0, s>>>(b.info, joint_desc, njoints, parent.p, status_dev, need.p);
    k_uf_flatten_awake<<<(n + TB - 1) / TB, TB, 0, s>>>(b.info, n, parent.p, awake.p, status_dev, need.p);
    k_uf_store_roots<<<(n + TB - 1) / TB, TB, 0, s>>>(n, parent.p, status_dev, need.p);
    if (npairs)
        k_kinematic_wake<<<(npairs + TB - 1) / TB, TB, 0, s>>>(b.info, b.linvel, b.angvel, pairs, npairs, parent.p,
                                                                awake.p, need.p);
    k_uf_apply<<<(n + TB - 1) / TB, TB, 0, s>>>(b.info, b.linvel, b.angvel, b.sleep, n, parent.p, awake.p, world_of,
                                                 simulate_flag, b.rec_flags, need.p);
}

}  // namespace bgpu
