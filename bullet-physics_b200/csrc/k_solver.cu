// Sequential-impulse (PGS) solve over graph-coloured row groups, and the
// post-solve manifold writeback / lifecycle prune.
//
// The reference solves rows one by one in pair order (solver/
// sequential_impulse.rs:692-735, 743-802). Here the row group of each pair
// (its <= 4 contacts, solved in order by one thread) is a graph vertex; two
// groups conflict when they share a body with nonzero inverse mass. A
// Jones-Plassmann colouring with first-fit colour choice splits the groups
// into batches of pairwise-independent groups. Within a batch no dynamic body
// is touched twice, so the result is bit-identical to the reference's
// sequential solve over the same rows taken in (colour, pair) order.
//
// The PGS kernel is a persistent cooperative launch split into two teams of
// blocks with their own grid barriers: the velocity team runs the warm start
// and the velocity sweeps, the split team the split-impulse sweeps, which
// touch only the push velocities and so run at the same time. The first
// sweep of each team computes the per-contact terms that stay fixed during the
// solve (tangent basis, Iw^-1 (r x d), the velocity couplings kn/kt1/kt2) once
// and stores them in a contact table in batch-slot order, so the later sweeps
// run only the impulse update, reading the table with coalesced loads.
//
// Rows store only the contact frame (normal, lever arms), the bias terms, the
// effective masses and the accumulated impulses; the tangent basis, the
// angular components Iw^-1 (r x d) and the velocity couplings are recomputed
// from the per-body world inverse inertia with the reference's arithmetic, so
// they equal the values the reference precomputes in prepare().
#include <algorithm>
#include <cooperative_groups.h>
#include <cub/cub.cuh>
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

constexpr uint32_t NO_COLOUR = 0xffffffffu;
constexpr int MAX_ROUNDS = 1024;

__device__ __forceinline__ uint32_t mix32(uint64_t k) {
    uint32_t h = uint32_t(k) ^ uint32_t(k >> 32) * 0x9E3779B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ float inv_mass_of(const float4* __restrict__ iw, uint32_t i) { return iw[3 * i + 2].y; }

__device__ __forceinline__ M3 load_iw(const float4* __restrict__ iw, uint32_t i, float& inv_mass) {
    float4 a = __ldg(&iw[3 * i]), b = __ldg(&iw[3 * i + 1]), c = __ldg(&iw[3 * i + 2]);
    inv_mass = c.y;
    return M3{V3{a.x, a.y, a.z}, V3{a.w, b.x, b.y}, V3{b.z, b.w, c.x}};
}

__global__ void k_flag_contact_pairs(uint32_t npairs, const uint32_t* __restrict__ row_count, uint32_t* flags) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < npairs) flags[p] = row_count[p] > 0 ? 1u : 0u;
}

struct ColourArgs {
    const uint32_t* count;  // number of contact pairs
    const uint32_t* contact_pairs;
    const uint64_t* pairs;
    const float4* iw;
    uint32_t* colour;
    unsigned long long* prio;
    unsigned long long* mask;
    unsigned long long* dup;      // 2 words per body: colours seeded twice at the body
    const float4* entries;        // this step's manifold entries (their meta carries last step's colour)
    uint32_t seed;                // 1: start from last step's colours
    unsigned int* bar;  // [0] barrier counter, [5] colour max, [6] [7] uncoloured-list lengths
    uint32_t* status;
};

__device__ __forceinline__ unsigned long long* colour_word(unsigned long long* m, uint32_t x, uint32_t c) {
    return &m[2 * x + (c >> 6)];
}

// Seeding, then Jones-Plassmann rounds. Seeding: a group whose pair kept its
// manifold starts from the colour it had last step (kept in the entry's meta
// bits); a seed is dropped, for every group that claims it, when two groups
// claim the same colour at one dynamic body - so the result does not depend on
// the order of the atomics. The bits of dropped seeds stay in the masks and
// only make those colours unavailable there. Jones-Plassmann: an uncoloured
// group wins when its priority is the maximum over the uncoloured groups at
// both of its dynamic bodies; winners take the lowest colour free at both.
//
// The rounds walk a list of the still-uncoloured groups (rebuilt by each round
// from its losers), so a round costs what is left to colour, not the whole
// set; once the list fits one block, that block finishes the rounds alone with
// block-local syncs and the rest of the grid exits. Which groups win in a
// round depends only on the priorities, so the colours do not depend on the
// list order or on which threads run the rounds.
struct JpList {
    uint32_t* items[2];
    unsigned int* len[2];
};

// Appends k to a list: one atomicAdd per group of lanes that append together.
__device__ __forceinline__ void list_append(uint32_t* items, unsigned int* len, uint32_t k) {
    cooperative_groups::coalesced_group g = cooperative_groups::coalesced_threads();
    unsigned int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(len, g.size());
    base = g.shfl(base, 0);
    items[base + g.thread_rank()] = k;
}

// One Jones-Plassmann round over list r & 1; losers go to list (r + 1) & 1.
// [lo, n) with step `step` is this thread's share of the list.
__device__ __forceinline__ void jp_clear(const ColourArgs& a, const uint32_t* list, uint32_t n, uint32_t lo, uint32_t step) {
    for (uint32_t i = lo; i < n; i += step) {
        const uint64_t key = a.pairs[a.contact_pairs[list[i]]];
        a.prio[key_lo(key)] = 0ull;
        a.prio[key_hi(key)] = 0ull;
    }
}

__device__ __forceinline__ void jp_bid(const ColourArgs& a, const uint32_t* list, uint32_t n, uint32_t lo, uint32_t step) {
    for (uint32_t i = lo; i < n; i += step) {
        const uint32_t k = list[i];
        const uint64_t key = a.pairs[a.contact_pairs[k]];
        const uint32_t u = key_lo(key), v = key_hi(key);
        const unsigned long long pr = (uint64_t(mix32(key)) << 32) | k;
        if (inv_mass_of(a.iw, u) > 0.0f) atomicMax(&a.prio[u], pr);
        if (inv_mass_of(a.iw, v) > 0.0f) atomicMax(&a.prio[v], pr);
    }
}

// The colour count (bar[5]) is raised once per block: each warp folds its lanes'
// colours into the block's shared maximum, which colour_max_flush publishes.
__device__ __forceinline__ void warp_colour_max(unsigned int* s_cmax, uint32_t top) {
    top = __reduce_max_sync(0xffffffffu, top);
    if ((threadIdx.x & 31u) == 0 && top) atomicMax(s_cmax, top);
}

__device__ __forceinline__ void colour_max_flush(const unsigned int* s_cmax, unsigned int* bar5) {
    __syncthreads();
    if (threadIdx.x == 0 && *s_cmax) atomicMax(bar5, *s_cmax);
}

__device__ __forceinline__ void jp_pick(const ColourArgs& a, const uint32_t* list, uint32_t n, uint32_t lo, uint32_t step,
                                        uint32_t* losers, unsigned int* nlosers, unsigned int* s_cmax) {
    uint32_t top = 0;
    for (uint32_t i = lo; i < n; i += step) {
        const uint32_t k = list[i];
        const uint64_t key = a.pairs[a.contact_pairs[k]];
        const uint32_t u = key_lo(key), v = key_hi(key);
        const unsigned long long pr = (uint64_t(mix32(key)) << 32) | k;
        const bool du = inv_mass_of(a.iw, u) > 0.0f, dv = inv_mass_of(a.iw, v) > 0.0f;
        const bool win = (!du || __ldcg(&a.prio[u]) == pr) && (!dv || __ldcg(&a.prio[v]) == pr);
        if (!win) {
            list_append(losers, nlosers, k);
            continue;
        }
        unsigned long long m0 = 0, m1 = 0;
        if (du) { m0 |= __ldcg(&a.mask[2 * u]); m1 |= __ldcg(&a.mask[2 * u + 1]); }
        if (dv) { m0 |= __ldcg(&a.mask[2 * v]); m1 |= __ldcg(&a.mask[2 * v + 1]); }
        uint32_t c;
        if (~m0) c = uint32_t(__ffsll((long long)~m0) - 1);
        else if (~m1) c = 64u + uint32_t(__ffsll((long long)~m1) - 1);
        else { c = MAX_COLOURS - 1; atomicOr(a.status, ST_COLOUR_OVERFLOW); }
        a.colour[k] = c;
        const unsigned long long b0 = c < 64 ? (1ull << c) : 0ull, b1 = c >= 64 ? (1ull << (c - 64)) : 0ull;
        if (du) { a.mask[2 * u] |= b0; a.mask[2 * u + 1] |= b1; }
        if (dv) { a.mask[2 * v] |= b0; a.mask[2 * v + 1] |= b1; }
        top = max(top, c + 1u);
    }
    warp_colour_max(s_cmax, top);
}

__global__ void k_colour(ColourArgs a, JpList wl) {
    const uint32_t K = *a.count;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const unsigned int nblocks = gridDim.x;
    unsigned int nbar = 0;
    __shared__ unsigned int s_cmax;
    if (threadIdx.x == 0) s_cmax = 0u;
    for (uint32_t k = tid; k < K; k += stride) {
        a.colour[k] = NO_COLOUR;
        uint64_t key = a.pairs[a.contact_pairs[k]];
        uint32_t u = key_lo(key), v = key_hi(key);
        a.mask[2 * u] = 0ull; a.mask[2 * u + 1] = 0ull;
        a.mask[2 * v] = 0ull; a.mask[2 * v + 1] = 0ull;
        if (a.seed) {
            a.dup[2 * u] = 0ull; a.dup[2 * u + 1] = 0ull;
            a.dup[2 * v] = 0ull; a.dup[2 * v + 1] = 0ull;
        } else {
            wl.items[0][k] = k;  // every group starts uncoloured
        }
    }
    if (tid == 0) {
        a.bar[5] = 0;
        *wl.len[0] = a.seed ? 0u : K;
        *wl.len[1] = 0u;
    }
    team_barrier(a.bar, ++nbar * nblocks, a.status);
    if (a.seed) {
        for (uint32_t k = tid; k < K; k += stride) {  // claim last step's colour at both bodies
            const uint32_t p = a.contact_pairs[k];
            const uint32_t cs = (__float_as_uint(a.entries[size_t(p) * ENTRY_F4 + 2].w) >> META_COLOUR_SHIFT) & 0xffu;
            if (cs == 0u || cs > MAX_COLOURS) continue;
            const uint32_t c = cs - 1u;
            const unsigned long long bit = 1ull << (c & 63u);
            const uint64_t key = a.pairs[p];
            const uint32_t u = key_lo(key), v = key_hi(key);
            if (inv_mass_of(a.iw, u) > 0.0f && (atomicOr(colour_word(a.mask, u, c), bit) & bit))
                atomicOr(colour_word(a.dup, u, c), bit);
            if (inv_mass_of(a.iw, v) > 0.0f && (atomicOr(colour_word(a.mask, v, c), bit) & bit))
                atomicOr(colour_word(a.dup, v, c), bit);
        }
        team_barrier(a.bar, ++nbar * nblocks, a.status);
        uint32_t top = 0;
        for (uint32_t k = tid; k < K; k += stride) {  // keep the seeds claimed once at each body
            const uint32_t p = a.contact_pairs[k];
            const uint32_t cs = (__float_as_uint(a.entries[size_t(p) * ENTRY_F4 + 2].w) >> META_COLOUR_SHIFT) & 0xffu;
            bool keep = false;
            uint32_t c = 0;
            if (cs != 0u && cs <= MAX_COLOURS) {
                c = cs - 1u;
                const unsigned long long bit = 1ull << (c & 63u);
                const uint64_t key = a.pairs[p];
                const uint32_t u = key_lo(key), v = key_hi(key);
                const bool du = inv_mass_of(a.iw, u) > 0.0f && (__ldcg(colour_word(a.dup, u, c)) & bit);
                const bool dv = inv_mass_of(a.iw, v) > 0.0f && (__ldcg(colour_word(a.dup, v, c)) & bit);
                keep = !du && !dv;
            }
            if (keep) {
                a.colour[k] = c;
                top = max(top, c + 1u);
            } else {
                list_append(wl.items[0], wl.len[0], k);
            }
        }
        warp_colour_max(&s_cmax, top);
        colour_max_flush(&s_cmax, &a.bar[5]);
        team_barrier(a.bar, ++nbar * nblocks, a.status);
    }
    // Rounds on the whole grid while the list is longer than one block. The list
    // length is read once per block, so every thread of a block takes the same path
    // (even after a barrier timeout, when lengths may still be changing).
    __shared__ unsigned int s_len;
    auto list_len = [&](uint32_t which) -> uint32_t {
        if (threadIdx.x == 0) s_len = *(volatile unsigned int*)wl.len[which];
        __syncthreads();
        const uint32_t v = s_len;
        __syncthreads();
        return v;
    };
    int round = 0;
    for (; round < MAX_ROUNDS; ++round) {
        const uint32_t cur = uint32_t(round) & 1u, nxt = cur ^ 1u;
        const uint32_t n = list_len(cur);
        if (n <= blockDim.x) break;
        jp_clear(a, wl.items[cur], n, tid, stride);
        if (tid == 0) *wl.len[nxt] = 0u;  // last read (as this list's length) before the previous barrier
        team_barrier(a.bar, ++nbar * nblocks, a.status);
        jp_bid(a, wl.items[cur], n, tid, stride);
        team_barrier(a.bar, ++nbar * nblocks, a.status);
        jp_pick(a, wl.items[cur], n, tid, stride, wl.items[nxt], wl.len[nxt], &s_cmax);
        colour_max_flush(&s_cmax, &a.bar[5]);
        team_barrier(a.bar, ++nbar * nblocks, a.status);
        if (__syncthreads_or((*(volatile uint32_t*)a.status & ST_BARRIER_TIMEOUT) != 0u)) return;
    }
    // The short tail: block 0 alone, one group per thread.
    if (blockIdx.x != 0) return;
    for (; round < MAX_ROUNDS; ++round) {
        const uint32_t cur = uint32_t(round) & 1u, nxt = cur ^ 1u;
        const uint32_t n = list_len(cur);
        if (n == 0) break;
        jp_clear(a, wl.items[cur], n, threadIdx.x, blockDim.x);
        if (threadIdx.x == 0) *wl.len[nxt] = 0u;
        __syncthreads();
        jp_bid(a, wl.items[cur], n, threadIdx.x, blockDim.x);
        __syncthreads();
        jp_pick(a, wl.items[cur], n, threadIdx.x, blockDim.x, wl.items[nxt], wl.len[nxt], &s_cmax);
        __syncthreads();
    }
    colour_max_flush(&s_cmax, &a.bar[5]);
    if (round >= MAX_ROUNDS && threadIdx.x == 0) atomicOr(a.status, ST_COLOUR_ROUNDS);
}

// Colour histograms of all groups and of the groups with split-active rows,
// plus the row and split-row totals.
__global__ void k_colour_hist(const uint32_t* __restrict__ count, const uint32_t* __restrict__ contact_pairs,
                              const uint32_t* __restrict__ colour, const uint32_t* __restrict__ row_count,
                              const float4* __restrict__ rows, uint32_t* hist, uint32_t* split_hist, uint32_t* split_flag,
                              uint32_t* sub_hist) {
    // Block-local histograms; [MAX_COLOURS] rows, [MAX_COLOURS + 1] split-active rows;
    // shc: groups per (colour, row count - 1).
    __shared__ uint32_t sh[MAX_COLOURS + 2], ssh[MAX_COLOURS], shc[MAX_COLOURS * 4];
    for (uint32_t i = threadIdx.x; i < MAX_COLOURS + 2; i += blockDim.x) sh[i] = 0;
    for (uint32_t i = threadIdx.x; i < MAX_COLOURS; i += blockDim.x) ssh[i] = 0;
    for (uint32_t i = threadIdx.x; i < MAX_COLOURS * 4; i += blockDim.x) shc[i] = 0;
    __syncthreads();
    uint32_t K = *count;
    uint32_t nrows = 0, nsplit_rows = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        uint32_t c = colour[k];
        if (c >= MAX_COLOURS) {  // colouring gave up (its status bit is set): the group is not solved
            split_flag[k] = 0u;
            continue;
        }
        atomicAdd(&sh[c], 1u);
        uint32_t p = contact_pairs[k];
        uint32_t n = row_count[p];
        atomicAdd(&shc[c * 4 + (n - 1)], 1u);
        nrows += n;
        uint32_t nsr = 0;  // split-active rows
        for (uint32_t r = 0; r < n; ++r) nsr += rows[(size_t(p) * 4 + r) * ROW_F4 + 5].z != 0.0f ? 1u : 0u;
        split_flag[k] = nsr ? 1u : 0u;
        if (nsr) {
            nsplit_rows += nsr;
            atomicAdd(&ssh[c], 1u);
        }
    }
    nrows = __reduce_add_sync(0xffffffffu, nrows);
    nsplit_rows = __reduce_add_sync(0xffffffffu, nsplit_rows);
    if ((threadIdx.x & 31u) == 0u) {
        if (nrows) atomicAdd(&sh[MAX_COLOURS], nrows);
        if (nsplit_rows) atomicAdd(&sh[MAX_COLOURS + 1], nsplit_rows);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < MAX_COLOURS; i += blockDim.x) {
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
        if (ssh[i]) atomicAdd(&split_hist[i], ssh[i]);
    }
    for (uint32_t i = threadIdx.x; i < MAX_COLOURS * 4; i += blockDim.x)
        if (shc[i]) atomicAdd(&sub_hist[i], shc[i]);
    if (threadIdx.x == 0) {
        if (sh[MAX_COLOURS]) atomicAdd(&hist[MAX_COLOURS + 1], sh[MAX_COLOURS]);
        if (sh[MAX_COLOURS + 1]) atomicAdd(&hist[MAX_COLOURS + 2], sh[MAX_COLOURS + 1]);
    }
}

// Offsets of the colour batches; scalars [3] rows [4] colours [5] split groups
// [10] split rows [11] largest split batch.
__global__ void k_colour_scan(uint32_t* hist, uint32_t* offset, uint32_t* cursor, uint32_t* split_hist,
                              uint32_t* split_offset, uint32_t* split_cursor, const unsigned int* bar, uint32_t* scalars,
                              uint32_t* remap, const uint32_t* sub_hist, uint32_t* sub_cursor) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t nraw = bar[5];
    uint32_t acc = 0, sacc = 0, smax = 0, split_groups = 0, d = 0;
    // Colours without groups are dropped (remap: colour -> dense colour), batches start on
    // multiples of 32 (one warp's slots never straddle two batches). Inside a batch the
    // groups with 4 rows come first, then 3, 2, 1 (sub_cursor: the scatter's cursor of each
    // part), so most warps hold groups of one size: their lanes run the same number of
    // contacts and read the table's contact planes without gaps. The split batches keep
    // their cursors; after the scatter they hold the split batch ends.
    for (uint32_t c = 0; c < nraw; ++c) {
        if (hist[c] == 0) continue;
        remap[c] = d;
        acc = (acc + 31u) & ~31u;
        offset[d] = acc;
        uint32_t part = acc;
        for (uint32_t n = 4; n >= 1; --n) {
            sub_cursor[d * 4 + (n - 1)] = part;
            part += sub_hist[c * 4 + (n - 1)];
        }
        acc += hist[c];
        cursor[d] = acc;  // the batch end
        sacc = (sacc + 31u) & ~31u;
        split_offset[d] = sacc;
        split_cursor[d] = sacc;
        sacc += split_hist[c];
        smax = max(smax, split_hist[c]);
        split_groups += split_hist[c];
        ++d;
    }
    offset[d] = acc;
    split_offset[d] = sacc;
    scalars[3] = hist[MAX_COLOURS + 1];
    scalars[4] = d;
    scalars[5] = split_groups;
    scalars[10] = hist[MAX_COLOURS + 2];
    scalars[11] = smax;
}

// One atomicAdd per distinct colour among the calling lanes of a warp.
__device__ __forceinline__ uint32_t claim_slot(uint32_t* cursor, uint32_t c) {
    uint32_t active = __activemask();
    uint32_t peers = __match_any_sync(active, c);
    uint32_t lane = threadIdx.x & 31u;
    uint32_t leader = uint32_t(__ffs(int(peers)) - 1);
    uint32_t rank = uint32_t(__popc(peers & ((1u << lane) - 1u)));
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cursor[c], uint32_t(__popc(int(peers))));
    base = __shfl_sync(peers, base, int(leader));
    return base + rank;
}

// Slot record of a group: its two bodies and its pair index with the row count
// in the top three bits.
__global__ void k_colour_scatter(const uint32_t* __restrict__ count, const uint32_t* __restrict__ contact_pairs,
                                 const uint64_t* __restrict__ pairs, const uint32_t* __restrict__ row_count,
                                 const uint32_t* __restrict__ colour, const uint32_t* __restrict__ split_flag,
                                 uint32_t* sub_cursor, uint32_t* split_cursor, uint4* batch_rec, uint4* split_rec,
                                 float4* entries, const uint32_t* __restrict__ remap) {
    uint32_t K = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        if (colour[k] >= MAX_COLOURS) continue;  // colouring gave up (its status bit is set)
        uint32_t c = remap[colour[k]];
        uint32_t p = contact_pairs[k];
        uint64_t key = pairs[p];
        uint4 rec = make_uint4(key_lo(key), key_hi(key), p | (row_count[p] << 29), 0u);
        // The colour rides in the manifold's meta bits to seed next step's colouring.
        float* mw = &entries[size_t(p) * ENTRY_F4 + 2].w;
        *mw = __uint_as_float((__float_as_uint(*mw) & ~(0xffu << META_COLOUR_SHIFT)) | ((c + 1u) << META_COLOUR_SHIFT));
        batch_rec[claim_slot(sub_cursor, c * 4 + (row_count[p] - 1))] = rec;
        if (split_flag[k]) split_rec[claim_slot(split_cursor, c)] = rec;
    }
}

struct SolveArgs {
    float4* rows;
    const uint4* batch_rec;
    const uint32_t* offset;   // colour batch starts (multiples of 32)
    const uint32_t* end;      // colour batch ends
    const uint4* split_rec;
    const uint32_t* split_offset;
    const uint32_t* split_end;
    const uint32_t* scalars;  // [4] colours [5] split groups [11] largest split batch
    float4* linvel;
    float4* angvel;
    float4* push_lin;
    float4* push_ang;
    const float4* iw;
    float4* vtab;             // velocity contact table (VT_PLANES planes)
    float4* stab;             // split contact table (ST_PLANES planes)
    float4* srec;             // adjoint recording (else null): per (sweep, slot, contact) vn, impulse, clamp bits
    unsigned int* bar;        // [0] velocity-team barrier counter, [1] split-team counter
    uint32_t* status;
    float inv_dt;
    float restitution_threshold;
    uint32_t iterations;
    JointsDev j;              // joint rows, solved after the contacts of each sweep (j.ncol == 0: none)
    float damping;            // joint rows (info.rs damping)
};

__device__ __forceinline__ void apply(V3& la, V3& wa, V3& lb, V3& wb, bool appa, bool appb, float ima, float imb, V3 d,
                                      V3 ca, V3 cb, float j) {
    if (appa) { la -= d * (j * ima); wa -= ca * j; }
    if (appb) { lb += d * (j * imb); wb += cb * j; }
}

enum Kind { WARM = 0, ITER = 1, SPLIT = 2 };

__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// warm_start (sequential_impulse.rs:710-717) for group slot t, which also
// fills the slot's velocity table with the prepared terms the sweeps use
// (sequential_impulse.rs:352-520 computes the same values in prepare()).
__device__ __forceinline__ void warm_group(const SolveArgs& a, uint32_t t, uint32_t p, uint32_t cnt, uint32_t ia,
                                           uint32_t ib, V3& la, V3& wa, V3& lb, V3& wb, bool& appa, bool& appb) {
    float ima, imb;
    const M3 iwa = load_iw(a.iw, ia, ima);
    const M3 iwb = load_iw(a.iw, ib, imb);
    appa = ima > 0.0f;
    appb = imb > 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) {
        float4* e = a.vtab + tix<VT_PLANES>(0, k, t);
        const float4* r = a.rows + (size_t(p) * 4 + k) * ROW_F4;
        const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
        const V3 n = from4(r0), ra = from4(r1), rb = from4(r2);
        V3 t1, t2;
        tangent_basis_dev(n, t1, t2);
        const V3 ana = mul(iwa, cross(ra, n)), anb = mul(iwb, cross(rb, n));
        const V3 a1a = mul(iwa, cross(ra, t1)), a1b = mul(iwb, cross(rb, t1));
        const V3 a2a = mul(iwa, cross(ra, t2)), a2b = mul(iwb, cross(rb, t2));
        apply(la, wa, lb, wb, appa, appb, ima, imb, n, ana, anb, r3.x);
        apply(la, wa, lb, wb, appa, appb, ima, imb, t1, a1a, a1b, r3.y);
        apply(la, wa, lb, wb, appa, appb, ima, imb, t2, a2a, a2b, r3.z);
        e[VT_N * PLANE_STRIDE] = r0;
        e[VT_RA * PLANE_STRIDE] = r1;
        e[VT_RB * PLANE_STRIDE] = r2;
        e[VT_T1 * PLANE_STRIDE] = f4(t1, ima);
        e[VT_ANA * PLANE_STRIDE] = f4(ana, r4.x);
        e[VT_ANB * PLANE_STRIDE] = f4(anb, r4.y);
        e[VT_A1A * PLANE_STRIDE] = f4(a1a, r4.z);
        e[VT_A1B * PLANE_STRIDE] = f4(a1b, r4.w);
        e[VT_A2A * PLANE_STRIDE] = f4(a2a, r3.w);
        e[VT_A2B * PLANE_STRIDE] = f4(a2b, imb);
        e[VT_IMP * PLANE_STRIDE] = r3;
    }
}



// One solve_contact sweep (sequential_impulse.rs:804-930) over group slot t;
// on the last sweep the impulses also go back to the pair's rows.
__device__ __forceinline__ void iter_group(const SolveArgs& a, uint32_t t, uint32_t p, uint32_t cnt, uint32_t sweep,
                                           bool last, V3& la, V3& wa, V3& lb, V3& wb, bool& appa, bool& appb) {
    const float4* e0 = a.vtab + tix<VT_PLANES>(0, 0, t);
    const float ima = e0[VT_T1 * PLANE_STRIDE].w, imb = e0[VT_A2B * PLANE_STRIDE].w;
    const float ims = ima + imb;
    appa = ima > 0.0f;
    appb = imb > 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) {
        float4* e = a.vtab + tix<VT_PLANES>(0, k, t);
        const float4 r0 = e[VT_N * PLANE_STRIDE], r1 = e[VT_RA * PLANE_STRIDE], r2 = e[VT_RB * PLANE_STRIDE];
        const float4 q3 = e[VT_T1 * PLANE_STRIDE];
        const float4 q5 = e[VT_ANA * PLANE_STRIDE], q6 = e[VT_ANB * PLANE_STRIDE];
        const float4 q7 = e[VT_A1A * PLANE_STRIDE], q8 = e[VT_A1B * PLANE_STRIDE];
        const float4 q9 = e[VT_A2A * PLANE_STRIDE], q10 = e[VT_A2B * PLANE_STRIDE];
        const float4 r3 = e[VT_IMP * PLANE_STRIDE];
        const V3 n = from4(r0), ra = from4(r1), rb = from4(r2), t1 = from4(q3);
        const V3 t2 = cross(n, t1);  // tangent_basis (sequential_impulse.rs:620-629), as warm_group made it
        const V3 ana = from4(q5), anb = from4(q6), a1a = from4(q7), a1b = from4(q8), a2a = from4(q9), a2b = from4(q10);
        // The velocity couplings of sequential_impulse.rs:352-520, in warm_group's operand order.
        const V3 kn = n * ims + cross(anb, rb) + cross(ana, ra);
        const V3 kt1 = t1 * ims + cross(a1b, rb) + cross(a1a, ra);
        const V3 kt2 = t2 * ims + cross(a2b, rb) + cross(a2a, ra);
        const float4 r4 = make_float4(q5.w, q6.w, q7.w, q8.w);
        V3 va = la + cross(wa, ra);
        V3 vb = lb + cross(wb, rb);
        V3 rel = vb - va;
        float vn = dot(rel, n);
        float bias = 0.0f;
        if (vn < -a.restitution_threshold) bias = -q9.w * vn;
        if (r1.w != 0.0f) bias += r1.w;
        if (r2.w != 0.0f) bias += r2.w;
        float lambda = r4.w != 0.0f ? r4.x * (bias - vn) - r4.w * r3.x : r4.x * (bias - vn);
        float old = r3.x;
        float nimp = fmaxf(old + lambda, 0.0f);
        float jn = nimp - old;
        apply(la, wa, lb, wb, appa, appb, ima, imb, n, ana, anb, jn);
        rel += kn * jn;
        float maxf = r0.w * nimp;
        float vt = dot(rel, t1);
        float lam = -r4.y * (vt - 0.0f * a.inv_dt);
        float o1 = r3.y;
        const float u1 = o1 + lam;
        float n1 = fminf(fmaxf(u1, -maxf), maxf);
        float j1 = n1 - o1;
        apply(la, wa, lb, wb, appa, appb, ima, imb, t1, a1a, a1b, j1);
        rel += kt1 * j1;
        vt = dot(rel, t2);
        lam = -r4.z * (vt - 0.0f * a.inv_dt);
        float o2 = r3.z;
        const float u2 = o2 + lam;
        float n2 = fminf(fmaxf(u2, -maxf), maxf);
        float j2 = n2 - o2;
        apply(la, wa, lb, wb, appa, appb, ima, imb, t2, a2a, a2b, j2);
        const float4 nr3 = make_float4(nimp, n1, n2, r3.w);
        if (a.srec) {  // the forward values the adjoint's frozen linearisation needs
            const uint32_t s1 = u1 > maxf ? 1u : (u1 < -maxf ? 2u : 0u);
            const uint32_t s2 = u2 > maxf ? 1u : (u2 < -maxf ? 2u : 0u);
            a.srec[sweep_index(sweep, k, t, a.iterations)] = make_float4(vn, nimp, __uint_as_float(s1 | (s2 << 2)), 0.0f);
        }
        e[VT_IMP * PLANE_STRIDE] = nr3;
        if (last) a.rows[(size_t(p) * 4 + k) * ROW_F4 + 3] = nr3;
    }
}

// split_impulse_pass body (sequential_impulse.rs:759-786) for split slot t; the
// first sweep fills the slot's split table, the last writes row 5 back.
__device__ __forceinline__ void split_group(const SolveArgs& a, uint32_t t, uint32_t p, uint32_t cnt, uint32_t ia,
                                            uint32_t ib, bool first, bool last, V3& pla, V3& pwa, V3& plb, V3& pwb,
                                            bool& appa, bool& appb) {
    const float4* e0 = a.stab + tix<ST_PLANES>(0, 0, t);
    float ima, imb;
    M3 iwa, iwb;
    if (first) {
        iwa = load_iw(a.iw, ia, ima);
        iwb = load_iw(a.iw, ib, imb);
    } else {
        ima = e0[3 * PLANE_STRIDE].w;
        imb = e0[4 * PLANE_STRIDE].w;
    }
    appa = ima > 0.0f;
    appb = imb > 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) {
        float4* e = a.stab + tix<ST_PLANES>(0, k, t);
        float4 q0, q1, q2, q3, q4, r5;
        if (first) {
            const float4* r = a.rows + (size_t(p) * 4 + k) * ROW_F4;
            const float4 r0 = r[0], r1 = r[1], r2 = r[2], r4 = r[4];
            r5 = r[5];
            const V3 n = from4(r0), ra = from4(r1), rb = from4(r2);
            const V3 ana = mul(iwa, cross(ra, n)), anb = mul(iwb, cross(rb, n));
            q0 = f4(n, r4.x);
            q1 = f4(ra, r4.w);
            q2 = f4(rb, 0.0f);
            q3 = f4(ana, ima);
            q4 = f4(anb, imb);
            e[0 * PLANE_STRIDE] = q0;
            e[1 * PLANE_STRIDE] = q1;
            e[2 * PLANE_STRIDE] = q2;
            e[3 * PLANE_STRIDE] = q3;
            e[4 * PLANE_STRIDE] = q4;
        } else {
            r5 = e[5 * PLANE_STRIDE];
        }
        if (r5.z == 0.0f) {
            if (first) e[5 * PLANE_STRIDE] = r5;
            continue;
        }
        if (!first) {
            q0 = e[0 * PLANE_STRIDE];
            q1 = e[1 * PLANE_STRIDE];
            q2 = e[2 * PLANE_STRIDE];
            q3 = e[3 * PLANE_STRIDE];
            q4 = e[4 * PLANE_STRIDE];
        }
        const V3 n = from4(q0), ra = from4(q1), rb = from4(q2), ana = from4(q3), anb = from4(q4);
        const float nmass = q0.w, cfm = q1.w;
        V3 pva = pla + cross(pwa, ra);
        V3 pvb = plb + cross(pwb, rb);
        float pvn = dot(pvb - pva, n);
        float delta = cfm != 0.0f ? r5.x - pvn * nmass - cfm * r5.y : r5.x - pvn * nmass;
        float old = r5.y;
        float np = fmaxf(old + delta, 0.0f);
        float j = np - old;
        if (j != 0.0f) {
            if (appa) { pla -= n * (j * ima); pwa -= ana * j; }
            if (appb) { plb += n * (j * imb); pwb += anb * j; }
        }
        const float4 nr5 = make_float4(r5.x, np, r5.z, r5.w);
        e[5 * PLANE_STRIDE] = nr5;
        if (last) a.rows[(size_t(p) * 4 + k) * ROW_F4 + 5] = nr5;
    }
}

// One group: velocities (or push velocities) from L2, the group's solve, the
// dynamic bodies' new velocities back to L2.
template <int KIND>
__device__ __forceinline__ void run_group(const SolveArgs& a, uint32_t t, uint4 rec, uint32_t sweep, uint32_t last) {
    const uint32_t ia = rec.x, ib = rec.y, p = rec.z & 0x1fffffffu, cnt = rec.z >> 29;
    float4* plin = KIND == SPLIT ? a.push_lin : a.linvel;
    float4* pang = KIND == SPLIT ? a.push_ang : a.angvel;
    V3 la = from4(__ldcg(&plin[ia])), wa = from4(__ldcg(&pang[ia]));
    V3 lb = from4(__ldcg(&plin[ib])), wb = from4(__ldcg(&pang[ib]));
    bool appa, appb;  // only dynamic bodies move
    if (KIND == WARM) warm_group(a, t, p, cnt, ia, ib, la, wa, lb, wb, appa, appb);
    else if (KIND == ITER) iter_group(a, t, p, cnt, sweep, sweep == last, la, wa, lb, wb, appa, appb);
    else split_group(a, t, p, cnt, ia, ib, sweep == 0, sweep == last, la, wa, lb, wb, appa, appb);
    if (appa) { __stcg(&plin[ia], to4(la, 0.0f)); __stcg(&pang[ia], to4(wa, 0.0f)); }
    if (appb) { __stcg(&plin[ib], to4(lb, 0.0f)); __stcg(&pang[ib], to4(wb, 0.0f)); }
}

// Bring all of a slot's table entries into L2 (the next phase's group, while the
// team waits at the barrier): the tables of a large pile outgrow L2, so without
// this the first loads after the barrier would wait for DRAM. (Into L1 instead
// measured the same: the barrier's acquire drops L1. Asking for a group's later
// contacts into L1 at the start of its solve measured slower.)
template <bool VELOCITY>
__device__ __forceinline__ void prefetch_slot_l2(const SolveArgs& a, uint32_t t, uint32_t cnt) {
    for (uint32_t k = 0; k < cnt; ++k) {
        if (VELOCITY) {
            const float4* e = a.vtab + tix<VT_PLANES>(0, k, t);
            for (uint32_t pl = 0; pl < VT_PLANES; ++pl) prefetch_l2(e + pl * PLANE_STRIDE);
        } else {
            const float4* e = a.stab + tix<ST_PLANES>(0, k, t);
            for (uint32_t pl = 0; pl < ST_PLANES; ++pl) prefetch_l2(e + pl * PLANE_STRIDE);
        }
    }
}

template <bool VELOCITY>
__device__ __forceinline__ void run_item(const SolveArgs& a, uint32_t sweep, uint32_t last, uint32_t t, uint4 rec) {
    if (!VELOCITY) run_group<SPLIT>(a, t, rec, sweep, last);
    else if (sweep == 0) run_group<WARM>(a, t, rec, sweep, last);
    else run_group<ITER>(a, t, rec, sweep, last);
}

// Phases 0 .. nphases-1 of a team: phase q is colour q % ncol of sweep q / ncol.
// The team's threads deal the batch slots of each phase among themselves and
// meet at the team barrier between phases; each thread reads its next slot
// record while it solves the current one.
//
// A colour with at most one block's worth of groups (the tail colours of a
// pile, or every colour of a small scene) is solved by the team's first block
// alone, one group per thread. Between two such colours the block syncs
// locally instead of the team meeting at a barrier: the other blocks go on to
// the next barrier and wait there.
template <bool VELOCITY>
__device__ __forceinline__ void run_phases(const SolveArgs& a, const uint4* __restrict__ recs, const uint32_t* soff,
                                           const uint32_t* send, uint32_t ncol, uint32_t nphases, uint32_t last, uint32_t tid,
                                           uint32_t stride, unsigned int* ctr, uint32_t team_blocks, uint32_t team_block,
                                           uint32_t& nbar, uint32_t sweep0 = 0) {
    if (ncol == 0 || nphases == 0) return;
    auto small = [&](uint32_t c) { return send[c] - soff[c] <= blockDim.x; };
    auto first_slot = [&](uint32_t c) -> uint32_t {
        if (!small(c)) return soff[c] + tid;
        return team_block == 0 ? soff[c] + threadIdx.x : send[c];
    };
    auto first_rec = [&](uint32_t c) -> uint4 {
        const uint32_t t = first_slot(c);
        return t < send[c] ? __ldg(&recs[t]) : make_uint4(0u, 0u, 0u, 0u);
    };
    uint4 rec = first_rec(0);  // rec.z == 0 (no rows): no slot for this thread
    for (uint32_t q = 0; q < nphases; ++q) {
        const uint32_t c = q % ncol, sweep = sweep0 + q / ncol;
        const uint4 next = q + 1 < nphases ? first_rec((q + 1) % ncol) : make_uint4(0u, 0u, 0u, 0u);
        if (rec.z) {
            const uint32_t t0 = first_slot(c);
            run_item<VELOCITY>(a, sweep, last, t0, rec);
            if (!small(c))
                for (uint32_t t = t0 + stride; t < send[c]; t += stride) run_item<VELOCITY>(a, sweep, last, t, __ldg(&recs[t]));
        }
        rec = next;
        if (q + 1 < nphases) {
            const uint32_t cn = (q + 1) % ncol;
            if (small(c) && small(cn)) {
                __syncthreads();  // global writes of the block are visible to the block after it
                continue;
            }
            // The next phase's table entries (written in sweep 0) head for L2 while the team waits.
            if (rec.z && (q + 1) >= ncol) prefetch_slot_l2<VELOCITY>(a, first_slot(cn), rec.z >> 29);
            team_barrier(ctr, ++nbar * team_blocks, a.status);
        }
    }
}

// One joint colour: slots [first, end) with the given stride.
__device__ __forceinline__ void joint_phase(JointsDev j, float4* linvel, float4* angvel, const float4* iw, float damping,
                                         uint32_t first, uint32_t end, uint32_t stride) {
    for (uint32_t t = first; t < end; t += stride) solve_joint_slot(j, t, linvel, angvel, iw, damping);
}

// The velocity team's sweeps in a world with joints: sweep by sweep, the contact phases,
// then (velocity sweeps only) one phase per joint colour (sequential_impulse.rs:720-735).
// Between two phases that block 0 runs alone (at most one block's worth of slots) the
// block syncs locally; otherwise the team meets at its barrier. Only the k_solve built
// for worlds with joints contains it.
__device__ __forceinline__ void velocity_sweeps_with_joints(const SolveArgs& a, const uint32_t* s_off, const uint32_t* s_end,
                                                         const uint32_t* s_joff, uint32_t ncol, uint32_t njcol,
                                                         uint32_t iters, uint32_t tid, uint32_t stride,
                                                         uint32_t team_blocks, uint32_t team_block, uint32_t& nbar) {
    auto csmall = [&](uint32_t c) { return s_end[c] - s_off[c] <= blockDim.x; };
    auto jsmall = [&](uint32_t c) { return s_joff[c + 1] - s_joff[c] <= blockDim.x; };
    auto sync = [&](bool local) {
        if (local) __syncthreads();
        else team_barrier(a.bar, ++nbar * team_blocks, a.status);
    };
    for (uint32_t sw = 0; sw <= iters; ++sw) {
        run_phases<true>(a, a.batch_rec, s_off, s_end, ncol, ncol, iters, tid, stride, a.bar, team_blocks, team_block,
                         nbar, sw);
        bool prev_small = ncol ? csmall(ncol - 1) : true;
        if (sw >= 1) {
            for (uint32_t jc = 0; jc < njcol; ++jc) {
                const bool small = jsmall(jc);
                sync(prev_small && small);
                const uint32_t lo = s_joff[jc], hi = s_joff[jc + 1];
                if (small) {
                    if (team_block == 0 && lo + threadIdx.x < hi)
                        joint_phase(a.j, a.linvel, a.angvel, a.iw, a.damping, lo + threadIdx.x, hi, blockDim.x);
                } else {
                    joint_phase(a.j, a.linvel, a.angvel, a.iw, a.damping, lo + tid, hi, stride);
                }
                prev_small = small;
            }
        }
        if (sw < iters) sync(prev_small && (ncol ? csmall(0) : true));
    }
}

// solve() (sequential_impulse.rs:692-705): warm start and velocity sweeps on
// the velocity team; the split sweeps on the split team, which has enough
// blocks for the largest split batch and at most a quarter of the grid (none
// on a grid too small to split, where the velocity team runs them last).
// JOINTS: the build for worlds with joints (the contact-only build carries none of their code).
template <bool JOINTS>
__global__ void __launch_bounds__(256, 2) k_solve(SolveArgs a) {
    const uint32_t ncol = a.scalars[4];
    const uint32_t nsplit = a.scalars[5];
    const uint32_t iters = a.iterations;
    const uint32_t G = gridDim.x;
    uint32_t split_blocks = 0;
    if (nsplit && iters && G >= 4) {
        uint32_t need = (a.scalars[11] + blockDim.x - 1) / blockDim.x;
        split_blocks = min(max(need, 1u), G / 4);
    }
    const bool split_team = blockIdx.x >= G - split_blocks;
    const uint32_t team_blocks = split_team ? split_blocks : G - split_blocks;
    const uint32_t team_block = split_team ? blockIdx.x - (G - split_blocks) : blockIdx.x;
    const uint32_t tid = team_block * blockDim.x + threadIdx.x;
    const uint32_t stride = team_blocks * blockDim.x;
    __shared__ uint32_t s_off[MAX_COLOURS], s_end[MAX_COLOURS], s_split_off[MAX_COLOURS], s_split_end[MAX_COLOURS];
    for (uint32_t c = threadIdx.x; c < ncol; c += blockDim.x) {
        s_off[c] = a.offset[c];
        s_end[c] = a.end[c];
        s_split_off[c] = a.split_offset[c];
        s_split_end[c] = a.split_end[c];
    }
    const uint32_t njcol = JOINTS ? a.j.ncol : 0u;
    __shared__ uint32_t s_joff[JOINTS ? MAX_COLOURS + 1 : 1];
    if (JOINTS)
        for (uint32_t c = threadIdx.x; c <= njcol && njcol; c += blockDim.x) s_joff[c] = a.j.coff[c];
    __syncthreads();  // the batch ranges above are read by every thread of the block
    uint32_t nbar = 0;
    if (split_team) {
        run_phases<false>(a, a.split_rec, s_split_off, s_split_end, ncol, iters * ncol, iters - 1u, tid, stride, a.bar + 1,
                          team_blocks, team_block, nbar);
        return;
    }
    if (!JOINTS || njcol == 0) {
        run_phases<true>(a, a.batch_rec, s_off, s_end, ncol, (iters + 1) * ncol, iters, tid, stride, a.bar, team_blocks,
                         team_block, nbar);
    } else {
        velocity_sweeps_with_joints(a, s_off, s_end, s_joff, ncol, njcol, iters, tid, stride, team_blocks, team_block, nbar);
    }
    if (nsplit && iters && split_blocks == 0) {
        team_barrier(a.bar, ++nbar * team_blocks, a.status);
        run_phases<false>(a, a.split_rec, s_split_off, s_split_end, ncol, iters * ncol, iters - 1u, tid, stride, a.bar, team_blocks,
                          team_block, nbar);
    }
}

// ---------------------------------------------------------------- per-world PGS (batched worlds)
// Every world of a batch is solved on its own by one CTA or one warp: its row groups are
// coloured in shared memory (Jones-Plassmann with the world's own priorities, colours from
// one 64-bit mask per body), sorted into colour batches, and solved phase by phase with only
// a block (or warp) sync between phases; its bodies' velocities and push velocities stay in
// shared memory for the whole solve. No barrier spans worlds. Within a world the order is the
// same (colour, pair) Gauss-Seidel order the global solver uses, so each world equals the
// reference's sequential solve over its rows in that order. The split sweeps touch only push
// velocities, so split sweep s runs in the phases of velocity sweep s + 1.
struct WorldSolveArgs {
    SolveArgs a;                       // rows, tables, adjoint sweep records, iw, constants
    const uint32_t* contact_pairs;     // pair ids with rows, ascending (so grouped by world)
    const uint32_t* ngroups;           // device count of contact_pairs
    const uint64_t* pairs;
    const uint32_t* row_count;
    const uint32_t* world_off;
    uint32_t* colour;                  // out: world-local colour per contact pair
    uint4* recs;                       // out: slot records, world by world, colour by colour
    uint32_t* wcol;                    // out: per world g0, ncol, offsets[ncol + 1]
    uint32_t* colour_count;            // out: groups per colour summed over worlds (stats)
    uint32_t* split_count;
    uint32_t* scalars;                 // out: [3] rows [4] colours (max) [5] split groups [10] split rows
    float4* linvel;
    float4* angvel;
    float4* push_lin;
    float4* push_ang;
    uint32_t* status;
    WorldPlanDev plan;
};

struct WorldCtx {  // per world being solved by a CTA or a warp
    uint32_t g0, g1, ncol, left, rows, split_groups, split_rows;
    uint32_t hist[WS_MAX_COLOURS], off[WS_MAX_COLOURS + 1], cur[WS_MAX_COLOURS], split_hist[WS_MAX_COLOURS];
};

template <bool WARP>
__device__ __forceinline__ void ws_sync() {
    if (WARP) __syncwarp();
    else __syncthreads();
}

__device__ __forceinline__ uint32_t lower_bound_lo(const uint64_t* __restrict__ pairs, const uint32_t* __restrict__ cp,
                                                   uint32_t n, uint32_t body) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key_lo(pairs[cp[mid]]) < body) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One group of a world: velocities from the world's shared-memory arrays (body i at i - b0).
template <int KIND>
__device__ __forceinline__ void run_group_shared(const SolveArgs& a, uint32_t t, uint4 rec, uint32_t sweep,
                                                 uint32_t last, float4* lin, float4* ang, uint32_t b0) {
    const uint32_t ia = rec.x, ib = rec.y, p = rec.z & 0x1fffffffu, cnt = rec.z >> 29;
    const uint32_t la_i = ia - b0, lb_i = ib - b0;
    V3 la = from4(lin[la_i]), wa = from4(ang[la_i]);
    V3 lb = from4(lin[lb_i]), wb = from4(ang[lb_i]);
    bool appa, appb;
    if (KIND == WARM) warm_group(a, t, p, cnt, ia, ib, la, wa, lb, wb, appa, appb);
    else if (KIND == ITER) iter_group(a, t, p, cnt, sweep, sweep == last, la, wa, lb, wb, appa, appb);
    else split_group(a, t, p, cnt, ia, ib, sweep == 0, sweep == last, la, wa, lb, wb, appa, appb);
    if (appa) { lin[la_i] = to4(la, 0.0f); ang[la_i] = to4(wa, 0.0f); }
    if (appb) { lin[lb_i] = to4(lb, 0.0f); ang[lb_i] = to4(wb, 0.0f); }
}

// The whole PGS of world w by `nt` threads (lane = 0 .. nt - 1), `sm` its 4 * nb float4 of
// shared memory, `C` its context. Every thread of the CTA (block mode) or of the warp (warp
// mode) calls it; every early return is taken by all of them together, so every sync is
// reached by all of them.
template <bool WARP>
__device__ void solve_world(const WorldSolveArgs& A, uint32_t w, uint32_t lane, uint32_t nt, float4* sm, WorldCtx& C) {
    const SolveArgs& a = A.a;
    const uint32_t b0 = A.world_off[w], nb = A.world_off[w + 1] - b0;
    float4* lin = sm;
    float4* ang = sm + nb;
    float4* plin = sm + 2 * nb;
    float4* pang = sm + 3 * nb;
    // Colouring scratch over the push-velocity region (24 of its 32 bytes per body).
    unsigned long long* mask = reinterpret_cast<unsigned long long*>(plin);
    unsigned long long* best0 = mask + nb;
    unsigned long long* best1 = best0 + nb;
    for (uint32_t i = lane; i < nb; i += nt) {
        lin[i] = __ldcg(&A.linvel[b0 + i]);
        ang[i] = __ldcg(&A.angvel[b0 + i]);
        mask[i] = 0ull;
        best0[i] = 0ull;
        best1[i] = 0ull;
    }
    if (lane == 0) {
        const uint32_t K = *A.ngroups;
        C.g0 = lower_bound_lo(A.pairs, A.contact_pairs, K, b0);
        C.g1 = lower_bound_lo(A.pairs, A.contact_pairs, K, b0 + nb);
        C.left = C.g1 - C.g0;
        C.ncol = 0;
        C.rows = C.split_groups = C.split_rows = 0;
    }
    for (uint32_t c = lane; c < WS_MAX_COLOURS; c += nt) {
        C.hist[c] = 0;
        C.split_hist[c] = 0;
    }
    ws_sync<WARP>();
    const uint32_t g0 = C.g0, g1 = C.g1;
    if (g0 == g1 && !a.j.ncol) {  // no rows in this world: its velocities stay as they are
        if (lane == 0) {  // an empty record (the adjoint's reverse pass reads every world's)
            A.wcol[size_t(w) * WS_STRIDE] = g0;
            A.wcol[size_t(w) * WS_STRIDE + 1] = 0;
        }
        return;
    }
    auto dyn = [&](uint32_t i) { return inv_mass_of(a.iw, i) > 0.0f; };
    // 1. Jones-Plassmann rounds: an uncoloured group wins when its priority is the largest
    //    among the uncoloured groups at each of its dynamic bodies; a winner takes the lowest
    //    colour free at both bodies (winners of one round share no dynamic body).
    for (uint32_t g = g0 + lane; g < g1; g += nt) A.colour[g] = NO_COLOUR;
    ws_sync<WARP>();
    for (uint32_t r = 0; C.left != 0; ++r) {
        if (r >= MAX_ROUNDS) {
            if (lane == 0) atomicOr(A.status, ST_COLOUR_ROUNDS);
            break;
        }
        unsigned long long* best = (r & 1) ? best1 : best0;
        unsigned long long* other = (r & 1) ? best0 : best1;
        for (uint32_t g = g0 + lane; g < g1; g += nt) {
            if (A.colour[g] != NO_COLOUR) continue;
            const uint64_t key = A.pairs[A.contact_pairs[g]];
            const unsigned long long v = (static_cast<unsigned long long>(mix32(key)) << 32) | (g - g0 + 1u);
            const uint32_t ia = key_lo(key), ib = key_hi(key);
            if (dyn(ia)) atomicMax(&best[ia - b0], v);
            if (dyn(ib)) atomicMax(&best[ib - b0], v);
        }
        ws_sync<WARP>();
        uint32_t won = 0;
        for (uint32_t g = g0 + lane; g < g1; g += nt) {
            if (A.colour[g] != NO_COLOUR) continue;
            const uint64_t key = A.pairs[A.contact_pairs[g]];
            const unsigned long long v = (static_cast<unsigned long long>(mix32(key)) << 32) | (g - g0 + 1u);
            const uint32_t ia = key_lo(key), ib = key_hi(key);
            const bool da = dyn(ia), db = dyn(ib);
            if ((da && best[ia - b0] != v) || (db && best[ib - b0] != v)) continue;
            const unsigned long long m = (da ? mask[ia - b0] : 0ull) | (db ? mask[ib - b0] : 0ull);
            int c = __ffsll(static_cast<long long>(~m)) - 1;
            if (c < 0) {  // 64 colours taken at one body
                atomicOr(A.status, ST_COLOUR_OVERFLOW);
                c = int(WS_MAX_COLOURS) - 1;
            }
            A.colour[g] = uint32_t(c);
            if (da) mask[ia - b0] |= 1ull << c;
            if (db) mask[ib - b0] |= 1ull << c;
            ++won;
        }
        for (uint32_t i = lane; i < nb; i += nt) other[i] = 0ull;
        if (won) atomicSub(&C.left, won);
        ws_sync<WARP>();
    }
    // 2. Colour batches: histogram, offsets, scatter of the slot records.
    for (uint32_t g = g0 + lane; g < g1; g += nt) {
        const uint32_t c = A.colour[g];
        if (c >= WS_MAX_COLOURS) continue;  // left uncoloured (round limit; the status word says so)
        atomicAdd(&C.hist[c], 1u);
        atomicMax(&C.ncol, c + 1u);
    }
    ws_sync<WARP>();
    const uint32_t ncol = C.ncol;
    if (lane == 0) {
        uint32_t acc = 0;
        uint32_t* rec = A.wcol + size_t(w) * WS_STRIDE;
        rec[0] = g0;
        rec[1] = ncol;
        for (uint32_t c = 0; c < ncol; ++c) {
            C.off[c] = acc;
            C.cur[c] = acc;
            rec[2 + c] = acc;
            acc += C.hist[c];
        }
        C.off[ncol] = acc;
        rec[2 + ncol] = acc;
        if (ncol) atomicMax(&A.scalars[4], ncol);
    }
    ws_sync<WARP>();
    uint32_t my_rows = 0, my_split_groups = 0, my_split_rows = 0;
    for (uint32_t g = g0 + lane; g < g1; g += nt) {
        const uint32_t c = A.colour[g];
        if (c >= WS_MAX_COLOURS) continue;
        const uint32_t slot = g0 + atomicAdd(&C.cur[c], 1u);
        const uint32_t p = A.contact_pairs[g];
        const uint64_t key = A.pairs[p];
        const uint32_t cnt = A.row_count[p];
        uint32_t nsplit = 0;
        for (uint32_t k = 0; k < cnt; ++k) nsplit += a.rows[(size_t(p) * 4 + k) * ROW_F4 + 5].z != 0.0f ? 1u : 0u;
        A.recs[slot] = make_uint4(key_lo(key), key_hi(key), p | (cnt << 29), nsplit ? 1u : 0u);
        my_rows += cnt;
        if (nsplit) {
            ++my_split_groups;
            my_split_rows += nsplit;
            atomicAdd(&C.split_hist[c], 1u);
        }
    }
    if (my_rows) atomicAdd(&C.rows, my_rows);
    if (my_split_groups) {
        atomicAdd(&C.split_groups, my_split_groups);
        atomicAdd(&C.split_rows, my_split_rows);
    }
    ws_sync<WARP>();  // the colouring scratch is free from here on
    for (uint32_t i = lane; i < nb; i += nt) {
        plin[i] = __ldcg(&A.push_lin[b0 + i]);
        pang[i] = __ldcg(&A.push_ang[b0 + i]);
    }
    if (lane == 0) {
        atomicAdd(&A.scalars[3], C.rows);
        if (C.split_groups) {
            atomicAdd(&A.scalars[5], C.split_groups);
            atomicAdd(&A.scalars[10], C.split_rows);
        }
    }
    for (uint32_t c = lane; c < ncol; c += nt) {
        atomicAdd(&A.colour_count[c], C.hist[c]);
        if (C.split_hist[c]) atomicAdd(&A.split_count[c], C.split_hist[c]);
    }
    ws_sync<WARP>();
    // 3. Warm start and velocity sweeps; split sweep s rides along velocity sweep s + 1.
    const uint32_t iters = a.iterations;
    for (uint32_t sweep = 0; sweep <= iters; ++sweep) {
        for (uint32_t c = 0; c < ncol; ++c) {
            const uint32_t hi = g0 + C.off[c + 1];
            for (uint32_t t = g0 + C.off[c] + lane; t < hi; t += nt) {
                const uint4 rec = A.recs[t];
                if (sweep == 0) run_group_shared<WARM>(a, t, rec, 0, iters, lin, ang, b0);
                else run_group_shared<ITER>(a, t, rec, sweep, iters, lin, ang, b0);
                if (sweep >= 1 && rec.w) run_group_shared<SPLIT>(a, t, rec, sweep - 1, iters - 1, plin, pang, b0);
            }
            ws_sync<WARP>();
        }
        // sequential_impulse.rs:720-735: a velocity sweep's joint rows follow its contacts (the
        // host allows joints here only for a plain world, whose bodies start at 0).
        if (sweep >= 1 && a.j.ncol) {
            for (uint32_t jc = 0; jc < a.j.ncol; ++jc) {
                const uint32_t hi = a.j.coff[jc + 1];
                for (uint32_t t = a.j.coff[jc] + lane; t < hi; t += nt)
                    solve_joint_slot<true>(a.j, t, lin, ang, a.iw, a.damping);
                ws_sync<WARP>();
            }
        }
    }
    // 4. The world's velocities and push velocities back to global memory.
    for (uint32_t i = lane; i < nb; i += nt) {
        __stcg(&A.linvel[b0 + i], lin[i]);
        __stcg(&A.angvel[b0 + i], ang[i]);
        __stcg(&A.push_lin[b0 + i], plin[i]);
        __stcg(&A.push_ang[b0 + i], pang[i]);
    }
}

__global__ void __launch_bounds__(256) k_world_solve(WorldSolveArgs A) {
    extern __shared__ float4 ws_dyn[];
    __shared__ WorldCtx ctx[WS_MAX_WARPS];
    const uint2 c = A.plan.cta[blockIdx.x];
    const bool block_mode = (c.y >> 31) != 0u;
    const uint32_t count = c.y & 0x7fffffffu;
    if (block_mode) {
        solve_world<false>(A, A.plan.list[c.x], threadIdx.x, blockDim.x, ws_dyn, ctx[0]);
        return;
    }
    const uint32_t wi = threadIdx.x >> 5;
    if (wi >= count) return;  // warp mode: warps never sync with each other
    uint32_t off = 0;
    for (uint32_t j = 0; j < wi; ++j) {
        const uint32_t wj = A.plan.list[c.x + j];
        off += A.world_off[wj + 1] - A.world_off[wj];
    }
    solve_world<true>(A, A.plan.list[c.x + wi], threadIdx.x & 31u, 32u, ws_dyn + 4 * size_t(off), ctx[wi]);
}

// ---------------------------------------------------------------- cache update
// step.rs:982-1005: the solved normal impulse goes back to its manifold point.
__global__ void k_writeback(uint32_t npairs, const uint32_t* __restrict__ row_count, const float4* __restrict__ rows,
                            float4* entries, uint32_t* valid_flags) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    float4* e = entries + size_t(p) * ENTRY_F4;
    uint32_t n = row_count[p];
    for (uint32_t k = 0; k < n; ++k) {
        float imp = rows[(size_t(p) * 4 + k) * ROW_F4 + 3].x;
        float4 y = e[5 + 3 * k];
        y.w = imp;
        e[5 + 3 * k] = y;
    }
    valid_flags[p] = (__float_as_uint(e[2].w) & META_VALID) ? 1u : 0u;
}

// step.rs:1006-1010: with prune = simulate && prev_simulate (of the manifold's world), manifolds
// whose pair vanished die; otherwise the unowned old manifolds survive.
__global__ void k_flag_unowned(uint32_t nold, const uint32_t* __restrict__ owned, const uint64_t* __restrict__ old_keys,
                               const uint32_t* __restrict__ world_of, const uint32_t* __restrict__ simulate,
                               const uint32_t* __restrict__ prev_simulate, uint32_t* flags) {
    uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nold) return;
    uint32_t w = world_of ? world_of[key_lo(old_keys[o])] : 0u;
    bool prune = (simulate[w] != 0) && (prev_simulate[w] != 0);
    flags[o] = (!prune && !owned[o]) ? 1u : 0u;
}

__device__ __forceinline__ uint32_t lower_bound_pairs(const uint64_t* __restrict__ pairs, const uint32_t* __restrict__ sel,
                                                      uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (pairs[sel[mid]] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t lower_bound_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ sel,
                                                     uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (keys[sel[mid]] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Merge the surviving current manifolds (A, pair order) with the surviving old ones (B, key order).
__global__ void k_merge(const uint64_t* __restrict__ pairs, const float4* __restrict__ cur_entries,
                        const uint32_t* __restrict__ sel_a, const uint32_t* __restrict__ na_ptr,
                        const uint64_t* __restrict__ old_keys, const float4* __restrict__ old_entries,
                        const uint32_t* __restrict__ sel_b, const uint32_t* __restrict__ nb_ptr, uint64_t* out_keys,
                        float4* out_entries, uint32_t* out_count, uint32_t* rec_merge_pos) {
    uint32_t na = *na_ptr, nb = *nb_ptr;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *out_count = na + nb;
    if (t < na) {
        uint32_t p = sel_a[t];
        uint64_t key = pairs[p];
        uint32_t pos = t + (nb ? lower_bound_keys(old_keys, sel_b, nb, key) : 0u);
        out_keys[pos] = key;
        if (rec_merge_pos) rec_merge_pos[p] = pos;
        const float4* src = cur_entries + size_t(p) * ENTRY_F4;
        float4* dst = out_entries + size_t(pos) * ENTRY_F4;
        for (int q = 0; q < ENTRY_F4; ++q) dst[q] = src[q];
    } else if (t < na + nb) {
        uint32_t b = t - na;
        uint32_t o = sel_b[b];
        uint64_t key = old_keys[o];
        uint32_t pos = b + lower_bound_pairs(pairs, sel_a, na, key);
        out_keys[pos] = key;
        const float4* src = old_entries + size_t(o) * ENTRY_F4;
        float4* dst = out_entries + size_t(pos) * ENTRY_F4;
        for (int q = 0; q < ENTRY_F4; ++q) dst[q] = src[q];
    }
}

// A barrier whose target counts one block more than the grid has: nothing completes it.
__global__ void k_wait_selftest(unsigned int* ctr, uint32_t* status, unsigned long long limit_ns) {
    team_barrier(ctr, gridDim.x + 1u, status, limit_ns);
}

int coop_grid(const void* fn, int block, size_t smem) {
    static int sms = -1;
    if (sms < 0) {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
    }
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem), "occupancy");
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

}  // namespace

// PGS (cooperative launch: the teams' barriers need every block resident).
static void launch_solve(const WorldView& w, PairData& pd, const StepParams& sp, uint32_t* status_dev, cudaStream_t s,
                         const JointsDev* joints) {
    const int TB = 256;
    check_cuda(cudaMemsetAsync(pd.barrier.p, 0, 2 * sizeof(unsigned int), s), "memset barrier");
    SolveArgs sa{pd.rows.p, pd.batch_rec.p, pd.colour_offset.p, pd.colour_cursor.p, pd.split_rec.p,
                 pd.split_offset.p, pd.split_cursor.p, pd.scalars.p, w.b.linvel, w.b.angvel, w.b.push_lin,
                 w.b.push_ang, w.b.iw, pd.vtab.p, pd.stab.p, pd.rec.sweeps,
                 pd.barrier.p, status_dev, sp.inv_dt, sp.info.restitution_velocity_threshold,
                 sp.info.num_iterations, joints ? *joints : JointsDev{}, sp.info.damping};
    const void* fn = joints ? (const void*)k_solve<true> : (const void*)k_solve<false>;
    static int solve_grid[2] = {0, 0};
    int& grid = solve_grid[joints ? 1 : 0];
    if (!grid) grid = coop_grid(fn, TB, 0);
    void* sargs[] = {&sa};
    check_cuda(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(TB), sargs, 0, s), "solve launch");
}

void run_wait_selftest(unsigned long long limit_ns, unsigned int* ctr, uint32_t* status, cudaStream_t s) {
    k_wait_selftest<<<2, 32, 0, s>>>(ctr, status, limit_ns);
}

void run_solver(const WorldView& w, const uint64_t* pairs, uint32_t npairs, PairData& pd, const StepParams& sp,
                uint32_t* status_dev, cudaStream_t s, const std::function<void(int)>& mark, bool seed_colours,
                const JointsDev* joints) {
    const bool with_joints = joints && joints->n && joints->ncol;
    if (npairs == 0) {
        check_cuda(cudaMemsetAsync(pd.scalars.p + 2, 0, 4 * sizeof(uint32_t), s), "memset");
        check_cuda(cudaMemsetAsync(pd.scalars.p + 10, 0, 2 * sizeof(uint32_t), s), "memset");
        mark(5);
        if (with_joints) launch_solve(w, pd, sp, status_dev, s, joints);
        mark(6);
        return;
    }
    const int TB = 256;
    if (npairs >= (1u << 29)) throw CudaError{cudaErrorInvalidValue, "more than 2^29 pairs for the solver's slot records"};
    // Contact pairs (ascending pair order).
    k_flag_contact_pairs<<<(npairs + TB - 1) / TB, TB, 0, s>>>(npairs, pd.row_count.p, pd.flags.p);
    size_t bytes = 0;
    cub::CountingInputIterator<uint32_t> it(0);
    check_cuda(cub::DeviceSelect::Flagged(nullptr, bytes, it, pd.flags.p, pd.contact_pairs.p, pd.scalars.p + 2,
                                          int(npairs), s), "select size");
    pd.cub_tmp.reserve(bytes);
    check_cuda(cub::DeviceSelect::Flagged(pd.cub_tmp.p, bytes, it, pd.flags.p, pd.contact_pairs.p, pd.scalars.p + 2,
                                          int(npairs), s), "select");
    // Colouring (cooperative launch).
    check_cuda(cudaMemsetAsync(pd.barrier.p, 0, 16 * sizeof(unsigned int), s), "memset barrier");
    ColourArgs ca{pd.scalars.p + 2, pd.contact_pairs.p, pairs, w.b.iw, pd.colour.p, pd.body_prio.p, pd.body_mask.p,
                  pd.body_dup.p, pd.entries.p, seed_colours ? 1u : 0u, pd.barrier.p, status_dev};
    static int colour_grid = 0;
    if (!colour_grid) colour_grid = coop_grid((const void*)k_colour, TB, 0);
    pd.colour_work.reserve(2 * size_t(npairs) + 2);
    JpList wl{{pd.colour_work.p, pd.colour_work.p + npairs}, {pd.barrier.p + 6, pd.barrier.p + 7}};
    void* cargs[] = {&ca, &wl};
    check_cuda(cudaLaunchCooperativeKernel((const void*)k_colour, dim3(colour_grid), dim3(TB), cargs, 0, s),
               "colour launch");
    // Batches.
    check_cuda(cudaMemsetAsync(pd.colour_count.p, 0, (MAX_COLOURS + 3) * sizeof(uint32_t), s), "memset");
    check_cuda(cudaMemsetAsync(pd.split_count.p, 0, (MAX_COLOURS + 3) * sizeof(uint32_t), s), "memset");
    pd.colour_sub.reserve(2 * 4 * MAX_COLOURS);
    uint32_t* sub_hist = pd.colour_sub.p;
    uint32_t* sub_cursor = pd.colour_sub.p + 4 * MAX_COLOURS;
    check_cuda(cudaMemsetAsync(sub_hist, 0, 4 * MAX_COLOURS * sizeof(uint32_t), s), "memset");
    uint32_t g = std::min<uint32_t>((npairs + TB - 1) / TB, 148u * 8u);
    k_colour_hist<<<g, TB, 0, s>>>(pd.scalars.p + 2, pd.contact_pairs.p, pd.colour.p, pd.row_count.p, pd.rows.p,
                                   pd.colour_count.p, pd.split_count.p, pd.flags.p, sub_hist);
    k_colour_scan<<<1, 32, 0, s>>>(pd.colour_count.p, pd.colour_offset.p, pd.colour_cursor.p, pd.split_count.p,
                                   pd.split_offset.p, pd.split_cursor.p, pd.barrier.p, pd.scalars.p, pd.colour_remap.p,
                                   sub_hist, sub_cursor);
    k_colour_scatter<<<g, TB, 0, s>>>(pd.scalars.p + 2, pd.contact_pairs.p, pairs, pd.row_count.p, pd.colour.p,
                                      pd.flags.p, sub_cursor, pd.split_cursor.p, pd.batch_rec.p,
                                      pd.split_rec.p, pd.entries.p, pd.colour_remap.p);
    mark(5);
    // Slot capacity: every group plus the 32-alignment padding of each batch.
    const size_t slots = (size_t(npairs) + 32u * (MAX_COLOURS + 1) + 31u) & ~size_t(31);
    pd.vtab.reserve(size_t(VT_PLANES) * 4 * slots);
    pd.stab.reserve(size_t(ST_PLANES) * 4 * slots);
    launch_solve(w, pd, sp, status_dev, s, with_joints ? joints : nullptr);
    mark(6);
}

bool build_world_plan(const std::vector<uint32_t>& world_off, uint32_t block, uint32_t tau, WorldPlan& plan,
                      cudaStream_t s) {
    plan.valid = false;
    if (block < 32 || block > 32 * WS_MAX_WARPS || block % 32) return false;
    const uint32_t nw = world_off.empty() ? 0u : uint32_t(world_off.size() - 1);
    std::vector<uint32_t> order(nw);
    for (uint32_t k = 0; k < nw; ++k) order[k] = k;
    auto size = [&](uint32_t k) { return world_off[k + 1] - world_off[k]; };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return size(x) > size(y); });
    const size_t smem_cap = 200u * 1024u;  // leaves room for the static contexts and L1
    std::vector<uint2> cta;
    size_t smem = 0;
    const uint32_t per_cta = block / 32;
    uint32_t k = 0;
    while (k < nw) {
        const uint32_t nb = size(order[k]);
        if (nb > tau) {  // block mode: one world per CTA
            if (size_t(nb) * WS_SMEM_PER_BODY > smem_cap) return false;
            cta.push_back(make_uint2(k, 1u | (1u << 31)));
            smem = std::max(smem, size_t(nb) * WS_SMEM_PER_BODY);
            ++k;
            continue;
        }
        uint32_t cnt = 0;
        size_t bodies = 0;
        while (k + cnt < nw && cnt < per_cta && (bodies + size(order[k + cnt])) * WS_SMEM_PER_BODY <= smem_cap) {
            bodies += size(order[k + cnt]);
            ++cnt;
        }
        if (cnt == 0) return false;
        cta.push_back(make_uint2(k, cnt));
        smem = std::max(smem, bodies * WS_SMEM_PER_BODY);
        k += cnt;
    }
    plan.cta.reserve(std::max<size_t>(cta.size(), 1));
    plan.list.reserve(std::max<uint32_t>(nw, 1));
    if (!cta.empty())
        check_cuda(cudaMemcpyAsync(plan.cta.p, cta.data(), cta.size() * sizeof(uint2), cudaMemcpyHostToDevice, s), "h2d");
    if (nw) check_cuda(cudaMemcpyAsync(plan.list.p, order.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "h2d");
    check_cuda(cudaStreamSynchronize(s), "sync");  // the host vectors go out of scope
    // Without this opt-in, dynamic shared memory is limited to 48 KB minus the kernel's static part.
    check_cuda(cudaFuncSetAttribute((const void*)k_world_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem)), "smem attribute");
    plan.ncta = uint32_t(cta.size());
    plan.block = block;
    plan.tau = tau;
    plan.smem = smem;
    plan.valid = true;
    return true;
}

void run_world_solver(const WorldView& w, const uint64_t* pairs, uint32_t npairs, PairData& pd, const StepParams& sp,
                      uint32_t* status_dev, cudaStream_t s, const std::function<void(int)>& mark,
                      const uint32_t* world_off, uint32_t nworlds, const WorldPlan& plan, uint32_t* wcol,
                      const JointsDev* joints) {
    const bool with_joints = joints && joints->n && joints->ncol;
    check_cuda(cudaMemsetAsync(pd.scalars.p + 2, 0, 4 * sizeof(uint32_t), s), "memset");
    check_cuda(cudaMemsetAsync(pd.scalars.p + 10, 0, 2 * sizeof(uint32_t), s), "memset");
    check_cuda(cudaMemsetAsync(pd.colour_count.p, 0, (MAX_COLOURS + 3) * sizeof(uint32_t), s), "memset");
    check_cuda(cudaMemsetAsync(pd.split_count.p, 0, (MAX_COLOURS + 3) * sizeof(uint32_t), s), "memset");
    if (nworlds == 0 || (npairs == 0 && !with_joints)) {
        mark(5);
        mark(6);
        return;
    }
    const int TB = 256;
    if (npairs >= (1u << 29)) throw CudaError{cudaErrorInvalidValue, "more than 2^29 pairs for the solver's slot records"};
    if (npairs)
        k_flag_contact_pairs<<<(npairs + TB - 1) / TB, TB, 0, s>>>(npairs, pd.row_count.p, pd.flags.p);
    size_t bytes = 0;
    cub::CountingInputIterator<uint32_t> it(0);
    if (npairs) {
        check_cuda(cub::DeviceSelect::Flagged(nullptr, bytes, it, pd.flags.p, pd.contact_pairs.p, pd.scalars.p + 2,
                                              int(npairs), s), "select size");
        pd.cub_tmp.reserve(bytes);
        check_cuda(cub::DeviceSelect::Flagged(pd.cub_tmp.p, bytes, it, pd.flags.p, pd.contact_pairs.p,
                                              pd.scalars.p + 2, int(npairs), s), "select");
    }
    mark(5);
    const size_t slots = (size_t(npairs) + 32u * (MAX_COLOURS + 1) + 31u) & ~size_t(31);
    pd.vtab.reserve(size_t(VT_PLANES) * 4 * slots);
    pd.stab.reserve(size_t(ST_PLANES) * 4 * slots);
    WorldSolveArgs A;
    A.a = SolveArgs{pd.rows.p, pd.batch_rec.p, pd.colour_offset.p, pd.colour_cursor.p, pd.split_rec.p,
                    pd.split_offset.p, pd.split_cursor.p, pd.scalars.p, w.b.linvel, w.b.angvel, w.b.push_lin,
                    w.b.push_ang, w.b.iw, pd.vtab.p, pd.stab.p, pd.rec.sweeps,
                    pd.barrier.p, status_dev, sp.inv_dt, sp.info.restitution_velocity_threshold,
                    sp.info.num_iterations, with_joints ? *joints : JointsDev{}, sp.info.damping};
    A.contact_pairs = pd.contact_pairs.p;
    A.ngroups = pd.scalars.p + 2;
    A.pairs = pairs;
    A.row_count = pd.row_count.p;
    A.world_off = world_off;
    A.colour = pd.colour.p;
    A.recs = pd.batch_rec.p;
    A.wcol = wcol;
    A.colour_count = pd.colour_count.p;
    A.split_count = pd.split_count.p;
    A.scalars = pd.scalars.p;
    A.linvel = w.b.linvel;
    A.angvel = w.b.angvel;
    A.push_lin = w.b.push_lin;
    A.push_ang = w.b.push_ang;
    A.status = status_dev;
    A.plan = plan.dev();
    k_world_solve<<<plan.ncta, plan.block, plan.smem, s>>>(A);
    check_cuda(cudaGetLastError(), "world solve launch");
    mark(6);
}

void run_cache_update(const uint64_t* pairs, uint32_t npairs, const Manifolds& old_cache, PairData& pd,
                      Manifolds& next, const uint32_t* world_of, const uint32_t* simulate_flag,
                      const uint32_t* prev_simulate, cudaStream_t s) {
    const int TB = 256;
    uint32_t nold_cap = old_cache.count_host;
    // A: surviving manifolds of the current pairs.
    if (npairs) k_writeback<<<(npairs + TB - 1) / TB, TB, 0, s>>>(npairs, pd.row_count.p, pd.rows.p, pd.entries.p,
                                                                  pd.flags.p);
    cub::CountingInputIterator<uint32_t> it(0);
    size_t bytes_a = 0, bytes_b = 0;
    uint32_t* na_dev = pd.scalars.p + 8;
    uint32_t* nb_dev = pd.scalars.p + 9;
    check_cuda(cudaMemsetAsync(na_dev, 0, 2 * sizeof(uint32_t), s), "memset");
    if (npairs)
        check_cuda(cub::DeviceSelect::Flagged(nullptr, bytes_a, it, pd.flags.p, pd.sel_a.p, na_dev, int(npairs), s), "sel");
    if (nold_cap)
        check_cuda(cub::DeviceSelect::Flagged(nullptr, bytes_b, it, pd.flags.p, pd.sel_b.p, nb_dev, int(nold_cap), s), "sel");
    pd.cub_tmp.reserve(std::max(bytes_a, bytes_b));
    if (npairs)
        check_cuda(cub::DeviceSelect::Flagged(pd.cub_tmp.p, bytes_a, it, pd.flags.p, pd.sel_a.p, na_dev, int(npairs), s),
                   "sel");
    // B: unowned old manifolds (only kept when this step does not prune).
    if (nold_cap) {
        // nold_cap is the exact old count: the world syncs on it before the step.
        k_flag_unowned<<<(nold_cap + TB - 1) / TB, TB, 0, s>>>(nold_cap, pd.old_owned.p, old_cache.keys.p, world_of,
                                                                simulate_flag, prev_simulate, pd.flags.p);
        check_cuda(cub::DeviceSelect::Flagged(pd.cub_tmp.p, bytes_b, it, pd.flags.p, pd.sel_b.p, nb_dev, int(nold_cap), s),
                   "sel");
    }
    size_t cap = size_t(npairs) + nold_cap + 1;
    next.keys.reserve(cap);
    next.entries.reserve(cap * ENTRY_F4);
    uint32_t total = npairs + nold_cap;
    if (total)
        k_merge<<<(total + TB - 1) / TB, TB, 0, s>>>(pairs, pd.entries.p, pd.sel_a.p, na_dev, old_cache.keys.p,
                                                      old_cache.entries.p, pd.sel_b.p, nb_dev, next.keys.p,
                                                      next.entries.p, next.count_dev, pd.rec.merge_pos);
    else
        check_cuda(cudaMemsetAsync(next.count_dev, 0, sizeof(uint32_t), s), "memset");
}

}  // namespace bgpu
