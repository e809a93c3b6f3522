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
// Worlds without joints use the chunked PGS (k_solve_chunks): the bodies are cut into
// Morton-ordered chunks, one per block of a cooperative launch, each block solves its own
// chunk's groups colour by colour, and between two phases it waits only for the blocks whose
// groups share a dynamic body with its own. A group's contacts are spread over lanes (one
// contact per lane, the velocities handed from lane to lane in contact order), and the split
// sweep s rides in the phases of velocity sweep s + 1. Worlds with joints use the team kernel
// (k_solve): a persistent cooperative launch split into two teams of blocks with their own
// grid barriers, the velocity team running the warm start, the velocity sweeps and the joint
// rows, the split team the split-impulse sweeps, which touch only the push velocities and so
// run at the same time. The warm start computes the per-contact terms that stay fixed during
// the solve (tangent basis, Iw^-1 (r x d)) once and stores them in a contact table in
// batch-slot order, so the later sweeps run only the impulse update, reading the table with
// coalesced loads.
//
// Rows store only the contact frame (normal, lever arms), the bias terms, the
// effective masses and the accumulated impulses; the tangent basis, the
// angular components Iw^-1 (r x d) and the velocity couplings are recomputed
// from the per-body world inverse inertia with the reference's arithmetic, so
// they equal the values the reference precomputes in prepare().
#include <algorithm>
#include <cstdlib>
#include <cstring>
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
// With chunk histograms (vhist non-null) the pass also counts each group into its (colour,
// chunk) bins and records its touch sets (chunk_count, with the chunked PGS's code below).
__device__ __forceinline__ void chunk_count(const uint64_t* __restrict__ pairs, uint32_t p, uint32_t c, uint32_t rows,
                                            bool split, const float4* __restrict__ iw,
                                            const uint32_t* __restrict__ chunk_of, uint32_t P, uint32_t* vhist,
                                            uint32_t* shist, uint32_t* touch, uint32_t* all_flag);

__global__ void k_colour_hist(const uint32_t* __restrict__ count, const uint32_t* __restrict__ contact_pairs,
                              const uint32_t* __restrict__ colour, const uint32_t* __restrict__ row_count,
                              const float4* __restrict__ rows, uint32_t* hist, uint32_t* split_hist, uint32_t* split_flag,
                              uint32_t* sub_hist, const uint64_t* __restrict__ pairs, const float4* __restrict__ iw,
                              const uint32_t* __restrict__ chunk_of, uint32_t P, uint32_t* vhist, uint32_t* shist,
                              uint32_t* touch, uint32_t* all_flag) {
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
        if (vhist) chunk_count(pairs, p, c, n, nsr != 0u, iw, chunk_of, P, vhist, shist, touch, all_flag);
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
// [10] split rows [11] largest split batch. One warp, four raw colours a lane.
// Colours without groups are dropped (remap: colour -> dense colour), batches start on
// multiples of 32 (one warp's slots never straddle two batches), so a batch's start is the sum
// of the earlier batches' sizes rounded up to 32. Inside a batch the groups with 4 rows come
// first, then 3, 2, 1 (sub_cursor: the scatter's cursor of each part), so most warps hold
// groups of one size: their lanes run the same number of contacts and read the table's contact
// planes without gaps. The split batches keep their cursors; after the scatter they hold the
// split batch ends. (chunked: the scatter takes per-(colour, chunk) cursors, so the batch ends
// are written here.)
__global__ void k_colour_scan(uint32_t* hist, uint32_t* offset, uint32_t* cursor, uint32_t* split_hist,
                              uint32_t* split_offset, uint32_t* split_cursor, const unsigned int* bar, uint32_t* scalars,
                              uint32_t* remap, const uint32_t* sub_hist, uint32_t* sub_cursor, uint32_t chunked) {
    static_assert(MAX_COLOURS == 128, "four raw colours a lane");
    if (blockIdx.x != 0 || threadIdx.x >= 32u) return;
    const uint32_t lane = threadIdx.x;
    const uint32_t nraw = bar[5];
    uint32_t h[4], sh[4], cnt = 0, pad = 0, spad = 0, smax = 0, sg = 0;
    for (uint32_t k = 0; k < 4; ++k) {
        const uint32_t c = 4u * lane + k;
        h[k] = c < nraw ? hist[c] : 0u;
        sh[k] = h[k] ? split_hist[c] : 0u;
        if (h[k]) {
            ++cnt;
            pad += (h[k] + 31u) & ~31u;
            spad += (sh[k] + 31u) & ~31u;
            smax = max(smax, sh[k]);
            sg += sh[k];
        }
    }
    uint32_t d = cnt, acc = pad, sacc = spad;  // inclusive scans, then exclusive
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, d, o), y = __shfl_up_sync(0xffffffffu, acc, o),
                       z = __shfl_up_sync(0xffffffffu, sacc, o);
        if (lane >= o) { d += x; acc += y; sacc += z; }
    }
    const uint32_t ncol = __shfl_sync(0xffffffffu, d, 31);
    d -= cnt;
    acc -= pad;
    sacc -= spad;
    for (uint32_t k = 0; k < 4; ++k) {
        if (!h[k]) continue;
        const uint32_t c = 4u * lane + k;
        remap[c] = d;
        offset[d] = acc;
        uint32_t part = acc;
        for (uint32_t n = 4; n >= 1; --n) {
            sub_cursor[d * 4 + (n - 1)] = part;
            part += sub_hist[c * 4 + (n - 1)];
        }
        cursor[d] = acc + h[k];  // the batch end
        split_offset[d] = sacc;
        split_cursor[d] = chunked ? sacc + sh[k] : sacc;
        if (d + 1u == ncol) {  // the last batch: the ends, unpadded
            offset[ncol] = acc + h[k];
            split_offset[ncol] = sacc + sh[k];
        }
        acc += (h[k] + 31u) & ~31u;
        sacc += (sh[k] + 31u) & ~31u;
        ++d;
    }
    for (uint32_t o = 16; o > 0; o >>= 1) {
        smax = max(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        sg += __shfl_xor_sync(0xffffffffu, sg, o);
    }
    if (lane == 0) {
        if (ncol == 0) {
            offset[0] = 0u;
            split_offset[0] = 0u;
        }
        scalars[3] = hist[MAX_COLOURS + 1];
        scalars[4] = ncol;
        scalars[5] = sg;
        scalars[10] = hist[MAX_COLOURS + 2];
        scalars[11] = smax;
    }
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

// ---------------------------------------------------------------- chunks (chunked PGS)
// The chunked PGS deals each colour batch to the blocks of the launch by chunk: a chunk is a
// run of bodies in Morton order (the broad phase's tree leaves), and a group belongs to the
// chunk of its first dynamic body. Block b solves chunk b's groups of every colour; before
// a phase it waits only for the blocks whose groups share a dynamic body with its own (its
// neighbours), not for the whole grid. Every block whose groups touch a body appears in the
// body's touch set (its own chunk plus the foreign chunks recorded by the histogram pass), so
// making every two chunks of each touch set neighbours covers every shared body.
constexpr uint32_t CHUNK_TOUCH = 8;          // foreign chunks recorded per body
constexpr uint32_t CHUNK_EMPTY = 0xffffffffu;
constexpr uint32_t CHUNK_MAX = 1024;         // blocks of a chunked launch
constexpr uint32_t CHUNK_CTR_STRIDE = 8;     // progress counters 32 bytes apart
constexpr uint32_t CHUNK_TB = 512;           // threads of a chunk block (one block per SM)

__device__ __forceinline__ uint32_t group_owner(uint32_t ia, uint32_t ib, const float4* __restrict__ iw,
                                                const uint32_t* __restrict__ chunk_of) {
    return chunk_of[inv_mass_of(iw, ia) > 0.0f ? ia : ib];
}

// Bodies in Morton order cut into P equal runs (bodies outside the tree keep chunk 0); with no
// tree, runs of body indices.
__global__ void k_chunk_of(uint32_t n, uint32_t P, const uint32_t* __restrict__ leaf, uint32_t m, uint32_t* chunk_of) {
    const uint32_t lim = leaf ? m : n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
        const uint32_t c = uint32_t(uint64_t(i) * P / lim);
        chunk_of[leaf ? leaf[i] : i] = c;
    }
}

// Records chunk B in the touch set of body x when B is not x's own chunk (slot values only
// ever go from empty to a chunk id, so a stale read of a filled slot is still correct).
__device__ __forceinline__ void chunk_touch(uint32_t* touch, uint32_t x, uint32_t B, uint32_t* all_flag) {
    uint32_t* t = touch + size_t(x) * CHUNK_TOUCH;
    for (uint32_t s = 0; s < CHUNK_TOUCH; ++s) {
        uint32_t v = t[s];
        if (v == B) return;
        if (v == CHUNK_EMPTY) {
            v = atomicCAS(&t[s], CHUNK_EMPTY, B);
            if (v == CHUNK_EMPTY || v == B) return;
        }
    }
    atomicOr(all_flag, 1u);  // more foreign chunks than slots: every block becomes every block's neighbour
}

// Groups per (colour, chunk, row count) and split groups per (colour, chunk), plus the
// touch sets of the groups' dynamic bodies (k_colour_hist's pass, for each group).
__device__ __forceinline__ void chunk_count(const uint64_t* __restrict__ pairs, uint32_t p, uint32_t c, uint32_t rows,
                                            bool split, const float4* __restrict__ iw,
                                            const uint32_t* __restrict__ chunk_of, uint32_t P, uint32_t* vhist,
                                            uint32_t* shist, uint32_t* touch, uint32_t* all_flag) {
    const uint64_t key = pairs[p];
    const uint32_t ia = key_lo(key), ib = key_hi(key);
    const uint32_t B = group_owner(ia, ib, iw, chunk_of);
    atomicAdd(&vhist[(size_t(c) * P + B) * 4 + (rows - 1)], 1u);
    if (split) atomicAdd(&shist[size_t(c) * P + B], 1u);
    if (inv_mass_of(iw, ia) > 0.0f && chunk_of[ia] != B) chunk_touch(touch, ia, B, all_flag);
    if (inv_mass_of(iw, ib) > 0.0f && chunk_of[ib] != B) chunk_touch(touch, ib, B, all_flag);
}

// One block per raw colour: the colour's batch is laid out chunk by chunk (inside a chunk the
// groups with 4 rows first, then 3, 2, 1), so the counts become the scatter's cursors and the
// chunk bins [voff[d (P + 1) + b], voff[d (P + 1) + b + 1]) of dense colour d with the bin's
// groups of 4, 3, 2 and 1 rows in vsec[(d P + b) 4 + 0..3]; the same for the split batch (one
// part per chunk).
template <int TB>
__global__ void __launch_bounds__(TB) k_chunk_scan(uint32_t P, const uint32_t* __restrict__ hist,
                                                   const uint32_t* __restrict__ remap,
                                                   const uint32_t* __restrict__ offset,
                                                   const uint32_t* __restrict__ split_offset,
                                                   const unsigned int* __restrict__ bar, uint32_t* vhist,
                                                   uint32_t* shist, uint32_t* voff, uint32_t* soff, uint32_t* vsec) {
    using Scan = cub::BlockScan<uint32_t, TB>;
    __shared__ typename Scan::TempStorage tmp;
    const uint32_t c = blockIdx.x;
    if (c >= bar[5] || hist[c] == 0) return;
    const uint32_t d = remap[c];
    const uint32_t per = (P + TB - 1) / TB;  // chunks per thread
    const uint32_t b0 = min(P, threadIdx.x * per), b1 = min(P, b0 + per);
    uint32_t* vh = vhist + size_t(c) * P * 4;
    uint32_t* sh = shist + size_t(c) * P;
    uint32_t vsum = 0, ssum = 0;
    for (uint32_t b = b0; b < b1; ++b) {
        for (uint32_t n = 0; n < 4; ++n) vsum += vh[b * 4 + n];
        ssum += sh[b];
    }
    uint32_t vx, sx;
    Scan(tmp).ExclusiveSum(vsum, vx);
    __syncthreads();  // the scan's temporary storage is reused
    Scan(tmp).ExclusiveSum(ssum, sx);
    uint32_t vpos = offset[d] + vx, spos = split_offset[d] + sx;
    for (uint32_t b = b0; b < b1; ++b) {
        voff[size_t(d) * (P + 1) + b] = vpos;
        for (int n = 3; n >= 0; --n) {  // 4 rows first
            const uint32_t cnt = vh[b * 4 + n];
            vsec[(size_t(d) * P + b) * 4 + (3 - n)] = cnt;
            vh[b * 4 + n] = vpos;
            vpos += cnt;
        }
        soff[size_t(d) * (P + 1) + b] = spos;
        const uint32_t cnt = sh[b];
        sh[b] = spos;
        spos += cnt;
    }
    if (threadIdx.x == TB - 1) {
        voff[size_t(d) * (P + 1) + P] = vpos;
        soff[size_t(d) * (P + 1) + P] = spos;
    }
}

// Neighbour bits: every two distinct chunks of a body's touch set (its own chunk included).
__global__ void k_chunk_adjacency(uint32_t n, const uint32_t* __restrict__ chunk_of, const uint32_t* __restrict__ touch,
                                  uint32_t W, uint32_t* adj) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t* t = touch + size_t(i) * CHUNK_TOUCH;
        if (t[0] == CHUNK_EMPTY) continue;  // touched by its own chunk only
        uint32_t v[CHUNK_TOUCH + 1];
        uint32_t m = 0;
        v[m++] = chunk_of[i];
#pragma unroll
        for (uint32_t s = 0; s < CHUNK_TOUCH; ++s)
            if (t[s] != CHUNK_EMPTY) v[m++] = t[s];
        for (uint32_t a = 0; a < m; ++a)
            for (uint32_t b = 0; b < m; ++b) {
                if (v[a] == v[b]) continue;
                uint32_t* w = &adj[size_t(v[a]) * W + (v[b] >> 5)];
                const uint32_t bit = 1u << (v[b] & 31u);
                if (!(*w & bit)) atomicOr(w, bit);
            }
    }
}

// Slot record of a group: its two bodies and its pair index with the row count
// in the top three bits. With chunk cursors (vcur / scur, by raw colour) the slot is taken
// in the group's (colour, chunk, row count) part.
__global__ void k_colour_scatter(const uint32_t* __restrict__ count, const uint32_t* __restrict__ contact_pairs,
                                 const uint64_t* __restrict__ pairs, const uint32_t* __restrict__ row_count,
                                 const uint32_t* __restrict__ colour, const uint32_t* __restrict__ split_flag,
                                 uint32_t* sub_cursor, uint32_t* split_cursor, uint4* batch_rec, uint4* split_rec,
                                 float4* entries, const uint32_t* __restrict__ remap,
                                 const uint32_t* __restrict__ chunk_of, const float4* __restrict__ iw, uint32_t P,
                                 uint32_t* vcur, uint32_t* scur) {
    uint32_t K = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        if (colour[k] >= MAX_COLOURS) continue;  // colouring gave up (its status bit is set)
        const uint32_t raw = colour[k];
        uint32_t c = remap[raw];
        uint32_t p = contact_pairs[k];
        uint64_t key = pairs[p];
        uint4 rec = make_uint4(key_lo(key), key_hi(key), p | (row_count[p] << 29), 0u);
        // The colour rides in the manifold's meta bits to seed next step's colouring.
        float* mw = &entries[size_t(p) * ENTRY_F4 + 2].w;
        *mw = __uint_as_float((__float_as_uint(*mw) & ~(0xffu << META_COLOUR_SHIFT)) | ((c + 1u) << META_COLOUR_SHIFT));
        if (vcur) {
            const uint32_t B = group_owner(rec.x, rec.y, iw, chunk_of);
            batch_rec[claim_slot(vcur, (raw * P + B) * 4 + (row_count[p] - 1))] = rec;
            if (split_flag[k]) split_rec[claim_slot(scur, raw * P + B)] = rec;
        } else {
            batch_rec[claim_slot(sub_cursor, c * 4 + (row_count[p] - 1))] = rec;
            if (split_flag[k]) split_rec[claim_slot(split_cursor, c)] = rec;
        }
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

// The per-contact terms of warm_start (sequential_impulse.rs:710-717) for contact k of pair p,
// written to the contact's velocity-table entries e (the terms sequential_impulse.rs:352-520
// computes in prepare()); the warm-start impulses are applied by warm_apply.
struct WarmTerms {
    V3 n, t1, t2, ana, anb, a1a, a1b, a2a, a2b;
    float4 r3;
};

__device__ __forceinline__ WarmTerms warm_terms(const SolveArgs& a, uint32_t p, uint32_t k, const M3& iwa,
                                                const M3& iwb, float ima, float imb, float4* e) {
    const float4* r = a.rows + (size_t(p) * 4 + k) * ROW_F4;
    const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
    WarmTerms w;
    w.n = from4(r0);
    const V3 ra = from4(r1), rb = from4(r2);
    tangent_basis_dev(w.n, w.t1, w.t2);
    w.ana = mul(iwa, cross(ra, w.n));
    w.anb = mul(iwb, cross(rb, w.n));
    w.a1a = mul(iwa, cross(ra, w.t1));
    w.a1b = mul(iwb, cross(rb, w.t1));
    w.a2a = mul(iwa, cross(ra, w.t2));
    w.a2b = mul(iwb, cross(rb, w.t2));
    w.r3 = r3;
    e[VT_N * PLANE_STRIDE] = r0;
    e[VT_RA * PLANE_STRIDE] = r1;
    e[VT_RB * PLANE_STRIDE] = r2;
    e[VT_T1 * PLANE_STRIDE] = f4(w.t1, ima);
    e[VT_ANA * PLANE_STRIDE] = f4(w.ana, r4.x);
    e[VT_ANB * PLANE_STRIDE] = f4(w.anb, r4.y);
    e[VT_A1A * PLANE_STRIDE] = f4(w.a1a, r4.z);
    e[VT_A1B * PLANE_STRIDE] = f4(w.a1b, r4.w);
    e[VT_A2A * PLANE_STRIDE] = f4(w.a2a, r3.w);
    e[VT_A2B * PLANE_STRIDE] = f4(w.a2b, imb);
    e[VT_IMP * PLANE_STRIDE] = r3;
    return w;
}

__device__ __forceinline__ void warm_apply(const WarmTerms& w, V3& la, V3& wa, V3& lb, V3& wb, bool appa, bool appb,
                                           float ima, float imb) {
    apply(la, wa, lb, wb, appa, appb, ima, imb, w.n, w.ana, w.anb, w.r3.x);
    apply(la, wa, lb, wb, appa, appb, ima, imb, w.t1, w.a1a, w.a1b, w.r3.y);
    apply(la, wa, lb, wb, appa, appb, ima, imb, w.t2, w.a2a, w.a2b, w.r3.z);
}

// warm_start for group slot t: every contact's terms into the slot's velocity table, its
// warm-start impulses onto the velocities in contact order.
__device__ __forceinline__ void warm_group(const SolveArgs& a, uint32_t t, uint32_t p, uint32_t cnt, uint32_t ia,
                                           uint32_t ib, V3& la, V3& wa, V3& lb, V3& wb, bool& appa, bool& appb) {
    float ima, imb;
    const M3 iwa = load_iw(a.iw, ia, ima);
    const M3 iwb = load_iw(a.iw, ib, imb);
    appa = ima > 0.0f;
    appb = imb > 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) {
        const WarmTerms w = warm_terms(a, p, k, iwa, iwb, ima, imb, a.vtab + tix<VT_PLANES>(0, k, t));
        warm_apply(w, la, wa, lb, wb, appa, appb, ima, imb);
    }
}

// The velocity-table entries of one contact.
struct VPlanes {
    float4 r0, r1, r2, q3, q5, q6, q7, q8, q9, q10, r3;
};

__device__ __forceinline__ VPlanes load_vplanes(const float4* e) {
    VPlanes v;
    v.r0 = e[VT_N * PLANE_STRIDE];
    v.r1 = e[VT_RA * PLANE_STRIDE];
    v.r2 = e[VT_RB * PLANE_STRIDE];
    v.q3 = e[VT_T1 * PLANE_STRIDE];
    v.q5 = e[VT_ANA * PLANE_STRIDE];
    v.q6 = e[VT_ANB * PLANE_STRIDE];
    v.q7 = e[VT_A1A * PLANE_STRIDE];
    v.q8 = e[VT_A1B * PLANE_STRIDE];
    v.q9 = e[VT_A2A * PLANE_STRIDE];
    v.q10 = e[VT_A2B * PLANE_STRIDE];
    v.r3 = e[VT_IMP * PLANE_STRIDE];
    return v;
}

// One solve_contact (sequential_impulse.rs:804-930) of contact k of slot t (pair p) from its
// table entries (plane pl at src[pl * st]: the table itself or a shared-memory copy); the new
// impulses go back to the table entry e (and, on the last sweep, to the pair's row).
__device__ __forceinline__ void iter_contact(const SolveArgs& a, const float4* src, uint32_t st, float ima, float imb,
                                             bool appa, bool appb, V3& la, V3& wa, V3& lb, V3& wb, float4* e,
                                             uint32_t sweep, uint32_t k, uint32_t t, bool last, uint32_t p) {
    const float ims = ima + imb;
    const float4 r0 = src[VT_N * st], r1 = src[VT_RA * st], r2 = src[VT_RB * st], q3 = src[VT_T1 * st],
                 q5 = src[VT_ANA * st], q6 = src[VT_ANB * st], q7 = src[VT_A1A * st], q8 = src[VT_A1B * st],
                 q9 = src[VT_A2A * st], q10 = src[VT_A2B * st], r3 = src[VT_IMP * st];
    const V3 n = from4(r0), ra = from4(r1), rb = from4(r2), t1 = from4(q3);
    const V3 t2 = cross(n, t1);  // tangent_basis (sequential_impulse.rs:620-629), as warm_terms made it
    const V3 ana = from4(q5), anb = from4(q6), a1a = from4(q7), a1b = from4(q8), a2a = from4(q9), a2b = from4(q10);
    // The velocity couplings of sequential_impulse.rs:352-520, in warm_terms's operand order.
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

// One solve_contact sweep (sequential_impulse.rs:804-930) over group slot t;
// on the last sweep the impulses also go back to the pair's rows.
__device__ __forceinline__ void iter_group(const SolveArgs& a, uint32_t t, uint32_t p, uint32_t cnt, uint32_t sweep,
                                           bool last, V3& la, V3& wa, V3& lb, V3& wb, bool& appa, bool& appb) {
    const float4* e0 = a.vtab + tix<VT_PLANES>(0, 0, t);
    const float ima = e0[VT_T1 * PLANE_STRIDE].w, imb = e0[VT_A2B * PLANE_STRIDE].w;
    appa = ima > 0.0f;
    appb = imb > 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) {
        float4* e = a.vtab + tix<VT_PLANES>(0, k, t);
        iter_contact(a, e, PLANE_STRIDE, ima, imb, appa, appb, la, wa, lb, wb, e, sweep, k, t, last, p);
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

__device__ __forceinline__ void shfl_v3(V3& v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    v.z = __shfl_sync(0xffffffffu, v.z, src);
}

// One group spread over a segment of lanes: lane k holds contact k of slot t (k < cnt; a
// segment of 4 lanes holding a 3-contact group keeps its last lane idle). Every lane loads
// its own contact's table entries (or, on the warm start, computes its contact's terms
// from the rows) at once, in lane_prepare, which reads nothing another block writes during
// the solve; lane_exec then loads the two bodies' velocities and solves the contacts in
// order k = 0, 1, ..., the lane of contact k updating the velocities and handing them to
// the segment by shuffles, so each contact sees exactly the velocities of the sequential
// solve. All 32 lanes of the warp call lane_exec together (lanes without a group have
// cnt = 0); seg0 is the lane of the segment's contact 0.
template <bool WARM>
struct LaneState {  // sweeps >= 1: the contact's table entries are in shared memory
    uint4 rec;
    float ima, imb;
};
template <>
struct LaneState<true> {
    uint4 rec;
    float ima, imb;
    WarmTerms W;  // the warm start
};

// Warm start: the slot record and the contact's terms (from the rows and the bodies' inverse
// inertia), written to the velocity table.
__device__ __forceinline__ void lane_prepare_warm(const SolveArgs& a, uint32_t t, uint32_t cnt, uint32_t k,
                                                  LaneState<true>& S) {
    S.rec = cnt ? __ldg(&a.batch_rec[t]) : make_uint4(0u, 0u, 0u, 0u);
    S.ima = S.imb = 0.0f;
    if (k >= cnt) return;
    const M3 iwa = load_iw(a.iw, S.rec.x, S.ima);
    const M3 iwb = load_iw(a.iw, S.rec.y, S.imb);
    S.W = warm_terms(a, S.rec.z & 0x1fffffffu, k, iwa, iwb, S.ima, S.imb, a.vtab + tix<VT_PLANES>(0, k, t));
}

template <bool WARM>
__device__ __forceinline__ void lane_exec(const SolveArgs& a, uint32_t t, uint32_t cnt, uint32_t k, uint32_t seg0,
                                          uint32_t sweep, uint32_t last, const LaneState<WARM>& S, const float4* sp) {
    const uint32_t jmax = __reduce_max_sync(0xffffffffu, cnt);
    if (jmax == 0) return;
    const uint32_t ia = S.rec.x, ib = S.rec.y, p = S.rec.z & 0x1fffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    V3 la{0.0f, 0.0f, 0.0f}, wa = la, lb = la, wb = la;
    if (cnt) {
        la = from4(__ldcg(&a.linvel[ia]));
        wa = from4(__ldcg(&a.angvel[ia]));
        lb = from4(__ldcg(&a.linvel[ib]));
        wb = from4(__ldcg(&a.angvel[ib]));
    }
    const bool mine = k < cnt;
    // Every lane of a segment holds the group's inverse masses except an idle fourth lane,
    // which only forwards velocities; the store below is lane 0's.
    const bool appa = S.ima > 0.0f, appb = S.imb > 0.0f;
    float4* e = a.vtab + tix<VT_PLANES>(0, mine ? k : 0u, t);
    for (uint32_t j = 0; j < jmax; ++j) {
        if (mine && k == j) {
            if constexpr (WARM) warm_apply(S.W, la, wa, lb, wb, appa, appb, S.ima, S.imb);
            else iter_contact(a, sp, blockDim.x, S.ima, S.imb, appa, appb, la, wa, lb, wb, e, sweep, k, t, sweep == last, p);
        }
        if (jmax > 1) {  // else every segment is one lane
            const int src = int(j < cnt ? seg0 + j : lane);
            shfl_v3(la, src);
            shfl_v3(wa, src);
            shfl_v3(lb, src);
            shfl_v3(wb, src);
        }
    }
    if (cnt && k == 0) {
        if (appa) { __stcg(&a.linvel[ia], to4(la, 0.0f)); __stcg(&a.angvel[ia], to4(wa, 0.0f)); }
        if (appb) { __stcg(&a.linvel[ib], to4(lb, 0.0f)); __stcg(&a.angvel[ib], to4(wb, 0.0f)); }
    }
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

// ---------------------------------------------------------------- chunked PGS
struct ChunkArgs {
    uint32_t P;                        // blocks of the launch = chunks
    uint32_t W;                        // words per adjacency row
    const uint32_t* voff;              // [d (P + 1) + b]: chunk b's part of colour batch d
    const uint32_t* soff;              // the same for the split batches
    const uint32_t* vsec;              // [(d P + b) 4 + i]: groups of 4 - i rows in chunk b's part of batch d
    const uint32_t* adj;               // [b W + w]: neighbour bits of chunk b
    const uint32_t* all_flag;          // nonzero: every chunk is every chunk's neighbour
    unsigned int* ctr;                 // [b CHUNK_CTR_STRIDE]: phases chunk b has finished
};

// Publishes that this block finished every phase before q. The block's global writes are
// ordered before the release store by the bar.sync.
__device__ __forceinline__ void chunk_arrive(const ChunkArgs& ch, uint32_t q) {
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(ch.ctr + blockIdx.x * CHUNK_CTR_STRIDE), "r"(q)
                     : "memory");
}

// Waits until each neighbour has finished every phase before q: one warp polls the
// neighbours' counters (acquire loads), and the closing bar.sync makes their writes visible
// to the block. The wait is bounded like team_barrier's.
__device__ __forceinline__ void chunk_poll(const ChunkArgs& ch, const uint16_t* nb, uint32_t nnb, uint32_t q,
                                           uint32_t* status) {
    if (threadIdx.x < 32u) {
        uint32_t spins = 0;
        unsigned long long t0 = 0;
        bool gave_up = false;
        for (uint32_t k = threadIdx.x; k < nnb && !gave_up; k += 32u) {
            const unsigned int* c = ch.ctr + uint32_t(nb[k]) * CHUNK_CTR_STRIDE;
            for (;;) {
                unsigned int v;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(c) : "memory");
                if (v >= q) break;
                if ((++spins & 63u) == 0u) {
                    const unsigned long long now = globaltimer_ns();
                    if (t0 == 0) t0 = now;
                    if ((*(volatile uint32_t*)status & ST_BARRIER_TIMEOUT) || now - t0 > BARRIER_TIMEOUT_NS ||
                        spins > BARRIER_SPIN_LIMIT) {
                        atomicOr(status, ST_BARRIER_TIMEOUT);
                        gave_up = true;
                        break;
                    }
                }
            }
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned int d = static_cast<unsigned int>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}

// One phase of a chunked block: velocity items are lanes (groups of 4 and 3 rows take 4 lanes,
// of 2 rows 2, of 1 row one: parts L4, L3, L2, L), padded to a whole warp; split items (one
// group per thread) follow from LV. Between publishing its progress and polling its
// neighbours the block starts round 0's loads (item threadIdx.x), which read nothing another
// block writes during the solve: its slot record and its contact's table entries (copied
// into shared memory, s_pl[plane][thread]) or its warm-start terms, or its split group's
// table entries (into L2). The loads come after the publishing bar.sync, which orders this
// thread's earlier table writes before them. The item-to-thread deal depends only on the
// bin's counts, so a contact's table entries are read by the thread that wrote them.
template <bool WARM>
__device__ __forceinline__ void chunk_phase(const SolveArgs& a, const ChunkArgs& ch, const uint16_t* nb, uint32_t nnb,
                                            uint32_t q, uint32_t sw, uint32_t iters, uint32_t v0, uint32_t nv,
                                            uint32_t n4, uint32_t n3, uint32_t n2, uint32_t s0, uint32_t ns,
                                            float4* s_pl) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t L4 = 4u * n4, L3 = L4 + 4u * n3, L2 = L3 + 2u * n2, L = L2 + (nv - n4 - n3 - n2);
    const uint32_t LV = (L + 31u) & ~31u;
    auto lane_item = [&](uint32_t i, uint32_t& g, uint32_t& k, uint32_t& cnt, uint32_t& seg0) {
        g = 0; k = 0; cnt = 0; seg0 = lane;
        if (i < L4) { g = i >> 2; k = i & 3u; cnt = 4; seg0 = lane & ~3u; }
        else if (i < L3) { g = n4 + ((i - L4) >> 2); k = i & 3u; cnt = 3; seg0 = lane & ~3u; }
        else if (i < L2) { g = n4 + n3 + ((i - L3) >> 1); k = i & 1u; cnt = 2; seg0 = lane & ~1u; }
        else if (i < L) { g = n4 + n3 + n2 + (i - L2); cnt = 1; }
    };
    const uint32_t first = threadIdx.x & ~31u;
    // Round r's table entries of this thread's contact go to s_pl by cp.async.
    auto stage = [&](uint32_t g, uint32_t k, uint32_t cnt) {
        if (k < cnt) {
            const float4* e = a.vtab + tix<VT_PLANES>(0, k, v0 + g);
            for (uint32_t pl = 0; pl < VT_PLANES; ++pl)
                cp_async16(&s_pl[pl * blockDim.x + threadIdx.x], e + pl * PLANE_STRIDE);
        }
    };
    if (q) chunk_arrive(ch, q);
    uint4 rec0 = make_uint4(0u, 0u, 0u, 0u);
    LaneState<WARM> S0;
    if (WARM && first < LV) {
        uint32_t g, k, cnt, seg0;
        lane_item(threadIdx.x, g, k, cnt, seg0);
        if constexpr (WARM) lane_prepare_warm(a, v0 + g, cnt, k, S0);
    } else if (!WARM && first < LV) {
        uint32_t g, k, cnt, seg0;
        lane_item(threadIdx.x, g, k, cnt, seg0);
        stage(g, k, cnt);
        if (cnt) rec0 = __ldg(&a.batch_rec[v0 + g]);
    } else if (threadIdx.x >= LV && threadIdx.x - LV < ns && sw >= 2) {
        prefetch_slot_l2<false>(a, s0 + threadIdx.x - LV, __ldg(&a.split_rec[s0 + threadIdx.x - LV]).z >> 29);
    }
    if (q) chunk_poll(ch, nb, nnb, q, a.status);
    for (uint32_t base = first; base < LV + ns; base += blockDim.x) {
        const uint32_t i = base + lane;
        if (base < LV) {  // warp-uniform: the whole warp runs velocity lanes
            uint32_t g, k, cnt, seg0;
            lane_item(i, g, k, cnt, seg0);
            LaneState<WARM> S;
            const float4* sp = s_pl + threadIdx.x;
            if constexpr (WARM) {
                if (base != first) lane_prepare_warm(a, v0 + g, cnt, k, S);
                else S = S0;
            } else {
                if (base != first) {
                    stage(g, k, cnt);
                    S.rec = cnt ? __ldg(&a.batch_rec[v0 + g]) : make_uint4(0u, 0u, 0u, 0u);
                } else {
                    S.rec = rec0;
                }
                asm volatile("cp.async.wait_all;" ::: "memory");
                S.ima = k < cnt ? sp[VT_T1 * blockDim.x].w : 0.0f;
                S.imb = k < cnt ? sp[VT_A2B * blockDim.x].w : 0.0f;
            }
            lane_exec<WARM>(a, v0 + g, cnt, k, seg0, sw, iters, S, sp);
        } else if (i - LV < ns) {
            run_item<false>(a, sw - 1u, iters - 1u, s0 + i - LV, __ldg(&a.split_rec[s0 + i - LV]));
        }
    }
}

// solve() (sequential_impulse.rs:692-705) for worlds without joints, one chunk per block:
// phase (s, c) runs velocity sweep s (s = 0: warm start) over the block's groups of colour c
// and split sweep s - 1 over its split groups of colour c (split sweeps touch only the push
// velocities, so they share the phase). Each block runs its phases in the team kernel's order
// and waits only on its neighbours, so every body sees the same sequence of updates as under
// grid barriers: the result is the sequential solve in (colour, pair) order. A block skips
// the phases it has no groups in. The warm start (phases 0 .. ncol - 1, WARM) and the sweeps
// (the rest) are two launches of their own code (each keeps its registers); the counters run
// on across the two, so the second launch starts with every neighbour past the warm start.
template <bool WARM>
__global__ void __launch_bounds__(CHUNK_TB, 512 / CHUNK_TB) k_solve_chunks(SolveArgs a, ChunkArgs ch) {
    const uint32_t ncol = a.scalars[4];
    const uint32_t iters = a.iterations;
    const uint32_t b = blockIdx.x;
    extern __shared__ float4 s_pl[];  // [VT_PLANES][blockDim.x]: round 0's table entries
    __shared__ uint32_t s_v[MAX_COLOURS][2], s_s[MAX_COLOURS][2], s_sec[MAX_COLOURS][3];
    __shared__ uint16_t s_nb[CHUNK_MAX];
    __shared__ unsigned int s_nnb;
    if (threadIdx.x == 0) s_nnb = 0;
    for (uint32_t c = threadIdx.x; c < ncol; c += blockDim.x) {
        s_v[c][0] = ch.voff[size_t(c) * (ch.P + 1) + b];
        s_v[c][1] = ch.voff[size_t(c) * (ch.P + 1) + b + 1];
        s_s[c][0] = ch.soff[size_t(c) * (ch.P + 1) + b];
        s_s[c][1] = ch.soff[size_t(c) * (ch.P + 1) + b + 1];
        for (uint32_t i = 0; i < 3; ++i) s_sec[c][i] = ch.vsec[(size_t(c) * ch.P + b) * 4 + i];
    }
    __syncthreads();  // s_nnb
    const bool all = *ch.all_flag != 0u;
    for (uint32_t w = threadIdx.x; w < ch.W; w += blockDim.x) {
        uint32_t bits = all ? 0xffffffffu : ch.adj[size_t(b) * ch.W + w];
        while (bits) {
            const uint32_t j = w * 32u + uint32_t(__ffs(int(bits)) - 1);
            bits &= bits - 1u;
            if (j < ch.P && j != b) s_nb[atomicAdd(&s_nnb, 1u)] = uint16_t(j);
        }
    }
    __syncthreads();  // the neighbour list
    const uint32_t nnb = s_nnb;
    const uint32_t nphases = WARM ? ncol : (iters + 1) * ncol;
    for (uint32_t q = WARM ? 0u : ncol; q < nphases; ++q) {
        const uint32_t c = q % ncol, sw = q / ncol;
        const uint32_t v0 = s_v[c][0], nv = s_v[c][1] - v0;
        const uint32_t s0 = s_s[c][0], ns = sw >= 1 ? s_s[c][1] - s0 : 0u;
        if (nv + ns == 0) continue;
        const uint32_t n4 = s_sec[c][0], n3 = s_sec[c][1], n2 = s_sec[c][2];
        chunk_phase<WARM>(a, ch, s_nb, nnb, q, sw, iters, v0, nv, n4, n3, n2, s0, ns, s_pl);
    }
    // Every later phase of this block is empty: publish the end.
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(ch.ctr + b * CHUNK_CTR_STRIDE), "r"(nphases)
                     : "memory");
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
    float4* entries;                   // the pairs' new manifolds: their meta bits carry the colour
    uint32_t seed;                     // nonzero: start from the colours the manifolds carry
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
    unsigned long long* dup = best1 + nb;  // seeded colours claimed twice at a body
    for (uint32_t i = lane; i < nb; i += nt) {
        lin[i] = __ldcg(&A.linvel[b0 + i]);
        ang[i] = __ldcg(&A.angvel[b0 + i]);
        mask[i] = 0ull;
        best0[i] = 0ull;
        best1[i] = 0ull;
        dup[i] = 0ull;
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
    auto seed_of = [&](uint32_t g) -> uint32_t {  // last step's colour + 1 (0: none)
        const uint32_t cs =
            (__float_as_uint(A.entries[size_t(A.contact_pairs[g]) * ENTRY_F4 + 2].w) >> META_COLOUR_SHIFT) & 0xffu;
        return cs <= WS_MAX_COLOURS ? cs : 0u;
    };
    if (A.seed) {
        //    Seeds: each group claims last step's colour at its dynamic bodies; a group keeps it
        //    when no other group claimed the same colour at either body. The others are coloured
        //    by the rounds below, first fit around every claimed colour.
        for (uint32_t g = g0 + lane; g < g1; g += nt) {
            const uint32_t cs = seed_of(g);
            if (cs == 0u) continue;
            const unsigned long long bit = 1ull << (cs - 1u);
            const uint64_t key = A.pairs[A.contact_pairs[g]];
            const uint32_t ia = key_lo(key), ib = key_hi(key);
            if (dyn(ia) && (atomicOr(&mask[ia - b0], bit) & bit)) atomicOr(&dup[ia - b0], bit);
            if (dyn(ib) && (atomicOr(&mask[ib - b0], bit) & bit)) atomicOr(&dup[ib - b0], bit);
        }
        ws_sync<WARP>();
        uint32_t kept = 0;
        for (uint32_t g = g0 + lane; g < g1; g += nt) {
            const uint32_t cs = seed_of(g);
            bool keep = false;
            if (cs != 0u) {
                const unsigned long long bit = 1ull << (cs - 1u);
                const uint64_t key = A.pairs[A.contact_pairs[g]];
                const uint32_t ia = key_lo(key), ib = key_hi(key);
                keep = !(dyn(ia) && (dup[ia - b0] & bit)) && !(dyn(ib) && (dup[ib - b0] & bit));
            }
            A.colour[g] = keep ? cs - 1u : NO_COLOUR;
            kept += keep ? 1u : 0u;
        }
        if (kept) atomicSub(&C.left, kept);
    } else {
        for (uint32_t g = g0 + lane; g < g1; g += nt) A.colour[g] = NO_COLOUR;
    }
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
        // The colour rides in the manifold's meta bits to seed next step's colouring.
        float* mw = &A.entries[size_t(p) * ENTRY_F4 + 2].w;
        *mw = __uint_as_float((__float_as_uint(*mw) & ~(0xffu << META_COLOUR_SHIFT)) | ((c + 1u) << META_COLOUR_SHIFT));
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

// MAXT: the launch's largest block. Plans of up to 256 threads a CTA mix block and warp modes;
// the 512-thread build runs only plans whose worlds are all in block mode (one large world).
template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_world_solve(WorldSolveArgs A) {
    extern __shared__ float4 ws_dyn[];
    __shared__ WorldCtx ctx[MAXT > 256 ? 1 : WS_MAX_WARPS];
    const uint2 c = A.plan.cta[blockIdx.x];
    const bool block_mode = (c.y >> 31) != 0u;
    const uint32_t count = c.y & 0x7fffffffu;
    if (block_mode) {
        solve_world<false>(A, A.plan.list[c.x], threadIdx.x, blockDim.x, ws_dyn, ctx[0]);
        return;
    }
    if (MAXT > 256) return;  // the plan builder gives this build block-mode plans only
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

int device_sms() {
    static int sms = -1;
    if (sms < 0) {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
    }
    return sms;
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

// The PGS kernel for worlds without joints is the chunked one; BGPU_PGS=team in the
// environment keeps the team-barrier kernel (which worlds with joints always use), for
// comparison.
static int pgs_mode() {
    static int mode = -1;
    if (mode < 0) {
        const char* e = std::getenv("BGPU_PGS");
        mode = (e && std::strcmp(e, "team") == 0) ? 1 : 2;
    }
    return mode;
}

static int g_last_solver_kind = 0;
int last_solver_kind() { return g_last_solver_kind; }

constexpr size_t CHUNK_SMEM = size_t(VT_PLANES) * CHUNK_TB * sizeof(float4);

static int chunk_grid() {
    static int grid = 0;
    if (!grid) {
        int g[2];
        const void* fns[2] = {(const void*)k_solve_chunks<true>, (const void*)k_solve_chunks<false>};
        for (int i = 0; i < 2; ++i) {
            check_cuda(cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize, int(CHUNK_SMEM)),
                       "smem attribute");
            g[i] = coop_grid(fns[i], CHUNK_TB, CHUNK_SMEM);
        }
        grid = std::min(g[0], g[1]);  // both launches cut the bodies into the same chunks
    }
    if (grid > int(CHUNK_MAX)) throw CudaError{cudaErrorInvalidValue, "chunked PGS: more blocks than chunk slots"};
    return grid;
}

void run_wait_selftest(unsigned long long limit_ns, unsigned int* ctr, uint32_t* status, cudaStream_t s) {
    k_wait_selftest<<<2, 32, 0, s>>>(ctr, status, limit_ns);
}

void run_solver(const WorldView& w, const uint64_t* pairs, uint32_t npairs, PairData& pd, const StepParams& sp,
                uint32_t* status_dev, cudaStream_t s, const std::function<void(int)>& mark, bool seed_colours,
                const JointsDev* joints, const uint32_t* morton_leaf, uint32_t tree_m) {
    const bool with_joints = joints && joints->n && joints->ncol;
    g_last_solver_kind = 0;
    if (npairs == 0) {
        check_cuda(cudaMemsetAsync(pd.scalars.p + 2, 0, 4 * sizeof(uint32_t), s), "memset");
        check_cuda(cudaMemsetAsync(pd.scalars.p + 10, 0, 2 * sizeof(uint32_t), s), "memset");
        mark(5);
        if (with_joints) {
            launch_solve(w, pd, sp, status_dev, s, joints);
            g_last_solver_kind = 1;
        }
        mark(6);
        return;
    }
    const int mode = with_joints ? 1 : pgs_mode();
    const bool chunked = mode == 2;
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
    // Two blocks per SM: enough threads for a pile's groups, and the rounds' grid barriers
    // are cheaper than with every block the SM could hold.
    static int colour_grid = 0;
    if (!colour_grid) colour_grid = std::min(coop_grid((const void*)k_colour, TB, 0), 2 * device_sms());
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
    // Chunks: each body's chunk; the (colour, chunk) counts and the touch sets come with the
    // colour histograms.
    uint32_t P = 0, W = 0;
    uint32_t *vhist = nullptr, *shist = nullptr, *all_flag = nullptr;
    if (chunked) {
        P = uint32_t(chunk_grid());
        W = (P + 31u) / 32u;
        const uint32_t n = w.nbodies;
        pd.chunk_of.reserve(std::max<uint32_t>(n, 1));
        pd.chunk_touch.reserve(size_t(std::max<uint32_t>(n, 1)) * CHUNK_TOUCH);
        pd.chunk_hist.reserve(size_t(MAX_COLOURS) * P * 5);
        pd.chunk_off.reserve(2 * size_t(MAX_COLOURS) * (P + 1) + size_t(MAX_COLOURS) * P * 4);
        pd.chunk_adj.reserve(size_t(P) * W + 1);
        pd.chunk_ctr.reserve(size_t(P) * CHUNK_CTR_STRIDE);
        vhist = pd.chunk_hist.p;
        shist = pd.chunk_hist.p + size_t(MAX_COLOURS) * P * 4;
        all_flag = pd.chunk_adj.p + size_t(P) * W;
        check_cuda(cudaMemsetAsync(pd.chunk_hist.p, 0, size_t(MAX_COLOURS) * P * 5 * sizeof(uint32_t), s), "memset");
        check_cuda(cudaMemsetAsync(pd.chunk_touch.p, 0xff, size_t(n) * CHUNK_TOUCH * sizeof(uint32_t), s), "memset");
        check_cuda(cudaMemsetAsync(pd.chunk_adj.p, 0, (size_t(P) * W + 1) * sizeof(uint32_t), s), "memset");
        check_cuda(cudaMemsetAsync(pd.chunk_of.p, 0, size_t(n) * sizeof(uint32_t), s), "memset");
        const uint32_t lim = (morton_leaf && tree_m) ? tree_m : n;
        k_chunk_of<<<std::min<uint32_t>((lim + TB - 1) / TB, 148u * 8u), TB, 0, s>>>(
            n, P, (morton_leaf && tree_m) ? morton_leaf : nullptr, tree_m, pd.chunk_of.p);
    }
    k_colour_hist<<<g, TB, 0, s>>>(pd.scalars.p + 2, pd.contact_pairs.p, pd.colour.p, pd.row_count.p, pd.rows.p,
                                   pd.colour_count.p, pd.split_count.p, pd.flags.p, sub_hist, pairs, w.b.iw,
                                   pd.chunk_of.p, P, vhist, shist, pd.chunk_touch.p, all_flag);
    k_colour_scan<<<1, 32, 0, s>>>(pd.colour_count.p, pd.colour_offset.p, pd.colour_cursor.p, pd.split_count.p,
                                   pd.split_offset.p, pd.split_cursor.p, pd.barrier.p, pd.scalars.p, pd.colour_remap.p,
                                   sub_hist, sub_cursor, chunked ? 1u : 0u);
    uint32_t *voff = nullptr, *soff = nullptr, *vsec = nullptr;
    if (chunked) {
        voff = pd.chunk_off.p;
        soff = pd.chunk_off.p + size_t(MAX_COLOURS) * (P + 1);
        vsec = pd.chunk_off.p + 2 * size_t(MAX_COLOURS) * (P + 1);
        k_chunk_scan<256><<<MAX_COLOURS, 256, 0, s>>>(P, pd.colour_count.p, pd.colour_remap.p, pd.colour_offset.p,
                                                      pd.split_offset.p, pd.barrier.p, vhist, shist, voff, soff, vsec);
    }
    k_colour_scatter<<<g, TB, 0, s>>>(pd.scalars.p + 2, pd.contact_pairs.p, pairs, pd.row_count.p, pd.colour.p,
                                      pd.flags.p, sub_cursor, pd.split_cursor.p, pd.batch_rec.p,
                                      pd.split_rec.p, pd.entries.p, pd.colour_remap.p, pd.chunk_of.p, w.b.iw, P,
                                      vhist, shist);
    if (chunked)
        k_chunk_adjacency<<<std::min<uint32_t>((w.nbodies + TB - 1) / TB, 148u * 8u), TB, 0, s>>>(
            w.nbodies, pd.chunk_of.p, pd.chunk_touch.p, W, pd.chunk_adj.p);
    mark(5);
    // Slot capacity: every group plus the 32-alignment padding of each batch.
    const size_t slots = (size_t(npairs) + 32u * (MAX_COLOURS + 1) + 31u) & ~size_t(31);
    pd.vtab.reserve(size_t(VT_PLANES) * 4 * slots);
    pd.stab.reserve(size_t(ST_PLANES) * 4 * slots);
    if (chunked) {
        check_cuda(cudaMemsetAsync(pd.chunk_ctr.p, 0, size_t(P) * CHUNK_CTR_STRIDE * sizeof(unsigned int), s),
                   "memset");
        SolveArgs sa{pd.rows.p, pd.batch_rec.p, pd.colour_offset.p, pd.colour_cursor.p, pd.split_rec.p,
                     pd.split_offset.p, pd.split_cursor.p, pd.scalars.p, w.b.linvel, w.b.angvel, w.b.push_lin,
                     w.b.push_ang, w.b.iw, pd.vtab.p, pd.stab.p, pd.rec.sweeps,
                     pd.barrier.p, status_dev, sp.inv_dt, sp.info.restitution_velocity_threshold,
                     sp.info.num_iterations, JointsDev{}, sp.info.damping};
        ChunkArgs ch{P, W, voff, soff, vsec, pd.chunk_adj.p, all_flag, pd.chunk_ctr.p};
        void* args[] = {&sa, &ch};
        check_cuda(cudaLaunchCooperativeKernel((const void*)k_solve_chunks<true>, dim3(P), dim3(CHUNK_TB), args,
                                               CHUNK_SMEM, s), "chunked warm-start launch");
        if (sp.info.num_iterations)
            check_cuda(cudaLaunchCooperativeKernel((const void*)k_solve_chunks<false>, dim3(P), dim3(CHUNK_TB), args,
                                                   CHUNK_SMEM, s), "chunked solve launch");
        g_last_solver_kind = 2;
    } else {
        launch_solve(w, pd, sp, status_dev, s, with_joints ? joints : nullptr);
        g_last_solver_kind = 1;
    }
    mark(6);
}

bool build_world_plan(const std::vector<uint32_t>& world_off, uint32_t block, uint32_t tau, WorldPlan& plan,
                      cudaStream_t s) {
    plan.valid = false;
    // Up to 256 threads a CTA; 512 when every world runs in block mode (tau 0).
    if (block < 32 || block > (tau == 0 ? 512u : 32u * WS_MAX_WARPS) || block % 32) return false;
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
    check_cuda(cudaFuncSetAttribute(block > 256 ? (const void*)k_world_solve<512> : (const void*)k_world_solve<256>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "smem attribute");
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
                      const JointsDev* joints, bool seed_colours) {
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
    A.entries = pd.entries.p;
    A.seed = seed_colours ? 1u : 0u;
    if (plan.block > 256) k_world_solve<512><<<plan.ncta, plan.block, plan.smem, s>>>(A);
    else k_world_solve<256><<<plan.ncta, plan.block, plan.smem, s>>>(A);
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
