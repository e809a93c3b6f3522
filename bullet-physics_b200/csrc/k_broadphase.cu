// Broad phase: Morton-ordered linear BVH (Karras 2012 radix-tree build,
// bottom-up refit) over the bounded proxies, queried once per proxy.
//
// Output contract (crates/bullet-collision/src/broadphase/mod.rs:94-130,
// brute_force.rs:54-68): every pair (i < j) whose closed AABBs overlap on all
// three axes (util.rs:28-38), sorted lexicographically. Each proxy i owns the
// segment of partners j > i. One tree walk per proxy counts its partners and
// keeps them, sorted, in a fixed number of stash slots; an exclusive scan of
// the counts places the segments and a copy pass moves the stashed ones into
// place, so no global pair sort is needed. The few proxies with more partners
// than slots walk the tree a second time and write their segment directly.
// Unbounded proxies (planes) are kept out of the tree and joined by an ordered
// flag/scan compaction.
#include <cub/cub.cuh>
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

constexpr int STACK_DEPTH = 64;
constexpr int LOCAL_SORT = 48;

__device__ __forceinline__ bool overlaps(float4 amin, float4 amax, float4 bmin, float4 bmax) {
    return amin.x <= bmax.x && amin.y <= bmax.y && amin.z <= bmax.z && bmin.x <= amax.x && bmin.y <= amax.y &&
           bmin.z <= amax.z;
}

__device__ __forceinline__ int float_to_ordered(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ordered_to_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_reset_bounds(int* bounds) {
    if (threadIdx.x < 3) bounds[threadIdx.x] = 0x7fffffff;
    else if (threadIdx.x < 6) bounds[threadIdx.x] = int(0x80000000);
}

__global__ void k_bounds(const float4* __restrict__ mn, const float4* __restrict__ mx, const uint32_t* __restrict__ is_unb,
                         uint32_t n, int* bounds) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float cx = INFINITY, cy = INFINITY, cz = INFINITY, dx = -INFINITY, dy = -INFINITY, dz = -INFINITY;
    if (i < n && !is_unb[i]) {
        float4 a = mn[i], b = mx[i];
        cx = dx = 0.5f * (a.x + b.x);
        cy = dy = 0.5f * (a.y + b.y);
        cz = dz = 0.5f * (a.z + b.z);
    }
    typedef cub::BlockReduce<float, 256> BR;
    __shared__ typename BR::TempStorage t;
    float r;
    r = BR(t).Reduce(cx, cub::Min()); __syncthreads(); if (threadIdx.x == 0 && r < INFINITY) atomicMin(&bounds[0], float_to_ordered(r));
    r = BR(t).Reduce(cy, cub::Min()); __syncthreads(); if (threadIdx.x == 0 && r < INFINITY) atomicMin(&bounds[1], float_to_ordered(r));
    r = BR(t).Reduce(cz, cub::Min()); __syncthreads(); if (threadIdx.x == 0 && r < INFINITY) atomicMin(&bounds[2], float_to_ordered(r));
    r = BR(t).Reduce(dx, cub::Max()); __syncthreads(); if (threadIdx.x == 0 && r > -INFINITY) atomicMax(&bounds[3], float_to_ordered(r));
    r = BR(t).Reduce(dy, cub::Max()); __syncthreads(); if (threadIdx.x == 0 && r > -INFINITY) atomicMax(&bounds[4], float_to_ordered(r));
    r = BR(t).Reduce(dz, cub::Max()); __syncthreads(); if (threadIdx.x == 0 && r > -INFINITY) atomicMax(&bounds[5], float_to_ordered(r));
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__device__ __forceinline__ uint32_t quantize(float c, float lo, float hi) {
    float ext = hi - lo;
    float t = ext > 0.0f ? (c - lo) / ext : 0.0f;
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    return uint32_t(t * 1023.0f);
}

// Morton code of each proxy's AABB centre (unbounded proxies: all ones, so they sort last),
// and the proxy index as the sort's value. A stable radix sort of the 32-bit codes with the
// indices as values orders the proxies exactly as sorting (code << 32 | index) would, in
// four 8-bit passes instead of eight.
__global__ void k_keys(const float4* __restrict__ mn, const float4* __restrict__ mx, const uint32_t* __restrict__ is_unb,
                       uint32_t n, const int* __restrict__ bounds, uint32_t* codes, uint32_t* index) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    index[i] = i;
    if (is_unb[i]) { codes[i] = 0xffffffffu; return; }
    float4 a = mn[i], b = mx[i];
    float lo0 = ordered_to_float(bounds[0]), lo1 = ordered_to_float(bounds[1]), lo2 = ordered_to_float(bounds[2]);
    float hi0 = ordered_to_float(bounds[3]), hi1 = ordered_to_float(bounds[4]), hi2 = ordered_to_float(bounds[5]);
    uint32_t x = quantize(0.5f * (a.x + b.x), lo0, hi0);
    uint32_t y = quantize(0.5f * (a.y + b.y), lo1, hi1);
    uint32_t z = quantize(0.5f * (a.z + b.z), lo2, hi2);
    codes[i] = (expand_bits(x) << 2) | (expand_bits(y) << 1) | expand_bits(z);
}

// Sorted leaves as unique 64-bit keys: code << 32 | proxy index.
struct LeafKeys {
    const uint32_t* __restrict__ code;
    const uint32_t* __restrict__ index;
    __device__ __forceinline__ uint64_t operator[](int i) const { return (uint64_t(code[i]) << 32) | index[i]; }
};

__device__ __forceinline__ int delta(const LeafKeys& k, int m, int i, int j) {
    if (j < 0 || j >= m) return -1;
    return __clzll(k[i] ^ k[j]);
}

// Karras 2012: internal node i spans a key range split at its highest differing bit.
__global__ void k_build(LeafKeys k, int m, uint32_t* left, uint32_t* right, uint32_t* parent,
                        uint32_t* leaf_body, uint32_t* refit_flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) leaf_body[i] = k.index[i];
    if (i >= m - 1) return;
    refit_flag[i] = 0;
    int d = (delta(k, m, i, i + 1) - delta(k, m, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(k, m, i, i - d);
    int lmax = 2;
    while (delta(k, m, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, m, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(k, m, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) / 2;
        if (delta(k, m, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    uint32_t lc = (lo == gamma) ? uint32_t(m - 1 + gamma) : uint32_t(gamma);
    uint32_t rc = (hi == gamma + 1) ? uint32_t(m - 1 + gamma + 1) : uint32_t(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    parent[lc] = uint32_t(i);
    parent[rc] = uint32_t(i);
}

// Leaf children are referenced as LEAF_REF | body index in the node records.
constexpr uint32_t LEAF_REF = 0x80000000u;

// Bottom-up refit: node boxes and the largest body index below each node; each internal
// node's record (4 float4: left child min | ref, left max | ref of right, right min | largest
// body index under left, right max | largest under right) is written by the thread that
// completes it, so a query reads one 64-byte record per node it visits.
__global__ void k_refit(int m, const uint32_t* __restrict__ leaf_body, const uint32_t* __restrict__ parent,
                        const uint32_t* __restrict__ left, const uint32_t* __restrict__ right, uint32_t* refit_flag,
                        const float4* __restrict__ bmin, const float4* __restrict__ bmax, float4* nmin, float4* nmax,
                        uint32_t* nid, float4* rec) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    uint32_t node = uint32_t(m - 1 + t);
    uint32_t body = leaf_body[t];
    nmin[node] = bmin[body];
    nmax[node] = bmax[body];
    nid[node] = body;
    if (m == 1) return;
    __threadfence();
    uint32_t cur = parent[node];
    for (int guard = 0; guard < 128; ++guard) {
        if (atomicAdd(&refit_flag[cur], 1u) == 0) return;  // first child to arrive stops
        __threadfence();
        uint32_t l = left[cur], r = right[cur];
        float4 a0 = __ldcg(&nmin[l]), a1 = __ldcg(&nmax[l]), b0 = __ldcg(&nmin[r]), b1 = __ldcg(&nmax[r]);
        const uint32_t il = __ldcg(&nid[l]), ir = __ldcg(&nid[r]);
        nmin[cur] = make_float4(fminf(a0.x, b0.x), fminf(a0.y, b0.y), fminf(a0.z, b0.z), 0.f);
        nmax[cur] = make_float4(fmaxf(a1.x, b1.x), fmaxf(a1.y, b1.y), fmaxf(a1.z, b1.z), 0.f);
        nid[cur] = il > ir ? il : ir;
        const uint32_t lref = l >= uint32_t(m - 1) ? (LEAF_REF | il) : l;
        const uint32_t rref = r >= uint32_t(m - 1) ? (LEAF_REF | ir) : r;
        float4* rc = rec + size_t(cur) * 4;
        rc[0] = make_float4(a0.x, a0.y, a0.z, __uint_as_float(lref));
        rc[1] = make_float4(a1.x, a1.y, a1.z, __uint_as_float(rref));
        rc[2] = make_float4(b0.x, b0.y, b0.z, __uint_as_float(il));
        rc[3] = make_float4(b1.x, b1.y, b1.z, __uint_as_float(ir));
        __threadfence();
        if (cur == 0) return;
        cur = parent[cur];
    }
}

// Partners j > i of bounded proxy i, in one of three modes:
//   Q_COUNT  counts[i] only;
//   Q_WRITE  the segment at offsets[i] (counts[i] from an earlier pass), sorted;
//   Q_STASH  counts[i], and when it is at most STASH_SLOTS the sorted partners in
//            stash slot a of Morton position t (stash[a * m + t], so a warp's
//            writes of one slot are contiguous); a proxy with more partners is
//            appended to `list` (its length in list_len) for a Q_WRITE pass.
// Q_COUNT and Q_WRITE take the proxies from `list` when it is given (t < list_len).
constexpr int Q_COUNT = 0, Q_WRITE = 1, Q_STASH = 2;
constexpr uint32_t STASH_SLOTS = 32;

template <int MODE>
__global__ void k_query(int m, uint32_t n, const uint32_t* __restrict__ is_unb, const float4* __restrict__ bmin,
                        const float4* __restrict__ bmax, const float4* __restrict__ rec,
                        const uint32_t* __restrict__ leaf_body, const uint32_t* __restrict__ unb, uint32_t nunb,
                        uint32_t* counts, const uint32_t* __restrict__ offsets, uint64_t* out, uint32_t* status,
                        uint32_t* list, uint32_t* list_len, uint32_t* stash) {
    constexpr bool WRITE = MODE == Q_WRITE;
    constexpr bool KEEP = MODE != Q_COUNT;
    // Threads take the bounded proxies in Morton (leaf) order, so a warp's
    // queries are neighbours in space and walk much the same part of the tree.
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i;
    if (MODE != Q_STASH && list) {
        if (t >= *list_len) return;
        i = list[t];
    } else {
        if (t >= uint32_t(m)) return;
        i = leaf_body[t];
    }
    float4 qmin = bmin[i], qmax = bmax[i];
    uint32_t cnt = 0;
    uint32_t local[LOCAL_SORT];
    uint64_t base = 0;
    uint32_t expected = 0;
    if (WRITE) {
        base = offsets[i];
        expected = counts[i];
    }
    auto emit = [&](uint32_t j) {
        if (MODE == Q_STASH) {
            if (cnt < STASH_SLOTS) local[cnt] = j;
        } else if (WRITE) {
            if (expected <= LOCAL_SORT) {
                if (cnt < LOCAL_SORT) local[cnt] = j;
            } else if (cnt < expected) {
                out[base + cnt] = (uint64_t(i) << 32) | j;
            }
        }
        ++cnt;
    };
    if (m == 1) {  // the root is the single leaf
        const uint32_t j = leaf_body[0];
        if (j > i && overlaps(qmin, qmax, bmin[j], bmax[j])) emit(j);
    } else if (m > 1) {
        // Subtrees whose largest body index is at most i hold no partner j > i and are skipped.
        uint32_t stack[STACK_DEPTH];
        int sp = 0;
        stack[sp++] = 0u;
        while (sp > 0) {
            const float4* r = rec + size_t(stack[--sp]) * 4;
            const float4 a = r[0], b = r[1], c = r[2], d = r[3];
            const uint32_t ref[2] = {__float_as_uint(a.w), __float_as_uint(b.w)};
            const bool hit[2] = {__float_as_uint(c.w) > i && overlaps(qmin, qmax, a, b),
                                 __float_as_uint(d.w) > i && overlaps(qmin, qmax, c, d)};
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (!hit[k]) continue;
                if (ref[k] & LEAF_REF) {
                    emit(ref[k] & ~LEAF_REF);
                } else if (sp < STACK_DEPTH) {
                    stack[sp++] = ref[k];
                } else {
                    atomicOr(status, ST_TRAVERSAL_STACK);
                }
            }
        }
    }
    for (uint32_t u = 0; u < nunb; ++u) {
        uint32_t h = unb[u];
        if (h > i && overlaps(qmin, qmax, bmin[h], bmax[h])) emit(h);
    }
    if (!KEEP) {
        counts[i] = cnt;
        return;
    }
    if (MODE == Q_STASH) {
        counts[i] = cnt;
        if (cnt > STASH_SLOTS) {
            list[atomicAdd(list_len, 1u)] = i;
            return;
        }
    }
    if (MODE == Q_STASH || expected <= LOCAL_SORT) {
        uint32_t c = cnt < LOCAL_SORT ? cnt : LOCAL_SORT;
        for (uint32_t a = 1; a < c; ++a) {
            uint32_t v = local[a];
            uint32_t b = a;
            while (b > 0 && local[b - 1] > v) { local[b] = local[b - 1]; --b; }
            local[b] = v;
        }
        if (MODE == Q_STASH)
            for (uint32_t a = 0; a < c; ++a) stash[size_t(a) * uint32_t(m) + t] = local[a];
        else
            for (uint32_t a = 0; a < c; ++a) out[base + a] = (uint64_t(i) << 32) | local[a];
    } else {
        uint32_t c = cnt < expected ? cnt : expected;
        for (uint32_t a = 1; a < c; ++a) {
            uint64_t v = out[base + a];
            uint32_t b = a;
            while (b > 0 && out[base + b - 1] > v) { out[base + b] = out[base + b - 1]; --b; }
            out[base + b] = v;
        }
    }
}

// Stashed segments (at most STASH_SLOTS partners) to their place in the pair list. Slot t
// belongs to proxy leaf_body[t] (to proxy t when leaf_body is null).
__global__ void k_stash_copy(int m, const uint32_t* __restrict__ leaf_body, const uint32_t* __restrict__ counts,
                             const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ stash, uint64_t* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= uint32_t(m)) return;
    const uint32_t i = leaf_body ? leaf_body[t] : t;
    const uint32_t c = counts[i];
    if (c > STASH_SLOTS) return;
    const uint64_t base = offsets[i];
    for (uint32_t a = 0; a < c; ++a) out[base + a] = (uint64_t(i) << 32) | stash[size_t(a) * uint32_t(m) + t];
}

// Unbounded proxy h: flags[j] = (j > h && overlap(h, j)) over all proxies.
__global__ void k_unb_flags(uint32_t h, uint32_t n, const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                            uint32_t* flags) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    flags[j] = (j > h && overlaps(bmin[h], bmax[h], bmin[j], bmax[j])) ? 1u : 0u;
}

__global__ void k_unb_count(uint32_t h, uint32_t n, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ scan,
                            uint32_t* counts) {
    if (blockIdx.x == 0 && threadIdx.x == 0) counts[h] = n ? scan[n - 1] + flags[n - 1] : 0u;
}

__global__ void k_unb_write(uint32_t h, uint32_t n, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ scan,
                            const uint32_t* __restrict__ offsets, uint64_t* out) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !flags[j]) return;
    out[uint64_t(offsets[h]) + scan[j]] = (uint64_t(h) << 32) | j;
}

__global__ void k_total(uint32_t n, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                        uint32_t* scalars) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        uint64_t t = n ? uint64_t(offsets[n - 1]) + counts[n - 1] : 0;
        scalars[0] = uint32_t(t > 0xffffffffull ? 0xffffffffull : t);
    }
}

__global__ void k_clear_u32(uint32_t n, uint32_t* a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0;
}

__global__ void k_set_unbounded(const uint32_t* __restrict__ unb, uint32_t nunb, uint32_t* is_unb) {
    uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < nunb) is_unb[unb[u]] = 1;
}

// Batched worlds: world k owns proxies [off[k], off[k + 1]) and pairs only form
// inside a world. One CTA per world tests every (i < j) of the world against
// the other proxies staged in shared memory, tile by tile in ascending j, so
// each proxy's partners come out in ascending order, as in the tree query. The
// pass fills counts[i] and stashes the partners of every proxy with at most
// STASH_SLOTS of them (stash[a * n + i]); a world with a proxy over that (a
// ground plane under a pile) sets wover[w] and adds one to *n_over.
constexpr int WP_TILE = 64;

__global__ void __launch_bounds__(WP_TILE) k_world_pairs(const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                                                           const uint32_t* __restrict__ off, uint32_t n_worlds, uint32_t n,
                                                           uint32_t* counts, uint32_t* stash, uint32_t* wover,
                                                           uint32_t* n_over) {
    __shared__ float4 smin[WP_TILE], smax[WP_TILE];
    for (uint32_t w = blockIdx.x; w < n_worlds; w += gridDim.x) {
        const uint32_t lo = off[w], hi = off[w + 1];
        bool over = false;
        for (uint32_t ibase = lo; ibase < hi; ibase += WP_TILE) {
            const uint32_t i = ibase + threadIdx.x;
            const bool has = i < hi;
            float4 qmin = make_float4(0.f, 0.f, 0.f, 0.f), qmax = qmin;
            if (has) { qmin = bmin[i]; qmax = bmax[i]; }
            uint32_t cnt = 0;
            for (uint32_t jbase = ibase; jbase < hi; jbase += WP_TILE) {
                __syncthreads();
                const uint32_t j = jbase + threadIdx.x;
                if (j < hi) { smin[threadIdx.x] = bmin[j]; smax[threadIdx.x] = bmax[j]; }
                __syncthreads();
                const uint32_t jn = min(uint32_t(WP_TILE), hi - jbase);
                if (!has) continue;
                for (uint32_t q = 0; q < jn; ++q) {
                    const uint32_t jj = jbase + q;
                    if (jj > i && overlaps(qmin, qmax, smin[q], smax[q])) {
                        if (cnt < STASH_SLOTS) stash[size_t(cnt) * n + i] = jj;
                        ++cnt;
                    }
                }
            }
            if (has) {
                counts[i] = cnt;
                over |= cnt > STASH_SLOTS;
            }
        }
        const int any = __syncthreads_or(over ? 1 : 0);
        if (threadIdx.x == 0) {
            wover[w] = any ? 1u : 0u;
            if (any) atomicAdd(n_over, 1u);
        }
    }
}

// The segments of the proxies that k_world_pairs could not stash, in the worlds it
// flagged. The CTA takes those proxies one at a time and tests 64 candidates j at
// once; a ballot per warp ranks the hits, so the segment is written in ascending j.
__global__ void __launch_bounds__(WP_TILE) k_world_pairs_write(const float4* __restrict__ bmin,
                                                                 const float4* __restrict__ bmax,
                                                                 const uint32_t* __restrict__ off, uint32_t n_worlds,
                                                                 const uint32_t* __restrict__ counts,
                                                                 const uint32_t* __restrict__ offsets,
                                                                 const uint32_t* __restrict__ wover, uint64_t* out) {
    static_assert(WP_TILE == 64, "two warps a CTA");
    __shared__ uint32_t s_mask[2], s_hits[2];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t w = blockIdx.x; w < n_worlds; w += gridDim.x) {
        if (!wover[w]) continue;  // uniform across the CTA
        const uint32_t lo = off[w], hi = off[w + 1];
        for (uint32_t ibase = lo; ibase < hi; ibase += WP_TILE) {
            const uint32_t me = ibase + threadIdx.x;
            const uint32_t m = __ballot_sync(0xffffffffu, me < hi && counts[me] > STASH_SLOTS);
            __syncthreads();  // the previous tile's readers of s_mask are done
            if (lane == 0) s_mask[warp] = m;
            __syncthreads();
            unsigned long long todo = (static_cast<unsigned long long>(s_mask[1]) << 32) | s_mask[0];
            while (todo) {
                const uint32_t i = ibase + uint32_t(__ffsll(static_cast<long long>(todo)) - 1);
                todo &= todo - 1ull;
                const float4 qmin = bmin[i], qmax = bmax[i];
                uint64_t pos = offsets[i];
                for (uint32_t jbase = i + 1; jbase < hi; jbase += WP_TILE) {
                    const uint32_t j = jbase + threadIdx.x;
                    const bool hit = j < hi && overlaps(qmin, qmax, bmin[j], bmax[j]);
                    const uint32_t b = __ballot_sync(0xffffffffu, hit);
                    if (lane == 0) s_hits[warp] = __popc(b);
                    __syncthreads();
                    const uint32_t h0 = s_hits[0], h1 = s_hits[1];
                    if (hit) out[pos + (warp ? h0 : 0u) + __popc(b & ((1u << lane) - 1u))] = (uint64_t(i) << 32) | j;
                    pos += h0 + h1;
                    __syncthreads();  // s_hits is rewritten next round
                }
            }
        }
    }
}

}  // namespace

uint64_t Broadphase::run_worlds(const float4* aabb_min, const float4* aabb_max, uint32_t n, const uint32_t* world_off,
                                uint32_t n_worlds, DevBuf<uint64_t>& out, cudaStream_t s) {
    if (n == 0 || n_worlds == 0) return 0;
    counts.reserve(n);
    offsets.reserve(n);
    scalars.reserve(4);
    stash.reserve(size_t(STASH_SLOTS) * n);
    overflow.reserve(n_worlds);
    check_cuda(cudaMemsetAsync(scalars.p + 1, 0, sizeof(uint32_t), s), "memset");
    const uint32_t grid = std::min<uint32_t>(n_worlds, 148u * 32u);
    k_world_pairs<<<grid, WP_TILE, 0, s>>>(aabb_min, aabb_max, world_off, n_worlds, n, counts.p, stash.p, overflow.p,
                                           scalars.p + 1);
    size_t scan_bytes = 0;
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.p, offsets.p, int(n), s), "scan size");
    cub_tmp.reserve(scan_bytes);
    check_cuda(cub::DeviceScan::ExclusiveSum(cub_tmp.p, scan_bytes, counts.p, offsets.p, int(n), s), "scan");
    k_total<<<1, 1, 0, s>>>(n, counts.p, offsets.p, scalars.p);
    check_cuda(cudaMemcpyAsync(host_scalars, scalars.p, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "total d2h");
    check_cuda(cudaStreamSynchronize(s), "broadphase sync");
    uint64_t total = host_scalars[0];
    const uint32_t n_over = host_scalars[1];
    out.reserve(total + 1);
    if (total) {
        k_stash_copy<<<(n + 255) / 256, 256, 0, s>>>(int(n), nullptr, counts.p, offsets.p, stash.p, out.p);
        if (n_over)
            k_world_pairs_write<<<grid, WP_TILE, 0, s>>>(aabb_min, aabb_max, world_off, n_worlds, counts.p, offsets.p,
                                                         overflow.p, out.p);
    }
    return total;
}

Broadphase::Broadphase() {
    check_cuda(cudaMallocHost(&host_scalars, 4 * sizeof(uint32_t)), "cudaMallocHost");
}

Broadphase::~Broadphase() {
    if (host_scalars) cudaFreeHost(host_scalars);
}

uint64_t Broadphase::run(const float4* aabb_min, const float4* aabb_max, uint32_t n,
                         const std::vector<uint32_t>& unbounded_host, DevBuf<uint64_t>& out, uint32_t* status_dev,
                         cudaStream_t s) {
    if (n == 0) return 0;
    const uint32_t nunb = uint32_t(unbounded_host.size());
    const int m = int(n - nunb);
    tree_m = m;
    this->nunb = nunb;
    const int TB = 256;
    const uint32_t grid = (n + TB - 1) / TB;
    keys.reserve(n);
    keys_alt.reserve(n);
    leaf_body.reserve(n);
    parent.reserve(2 * size_t(n));
    left.reserve(n);
    right.reserve(n);
    refit_flag.reserve(n);
    node_min.reserve(2 * size_t(n));
    node_max.reserve(2 * size_t(n));
    node_maxid.reserve(2 * size_t(n));
    node_rec.reserve(4 * size_t(n));
    counts.reserve(n);
    offsets.reserve(n);
    flags.reserve(n);
    scan_out.reserve(n);
    bounds.reserve(6);
    scalars.reserve(4);
    unbounded.reserve(nunb + 1);
    if (nunb) check_cuda(cudaMemcpyAsync(unbounded.p, unbounded_host.data(), nunb * sizeof(uint32_t),
                                         cudaMemcpyHostToDevice, s), "upload unbounded");
    // flags doubles as the "is unbounded" marker until the unbounded pass.
    k_clear_u32<<<grid, TB, 0, s>>>(n, flags.p);
    if (nunb) k_set_unbounded<<<(nunb + TB - 1) / TB, TB, 0, s>>>(unbounded.p, nunb, flags.p);
    k_reset_bounds<<<1, 32, 0, s>>>(bounds.p);
    k_bounds<<<grid, TB, 0, s>>>(aabb_min, aabb_max, flags.p, n, bounds.p);
    // keys / keys_alt (n x 8 bytes each) hold the codes and indices and their sort buffers.
    uint32_t* codes = reinterpret_cast<uint32_t*>(keys.p);
    uint32_t* codes_alt = reinterpret_cast<uint32_t*>(keys_alt.p);
    k_keys<<<grid, TB, 0, s>>>(aabb_min, aabb_max, flags.p, n, bounds.p, codes, codes + n);

    size_t tmp_bytes = 0;
    cub::DoubleBuffer<uint32_t> dk(codes, codes_alt), dv(codes + n, codes_alt + n);
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dv, int(n), 0, 32, s), "sort size");
    size_t scan_bytes = 0;
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.p, offsets.p, int(n), s), "scan size");
    cub_tmp.reserve(std::max(tmp_bytes, scan_bytes));
    check_cuda(cub::DeviceRadixSort::SortPairs(cub_tmp.p, tmp_bytes, dk, dv, int(n), 0, 32, s), "sort");
    const LeafKeys sorted{dk.Current(), dv.Current()};

    if (m > 0) {
        k_build<<<(m + TB - 1) / TB, TB, 0, s>>>(sorted, m, left.p, right.p, parent.p, leaf_body.p, refit_flag.p);
        k_refit<<<(m + TB - 1) / TB, TB, 0, s>>>(m, leaf_body.p, parent.p, left.p, right.p, refit_flag.p, aabb_min,
                                                 aabb_max, node_min.p, node_max.p, node_maxid.p, node_rec.p);
    }
    const uint32_t qgrid = m > 0 ? (uint32_t(m) + TB - 1) / TB : 1u;
    // One traversal per proxy: counts, plus the sorted partners of every proxy with at
    // most STASH_SLOTS of them; the rest are listed and walk the tree again below.
    stash.reserve(size_t(STASH_SLOTS) * uint32_t(m > 0 ? m : 1));
    overflow.reserve(uint32_t(m > 0 ? m : 1));
    check_cuda(cudaMemsetAsync(scalars.p, 0, 2 * sizeof(uint32_t), s), "memset");
    k_query<Q_STASH><<<qgrid, TB, 0, s>>>(m, n, flags.p, aabb_min, aabb_max, node_rec.p, leaf_body.p, unbounded.p,
                                          nunb, counts.p, nullptr, nullptr, status_dev, overflow.p, scalars.p + 1,
                                          stash.p);
    // Unbounded proxies: count their segments by flag + scan.
    for (uint32_t u = 0; u < nunb; ++u) {
        uint32_t h = unbounded_host[u];
        // scan_out holds the flags; the key scratch (no longer needed after the build) holds the scan.
        k_unb_flags<<<grid, TB, 0, s>>>(h, n, aabb_min, aabb_max, scan_out.p);
        check_cuda(cub::DeviceScan::ExclusiveSum(cub_tmp.p, scan_bytes, scan_out.p, (uint32_t*)keys_alt.p, int(n), s), "scan");
        k_unb_count<<<1, 1, 0, s>>>(h, n, scan_out.p, (uint32_t*)keys_alt.p, counts.p);
    }
    check_cuda(cub::DeviceScan::ExclusiveSum(cub_tmp.p, scan_bytes, counts.p, offsets.p, int(n), s), "scan");
    k_total<<<1, 1, 0, s>>>(n, counts.p, offsets.p, scalars.p);
    check_cuda(cudaMemcpyAsync(host_scalars, scalars.p, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "total d2h");
    check_cuda(cudaStreamSynchronize(s), "broadphase sync");
    uint64_t total = host_scalars[0];
    const uint32_t n_overflow = host_scalars[1];
    out.reserve(total + 1);
    if (total) {
        if (m > 0) k_stash_copy<<<qgrid, TB, 0, s>>>(m, leaf_body.p, counts.p, offsets.p, stash.p, out.p);
        if (n_overflow)
            k_query<Q_WRITE><<<(n_overflow + TB - 1) / TB, TB, 0, s>>>(
                m, n, flags.p, aabb_min, aabb_max, node_rec.p, leaf_body.p, unbounded.p, nunb, counts.p, offsets.p,
                out.p, status_dev, overflow.p, scalars.p + 1, nullptr);
        for (uint32_t u = 0; u < nunb; ++u) {
            uint32_t h = unbounded_host[u];
            k_unb_flags<<<grid, TB, 0, s>>>(h, n, aabb_min, aabb_max, scan_out.p);
            check_cuda(cub::DeviceScan::ExclusiveSum(cub_tmp.p, scan_bytes, scan_out.p, (uint32_t*)keys_alt.p, int(n), s), "scan");
            k_unb_write<<<grid, TB, 0, s>>>(h, n, scan_out.p, (uint32_t*)keys_alt.p, offsets.p, out.p);
        }
    }
    return total;
}

}  // namespace bgpu

// ---------------------------------------------------------------- allocation-free entry point
//
// For callers that cannot allocate device memory while they run: game and robotics
// loops with a fixed device-memory budget, code running inside another runtime
// that owns the allocator, or callers on a hard deadline that cannot afford a
// cudaMalloc / cudaFree round trip (both may synchronise the device). They pass
// device buffers for the input AABBs and the output pairs; every scratch array
// of the broad phase lives in one fixed file-scope device array instead.
//
// Limits: at most BGPU_NOALLOC_MAX_PROXIES proxies and BGPU_NOALLOC_MAX_UNBOUNDED
// unbounded proxies (extent >= 1e15, e.g. planes); larger inputs are rejected.
// The array is shared by every call in the process and keeps the last call's
// contents, so two calls that overlap on the GPU (different streams, or
// different host threads) race on it and must be serialised by the caller.
// Each GPU that loads the library holds the array until the process exits.
#include <mutex>
#include "../../include/bgpu.h"

namespace bgpu {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(24) << 20;
// Bytes per proxy of the arrays taken below (AABBs 32, sort keys 16, flags / scans / counts /
// offsets / tree links 36, parents 8, node boxes 64, node records 64, node index bounds 8),
// plus 256 B of alignment per array and room for CUB's sort / scan scratch (a few hundred KB
// at 65,536 keys; 4 MiB allowed). Each take() is also checked when the call runs.
constexpr size_t NOALLOC_PER_PROXY_BYTES = 228;
static_assert(NOALLOC_PER_PROXY_BYTES * BGPU_NOALLOC_MAX_PROXIES + 32 * 256 + (size_t(4) << 20) <= NOALLOC_SCRATCH_BYTES,
              "the allocation-free broad phase's scratch array is too small for its proxy limit");
static __device__ __align__(256) unsigned char g_bp_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_bp_scratch_mutex;
constexpr int NOALLOC_MAX_DEVICES = 64;
unsigned char* g_bp_scratch_addr[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array for the current device. In host code the
// array's name is only a stand-in, so the address comes from the runtime, once
// per device (the first call on a device does this lookup).
unsigned char* noalloc_scratch_address(int dev) {
    std::lock_guard<std::mutex> lock(g_bp_scratch_mutex);
    if (!g_bp_scratch_addr[dev]) {
        void* ptr = nullptr;
        check_cuda(cudaGetSymbolAddress(&ptr, g_bp_scratch), "cudaGetSymbolAddress(g_bp_scratch)");
        g_bp_scratch_addr[dev] = static_cast<unsigned char*>(ptr);
    }
    return g_bp_scratch_addr[dev];
}

struct Bump {
    unsigned char* base;
    size_t used, cap;
    template <class T>
    T* take(size_t n) {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = n * sizeof(T);
        if (off + bytes > cap) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

__global__ void k_noalloc_unpack(const float* __restrict__ aabbs, uint32_t n, float4* mn, float4* mx,
                                 uint32_t* is_unb) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = aabbs + 6 * size_t(i);
    mn[i] = make_float4(a[0], a[1], a[2], 0.0f);
    mx[i] = make_float4(a[3], a[4], a[5], 0.0f);
    bool huge = !(a[3] - a[0] < 1e15f) || !(a[4] - a[1] < 1e15f) || !(a[5] - a[2] < 1e15f);
    is_unb[i] = huge ? 1u : 0u;
}

__global__ void k_unb_write_list(uint32_t n, const uint32_t* __restrict__ is_unb, const uint32_t* __restrict__ scan,
                                 uint32_t* list) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && is_unb[i]) list[scan[i]] = i;
}

// Keys (lo << 32 | hi) become (lo, hi) uint32 pairs in place.
__global__ void k_noalloc_keys_to_pairs(uint64_t* buf, uint64_t n) {
    uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint64_t key = buf[k];
    uint32_t* p = reinterpret_cast<uint32_t*>(buf + k);
    p[0] = uint32_t(key >> 32);
    p[1] = uint32_t(key & 0xffffffffu);
}

}  // namespace
}  // namespace bgpu

extern "C" bgpu_status bgpu_broadphase_pairs_noalloc(const float* aabbs_dev, uint32_t n, uint32_t* pairs_dev,
                                                     uint64_t cap, uint64_t* out_n, void* stream) {
    using namespace bgpu;
    if (out_n) *out_n = 0;
    if ((n && !aabbs_dev) || (cap && !pairs_dev) || (reinterpret_cast<uintptr_t>(pairs_dev) & 7u)) {
        set_last_error("allocation-free broad phase: NULL buffer or pairs buffer not 8-byte aligned");
        return BGPU_ERR_INVALID_ARGUMENT;
    }
    if (n > BGPU_NOALLOC_MAX_PROXIES) {
        set_last_error("allocation-free broad phase: more than BGPU_NOALLOC_MAX_PROXIES (65536) proxies");
        return BGPU_ERR_CAPACITY;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    try {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
            set_last_error("allocation-free broad phase: device ordinal out of range");
            return BGPU_ERR_CAPACITY;
        }
        if (n == 0) return BGPU_OK;
        Bump sb{noalloc_scratch_address(dev), 0, NOALLOC_SCRATCH_BYTES};
        float4* mn = sb.take<float4>(n);
        float4* mx = sb.take<float4>(n);
        uint64_t* keys = sb.take<uint64_t>(n);
        uint64_t* keys_alt = sb.take<uint64_t>(n);
        uint32_t* is_unb = sb.take<uint32_t>(n);
        uint32_t* leaf_body = sb.take<uint32_t>(n);
        uint32_t* parent = sb.take<uint32_t>(2 * size_t(n));
        uint32_t* left = sb.take<uint32_t>(n);
        uint32_t* right = sb.take<uint32_t>(n);
        uint32_t* refit_flag = sb.take<uint32_t>(n);
        uint32_t* counts = sb.take<uint32_t>(n);
        uint32_t* offsets = sb.take<uint32_t>(n);
        uint32_t* flags = sb.take<uint32_t>(n);
        uint32_t* scan = sb.take<uint32_t>(n);
        uint32_t* unb_list = sb.take<uint32_t>(BGPU_NOALLOC_MAX_UNBOUNDED + 1);
        float4* node_min = sb.take<float4>(2 * size_t(n));
        float4* node_max = sb.take<float4>(2 * size_t(n));
        float4* node_rec = sb.take<float4>(4 * size_t(n));
        uint32_t* node_maxid = sb.take<uint32_t>(2 * size_t(n));
        int* bounds = sb.take<int>(8);
        uint32_t* scalars = sb.take<uint32_t>(8);
        const void* taken[] = {mn, mx, keys, keys_alt, is_unb, leaf_body, parent, left, right, refit_flag, counts,
                               offsets, flags, scan, unb_list, node_min, node_max, node_rec, node_maxid, bounds, scalars};
        for (const void* t : taken)
            if (!t) {
                set_last_error("allocation-free broad phase: scratch array too small");
                return BGPU_ERR_CAPACITY;
            }
        size_t sort_bytes = 0, scan_bytes = 0;
        uint32_t* codes = reinterpret_cast<uint32_t*>(keys);
        uint32_t* codes_alt = reinterpret_cast<uint32_t*>(keys_alt);
        cub::DoubleBuffer<uint32_t> dk(codes, codes_alt), dv(codes + n, codes_alt + n);
        check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, dk, dv, int(n), 0, 32, s), "sort size");
        check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, offsets, int(n), s), "scan size");
        size_t tmp_bytes = std::max(sort_bytes, scan_bytes);
        unsigned char* tmp = sb.take<unsigned char>(tmp_bytes);
        if (!tmp) {
            set_last_error("allocation-free broad phase: scratch array too small");
            return BGPU_ERR_CAPACITY;
        }
        const int TB = 256;
        const uint32_t grid = (n + TB - 1) / TB;
        // Nothing below relies on the previous call's contents; the status word and the
        // counters are cleared here, every other array is fully rewritten before it is read.
        check_cuda(cudaMemsetAsync(scalars, 0, 8 * sizeof(uint32_t), s), "memset");
        k_noalloc_unpack<<<grid, TB, 0, s>>>(aabbs_dev, n, mn, mx, is_unb);
        // Unbounded proxies, listed in index order (few by contract).
        check_cuda(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, is_unb, scan, int(n), s), "scan");
        uint32_t host_scan_last[2] = {0, 0};
        check_cuda(cudaMemcpyAsync(&host_scan_last[0], scan + (n - 1), 4, cudaMemcpyDeviceToHost, s), "d2h");
        check_cuda(cudaMemcpyAsync(&host_scan_last[1], is_unb + (n - 1), 4, cudaMemcpyDeviceToHost, s), "d2h");
        check_cuda(cudaStreamSynchronize(s), "sync");
        uint32_t nunb = host_scan_last[0] + host_scan_last[1];
        if (nunb > BGPU_NOALLOC_MAX_UNBOUNDED) {
            set_last_error("allocation-free broad phase: more than BGPU_NOALLOC_MAX_UNBOUNDED (16) unbounded proxies");
            return BGPU_ERR_CAPACITY;
        }
        uint32_t unb_host[BGPU_NOALLOC_MAX_UNBOUNDED + 1];
        if (nunb) {
            k_unb_write_list<<<grid, TB, 0, s>>>(n, is_unb, scan, unb_list);
            check_cuda(cudaMemcpyAsync(unb_host, unb_list, nunb * 4, cudaMemcpyDeviceToHost, s), "d2h");
        }
        const int m = int(n - nunb);
        k_reset_bounds<<<1, 32, 0, s>>>(bounds);
        k_bounds<<<grid, TB, 0, s>>>(mn, mx, is_unb, n, bounds);
        k_keys<<<grid, TB, 0, s>>>(mn, mx, is_unb, n, bounds, codes, codes + n);
        check_cuda(cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, dk, dv, int(n), 0, 32, s), "sort");
        const LeafKeys sorted{dk.Current(), dv.Current()};
        if (m > 0) {
            k_build<<<(m + TB - 1) / TB, TB, 0, s>>>(sorted, m, left, right, parent, leaf_body, refit_flag);
            k_refit<<<(m + TB - 1) / TB, TB, 0, s>>>(m, leaf_body, parent, left, right, refit_flag, mn, mx, node_min,
                                                     node_max, node_maxid, node_rec);
        }
        uint32_t* status = scalars + 1;
        const uint32_t qgrid = m > 0 ? (uint32_t(m) + TB - 1) / TB : 1u;
        k_query<Q_COUNT><<<qgrid, TB, 0, s>>>(m, n, is_unb, mn, mx, node_rec, leaf_body, unb_list, nunb, counts,
                                              nullptr, nullptr, status, nullptr, nullptr, nullptr);
        uint32_t* unb_scan = dk.Alternate();  // free after the build
        check_cuda(cudaStreamSynchronize(s), "sync");
        for (uint32_t u = 0; u < nunb; ++u) {
            uint32_t h = unb_host[u];
            k_unb_flags<<<grid, TB, 0, s>>>(h, n, mn, mx, flags);
            check_cuda(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, flags, unb_scan, int(n), s), "scan");
            k_unb_count<<<1, 1, 0, s>>>(h, n, flags, unb_scan, counts);
        }
        check_cuda(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, counts, offsets, int(n), s), "scan");
        k_total<<<1, 1, 0, s>>>(n, counts, offsets, scalars);
        uint32_t host_scalars[2] = {0, 0};
        check_cuda(cudaMemcpyAsync(host_scalars, scalars, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "d2h");
        check_cuda(cudaStreamSynchronize(s), "sync");
        if (host_scalars[1]) {  // the count walk overflowed its stack: the total is not a pair count
            set_last_error("allocation-free broad phase: traversal stack overflow");
            return BGPU_ERR_DEVICE_STATUS;
        }
        uint64_t total = host_scalars[0];
        if (out_n) *out_n = total;
        if (total > cap) {
            set_last_error("allocation-free broad phase: output capacity too small (out_n holds the pair count)");
            return BGPU_ERR_CAPACITY;
        }
        uint64_t* out = reinterpret_cast<uint64_t*>(pairs_dev);
        if (total) {
            k_query<Q_WRITE><<<qgrid, TB, 0, s>>>(m, n, is_unb, mn, mx, node_rec, leaf_body, unb_list, nunb, counts,
                                                  offsets, out, status, nullptr, nullptr, nullptr);
            for (uint32_t u = 0; u < nunb; ++u) {
                uint32_t h = unb_host[u];
                k_unb_flags<<<grid, TB, 0, s>>>(h, n, mn, mx, flags);
                check_cuda(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, flags, unb_scan, int(n), s), "scan");
                k_unb_write<<<grid, TB, 0, s>>>(h, n, flags, unb_scan, offsets, out);
            }
            k_noalloc_keys_to_pairs<<<uint32_t((total + TB - 1) / TB), TB, 0, s>>>(out, total);
        }
        uint32_t st = 0;
        check_cuda(cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s), "d2h");
        check_cuda(cudaStreamSynchronize(s), "sync");
        check_cuda(cudaGetLastError(), "launch");
        if (st) {
            set_last_error("allocation-free broad phase: traversal stack overflow");
            return BGPU_ERR_DEVICE_STATUS;
        }
        return BGPU_OK;
    } catch (const CudaError& e) {
        set_last_error(e.where);
        return BGPU_ERR_CUDA;
    }
}
