// Reverse mode of a recorded step (the adjoint; the reference has no
// counterpart: its world is not differentiable).
//
// The differentiated model holds each step's contact geometry fixed at its
// forward values: the rows' normals, lever arms, tangent basis, the terms
// Iw^-1 (r x d), effective masses and bias terms, and the bodies' world inverse
// inertia. The solve's clamp decisions (normal impulse at zero, friction at
// +-mu * normal impulse or inside, restitution branch) and the sleep decisions
// are the forward pass's. With those frozen, a step is piecewise linear in the
// velocities, the accumulated impulses and the material products mu_a * mu_b
// and e_a * e_b, and this file runs its exact transpose:
//
//   positions   x' = x + v dt                  (integrate_position, body.rs:1156)
//   solve       the PGS sweeps in reverse order (sequential_impulse.rs:692-930),
//               the warm start of each row taken from the previous step's final
//               normal impulse of the same manifold point times the warm-start
//               factor (step.rs:751, 821), and so chained across steps
//   islands     velocities of a body whose island fell asleep were zeroed
//   velocities  v' = s_lin v + g dt, w' = s_ang w (+ the gyroscopic term, frozen)
//
// The split-impulse pass and the push velocities do not depend on velocities
// or materials, so they carry no adjoint.
#include "bgpu_kernels.cuh"

namespace bgpu {

namespace {

__global__ void k_adj_positions(uint32_t n, float dt, const uint8_t* __restrict__ flags,
                                const float4* __restrict__ xbar, float4* vbar) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !(flags[i] & RF_MOVED)) return;
    float4 x = xbar[i], v = vbar[i];
    vbar[i] = make_float4(v.x + x.x * dt, v.y + x.y * dt, v.z + x.z * dt, 0.0f);
}

__global__ void k_adj_velocities(uint32_t n, float dt, const uint8_t* __restrict__ flags,
                                 const float4* __restrict__ material, float4* vbar, float4* wbar) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t f = flags[i];
    if (f & RF_ZEROED) {
        vbar[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        wbar[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    if (!(f & RF_INTEGRATED)) return;
    float4 m = material[i];
    // apply_damping (body.rs:1066-1070): v *= (1 - d)^dt when d != 0.
    if (m.z != 0.0f) {
        float s = powf(1.0f - m.z, dt);
        float4 v = vbar[i];
        vbar[i] = make_float4(v.x * s, v.y * s, v.z * s, 0.0f);
    }
    if (m.w != 0.0f) {
        float s = powf(1.0f - m.w, dt);
        float4 w = wbar[i];
        wbar[i] = make_float4(w.x * s, w.y * s, w.z * s, 0.0f);
    }
}

struct AdjArgs {
    const uint4* recs;         // the step's batch slot records
    const uint32_t* off;       // colour batch starts / ends
    const uint32_t* end;
    uint32_t ncol;
    uint32_t iters;
    const float4* tab;         // the step's velocity contact table
    const float4* sweeps;      // the step's sweep records
    float4* lbar;              // adjoint of each row's accumulated impulses (normal, t1, t2)
    float4* vbar;
    float4* wbar;
    float* mubar;
    float* ebar;
    const float4* material;
    const uint32_t* merge_pos;  // pair -> position of its manifold in the merged cache
    const float* carry_in;      // adjoint of the final normal impulses, by merged position * 4 + point
    const uint32_t* row_src;    // row -> old cache position * 4 + point of its warm start
    float* carry_out;           // adjoint of the previous step's final normal impulses (same indexing)
    float restitution_threshold;
    float warm_factor;
    unsigned int* bar;
    uint32_t* status;
};

__device__ __forceinline__ size_t lix(uint32_t k, uint32_t t) { return tix<1>(0, k, t); }

// One row group of one sweep, in reverse.
__device__ __forceinline__ void reverse_group(const AdjArgs& a, uint32_t t, uint32_t sweep) {
    const uint4 rec = a.recs[t];
    const uint32_t ia = rec.x, ib = rec.y, p = rec.z & 0x1fffffffu, cnt = rec.z >> 29;
    const float4* e0 = a.tab + tix<VT_PLANES>(0, 0, t);
    const float ima = e0[VT_T1 * PLANE_STRIDE].w, imb = e0[VT_A2B * PLANE_STRIDE].w;
    const float ims = ima + imb;
    const bool appa = ima > 0.0f, appb = imb > 0.0f;
    V3 La = from4(__ldcg(&a.vbar[ia])), Wa = from4(__ldcg(&a.wbar[ia]));
    V3 Lb = from4(__ldcg(&a.vbar[ib])), Wb = from4(__ldcg(&a.wbar[ib]));
    // Velocity-side adjoint of an impulse j applied along (d, ca, cb).
    auto japp = [&](V3 d, V3 ca, V3 cb) {
        float s = 0.0f;
        if (appa) s += -dot(d, La) * ima - dot(ca, Wa);
        if (appb) s += dot(d, Lb) * imb + dot(cb, Wb);
        return s;
    };
    if (sweep == a.iters) {  // first touch of this slot: the final impulses' adjoint
        const uint32_t mp = a.merge_pos ? a.merge_pos[p] : REC_NONE;
        for (uint32_t k = 0; k < cnt; ++k) {
            const float c = (a.carry_in && mp != REC_NONE) ? a.carry_in[size_t(mp) * 4 + k] : 0.0f;
            a.lbar[lix(k, t)] = make_float4(c, 0.0f, 0.0f, 0.0f);
        }
    }
    float mub = 0.0f, eb = 0.0f;
    for (int kk = int(cnt) - 1; kk >= 0; --kk) {
        const uint32_t k = uint32_t(kk);
        const float4* e = a.tab + tix<VT_PLANES>(0, k, t);
        const V3 n = from4(e[VT_N * PLANE_STRIDE]);
        const V3 ana = from4(e[VT_ANA * PLANE_STRIDE]), anb = from4(e[VT_ANB * PLANE_STRIDE]);
        float4 lb = a.lbar[lix(k, t)];
        if (sweep == 0) {  // warm start: only the normal impulse is nonzero (step.rs:751)
            const float lin = lb.x + japp(n, ana, anb);
            const uint32_t src = a.row_src[size_t(p) * 4 + k];
            if (src != REC_NONE && a.carry_out) atomicAdd(&a.carry_out[src], a.warm_factor * lin);
            continue;
        }
        const float4 r0 = e[VT_N * PLANE_STRIDE], r1 = e[VT_RA * PLANE_STRIDE], r2 = e[VT_RB * PLANE_STRIDE];
        const float4 q3 = e[VT_T1 * PLANE_STRIDE];
        const float4 q5 = e[VT_ANA * PLANE_STRIDE], q6 = e[VT_ANB * PLANE_STRIDE];
        const float4 q7 = e[VT_A1A * PLANE_STRIDE], q8 = e[VT_A1B * PLANE_STRIDE];
        const float4 q9 = e[VT_A2A * PLANE_STRIDE], q10 = e[VT_A2B * PLANE_STRIDE];
        const V3 ra = from4(r1), rb = from4(r2), t1 = from4(q3), t2 = cross(n, t1);
        const V3 a1a = from4(q7), a1b = from4(q8), a2a = from4(q9), a2b = from4(q10);
        const V3 kn = n * ims + cross(anb, rb) + cross(ana, ra);  // as the forward sweep makes them
        const V3 kt1 = t1 * ims + cross(a1b, rb) + cross(a1a, ra);
        const float mn = q5.w, m1 = q6.w, m2 = q7.w, cfm = q8.w, e_ab = q9.w, mu_ab = r0.w;
        const float4 sr = a.sweeps[sweep_index(sweep, k, t, a.iters)];
        const float vn = sr.x, nimp = sr.y;
        const uint32_t bits = __float_as_uint(sr.z), s1 = bits & 3u, s2 = (bits >> 2) & 3u;
        // friction 2: n2 = clamp(o2 - m2 t2.rel2, +-mu nimp)
        const float jb2 = japp(t2, a2a, a2b);
        const float n2b = lb.z + jb2;
        float o2b = -jb2, maxfb = 0.0f, u2b = 0.0f;
        if (s2 == 0u) u2b = n2b;
        else if (s2 == 1u) maxfb += n2b;
        else maxfb -= n2b;
        o2b += u2b;
        V3 relb = t2 * (-m2 * u2b);
        // friction 1 (rel2 = rel1 + kt1 j1)
        const float jb1 = dot(kt1, relb) + japp(t1, a1a, a1b);
        const float n1b = lb.y + jb1;
        float o1b = -jb1, u1b = 0.0f;
        if (s1 == 0u) u1b = n1b;
        else if (s1 == 1u) maxfb += n1b;
        else maxfb -= n1b;
        o1b += u1b;
        relb += t1 * (-m1 * u1b);
        // the friction bound mu_ab * nimp
        mub += maxfb * nimp;
        // normal (rel1 = rel0 + kn jn)
        const float jbn = dot(kn, relb) + japp(n, ana, anb);
        const float nimpb = lb.x + maxfb * mu_ab + jbn;
        float onb = -jbn;
        if (nimp > 0.0f) {
            onb += nimpb;
            const float biasb = mn * nimpb;
            float vnb = -mn * nimpb;
            onb -= cfm * nimpb;
            if (vn < -a.restitution_threshold) {  // bias = -e_ab vn
                eb += biasb * (-vn);
                vnb += biasb * (-e_ab);
            }
            relb += n * vnb;
        }
        // rel0 = (lb + wb x rb) - (la + wa x ra)
        Lb += relb;
        Wb += cross(rb, relb);
        La -= relb;
        Wa -= cross(ra, relb);
        a.lbar[lix(k, t)] = make_float4(onb, o1b, o2b, 0.0f);
    }
    if (appa) { __stcg(&a.vbar[ia], to4(La, 0.0f)); __stcg(&a.wbar[ia], to4(Wa, 0.0f)); }
    if (appb) { __stcg(&a.vbar[ib], to4(Lb, 0.0f)); __stcg(&a.wbar[ib], to4(Wb, 0.0f)); }
    // friction = mu_a mu_b, restitution = e_a e_b (sequential_impulse.rs:417-419)
    if (mub != 0.0f || eb != 0.0f) {
        const float4 ma = a.material[ia], mb = a.material[ib];
        atomicAdd(&a.mubar[ia], mub * mb.x);
        atomicAdd(&a.mubar[ib], mub * ma.x);
        atomicAdd(&a.ebar[ia], eb * mb.y);
        atomicAdd(&a.ebar[ib], eb * ma.y);
    }
}

// The forward phases (sweep, colour) in reverse order, one team barrier
// between phases; within a phase no dynamic body appears twice, so the body
// adjoints are gathered and scattered without atomics.
__global__ void __launch_bounds__(256, 2) k_adj_solve(AdjArgs a) {
    const uint32_t ncol = a.ncol;
    const uint32_t nphases = (a.iters + 1) * ncol;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    __shared__ uint32_t s_off[128], s_end[128];
    for (uint32_t c = threadIdx.x; c < ncol; c += blockDim.x) {
        s_off[c] = a.off[c];
        s_end[c] = a.end[c];
    }
    __syncthreads();
    uint32_t nbar = 0;
    for (uint32_t qq = nphases; qq-- > 0;) {
        const uint32_t c = qq % ncol, sweep = qq / ncol;
        for (uint32_t t = s_off[c] + tid; t < s_end[c]; t += stride) reverse_group(a, t, sweep);
        if (qq > 0) team_barrier(a.bar, ++nbar * gridDim.x, a.status);
    }
}

// A step of the per-world solver in reverse: each world's phases (sweep, colour) run backwards
// inside the CTA or warp the plan gives it (the same deal as the forward kernel, k_solver.cu),
// with a block or warp sync between phases. Worlds share no body, so no barrier spans them.
// wrec: per world g0, ncol, offsets[ncol + 1] (WS_STRIDE words).
template <bool WARP>
__device__ void reverse_world(const AdjArgs& a, const uint32_t* __restrict__ wrec, uint32_t w, uint32_t lane,
                              uint32_t nt) {
    const uint32_t* r = wrec + size_t(w) * WS_STRIDE;
    const uint32_t g0 = r[0], ncol = min(r[1], WS_MAX_COLOURS);
    for (uint32_t sweep = a.iters + 1; sweep-- > 0;) {
        for (uint32_t c = ncol; c-- > 0;) {
            const uint32_t hi = g0 + r[3 + c];
            for (uint32_t t = g0 + r[2 + c] + lane; t < hi; t += nt) reverse_group(a, t, sweep);
            if (WARP) __syncwarp();
            else __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(256) k_adj_solve_worlds(AdjArgs a, WorldPlanDev plan, const uint32_t* wrec) {
    const uint2 c = plan.cta[blockIdx.x];
    const bool block_mode = (c.y >> 31) != 0u;
    const uint32_t count = c.y & 0x7fffffffu;
    if (block_mode) {
        reverse_world<false>(a, wrec, plan.list[c.x], threadIdx.x, blockDim.x);
        return;
    }
    const uint32_t wi = threadIdx.x >> 5;
    if (wi < count) reverse_world<true>(a, wrec, plan.list[c.x + wi], threadIdx.x & 31u, 32u);
}

int adj_grid() {
    static int grid = 0;
    if (!grid) {
        int dev = 0, sms = 0, per_sm = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
        check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_adj_solve, 256, 0), "occupancy");
        grid = sms * (per_sm < 1 ? 1 : per_sm);
    }
    return grid;
}

}  // namespace

void launch_adj_positions(uint32_t n, float dt, const uint8_t* flags, const float4* xbar, float4* vbar, cudaStream_t s) {
    if (n) k_adj_positions<<<(n + 255) / 256, 256, 0, s>>>(n, dt, flags, xbar, vbar);
}

void launch_adj_velocities(uint32_t n, float dt, const uint8_t* flags, const float4* material, float4* vbar,
                           float4* wbar, cudaStream_t s) {
    if (n) k_adj_velocities<<<(n + 255) / 256, 256, 0, s>>>(n, dt, flags, material, vbar, wbar);
}

void run_adj_solve(const AdjStep& st, float4* lbar, float4* vbar, float4* wbar, float* mubar, float* ebar,
                   const float4* material, const float* carry_in, float* carry_out, float restitution_threshold,
                   float warm_factor, unsigned int* bar, uint32_t* status_dev, cudaStream_t s) {
    if (st.ncol == 0) return;
    check_cuda(cudaMemsetAsync(bar, 0, sizeof(unsigned int), s), "memset barrier");
    AdjArgs a{st.recs, st.off, st.end, st.ncol, st.iters, st.tab, st.sweeps, lbar, vbar, wbar, mubar, ebar, material,
              st.merge_pos, carry_in, st.row_src, carry_out, restitution_threshold, warm_factor, bar, status_dev};
    void* args[] = {&a};
    check_cuda(cudaLaunchCooperativeKernel((const void*)k_adj_solve, dim3(adj_grid()), dim3(256), args, 0, s),
               "adjoint solve launch");
}

void run_adj_solve_worlds(const AdjStep& st, const WorldPlan& plan, float4* lbar, float4* vbar, float4* wbar,
                          float* mubar, float* ebar, const float4* material, const float* carry_in, float* carry_out,
                          float restitution_threshold, float warm_factor, uint32_t* status_dev, cudaStream_t s) {
    if (st.ncol == 0) return;
    if (!plan.valid || plan.ncta == 0)
        throw CudaError{cudaErrorInvalidValue, "the batch's solver launch shape changed between forward and backward"};
    AdjArgs a{st.recs, st.off, st.end, st.ncol, st.iters, st.tab, st.sweeps, lbar, vbar, wbar, mubar, ebar, material,
              st.merge_pos, carry_in, st.row_src, carry_out, restitution_threshold, warm_factor, nullptr, status_dev};
    // A plan of more than 256 threads a CTA has block-mode worlds only, which run on any block size.
    k_adj_solve_worlds<<<plan.ncta, plan.block > 256 ? 256u : plan.block, 0, s>>>(a, plan.dev(), st.off);
    check_cuda(cudaGetLastError(), "adjoint world solve launch");
}

}  // namespace bgpu
