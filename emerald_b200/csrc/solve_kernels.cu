// Solver kernels of the 2D SPH sub-step: one thread per fluid particle,
// neighbour lists streamed slot-major, neighbour state gathered by index.
//
// Each kernel fuses the reference's fluid pass and boundary pass of one
// sph_common / sph2d_box function (they only read state the other pass does
// not write) and, where the reference runs a per-particle step right after,
// that step too. Sums run in neighbour-list order with the reference's
// operator order, so every value is bit-identical to the CPU reference.
//
// Convergence loops stay on the device: iteration kernels accumulate the
// reference's error reductions per scene (integer sum of error*1000 and the
// maximum), and a one-block check kernel applies the reference's exit test
// and marks finished scenes, whose later iteration launches return at once.
#include <algorithm>

#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr double kFlicksPerSecond = 705600000.0;

// Block-level setup shared by the per-particle kernels. A tile belongs to
// one scene, so the scene checks are uniform across the block.
struct Ctx {
    int32_t s;
    uint32_t i;
    bool live;
};

__device__ __forceinline__ bool enter(Arena const& a, bool skip_done, Ctx& c) {
    c.s = a.tile_scene[blockIdx.x];
    if (c.s < 0) return false;
    SceneState const& S = a.ss[c.s];
    if (!S.active) return false;
    if (skip_done && S.done) return false;
    SceneParams const& P = a.sp[c.s];
    c.i = blockIdx.x * kTile + threadIdx.x;
    c.live = (c.i - P.fluid_begin) < P.fluid_count;
    return true;
}

// Adds a per-thread error contribution to the scene's accumulators: the
// integer sum and the maximum of non-negative floats (bit order equals value
// order for them). NaN contributions are dropped, as std::max and the
// compare-exchange loop of update_atomic_max drop them.
__device__ void accumulate_error(SceneState* S, unsigned long long v, float m, bool live,
                                 bool exact = false) {
    uint32_t mb = (live && m == m && m > 0.0f) ? __float_as_uint(m) : 0u;
    if (!live) v = 0ull;
    double ed = (exact && live && m == m && m > 0.0f) ? static_cast<double>(m) : 0.0;
    for (int o = 16; o; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        if (exact) ed += __shfl_xor_sync(0xffffffffu, ed, o);
    }
    __shared__ unsigned long long ws[kTile / 32];
    __shared__ uint32_t wm[kTile / 32];
    __shared__ double wd[kTile / 32];
    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    if (lane == 0) {
        ws[warp] = v;
        wm[warp] = mb;
        wd[warp] = ed;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        uint32_t tm = 0;
        double td = 0.0;
        for (int w = 0; w < kTile / 32; ++w) {
            t += ws[w];
            tm = max(tm, wm[w]);
            td += wd[w];
        }
        if (t) atomicAdd(&S->err_sum, t);
        if (tm) atomicMax(&S->err_max, tm);
        if (exact && td != 0.0) atomicAdd(&S->err_sum_d, td);
    }
}

__device__ __forceinline__ float* pressures_cur(Arena const& a, SceneState const& S) {
    return (S.iter & 1) ? a.pbuf1 : a.pbuf0;
}
__device__ __forceinline__ float* pressures_next(Arena const& a, SceneState const& S) {
    return (S.iter & 1) ? a.pbuf0 : a.pbuf1;
}

// ------------------------------------------------------------ frame control

// max_vector_squared_magnitude over the velocities (common.cpp:87-92), per scene.
__global__ void k_max_v2(Arena a) {
    Ctx c;
    if (!enter(a, false, c)) return;
    float d = 0.0f;
    if (c.live) {
        float2 const v = a.v[c.i];
        d = v.x * v.x + v.y * v.y;
    }
    uint32_t mb = (c.live && d == d && d > 0.0f) ? __float_as_uint(d) : 0u;
    for (int o = 16; o; o >>= 1) mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    // one atomic per tile (a block is one scene's tile)
    __shared__ uint32_t wmax[kTile / 32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mb;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kTile / 32; ++w) t = max(t, wmax[w]);
        if (t) atomicMax(&a.ss[c.s].max_v2, t);
    }
}

__device__ int64_t to_flicks_x86(double s) {
    double const f = s * kFlicksPerSecond;
    if (!(f > -9.2233720368547758e18 && f < 9.2233720368547758e18)) return INT64_MIN;
    return static_cast<int64_t>(f);
}

__device__ int to_int_x86(double d) {
    if (!(d > -2147483649.0 && d < 2147483648.0)) return INT32_MIN;
    return static_cast<int>(d);
}

// One thread per scene: picks the sub-step dt exactly as
// std_adaptive_time_step (emerald/sph2d_box/adaptive_time_step.h:63-103) with
// cfl_maximum_time_step (emerald/sph_common/cfl.cpp:12-21), or the fixed
// PCISPH sub-step (emerald/sph2d_box/pcisph.cpp:166-204), or the caller's dt.
__global__ void k_begin_substep(Arena a, int nscenes) {
    int const s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nscenes) return;
    SceneParams const& P = a.sp[s];
    SceneState& S = a.ss[s];
    if (!S.active) return;
    S.error &= ~kErrNonFinite;
    if (P.mode == kFixedDt) {
        S.dt = P.fixed_dt;
        S.t = P.fixed_t;
        S.new_frame = 0;
        S.max_v2 = 0;
        S.substeps_total += 1;
        return;
    }
    if (S.remaining == 0) {
        S.remaining = (P.method == kPcisph) ? P.sub_steps : P.min_denom;
        S.elapsed = 0;
        S.frame_substeps = 0;
        S.new_frame = 1;
    } else {
        S.new_frame = 0;
    }
    int num;
    int64_t sub;
    float dt;
    if (P.method == kPcisph) {
        num = 1;
        sub = P.time_per_step / P.sub_steps;
        dt = P.seconds_per_sub_step;
    } else {
        double const numer = static_cast<double>(P.cfl_factor * P.support);
        double const denom = sqrt(static_cast<double>(__uint_as_float(S.max_v2)));
        double const r = safe_d(numer, denom) ? numer / denom : static_cast<double>(1.0f);
        int64_t const cfl = to_flicks_x86(r);
        int64_t const tpss = P.time_per_step / P.min_denom;
        num = to_int_x86(ceil((static_cast<double>(cfl) / kFlicksPerSecond) /
                              (static_cast<double>(tpss) / kFlicksPerSecond)));
        int const divisor = P.min_denom / P.max_denom;
        num = num < 1 ? 1 : (num > divisor ? divisor : num);
        num = num < S.remaining ? num : S.remaining;
        sub = static_cast<int64_t>(num) * tpss;
        dt = static_cast<float>(static_cast<double>(sub) / kFlicksPerSecond);
    }
    S.t = static_cast<float>(static_cast<double>(S.frame_time + S.elapsed) / kFlicksPerSecond);
    S.dt = dt;
    S.elapsed += sub;
    S.remaining -= num;
    S.frame_substeps += 1;
    S.substeps_total += 1;
    if (S.remaining == 0) {
        S.frame_time += P.time_per_step;
        S.elapsed = 0;
    }
    S.max_v2 = 0;
}

// Start of a frame-graph launch: no sub-step of it has run yet.
__global__ void k_frame_begin(Arena a, int nscenes) {
    int const s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nscenes) a.ss[s].call_substeps = 0;
}

// End of one sub-step inside a frame graph: counts it, and keeps the frame
// loop going while an active scene's frame has sub-steps left (the host
// loop of std_adaptive_time_step, emerald/sph2d_box/adaptive_time_step.h:74-103,
// as a while node).
__global__ void k_frame_check(Arena a, int nscenes, int method, cudaGraphConditionalHandle cond) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < nscenes; s += blockDim.x) {
        SceneState& S = a.ss[s];
        if (!S.active) continue;
        S.call_substeps += 1;
        if (S.remaining > 0) any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a.loop_iterations[4 + method] += 1ull;
        cudaGraphSetConditional(cond, any ? 1u : 0u);
    }
}

// Per-frame reset of the DFSPH kappas (dfsph_p.cpp:214-229), fixed-dt mode.
__global__ void k_zero_kappas(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    a.kdiv[c.i] = 0.0f;
    a.kdens[c.i] = 0.0f;
}

__device__ __forceinline__ int iteration_cap(SceneParams const& P, int kind) {
    return kind == 0 ? P.iisph_max_iter : (kind == 3 ? 6 : P.dfsph_max_iter);
}

// Rebuilds the solver-loop work list (Arena::loop_scene, loop_wt0,
// loop_n): the active scenes whose loop still runs and have particles, in
// scene order, with the exclusive prefix of their warp tiles (32 particles
// each). Run by every thread of one block after the scenes' done flags are
// final; a block-wide scan over the scenes, blockDim.x at a time.
__device__ void build_loop_list(Arena const& a, int nscenes) {
    __shared__ uint32_t base_wt, base_n;
    __shared__ uint32_t warp_wt[32], warp_n[32];
    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    int const nwarps = (blockDim.x + 31) >> 5;
    if (threadIdx.x == 0) {
        base_wt = 0u;
        base_n = 0u;
    }
    __syncthreads();
    for (int s0 = 0; s0 < nscenes; s0 += blockDim.x) {
        int const s = s0 + threadIdx.x;
        uint32_t wt = 0u;
        if (s < nscenes) {
            SceneState const& S = a.ss[s];
            if (S.active && !S.done) wt = (a.sp[s].fluid_count + 31u) / 32u;
        }
        uint32_t const on = wt ? 1u : 0u;
        // inclusive scans of (wt, on) within the warp, then across warps
        uint32_t iw = wt, in = on;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t const yw = __shfl_up_sync(0xffffffffu, iw, o);
            uint32_t const yn = __shfl_up_sync(0xffffffffu, in, o);
            if (lane >= o) {
                iw += yw;
                in += yn;
            }
        }
        if (lane == 31) {
            warp_wt[warp] = iw;
            warp_n[warp] = in;
        }
        __syncthreads();
        uint32_t pw = 0u, pn = 0u, tw = 0u, tn = 0u;
        for (int w = 0; w < nwarps; ++w) {
            if (w < warp) {
                pw += warp_wt[w];
                pn += warp_n[w];
            }
            tw += warp_wt[w];
            tn += warp_n[w];
        }
        if (on) {
            uint32_t const k = base_n + pn + in - 1u;
            a.loop_scene[k] = s;
            a.loop_wt0[k] = base_wt + pw + iw - wt;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            base_wt += tw;
            base_n += tn;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.loop_wt0[base_n] = base_wt;
        *a.loop_n = base_n;
    }
}

// Starts a solver loop; a scene whose cap is zero runs no iteration, as the
// reference's for-loop would. Inside a captured graph it also opens the
// loop's while node: a condition handle's default is applied when the graph
// that owns it is launched, and a loop nested in a frame graph's sub-step
// loop is reached once per sub-step of one launch, after the previous
// sub-step's exit test closed it. One block: in a batch it also builds the
// loop's first work list.
__global__ void k_iter_reset(Arena a, int nscenes, int kind, cudaGraphConditionalHandle cond,
                             int use_cond) {
    if (use_cond && threadIdx.x == 0) cudaGraphSetConditional(cond, 1u);
    for (int s = threadIdx.x; s < nscenes; s += blockDim.x) {
        SceneState& S = a.ss[s];
        S.iter = 0;
        S.done = (S.active && iteration_cap(a.sp[s], kind) > 0) ? 0 : 1;
        S.err_sum = 0ull;
        S.err_max = 0u;
        S.err_sum_d = 0.0;
    }
    __syncthreads();
    if (a.batch) build_loop_list(a, nscenes);
}

// Exit test after one solver iteration. kind 0: IISPH family
// (iisph.cpp:119-128), 1: DFSPH density (dfsph_p.cpp:113-133),
// 2: DFSPH divergence (:187-211), 3: PCISPH (pcisph.cpp:144-148).
// One block; *running is set when any scene still iterates and, inside a
// captured graph, the loop's while condition takes the same value.
// The exit test of one solver iteration for every scene (kind 0: IISPH
// family, iisph.cpp:119-128; 1: DFSPH density, dfsph_p.cpp:113-133; 2: DFSPH
// divergence, :187-211; 3: PCISPH, pcisph.cpp:144-148), run by one block.
// With `fresh`, the scenes' error accumulators were written by other blocks
// of the same kernel and are read through atomics (L2), not L1.
__device__ void exit_test(Arena const& a, int nscenes, int kind, int* running,
                          cudaGraphConditionalHandle cond, int use_cond, bool fresh) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < nscenes; s += blockDim.x) {
        SceneParams const& P = a.sp[s];
        SceneState& S = a.ss[s];
        if (!S.active || S.done) continue;
        unsigned long long const err_sum = fresh ? atomicAdd(&S.err_sum, 0ull) : S.err_sum;
        uint32_t const err_max = fresh ? atomicMax(&S.err_max, 0u) : S.err_max;
        double const err_sum_d = fresh ? atomicAdd(&S.err_sum_d, 0.0) : S.err_sum_d;
        double const n = static_cast<double>(1000ull * P.fluid_count);
        float const avg = P.fluid_count
                            ? static_cast<float>(static_cast<double>(err_sum) / n)
                            : 0.0f;
        // the exact mean of the errors, reported beside the reference's
        // metric (which drops each particle's error below 0.1%)
        double const exact = P.fluid_count ? err_sum_d / static_cast<double>(P.fluid_count) : 0.0;
        float const mx = __uint_as_float(err_max);
        bool conv = false;
        int const max_iter = iteration_cap(P, kind);
        if (kind == 0) {
            conv = S.iter > 1 && avg <= P.iisph_err_avg && mx <= P.iisph_err_max;
            S.stat_avg = avg;
            S.stat_max = mx;
        } else if (kind == 1) {
            if (S.iter > 1) {
                conv = avg <= P.dfsph_dens_avg && mx <= P.dfsph_dens_max;
                S.stat_avg = avg;
                S.stat_max = mx;
                S.stat_avg_exact = exact;
            }
        } else if (kind == 2) {
            if (S.iter > 0) {
                conv = avg <= P.dfsph_div_avg && mx <= P.dfsph_div_max;
                S.stat_div_avg = avg;
                S.stat_div_max = mx;
                S.stat_div_avg_exact = exact;
            }
        } else {
            if (S.iter > 1) {
                conv = (mx / P.rho0) <= 0.01f;
                S.stat_max = mx / P.rho0;
            }
        }
        S.iter += 1;
        S.err_sum = 0ull;
        S.err_max = 0u;
        S.err_sum_d = 0.0;
        if (conv || S.iter >= max_iter) {
            S.done = 1;
            if (kind == 2) {
                S.stat_div_iters = S.iter;
            } else {
                S.stat_iters = S.iter;
            }
        } else {
            any = 1;
        }
    }
    __syncthreads();
    if (a.batch) build_loop_list(a, nscenes);
    if (threadIdx.x == 0) {
        a.loop_iterations[kind] += 1ull;
        *running = any;
        if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
    }
}

// Exit test after one solver iteration, as its own one-block launch.
// *running is set when any scene still iterates and, inside a captured
// graph, the loop's while condition takes the same value.
__global__ void k_iter_check(Arena a, int nscenes, int kind, int* running,
                             cudaGraphConditionalHandle cond, int use_cond) {
    exit_test(a, nscenes, kind, running, cond, use_cond, false);
}

// The exit test run by the last block of an iteration's final
// persistent-warp kernel instead of its own launch: each block counts
// itself done; the one that completes the count runs exit_test and resets
// the counter for the next launch. `fence`: this kernel itself wrote the
// error accumulators the test reads (IISPH's beta pass), so the blocks'
// writes are fenced before they count themselves done.
__device__ __forceinline__ void fused_exit_test(Arena const& a, LoopCheck const& lc, bool fence) {
    if (!lc.counter) return;
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (fence) __threadfence();
        last = atomicAdd(lc.counter, 1u) == gridDim.x - 1 ? 1 : 0;
        if (last) __threadfence();
    }
    __syncthreads();
    if (last) {
        exit_test(a, lc.nscenes, lc.kind, lc.running, lc.cond, lc.use_cond, true);
        if (threadIdx.x == 0) *lc.counter = 0u;
    }
}

// --------------------------------------------------------- shared SPH sums

// Visits particle i's fluid list in list order, CH entries at a time: a
// chunk first loads its indices and kernel gradients, then every gathered
// neighbour value, then folds them into the sum in order. The loads of a
// chunk are independent, so they are in flight together; the sum is the
// same sequence of operations as a plain loop. The chunk of each kernel is
// a launch-time choice among 1, 4 and 8 (Tuning, set by the autotuner).
// These two are the chunks of callers that pass none (the IISPH final
// velocity update); the engine's DFSPH launches pass their Tuning's.
constexpr int kDivergenceChunk = 8;
constexpr int kPressureChunk = 4;

// Each warp of a gather kernel may first ask L2 for its fluid list rows
// (lane k: slot k's 128 index bytes and 256 gradient bytes), so that the
// sums' list loads find them there. Every lane of the warp calls it; lanes
// without a live particle pass count 0.
__device__ __forceinline__ void prefetch_fluid_lists(Arena const& a, int count) {
    int const lane = threadIdx.x & 31;
    int const slots = static_cast<int>(__reduce_max_sync(0xffffffffu, uint32_t(count)));
    if (lane < slots) {
        size_t const e = static_cast<size_t>(lane) * a.stride +
                         static_cast<size_t>(blockIdx.x) * kTile + (threadIdx.x & ~31u);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.nf_idx + e));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.nf_gw + e));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.nf_gw + e + 16));
    }
}

// Neighbour values the IISPH beta sum gathers.
struct IisphNeighbor {
    float rho, p;
    float2 sdp, dii;
};

template <int CH, class Gather, class Fold>
__device__ __forceinline__ void fold_fluid_list(Arena const& a, uint32_t i, int c, Gather gather,
                                                Fold fold) {
    size_t const stride = a.stride;
    using T = decltype(gather(0u));
    for (int k0 = 0; k0 < c; k0 += CH) {
        uint32_t jj[CH];
        float2 gw[CH];
        T val[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            if (k0 + u < c) {
                size_t const e = static_cast<size_t>(k0 + u) * stride + i;
                jj[u] = a.nf_idx[e];
                gw[u] = a.nf_gw[e];
            }
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            if (k0 + u < c) val[u] = gather(jj[u]);
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            if (k0 + u < c) fold(val[u], gw[u]);
        }
    }
}

// compute_densities (emerald/sph_common/density.cpp:10-73); with K each
// sum is Kahan-compensated.
template <bool K = false>
__device__ __forceinline__ float density_of(Arena const& a, SceneParams const& P, uint32_t i) {
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    float const fmass = rho0 * P.fluid_volume;
    SumF<K> d(P.fluid_volume * rho0 * P.w0);
    int const c = a.nf_cnt[i];
    #pragma unroll 4

    for (int k = 0; k < c; ++k) d.add(a.nf_w[k * stride + i] * fmass);
    float out = d.get();
    int const cs = a.ns_cnt[i];
    if (cs) {
        SumF<K> db;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            db.add(a.ns_w[e] * (rho0 * a.vols[a.ns_idx[e]]));
        }
        out += db.get();
    }
    return out;
}

// compute_divergences (emerald/sph_common/divergence.cpp:5-74).
// With K, the fluid and boundary terms go into one Kahan-compensated sum.
template <bool K = false, int CH = kDivergenceChunk>
__device__ __forceinline__ float divergence_of(Arena const& a, SceneParams const& P, uint32_t i) {
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    float const fmass = rho0 * P.fluid_volume;
    float2 const vi = a.v[i];
    int const c = a.nf_cnt[i];
    if (K) {
        KahanF acc{0.0f, 0.0f};
        for (int k = 0; k < c; ++k) {
            size_t const e = k * stride + i;
            kahan_add(acc, fmass * dot2(sub2(vi, a.v[a.nf_idx[e]]), a.nf_gw[e]));
        }
        int const cs = a.ns_cnt[i];
        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            uint32_t const j = a.ns_idx[e];
            kahan_add(acc, (rho0 * a.vols[j]) * dot2(sub2(vi, a.vs[j]), a.ns_gw[e]));
        }
        return acc.s;
    }
    float d = 0.0f;
    fold_fluid_list<CH>(
      a, i, c, [&](uint32_t j) { return a.v[j]; },
      [&](float2 vj, float2 g) { d += fmass * dot2(sub2(vi, vj), g); });
    int const cs = a.ns_cnt[i];
    if (cs) {
        float db = 0.0f;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            uint32_t const j = a.ns_idx[e];
            db += (rho0 * a.vols[j]) * dot2(sub2(vi, a.vs[j]), a.ns_gw[e]);
        }
        d += db;
    }
    return d;
}

// apply_pressures_in_place (emerald/sph_common/pressure.cpp:9-80) for one
// particle, with q = safe_divide(p, rho^2) precomputed per particle. With K,
// each sum is Kahan-compensated.
template <bool K = false, int CH = kPressureChunk>
__device__ __forceinline__ float2 apply_pressure_of(Arena const& a, SceneParams const& P, uint32_t i,
                                                    float2 v, float const* q, float dt) {
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    float const neg_fmass = -(rho0 * P.fluid_volume);
    float const qi = q[i];
    int const c = a.nf_cnt[i];
    if (K) {
        if (c) {
            KahanF2 acc{{0.0f, 0.0f}, {0.0f, 0.0f}};
            for (int k = 0; k < c; ++k) {
                size_t const e = k * stride + i;
                kahan_add(acc, scl2(neg_fmass * (qi + q[a.nf_idx[e]]), a.nf_gw[e]));
            }
            v = add2(v, scl2(dt, mk2(acc.x.s, acc.y.s)));
        }
        int const cs = a.ns_cnt[i];
        if (cs) {
            KahanF2 acc{{0.0f, 0.0f}, {0.0f, 0.0f}};
            for (int k = 0; k < cs; ++k) {
                size_t const e = k * stride + i;
                kahan_add(acc, scl2(-(rho0 * a.vols[a.ns_idx[e]]) * qi, a.ns_gw[e]));
            }
            v = add2(v, scl2(dt, mk2(acc.x.s, acc.y.s)));
        }
        return v;
    }
    if (c) {
        float2 acc = mk2(0.0f, 0.0f);
        fold_fluid_list<CH>(
          a, i, c, [&](uint32_t j) { return q[j]; },
          [&](float qj, float2 g) { acc = add2(acc, scl2(neg_fmass * (qi + qj), g)); });
        v = add2(v, scl2(dt, acc));
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        float2 acc = mk2(0.0f, 0.0f);
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            acc = add2(acc, scl2(-(rho0 * a.vols[a.ns_idx[e]]) * qi, a.ns_gw[e]));
        }
        v = add2(v, scl2(dt, acc));
    }
    return v;
}

// compute_pressure_accelerations (emerald/sph_common/pressure.cpp:83-178);
// with K each sum is Kahan-compensated.
template <bool K = false>
__device__ __forceinline__ float2 pressure_accel_of(Arena const& a, SceneParams const& P, uint32_t i,
                                                    float const* q) {
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    float const neg_fmass = -(rho0 * P.fluid_volume);
    float const qi = q[i];
    float2 out = mk2(0.0f, 0.0f);
    int const c = a.nf_cnt[i];
    if (c) {
        SumF2<K> acc;
        #pragma unroll 4

        for (int k = 0; k < c; ++k) {
            size_t const e = k * stride + i;
            acc.add(scl2(neg_fmass * (qi + q[a.nf_idx[e]]), a.nf_gw[e]));
        }
        out = acc.get();
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        SumF2<K> acc;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            acc.add(scl2(-(rho0 * a.vols[a.ns_idx[e]]) * qi, a.ns_gw[e]));
        }
        out = add2(out, acc.get());
    }
    return out;
}

// compute_all_external_forces (emerald/sph2d_box/forces.cpp:11-33) for one
// particle: the force starts at zero and takes the scene's terms in order,
// each with the reference function's own arithmetic; a scene driven by a
// host callback reads the callback's forces instead. v is the velocity at
// the point of the sub-step where the solver computes the forces.
__device__ __forceinline__ float2 external_force(Arena const& a, SceneParams const& P,
                                                 uint32_t i, float2 v) {
    if (P.force_array) return a.ext_f[i];
    float2 f = mk2(0.0f, 0.0f);
    for (int k = 0; k < P.force_count; ++k) {
        ForceTerm const t = P.force_terms[k];
        if (t.kind == kForceGravity) {
            // accumulate_gravity_forces (forces.cpp:63-71)
            f.y -= P.mass * t.a;
        } else if (t.kind == kForcePole) {
            // accumulate_constant_pole_attraction_forces (forces.cpp:85-101):
            // pull along the unit vector to the pole (Imath normalized(),
            // zero at the pole), plus the swirl (0, 0, magnitude / 8) x
            // (rN, 0) written out component by component.
            float2 const r = sub2(a.x[i], mk2(t.b, t.c));
            float const l = length2f(r);
            float2 const rn = (l == 0.0f) ? mk2(0.0f, 0.0f) : mk2(r.x / l, r.y / l);
            f = sub2(f, mk2(t.a * rn.x, t.a * rn.y));
            float const tz = 0.125f * t.a;
            float const zero = 0.0f;
            f = add2(f, mk2(zero * zero - tz * rn.y, tz * rn.x - zero * zero));
        } else if (t.kind == kForceDrag) {
            // accumulate_simple_drag_forces (forces.cpp:104-111)
            float const m = -t.a * t.b;
            f = add2(f, mk2(m * v.x, m * v.y));
        }
    }
    return f;
}

// integrate_velocities_in_place (dynamics.cpp:24-37) with the scene's
// external forces.
__device__ __forceinline__ float2 integrate_external(Arena const& a, SceneParams const& P,
                                                     uint32_t i, float2 v, float dt) {
    float2 const f = external_force(a, P, i, v);
    float const denom = P.rho0 * P.fluid_volume;
    float2 const numer = scl2(dt, f);
    if (safe_v(numer, denom)) v = add2(v, div2(numer, denom));
    return v;
}

// ------------------------------------------------------------------- DFSPH

// compute_densities + dfsph_p_compute_shared_coeffs (dfsph_p_ops.cpp:19-72),
// the per-frame kappa reset, and the p/rho^2 caches of both warm starts.
// With K, the density and the two alpha sums are Kahan-compensated.
template <bool K>
__device__ __forceinline__ void dfsph_density_alpha(Arena const& a, Ctx const& c) {
    SceneParams const& P = a.sp[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    float const fvol = P.fluid_volume;
    float d = fvol * rho0 * P.w0;
    float2 sum = mk2(0.0f, 0.0f);
    float sdot = 0.0f;
    KahanF kd{d, 0.0f}, ksdot{0.0f, 0.0f};
    KahanF2 ksum{{0.0f, 0.0f}, {0.0f, 0.0f}};
    int const cf = a.nf_cnt[i];
    float const fmass = rho0 * fvol;
    float const fmass_a = fvol * rho0;
    #pragma unroll 4

    for (int k = 0; k < cf; ++k) {
        size_t const e = k * stride + i;
        float2 const m = scl2(fmass_a, a.nf_gw[e]);
        if (K) {
            kahan_add(kd, a.nf_w[e] * fmass);
            kahan_add(ksum, m);
            kahan_add(ksdot, dot2(m, m));
        } else {
            d += a.nf_w[e] * fmass;
            sum = add2(sum, m);
            sdot += dot2(m, m);
        }
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        float db = 0.0f;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            float const vs = a.vols[a.ns_idx[e]];
            if (K) {
                kahan_add(kd, a.ns_w[e] * (rho0 * vs));
                kahan_add(ksum, scl2(vs * rho0, a.ns_gw[e]));
            } else {
                db += a.ns_w[e] * (rho0 * vs);
                sum = add2(sum, scl2(vs * rho0, a.ns_gw[e]));
            }
        }
        if (!K) d += db;
    }
    if (K) {
        d = kd.s;
        sum = mk2(ksum.x.s, ksum.y.s);
        sdot = ksdot.s;
    }
    a.rho[i] = d;
    float alpha = 0.0f;
    if (cf + cs) {
        float const numer = sqrf(d);
        float const denom = dot2(sum, sum) + sdot;
        alpha = safe_f(numer, denom) ? numer / denom : 0.0f;
    }
    a.alpha[i] = alpha;
    float kd0 = a.kdiv[i];
    float kn = a.kdens[i];
    if (a.ss[c.s].new_frame) {
        kd0 = 0.0f;
        kn = 0.0f;
        a.kdiv[i] = kd0;
        a.kdens[i] = kn;
    }
    a.qdiv[i] = p_over_rho2(kd0, d);
    a.qdens[i] = p_over_rho2(kn, d);
}

// MODE 0 launches carry only the reference arithmetic; MODE 1 launches
// (when some resident scene is in compensated mode) choose per scene.
template <int MODE>
__global__ void k_dfsph_density_alpha(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    if (MODE && a.sp[c.s].precision) {
        dfsph_density_alpha<true>(a, c);
    } else {
        dfsph_density_alpha<false>(a, c);
    }
}

// apply_pressures_in_place over the cached q; with `external`, the velocity
// first takes the external-force step (the DFSPH density warm start follows
// integrate_velocities_in_place, dfsph_p.cpp:349-365).
template <int MODE, int CH, int PF>
__global__ void k_apply_pressures(Arena a, int which_q, int external, int skip_done) {
    Ctx c;
    if (!enter(a, skip_done != 0, c)) return;
    if (PF) prefetch_fluid_lists(a, c.live ? int(a.nf_cnt[c.i]) : 0);
    if (!c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    float2 v = a.v[c.i];
    if (external) v = integrate_external(a, P, c.i, v, dt);
    float const* q = which_q ? a.qdens : a.qdiv;
    a.v[c.i] = (MODE && P.precision) ? apply_pressure_of<true, CH>(a, P, c.i, v, q, dt)
                                     : apply_pressure_of<false, CH>(a, P, c.i, v, q, dt);
}

// compute_divergences + dfsph_p_compute_divergence_pseudo_pressures
// (dfsph_p_ops.cpp:100-126) + the divergence error of dfsph_p.cpp:187-200.
template <int MODE, int CH, int PF>
__global__ void k_dfsph_divergence(Arena a) {
    Ctx c;
    if (!enter(a, true, c)) return;
    SceneParams const& P = a.sp[c.s];
    SceneState* S = &a.ss[c.s];
    float const dt = S->dt;
    float err = 0.0f;
    if (PF) prefetch_fluid_lists(a, c.live ? int(a.nf_cnt[c.i]) : 0);
    if (c.live) {
        uint32_t const i = c.i;
        float const d = (MODE && P.precision) ? divergence_of<true, CH>(a, P, i)
                                              : divergence_of<false, CH>(a, P, i);
        a.rho_star[i] = d;
        float kappa = 0.0f;
        if (!(d <= 0.0f)) {
            float const numer = d * a.alpha[i];
            kappa = safe_f(numer, dt) ? numer / dt : 0.0f;
        }
        a.kdiv[i] = kappa;
        a.qdiv[i] = p_over_rho2(kappa, a.rho[i]);
        err = d <= 0.0f ? 0.0f : (dt * d / P.rho0);
    }
    accumulate_error(S, static_cast<unsigned long long>(static_cast<long long>(err * 1000.0f)),
                     err, c.live, true);
}

// predict_density_stars (density.cpp:75-109) +
// dfsph_p_compute_density_pseudo_pressures (dfsph_p_ops.cpp:74-98) + the
// density error of dfsph_p.cpp:134-148.
template <int MODE, int CH, int PF>
__global__ void k_dfsph_density(Arena a) {
    Ctx c;
    if (!enter(a, true, c)) return;
    SceneParams const& P = a.sp[c.s];
    SceneState* S = &a.ss[c.s];
    float const dt = S->dt;
    float const rho0 = P.rho0;
    float err = 0.0f;
    if (PF) prefetch_fluid_lists(a, c.live ? int(a.nf_cnt[c.i]) : 0);
    if (c.live) {
        uint32_t const i = c.i;
        float const rho = a.rho[i];
        float const div = (MODE && P.precision) ? divergence_of<true, CH>(a, P, i)
                                                : divergence_of<false, CH>(a, P, i);
        float const star = max_0x(rho + (dt * div));
        a.rho_star[i] = star;
        float const delta = star - rho0;
        float kappa = 0.0f;
        if (!(delta <= 0.0f)) {
            float const numer = delta * a.alpha[i];
            float const dd = sqrf(dt);
            kappa = safe_f(numer, dd) ? numer / dd : 0.0f;
        }
        a.kdens[i] = kappa;
        a.qdens[i] = p_over_rho2(kappa, rho);
        err = delta <= 0.0f ? 0.0f : (delta / rho0);
    }
    accumulate_error(S, static_cast<unsigned long long>(static_cast<long long>(err * 1000.0f)),
                     err, c.live, true);
}

// ------------------------------------------ persistent-warp gather kernels
//
// The DFSPH sums above, launched as one grid of resident blocks: warp w of
// the G warps folds the 32-particle warp tiles w, w + G, w + 2G, ... (a warp
// tile lies inside one 128-particle tile, so in one scene). While it folds
// tile t, the list rows, count bytes and per-particle inputs of tile t + G
// are already on their way into L2 (asked for with the counts it loaded one
// tile earlier) and the counts of tile t + 2G are loading, so the lists
// stream from HBM behind the folds instead of in front of them. Each
// particle's sums are the same operations in the same order as in the
// block-per-tile kernels, so the bits are theirs. Error sums gather per warp
// and go to the scene's accumulators when the warp's next tile belongs to
// another scene, and at the end.

__device__ __forceinline__ void prefetch_l2(void const* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// L2 requests for a warp tile's fluid list rows (rows below the warp's
// largest count; kernel values or indices, and the gradients) and for up to
// five 128-byte lines of per-particle data, lane k asking for line k.
template <bool W>
__device__ __forceinline__ void prefetch_warp_tile(Arena const& a, uint32_t base, int count,
                                                   void const* l0, void const* l1, void const* l2,
                                                   void const* l3 = nullptr,
                                                   void const* l4 = nullptr) {
    int const lane = threadIdx.x & 31;
    int const rows = static_cast<int>(__reduce_max_sync(0xffffffffu, uint32_t(count)));
    if (lane < rows) {
        size_t const e = static_cast<size_t>(lane) * a.stride + base;
        prefetch_l2(W ? static_cast<void const*>(a.nf_w + e) : static_cast<void const*>(a.nf_idx + e));
        prefetch_l2(a.nf_gw + e);
        prefetch_l2(a.nf_gw + e + 16);
    }
    void const* const p = lane == 0 ? l0
                        : lane == 1 ? l1
                        : lane == 2 ? l2
                        : lane == 3 ? l3
                        : lane == 4 ? l4
                                    : nullptr;
    if (p) prefetch_l2(p);
}

struct WarpErr {
    int32_t scene;
    unsigned long long sum;
    uint32_t max;
    double exact;
};

__device__ __forceinline__ void flush_err(Arena const& a, WarpErr& e) {
    if (e.scene >= 0) {
        unsigned long long v = e.sum;
        uint32_t m = e.max;
        double d = e.exact;
        for (int o = 16; o; o >>= 1) {
            v += __shfl_xor_sync(0xffffffffu, v, o);
            m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
            d += __shfl_xor_sync(0xffffffffu, d, o);
        }
        if ((threadIdx.x & 31) == 0) {
            SceneState* S = &a.ss[e.scene];
            if (v) atomicAdd(&S->err_sum, v);
            if (m) atomicMax(&S->err_max, m);
            if (d != 0.0) atomicAdd(&S->err_sum_d, d);
        }
    }
    e = WarpErr{-1, 0ull, 0u, 0.0};
}

// The warps' remaining sums, combined per block in shared memory and sent
// to the scene's accumulators with one set of atomics per block (a warp
// whose scene differs from the block's first flushing warp sends its own).
// Every thread of the block calls it.
__device__ __forceinline__ void flush_err_block(Arena const& a, WarpErr& e) {
    __shared__ unsigned long long b_sum;
    __shared__ uint32_t b_max;
    __shared__ double b_exact;
    __shared__ int b_scene;
    if (threadIdx.x == 0) {
        b_sum = 0ull;
        b_max = 0u;
        b_exact = 0.0;
        b_scene = -1;
    }
    __syncthreads();
    unsigned long long v = e.sum;
    uint32_t m = e.max;
    double d = e.exact;
    for (int o = 16; o; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        d += __shfl_xor_sync(0xffffffffu, d, o);
    }
    if ((threadIdx.x & 31) == 0 && e.scene >= 0) {
        int const prev = atomicCAS(&b_scene, -1, e.scene);
        if (prev == -1 || prev == e.scene) {
            atomicAdd(&b_sum, v);
            atomicMax(&b_max, m);
            atomicAdd(&b_exact, d);
        } else {
            SceneState* S = &a.ss[e.scene];
            if (v) atomicAdd(&S->err_sum, v);
            if (m) atomicMax(&S->err_max, m);
            if (d != 0.0) atomicAdd(&S->err_sum_d, d);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && b_scene >= 0) {
        SceneState* S = &a.ss[b_scene];
        if (b_sum) atomicAdd(&S->err_sum, b_sum);
        if (b_max) atomicMax(&S->err_max, b_max);
        if (b_exact != 0.0) atomicAdd(&S->err_sum_d, b_exact);
    }
    e = WarpErr{-1, 0ull, 0u, 0.0};
}

// accumulate_error's contribution of one particle (its integer v and
// error m, the exact sum too when `exact`), kept in the warp.
__device__ __forceinline__ void add_err(Arena const& a, WarpErr& e, int32_t scene,
                                        unsigned long long v, float m, bool live, bool exact) {
    if (scene != e.scene) {
        flush_err(a, e);
        e.scene = scene;
    }
    if (live) {
        e.sum += v;
        if (m == m && m > 0.0f) {
            e.max = max(e.max, __float_as_uint(m));
            if (exact) e.exact += static_cast<double>(m);
        }
    }
}

// The scene of warp tile t when it takes part in this launch (active), else
// -1.
__device__ __forceinline__ int32_t live_tile_scene(Arena const& a, uint32_t t, bool skip_done) {
    int32_t const s = a.tile_scene[t / (kTile / 32)];
    if (s < 0) return -1;
    SceneState const& S = a.ss[s];
    return (S.active && !(skip_done && S.done)) ? s : -1;
}

// Warp tile w of the solver-loop work list (w < the list's total): its scene
// and its warp tile in the arena, by bisection of the prefix loop_wt0.
__device__ __forceinline__ void loop_list_tile(Arena const& a, uint32_t n, uint32_t w,
                                               int32_t& s, uint32_t& t) {
    uint32_t lo = 0u, hi = n;  // loop_wt0[lo] <= w < loop_wt0[hi]
    while (hi - lo > 1u) {
        uint32_t const mid = (lo + hi) >> 1;
        if (a.loop_wt0[mid] <= w) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    s = a.loop_scene[lo];
    t = a.sp[s].fluid_begin / 32u + (w - a.loop_wt0[lo]);
}

// Walks this warp's tiles: prefetch(base, count) asks L2 for a tile's data,
// body(scene, i, live) folds particle i of the tile. LIST (the solver-loop
// kernels of a batch) walks the warp tiles of the loop's work list only, so
// the scenes that have converged cost nothing; otherwise the walk covers
// every tile and skips those of inactive scenes (and, with skip_done, of
// scenes whose loop has ended). The list walk holds more registers, so
// single scenes keep the plain walk. Every lane of the warp runs every
// iteration (tile choices are warp-uniform), and every thread of the block
// returns from it (no early exit, so the kernels can meet at a block
// barrier afterwards).
template <bool LIST, class Prefetch, class Body>
__device__ __forceinline__ void walk_warp_tiles(Arena const& a, uint32_t wtiles, bool skip_done,
                                                Prefetch prefetch, Body body) {
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const G = (gridDim.x * blockDim.x) >> 5;
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if constexpr (LIST) {
        // one tile ahead (fewer registers than the plain walk's two)
        uint32_t const n = *a.loop_n;
        uint32_t const total = a.loop_wt0[n];
        int32_t s_cur = -1;
        uint32_t t_cur = 0u;
        if (w < total) {
            loop_list_tile(a, n, w, s_cur, t_cur);
            prefetch(t_cur * 32u, int(a.nf_cnt[t_cur * 32u + lane]));
        }
        for (; w < total; w += G) {
            int32_t s_next = -1;
            uint32_t t_next = 0u;
            if (w + G < total) {
                loop_list_tile(a, n, w + G, s_next, t_next);
                prefetch(t_next * 32u, int(a.nf_cnt[t_next * 32u + lane]));
            }
            SceneParams const& P = a.sp[s_cur];
            uint32_t const i = t_cur * 32u + lane;
            body(s_cur, i, (i - P.fluid_begin) < P.fluid_count);
            s_cur = s_next;
            t_cur = t_next;
        }
    } else {
        int32_t s_cur = w < wtiles ? live_tile_scene(a, w, skip_done) : -1;
        int32_t s_next = w + G < wtiles ? live_tile_scene(a, w + G, skip_done) : -1;
        int cnt_next = s_next >= 0 ? int(a.nf_cnt[(w + G) * 32u + lane]) : 0;
        if (s_cur >= 0) prefetch(w * 32u, int(a.nf_cnt[w * 32u + lane]));
        for (; w < wtiles; w += G) {
            uint32_t const wn = w + G;
            int32_t s_after = -1;
            int cnt_after = 0;
            if (wn < wtiles) {
                if (s_next >= 0) prefetch(wn * 32u, cnt_next);
                if (wn + G < wtiles) {
                    s_after = live_tile_scene(a, wn + G, skip_done);
                    if (s_after >= 0) cnt_after = int(a.nf_cnt[(wn + G) * 32u + lane]);
                }
            }
            if (s_cur >= 0) {
                SceneParams const& P = a.sp[s_cur];
                uint32_t const i = w * 32u + lane;
                body(s_cur, i, (i - P.fluid_begin) < P.fluid_count);
            }
            s_cur = s_next;
            s_next = s_after;
            cnt_next = cnt_after;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_dfsph_density_alpha_pw(Arena a, uint32_t wtiles) {
    walk_warp_tiles<false>(
      a, wtiles, false,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<true>(a, base, count, a.ns_cnt + base, a.kdiv + base, a.kdens + base);
      },
      [&](int32_t s, uint32_t i, bool live) {
          if (!live) return;
          Ctx const c{s, i, true};
          if (MODE && a.sp[s].precision) {
              dfsph_density_alpha<true>(a, c);
          } else {
              dfsph_density_alpha<false>(a, c);
          }
      });
}

template <int MODE, int CH, bool LIST>
__global__ void __launch_bounds__(256) k_apply_pressures_pw(Arena a, uint32_t wtiles, int which_q,
                                                            int external, int skip_done,
                                                            LoopCheck lc) {
    float const* q = which_q ? a.qdens : a.qdiv;
    walk_warp_tiles<LIST>(
      a, wtiles, skip_done != 0,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<false>(a, base, count, a.ns_cnt + base, a.v + base, a.v + base + 16,
                                    q + base);
      },
      [&](int32_t s, uint32_t i, bool live) {
          if (!live) return;
          SceneParams const& P = a.sp[s];
          float const dt = a.ss[s].dt;
          float2 v = a.v[i];
          if (external) v = integrate_external(a, P, i, v, dt);
          a.v[i] = (MODE && P.precision) ? apply_pressure_of<true, CH>(a, P, i, v, q, dt)
                                         : apply_pressure_of<false, CH>(a, P, i, v, q, dt);
      });
    fused_exit_test(a, lc, false);
}

template <int MODE, int CH, bool LIST>
__global__ void __launch_bounds__(256) k_dfsph_divergence_pw(Arena a, uint32_t wtiles) {
    WarpErr e{-1, 0ull, 0u, 0.0};
    walk_warp_tiles<LIST>(
      a, wtiles, true,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<false>(a, base, count, a.ns_cnt + base, a.v + base, a.v + base + 16,
                                    a.alpha + base, a.rho + base);
      },
      [&](int32_t s, uint32_t i, bool live) {
          SceneParams const& P = a.sp[s];
          float const dt = a.ss[s].dt;
          float err = 0.0f;
          if (live) {
              float const d = (MODE && P.precision) ? divergence_of<true, CH>(a, P, i)
                                                    : divergence_of<false, CH>(a, P, i);
              a.rho_star[i] = d;
              float kappa = 0.0f;
              if (!(d <= 0.0f)) {
                  float const numer = d * a.alpha[i];
                  kappa = safe_f(numer, dt) ? numer / dt : 0.0f;
              }
              a.kdiv[i] = kappa;
              a.qdiv[i] = p_over_rho2(kappa, a.rho[i]);
              err = d <= 0.0f ? 0.0f : (dt * d / P.rho0);
          }
          add_err(a, e, s,
                  static_cast<unsigned long long>(static_cast<long long>(err * 1000.0f)), err,
                  live, true);
      });
    flush_err_block(a, e);
}

template <int MODE, int CH, bool LIST>
__global__ void __launch_bounds__(256, LIST ? 3 : 1) k_dfsph_density_pw(Arena a, uint32_t wtiles) {
    WarpErr e{-1, 0ull, 0u, 0.0};
    walk_warp_tiles<LIST>(
      a, wtiles, true,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<false>(a, base, count, a.ns_cnt + base, a.v + base, a.v + base + 16,
                                    a.alpha + base, a.rho + base);
      },
      [&](int32_t s, uint32_t i, bool live) {
          SceneParams const& P = a.sp[s];
          float const dt = a.ss[s].dt;
          float const rho0 = P.rho0;
          float err = 0.0f;
          if (live) {
              float const rho = a.rho[i];
              float const div = (MODE && P.precision) ? divergence_of<true, CH>(a, P, i)
                                                      : divergence_of<false, CH>(a, P, i);
              float const star = max_0x(rho + (dt * div));
              a.rho_star[i] = star;
              float const delta = star - rho0;
              float kappa = 0.0f;
              if (!(delta <= 0.0f)) {
                  float const numer = delta * a.alpha[i];
                  float const dd = sqrf(dt);
                  kappa = safe_f(numer, dd) ? numer / dd : 0.0f;
              }
              a.kdens[i] = kappa;
              a.qdens[i] = p_over_rho2(kappa, rho);
              err = delta <= 0.0f ? 0.0f : (delta / rho0);
          }
          add_err(a, e, s,
                  static_cast<unsigned long long>(static_cast<long long>(err * 1000.0f)), err,
                  live, true);
      });
    flush_err_block(a, e);
}

// integrate_positions_in_place (dynamics.cpp:46-51). Compensated mode
// accumulates the positions in double and stores their float rounding.
// x_i += dt * v (+ shift): the reference's FP32 update, or for a
// compensated scene the FP64 accumulator (the positions the neighbour search
// takes its vectors from) rounded once into x_i. Every method's position
// update goes through here, so a compensated scene's FP64 positions stay
// current whichever method advances it.
__device__ __forceinline__ void advance_position(Arena const& a, SceneParams const& P,
                                                 uint32_t i, float dt, float2 v,
                                                 float2 shift = {0.0f, 0.0f}, bool shifted = false) {
    if (P.precision) {
        double2 x = a.x64[i];
        x.x += static_cast<double>(dt) * static_cast<double>(v.x);
        x.y += static_cast<double>(dt) * static_cast<double>(v.y);
        if (shifted) {
            x.x += static_cast<double>(shift.x);
            x.y += static_cast<double>(shift.y);
        }
        a.x64[i] = x;
        a.x[i] = mk2(static_cast<float>(x.x), static_cast<float>(x.y));
        return;
    }
    float2 const x = add2(a.x[i], scl2(dt, v));
    a.x[i] = shifted ? add2(x, shift) : x;
}

template <int MODE>
__global__ void k_integrate_positions(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    float const dt = a.ss[c.s].dt;
    if (MODE && a.sp[c.s].precision) {
        advance_position(a, a.sp[c.s], c.i, dt, a.v[c.i]);
        return;
    }
    a.x[c.i] = add2(a.x[c.i], scl2(dt, a.v[c.i]));
}

// -------------------------------------------------------------------- IISPH

// compute_densities, integrate_velocities_in_place and iisph_compute_diis
// (iisph_ops.cpp:20-90), plus the zero initial pressures (iisph.cpp:76).
// MODE 1 launches (some resident scene in compensated mode) Kahan-compensate
// the sums of compensated scenes, here and in the kernels below.
template <bool K>
__device__ __forceinline__ void iisph_density_dii(Arena const& a, Ctx const& c) {
    SceneParams const& P = a.sp[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const dt = a.ss[c.s].dt;
    float const rho0 = P.rho0;
    float const d = density_of<K>(a, P, i);
    a.rho[i] = d;
    a.v[i] = integrate_external(a, P, i, a.v[i], dt);
    float const neg_dt2 = -sqrf(dt);
    float const denom = sqrf(d);
    float2 dii = mk2(0.0f, 0.0f);
    int const cf = a.nf_cnt[i];
    if (cf) {
        float const fmass = rho0 * P.fluid_volume;
        SumF2<K> g;
        #pragma unroll 4

        for (int k = 0; k < cf; ++k) g.add(scl2(fmass, a.nf_gw[k * stride + i]));
        float2 const numer = scl2(neg_dt2, g.get());
        dii = safe_v(numer, denom) ? div2(numer, denom) : mk2(0.0f, 0.0f);
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        SumF2<K> g;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            g.add(scl2(rho0 * a.vols[a.ns_idx[e]], a.ns_gw[e]));
        }
        float2 const numer = scl2(neg_dt2, g.get());
        dii = add2(dii, safe_v(numer, denom) ? div2(numer, denom) : mk2(0.0f, 0.0f));
    }
    a.dii[i] = dii;
    a.pbuf0[i] = 0.0f;
}

template <int MODE>
__global__ void k_iisph_density_dii(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    if (MODE && a.sp[c.s].precision) {
        iisph_density_dii<true>(a, c);
    } else {
        iisph_density_dii<false>(a, c);
    }
}

// iisph_compute_aiis_and_density_stars (iisph_ops.cpp:92-200).
template <bool K>
__device__ __forceinline__ void iisph_aii(Arena const& a, Ctx const& c) {
    SceneParams const& P = a.sp[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const dt = a.ss[c.s].dt;
    float const rho0 = P.rho0;
    float2 const dii = a.dii[i];
    float2 const vi = a.v[i];
    float const neg_dt2 = -sqrf(dt);
    float aii = 0.0f;
    float star = a.rho[i];
    int const cf = a.nf_cnt[i];
    if (cf) {
        float const mass = P.fluid_volume * rho0;
        SumF<K> af, dd;
        #pragma unroll 4

        for (int k = 0; k < cf; ++k) {
            size_t const e = k * stride + i;
            uint32_t const j = a.nf_idx[e];
            float2 const gw = a.nf_gw[e];
            float2 const numer = scl2(neg_dt2 * mass, gw);
            float const denom = sqrf(a.rho[j]);
            if (safe_v(numer, denom)) {
                float2 const dji = neg2(div2(numer, denom));
                af.add(mass * dot2(sub2(dii, dji), gw));
            }
            dd.add(dt * mass * dot2(sub2(vi, a.v[j]), gw));
        }
        aii = af.get();
        star = a.rho[i] + dd.get();
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        SumF<K> ab, dd;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            size_t const e = k * stride + i;
            uint32_t const j = a.ns_idx[e];
            float2 const gw = a.ns_gw[e];
            float const mass = a.vols[j] * rho0;
            ab.add(mass * dot2(dii, gw));
            dd.add(dt * mass * dot2(sub2(vi, a.vs[j]), gw));
        }
        aii += ab.get();
        star += dd.get();
    }
    a.aii[i] = aii;
    a.rho_star[i] = star;
}

template <int MODE>
__global__ void k_iisph_aii(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    if (MODE && a.sp[c.s].precision) {
        iisph_aii<true>(a, c);
    } else {
        iisph_aii<false>(a, c);
    }
}

// iisph_compute_sum_dij_pjs (iisph_ops.cpp:202-235).
template <bool K, int CH>
__device__ __forceinline__ void iisph_sum_dij(Arena const& a, Ctx const& c) {
    SceneParams const& P = a.sp[c.s];
    SceneState const& S = a.ss[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const dt = S.dt;
    float const* p = pressures_cur(a, S);
    float const mass = P.fluid_volume * P.rho0;
    float const neg_dt2 = -sqrf(dt);
    SumF2<K> sum;
    int const cf = a.nf_cnt[i];
    (void)stride;
    fold_fluid_list<CH>(
      a, i, cf, [&](uint32_t j) { return mk2(p[j], a.rho[j]); },
      [&](float2 prho, float2 g) {
          float2 const numer = scl2(neg_dt2 * mass * prho.x, g);
          float const denom = sqrf(prho.y);
          if (safe_v(numer, denom)) sum.add(div2(numer, denom));
      });
    a.sdp[i] = sum.get();
}

template <int MODE, int CH, int PF>
__global__ void k_iisph_sum_dij(Arena a) {
    Ctx c;
    if (!enter(a, true, c)) return;
    if (PF) prefetch_fluid_lists(a, c.live ? int(a.nf_cnt[c.i]) : 0);
    if (!c.live) return;
    if (MODE && a.sp[c.s].precision) {
        iisph_sum_dij<true, CH>(a, c);
    } else {
        iisph_sum_dij<false, CH>(a, c);
    }
}

// iisph_compute_betas (iisph_ops.cpp:237-330) followed by
// iisph_compute_new_pressures for the same particle (iisph_ops.cpp:332-425).
// Returns whether the particle's error counts (a_ii != 0).
template <bool K, int CH>
__device__ __forceinline__ bool iisph_beta_pressure(Arena const& a, Ctx const& c, SceneState* S,
                                                    float& err) {
    SceneParams const& P = a.sp[c.s];
    bool counted = false;
    {
        uint32_t const i = c.i;
        size_t const stride = a.stride;
        float const dt = S->dt;
        float const rho0 = P.rho0;
        float const* p = pressures_cur(a, *S);
        float* pn = pressures_next(a, *S);
        float const pi = p[i];
        float2 const si = a.sdp[i];
        float const neg_dt2 = -sqrf(dt);
        float beta = 0.0f;
        int const cf = a.nf_cnt[i];
        if (cf) {
            float const mass = rho0 * P.fluid_volume;
            SumF<K> bf;
            fold_fluid_list<CH>(
              a, i, cf,
              [&](uint32_t j) { return IisphNeighbor{a.rho[j], p[j], a.sdp[j], a.dii[j]}; },
              [&](IisphNeighbor const& nb, float2 gw) {
                  float2 const numer = scl2(neg_dt2 * mass, gw);
                  float const denom = sqrf(nb.rho);
                  float2 const dij = safe_v(numer, denom) ? div2(numer, denom) : mk2(0.0f, 0.0f);
                  float2 const dji = neg2(dij);
                  float2 const skni = sub2(nb.sdp, scl2(pi, dji));
                  float2 const t = sub2(sub2(si, scl2(nb.p, nb.dii)), skni);
                  bf.add(mass * dot2(t, gw));
              });
            beta = bf.get();
        }
        int const cs = a.ns_cnt[i];
        if (cs) {
            SumF<K> bb;
            #pragma unroll 4

            for (int k = 0; k < cs; ++k) {
                size_t const e = k * stride + i;
                bb.add((rho0 * a.vols[a.ns_idx[e]]) * dot2(si, a.ns_gw[e]));
            }
            beta += bb.get();
        }
        float const alpha = a.aii[i];
        float out = pi;
        if (alpha != 0.0f) {
            float const numer = rho0 - a.rho_star[i] - beta;
            if (safe_f(numer, alpha)) {
                err = max_0x(-(numer - (alpha * pi)) / rho0);
                counted = true;
                out = max_0x(mix1(pi, numer / alpha, P.iisph_omega));
            } else {
                atomicOr(&S->error, kErrNonFinite);
            }
        }
        pn[i] = out;
    }
    return counted;
}

template <int MODE, int CH, int PF>
__global__ void k_iisph_beta_pressure(Arena a) {
    Ctx c;
    if (!enter(a, true, c)) return;
    SceneState* S = &a.ss[c.s];
    float err = 0.0f;
    bool counted = false;
    if (PF) prefetch_fluid_lists(a, c.live ? int(a.nf_cnt[c.i]) : 0);
    if (c.live) {
        counted = (MODE && a.sp[c.s].precision) ? iisph_beta_pressure<true, CH>(a, c, S, err)
                                                : iisph_beta_pressure<false, CH>(a, c, S, err);
    }
    accumulate_error(S, counted ? static_cast<unsigned long long>(err * 1000.0f) : 0ull, err,
                     c.live && counted);
}

// The two IISPH gather kernels as persistent warps (see the DFSPH ones
// above): the batched workload's per-iteration sums.
template <int MODE, int CH, bool LIST>
__global__ void __launch_bounds__(256) k_iisph_sum_dij_pw(Arena a, uint32_t wtiles) {
    walk_warp_tiles<LIST>(
      a, wtiles, true,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<false>(a, base, count, nullptr, nullptr, nullptr);
      },
      [&](int32_t s, uint32_t i, bool live) {
          if (!live) return;
          Ctx const c{s, i, true};
          if (MODE && a.sp[s].precision) {
              iisph_sum_dij<true, CH>(a, c);
          } else {
              iisph_sum_dij<false, CH>(a, c);
          }
      });
}

template <int MODE, int CH, bool LIST>
__global__ void __launch_bounds__(256, LIST ? 3 : 1) k_iisph_beta_pressure_pw(Arena a, uint32_t wtiles,
                                                                LoopCheck lc) {
    WarpErr e{-1, 0ull, 0u, 0.0};
    walk_warp_tiles<LIST>(
      a, wtiles, true,
      [&](uint32_t base, int count) {
          prefetch_warp_tile<false>(a, base, count, a.ns_cnt + base, a.sdp + base,
                                    a.sdp + base + 16, a.aii + base, a.rho_star + base);
      },
      [&](int32_t s, uint32_t i, bool live) {
          SceneState* S = &a.ss[s];
          float err = 0.0f;
          bool counted = false;
          if (live) {
              Ctx const c{s, i, true};
              counted = (MODE && a.sp[s].precision) ? iisph_beta_pressure<true, CH>(a, c, S, err)
                                                    : iisph_beta_pressure<false, CH>(a, c, S, err);
          }
          add_err(a, e, s, counted ? static_cast<unsigned long long>(err * 1000.0f) : 0ull, err,
                  live && counted, false);
      });
    flush_err_block(a, e);
    fused_exit_test(a, lc, true);
}

// q = safe_divide(p, rho^2) of the final pressures, for apply_pressures.
__global__ void k_make_q(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneState const& S = a.ss[c.s];
    a.qdens[c.i] = p_over_rho2(pressures_cur(a, S)[c.i], a.rho[c.i]);
}

// apply_pressures_in_place then integrate_positions_in_place
// (iisph.cpp:138-150).
template <int MODE>
__global__ void k_apply_integrate(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    float2 const v = (MODE && P.precision) ? apply_pressure_of<true>(a, P, c.i, a.v[c.i], a.qdens, dt)
                                           : apply_pressure_of<false>(a, P, c.i, a.v[c.i], a.qdens, dt);
    a.v[c.i] = v;
    advance_position(a, P, c.i, dt, v);
}

// ------------------------------------------------- IISPH_AP / PSEUDO_AP

// compute_densities, integrate_velocities_in_place, zero pressures.
template <int MODE>
__global__ void k_ap_density(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    a.rho[c.i] = (MODE && P.precision) ? density_of<true>(a, P, c.i) : density_of<false>(a, P, c.i);
    a.v[c.i] = integrate_external(a, P, c.i, a.v[c.i], dt);
    a.pbuf0[c.i] = 0.0f;
    a.qdens[c.i] = 0.0f;
}

// iisph_ap_density_stars_and_diagonals (iisph_ap_ops.cpp:19-103) and the
// pseudo variant (iisph_pseudo_ap_ops.cpp:19-117).
template <bool K>
__device__ __forceinline__ void ap_diag(Arena const& a, Ctx const& c, int pseudo) {
    SceneParams const& P = a.sp[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const dt = a.ss[c.s].dt;
    float const rho0 = P.rho0;
    int const cf = a.nf_cnt[i];
    int const cs = a.ns_cnt[i];
    float const rho = a.rho[i];
    if (!(cf + cs)) {
        a.rho_star[i] = rho;
        a.aii[i] = 0.0f;
        return;
    }
    float const self_mass = P.fluid_volume * rho0;
    float2 const vi = a.v[i];
    SumF2<K> sum_acc;
    SumF<K> sdot_acc, div_acc;
    float const fmass = P.fluid_volume * rho0;
    #pragma unroll 4

    for (int k = 0; k < cf; ++k) {
        size_t const e = k * stride + i;
        float2 const gw = a.nf_gw[e];
        sum_acc.add(scl2(fmass, gw));
        sdot_acc.add(fmass * dot2(gw, gw));
        div_acc.add(fmass * dot2(sub2(vi, a.v[a.nf_idx[e]]), gw));
    }
    #pragma unroll 4

    for (int k = 0; k < cs; ++k) {
        size_t const e = k * stride + i;
        uint32_t const j = a.ns_idx[e];
        float2 const gw = a.ns_gw[e];
        float const mass = a.vols[j] * rho0;
        sum_acc.add(scl2(mass, gw));
        div_acc.add(mass * dot2(sub2(vi, a.vs[j]), gw));
    }
    float2 const sum = sum_acc.get();
    float const sdot = sdot_acc.get();
    float const div = div_acc.get();
    float const denom = sqrf(rho);
    float const numer = pseudo ? -(dot2(sum, sum) + self_mass * sdot)
                               : -sqrf(dt) * (dot2(sum, sum) + self_mass * sdot);
    a.aii[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
    a.rho_star[i] = rho + dt * div;
}

template <int MODE>
__global__ void k_ap_diag(Arena a, int pseudo) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    if (MODE && a.sp[c.s].precision) {
        ap_diag<true>(a, c, pseudo);
    } else {
        ap_diag<false>(a, c, pseudo);
    }
}

// compute_pressure_accelerations over the cached p/rho^2 (also the pseudo
// pressure displacements, iisph_pseudo_ap_ops.cpp:119-224).
template <int MODE>
__global__ void k_pressure_accel(Arena a) {
    Ctx c;
    if (!enter(a, true, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    a.acc[c.i] = (MODE && P.precision) ? pressure_accel_of<true>(a, P, c.i, a.qdens)
                                       : pressure_accel_of<false>(a, P, c.i, a.qdens);
}

// iisph_ap_iterate_pressures_in_place (iisph_ap_ops.cpp:105-194) and the
// pseudo variant (iisph_pseudo_ap_ops.cpp:226-323).
template <bool K>
__device__ __forceinline__ float ap_neighbor_sum(Arena const& a, SceneParams const& P, uint32_t i,
                                                 int cf, int cs) {
    size_t const stride = a.stride;
    float const rho0 = P.rho0;
    SumF<K> api;
    float2 const ai = a.acc[i];
    float const fmass = rho0 * P.fluid_volume;
    #pragma unroll 4

    for (int k = 0; k < cf; ++k) {
        size_t const e = k * stride + i;
        api.add(fmass * dot2(sub2(ai, a.acc[a.nf_idx[e]]), a.nf_gw[e]));
    }
    #pragma unroll 4

    for (int k = 0; k < cs; ++k) {
        size_t const e = k * stride + i;
        api.add((rho0 * a.vols[a.ns_idx[e]]) * dot2(ai, a.ns_gw[e]));
    }
    return api.get();
}

template <int MODE>
__global__ void k_ap_iterate(Arena a, int pseudo) {
    Ctx c;
    if (!enter(a, true, c)) return;
    SceneParams const& P = a.sp[c.s];
    SceneState* S = &a.ss[c.s];
    float err = 0.0f;
    bool counted = false;
    if (c.live) {
        uint32_t const i = c.i;
        float const rho0 = P.rho0;
        int const cf = a.nf_cnt[i];
        int const cs = a.ns_cnt[i];
        float const diag = a.aii[i];
        float pnew;
        if (!cf && !cs) {
            pnew = 0.0f;
        } else if (pseudo && diag == 0.0f) {
            pnew = 0.0f;
        } else {
            float api = (MODE && P.precision) ? ap_neighbor_sum<true>(a, P, i, cf, cs)
                                              : ap_neighbor_sum<false>(a, P, i, cf, cs);
            if (!pseudo) api *= sqrf(S->dt);
            float const source = rho0 - a.rho_star[i];
            float const r = api - source;
            err = max_0x(safe_f(r, rho0) ? r / rho0 : 0.0f);
            counted = true;
            float const old = a.pbuf0[i];
            float const numer = P.iisph_omega * (source - api);
            pnew = max_0x(old + (safe_f(numer, diag) ? numer / diag : 0.0f));
        }
        a.pbuf0[i] = pnew;
        a.qdens[i] = p_over_rho2(pnew, a.rho[i]);
    }
    accumulate_error(S, counted ? static_cast<unsigned long long>(err * 1000.0f) : 0ull, err,
                     c.live && counted);
}

// Final pressure accelerations and the integration of iisph_ap.cpp:138-153
// (integrate_velocities_and_positions_in_place, dynamics.cpp:53-63) or
// iisph_pseudo_ap_integrate_velocities_and_positions_in_place
// (iisph_pseudo_ap_ops.cpp:325-343).
template <int MODE>
__global__ void k_ap_finish(Arena a, int pseudo) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    uint32_t const i = c.i;
    float2 const acc = (MODE && P.precision) ? pressure_accel_of<true>(a, P, i, a.qdens)
                                             : pressure_accel_of<false>(a, P, i, a.qdens);
    a.acc[i] = acc;
    if (!pseudo) {
        float2 const v = add2(a.v[i], scl2(dt, acc));
        a.v[i] = v;
        advance_position(a, P, i, dt, v);
    } else {
        float2 const vstar = a.v[i];
        advance_position(a, P, i, dt, vstar, acc, true);
        if (safe_v(vstar, dt)) a.v[i] = add2(vstar, div2(acc, dt));
    }
}

// ------------------------------------------------------------------- PCISPH

// Velocity from external forces only (pcisph.cpp:54-65).
__global__ void k_pc_init(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    float const mult = dt / P.mass;
    float2 const v = a.v[c.i];
    float2 const f = external_force(a, P, c.i, v);
    a.vext[c.i] = add2(v, scl2(mult, f));
    a.pbuf0[c.i] = 0.0f;
}

// Predicted velocity and position of one predictor pass (pcisph.cpp:72-88).
__global__ void k_pc_predict(Arena a) {
    Ctx c;
    if (!enter(a, true, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    SceneState const& S = a.ss[c.s];
    float const dt = S.dt;
    float2 vs = a.vext[c.i];
    if (S.iter > 0) vs = add2(vs, scl2(dt / P.mass, a.fp[c.i]));
    a.vstar[c.i] = vs;
    a.xstar[c.i] = add2(a.x[c.i], scl2(dt, vs));
}

// Densities at the predicted positions with the kernel values recomputed
// (compute_neighbor_distances_and_vectors_to + compute_neighbor_kernels,
// neighborhoods_from_state.cpp:103-128), pcisph_compute_densities,
// pcisph_accumulate_density_from_solids and pcisph_update_pressures
// (pcisph_ops.cpp:18-76), plus the max density error (common.cpp:78-85).
template <bool K>
__device__ __forceinline__ float pc_density_of(Arena const& a, SceneParams const& P, uint32_t i) {
    size_t const stride = a.stride;
    float const h = P.support;
    float2 const pos = a.xstar[i];
    int const cf = a.nf_cnt[i];
    SumF<K> ws(P.w0);
    #pragma unroll 4

    for (int k = 0; k < cf; ++k) {
        uint32_t const j = a.nf_idx[k * stride + i];
        ws.add(kernel_w(length2f(sub2(a.xstar[j], pos)), h));
    }
    float d = P.mass * ws.get();
    int const cs = a.ns_cnt[i];
    if (cs) {
        SumF<K> vf;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            uint32_t const j = a.ns_idx[k * stride + i];
            vf.add(a.vols[j] * kernel_w(length2f(sub2(a.xs[j], pos)), h));
        }
        d += P.rho0 * vf.get();
    }
    return d;
}

template <int MODE>
__global__ void k_pc_density(Arena a) {
    Ctx c;
    if (!enter(a, true, c)) return;
    SceneParams const& P = a.sp[c.s];
    SceneState* S = &a.ss[c.s];
    float err = 0.0f;
    if (c.live) {
        uint32_t const i = c.i;
        float const d = (MODE && P.precision) ? pc_density_of<true>(a, P, i)
                                              : pc_density_of<false>(a, P, i);
        a.rho[i] = d;
        float const p = a.pbuf0[i] + max_x0(d - P.rho0) / P.pcisph_denom;
        a.pbuf0[i] = p;
        a.qdens[i] = p / sqrf(d);
        err = max_0x(d - P.rho0);
    }
    accumulate_error(S, 0ull, err, c.live);
}

// pcisph_accumulate_pressure_forces and ..._from_solids (pcisph_ops.cpp:78-178)
// on the fixed neighbour lists at the predicted positions.
template <bool K>
__device__ __forceinline__ void pc_forces(Arena const& a, Ctx const& c) {
    SceneParams const& P = a.sp[c.s];
    uint32_t const i = c.i;
    size_t const stride = a.stride;
    float const h = P.support;
    float const m = P.mass;
    float const N2 = 0.01f * h * h;
    float2 const pos = a.xstar[i];
    float2 f = mk2(0.0f, 0.0f);
    int const cf = a.nf_cnt[i];
    if (cf) {
        float2 const vi = a.vstar[i];
        float const rho = a.rho[i];
        float const pors = a.qdens[i];
        SumF2<K> pf;
        #pragma unroll 4

        for (int k = 0; k < cf; ++k) {
            uint32_t const j = a.nf_idx[k * stride + i];
            float2 const vto = sub2(a.xstar[j], pos);
            float const dist = length2f(vto);
            float2 const gw = kernel_grad_w(neg2(vto), h);
            float const rho_j = a.rho[j];
            pf.add(scl2(pors + a.qdens[j], gw));
            float2 const dv = sub2(a.vstar[j], vi);
            float const dvr = dot2(vto, dv);
            if (dvr < 0.0f) {
                float const mu = h * dvr / (dist + N2);
                float const den = (rho + rho_j) / 2.0f;
                pf.add(scl2(((-1.0f * P.viscosity * mu) + (2.0f * sqrf(mu))) / den, gw));
            }
        }
        f = add2(f, scl2(-(m * m), pf.get()));
    }
    int const cs = a.ns_cnt[i];
    if (cs) {
        float const pors = a.pbuf0[i] / sqrf(a.rho[i]);
        SumF2<K> vg;
        #pragma unroll 4

        for (int k = 0; k < cs; ++k) {
            uint32_t const j = a.ns_idx[k * stride + i];
            float2 const gw = kernel_grad_w(neg2(sub2(a.xs[j], pos)), h);
            vg.add(scl2(a.vols[j], gw));
        }
        f = add2(f, scl2(-m * P.rho0 * pors, vg.get()));
    }
    a.fp[i] = f;
}

template <int MODE>
__global__ void k_pc_forces(Arena a) {
    Ctx c;
    if (!enter(a, true, c) || !c.live) return;
    if (MODE && a.sp[c.s].precision) {
        pc_forces<true>(a, c);
    } else {
        pc_forces<false>(a, c);
    }
}

// Final velocity and position update (pcisph.cpp:151-163).
__global__ void k_pc_final(Arena a) {
    Ctx c;
    if (!enter(a, false, c) || !c.live) return;
    SceneParams const& P = a.sp[c.s];
    float const dt = a.ss[c.s].dt;
    float2 const v = add2(a.vext[c.i], scl2(dt / P.mass, a.fp[c.i]));
    a.v[c.i] = v;
    advance_position(a, P, c.i, dt, v);
}

}  // namespace

// ------------------------------------------------------------ launchers

// Launches K(mode, chunk, prefetch) for the runtime choice: mode 1 when
// `comp`, chunk 1, 4 or 8 (anything else: 8), prefetch 0 or 1.
// Blocks of a persistent-warp launch: the resident blocks of `kernel` on
// every multiprocessor, no more than the tiles to cover.
template <class K>
unsigned persistent_grid(K kernel, uint32_t tiles, int threads = kTile) {
    static thread_local int dev_cached = -1;
    static thread_local int sms = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != dev_cached) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        dev_cached = dev;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    uint64_t const resident = uint64_t(std::max(per_sm, 1)) * uint64_t(std::max(sms, 1));
    // The fewest blocks that still give no warp more warp tiles than the
    // resident grid would: every warp then walks the same number of tiles
    // (8,192 warp tiles on 5,328 resident warps are 2 each on 4,096 warps,
    // not 2 on some and 1 on the rest).
    uint64_t const wpb = uint64_t(threads / 32);
    uint64_t const wtiles = uint64_t(tiles) * (kTile / 32);
    uint64_t const per_warp = (wtiles + resident * wpb - 1) / (resident * wpb);
    uint64_t const warps = (wtiles + per_warp - 1) / per_warp;
    uint64_t const blocks = (warps + wpb - 1) / wpb;
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(resident, blocks)));
}

#define EMLD_DISPATCH(K, comp, ch, pf)                                        \
    do {                                                                      \
        if (comp) {                                                           \
            if (pf) {                                                         \
                if ((ch) == 1) K(1, 1, 1); else if ((ch) == 4) K(1, 4, 1); else K(1, 8, 1); \
            } else {                                                          \
                if ((ch) == 1) K(1, 1, 0); else if ((ch) == 4) K(1, 4, 0); else K(1, 8, 0); \
            }                                                                 \
        } else {                                                              \
            if (pf) {                                                         \
                if ((ch) == 1) K(0, 1, 1); else if ((ch) == 4) K(0, 4, 1); else K(0, 8, 1); \
            } else {                                                          \
                if ((ch) == 1) K(0, 1, 0); else if ((ch) == 4) K(0, 4, 0); else K(0, 8, 0); \
            }                                                                 \
        }                                                                     \
    } while (0)

void launch_frame_begin(Arena const& a, int nscenes, cudaStream_t st) {
    k_frame_begin<<<(nscenes + 127) / 128, 128, 0, st>>>(a, nscenes);
}
void launch_frame_check(Arena const& a, int nscenes, int method, cudaGraphConditionalHandle cond,
                        cudaStream_t st) {
    k_frame_check<<<1, 128, 0, st>>>(a, nscenes, method, cond);
}
void launch_max_v2(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_max_v2<<<tiles, kTile, 0, st>>>(a);
}
void launch_begin_substep(Arena const& a, int nscenes, cudaStream_t st) {
    k_begin_substep<<<(nscenes + 127) / 128, 128, 0, st>>>(a, nscenes);
}
void launch_zero_kappas(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_zero_kappas<<<tiles, kTile, 0, st>>>(a);
}
void launch_iter_reset(Arena const& a, int nscenes, int kind, cudaStream_t st,
                       cudaGraphConditionalHandle cond, int use_cond) {
    k_iter_reset<<<1, 256, 0, st>>>(a, nscenes, kind, cond, use_cond);
}
void launch_iter_check(Arena const& a, int nscenes, int kind, int* running,
                       cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    k_iter_check<<<1, 256, 0, st>>>(a, nscenes, kind, running, cond, use_cond);
}
void launch_dfsph_density_alpha(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st,
                                int mode) {
    if (!tiles) return;
    if (mode & kPersistentWarps) {
        uint32_t const wt = tiles * (kTile / 32);
        int const th = (mode & kPersistentBlocks256) ? 256 : kTile;
        if (comp) {
            k_dfsph_density_alpha_pw<1>
              <<<persistent_grid(k_dfsph_density_alpha_pw<1>, tiles, th), th, 0, st>>>(a, wt);
        } else {
            k_dfsph_density_alpha_pw<0>
              <<<persistent_grid(k_dfsph_density_alpha_pw<0>, tiles, th), th, 0, st>>>(a, wt);
        }
        return;
    }
    if (comp) {
        k_dfsph_density_alpha<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_dfsph_density_alpha<0><<<tiles, kTile, 0, st>>>(a);
    }
}
// A persistent-warp loop kernel with the work-list walk (`list`: the
// solver loops of a batch) or the plain walk.
#define EMLD_PW_LAUNCH(KERNEL, M, C, ...)                                                      \
    do {                                                                                       \
        if (list) {                                                                            \
            KERNEL<M, C, true>                                                                 \
              <<<persistent_grid(KERNEL<M, C, true>, tiles, th), th, 0, st>>>(__VA_ARGS__);    \
        } else {                                                                               \
            KERNEL<M, C, false>                                                                \
              <<<persistent_grid(KERNEL<M, C, false>, tiles, th), th, 0, st>>>(__VA_ARGS__);   \
        }                                                                                      \
    } while (0)

#define EMLD_PW_DISPATCH(K, comp, ch)                                          \
    do {                                                                      \
        if (comp) {                                                           \
            if ((ch) == 1) K(1, 1); else if ((ch) == 4) K(1, 4); else K(1, 8); \
        } else {                                                              \
            if ((ch) == 1) K(0, 1); else if ((ch) == 4) K(0, 4); else K(0, 8); \
        }                                                                     \
    } while (0)

void launch_apply_pressures(Arena const& a, uint32_t tiles, int which_q, int external,
                            int skip_done, bool comp, cudaStream_t st, int chunk, LoopCheck lc) {
    if (!tiles) return;
    bool const pf = (chunk & kPrefetchLists) != 0;
    int const ch = chunk & kChunkMask;
    if (chunk & kPersistentWarps) {
        int const th = (chunk & kPersistentBlocks256) ? 256 : kTile;
        bool const list = a.batch && skip_done;
#define EMLD_APPLY_PW(M, C)                                                                     \
    EMLD_PW_LAUNCH(k_apply_pressures_pw, M, C, a, tiles * (kTile / 32), which_q, external,     \
                   skip_done, lc)
        EMLD_PW_DISPATCH(EMLD_APPLY_PW, comp, ch);
#undef EMLD_APPLY_PW
        return;
    }
#define EMLD_APPLY(M, C, F) k_apply_pressures<M, C, F><<<tiles, kTile, 0, st>>>(a, which_q, external, skip_done)
    EMLD_DISPATCH(EMLD_APPLY, comp, ch, pf);
#undef EMLD_APPLY
}
void launch_dfsph_divergence(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st, int chunk) {
    if (!tiles) return;
    bool const pf = (chunk & kPrefetchLists) != 0;
    int const ch = chunk & kChunkMask;
    if (chunk & kPersistentWarps) {
        int const th = (chunk & kPersistentBlocks256) ? 256 : kTile;
        bool const list = a.batch != 0;
#define EMLD_DIV_PW(M, C) EMLD_PW_LAUNCH(k_dfsph_divergence_pw, M, C, a, tiles * (kTile / 32))
        EMLD_PW_DISPATCH(EMLD_DIV_PW, comp, ch);
#undef EMLD_DIV_PW
        return;
    }
#define EMLD_DIV(M, C, F) k_dfsph_divergence<M, C, F><<<tiles, kTile, 0, st>>>(a)
    EMLD_DISPATCH(EMLD_DIV, comp, ch, pf);
#undef EMLD_DIV
}
void launch_dfsph_density(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st, int chunk) {
    if (!tiles) return;
    bool const pf = (chunk & kPrefetchLists) != 0;
    int const ch = chunk & kChunkMask;
    if (chunk & kPersistentWarps) {
        int const th = (chunk & kPersistentBlocks256) ? 256 : kTile;
        bool const list = a.batch != 0;
#define EMLD_DENS_PW(M, C) EMLD_PW_LAUNCH(k_dfsph_density_pw, M, C, a, tiles * (kTile / 32))
        EMLD_PW_DISPATCH(EMLD_DENS_PW, comp, ch);
#undef EMLD_DENS_PW
        return;
    }
#define EMLD_DENS(M, C, F) k_dfsph_density<M, C, F><<<tiles, kTile, 0, st>>>(a)
    EMLD_DISPATCH(EMLD_DENS, comp, ch, pf);
#undef EMLD_DENS
}
void launch_integrate_positions(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st) {
    if (comp) {
        k_integrate_positions<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_integrate_positions<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_iisph_density_dii(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_iisph_density_dii<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_iisph_density_dii<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_iisph_aii(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_iisph_aii<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_iisph_aii<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_iisph_sum_dij(Arena const& a, uint32_t tiles, cudaStream_t st, int chunk, bool comp) {
    if (!tiles) return;
    bool const pf = (chunk & kPrefetchLists) != 0;
    int const ch = chunk & kChunkMask;
    if (chunk & kPersistentWarps) {
        int const th = (chunk & kPersistentBlocks256) ? 256 : kTile;
        bool const list = a.batch != 0;
#define EMLD_SUM_PW(M, C) EMLD_PW_LAUNCH(k_iisph_sum_dij_pw, M, C, a, tiles * (kTile / 32))
        EMLD_PW_DISPATCH(EMLD_SUM_PW, comp, ch);
#undef EMLD_SUM_PW
        return;
    }
#define EMLD_SUM(M, C, F) k_iisph_sum_dij<M, C, F><<<tiles, kTile, 0, st>>>(a)
    EMLD_DISPATCH(EMLD_SUM, comp, ch, pf);
#undef EMLD_SUM
}
void launch_iisph_beta_pressure(Arena const& a, uint32_t tiles, cudaStream_t st, int chunk,
                                bool comp, LoopCheck lc) {
    if (!tiles) return;
    bool const pf = (chunk & kPrefetchLists) != 0;
    int const ch = chunk & kChunkMask;
    if (chunk & kPersistentWarps) {
        int const th = (chunk & kPersistentBlocks256) ? 256 : kTile;
        bool const list = a.batch != 0;
#define EMLD_BETA_PW(M, C)                                                                   \
    EMLD_PW_LAUNCH(k_iisph_beta_pressure_pw, M, C, a, tiles * (kTile / 32), lc)
        EMLD_PW_DISPATCH(EMLD_BETA_PW, comp, ch);
#undef EMLD_BETA_PW
        return;
    }
#define EMLD_BETA(M, C, F) k_iisph_beta_pressure<M, C, F><<<tiles, kTile, 0, st>>>(a)
    EMLD_DISPATCH(EMLD_BETA, comp, ch, pf);
#undef EMLD_BETA
}
void launch_make_q(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_make_q<<<tiles, kTile, 0, st>>>(a);
}
void launch_apply_integrate(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_apply_integrate<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_apply_integrate<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_ap_density(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_ap_density<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_ap_density<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_ap_diag(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp) {
    if (comp) {
        k_ap_diag<1><<<tiles, kTile, 0, st>>>(a, pseudo);
    } else {
        k_ap_diag<0><<<tiles, kTile, 0, st>>>(a, pseudo);
    }
}
void launch_pressure_accel(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_pressure_accel<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_pressure_accel<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_ap_iterate(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp) {
    if (comp) {
        k_ap_iterate<1><<<tiles, kTile, 0, st>>>(a, pseudo);
    } else {
        k_ap_iterate<0><<<tiles, kTile, 0, st>>>(a, pseudo);
    }
}
void launch_ap_finish(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp) {
    if (comp) {
        k_ap_finish<1><<<tiles, kTile, 0, st>>>(a, pseudo);
    } else {
        k_ap_finish<0><<<tiles, kTile, 0, st>>>(a, pseudo);
    }
}
void launch_pc_init(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_pc_init<<<tiles, kTile, 0, st>>>(a);
}
void launch_pc_predict(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_pc_predict<<<tiles, kTile, 0, st>>>(a);
}
void launch_pc_density(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_pc_density<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_pc_density<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_pc_forces(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp) {
    if (comp) {
        k_pc_forces<1><<<tiles, kTile, 0, st>>>(a);
    } else {
        k_pc_forces<0><<<tiles, kTile, 0, st>>>(a);
    }
}
void launch_pc_final(Arena const& a, uint32_t tiles, cudaStream_t st) {
    k_pc_final<<<tiles, kTile, 0, st>>>(a);
}

}  // namespace emerald
