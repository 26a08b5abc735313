// The sph2d_box solver operators on device memory: one C entry point per
// reference function of iisph_ops, dfsph_p_ops, pcisph_ops, iisph_ap_ops and
// iisph_pseudo_ap_ops, in the reference's argument order (count first,
// outputs before inputs) and arithmetic order, so that results are
// bit-identical to the reference's for the same inputs. Neighbour lists are
// the reference's Neighborhood_pointers layout (64 entries per particle,
// row-major, 64-bit indices).
//
// Where the reference runs a fluid pass that assigns and then a boundary pass
// that adds (the `_partial(boundary)` pairs), one thread here computes both
// sums of its particle and adds the boundary sum to the finished fluid
// value: the same two roundings in the same order, one launch instead of
// two, and no read-back of the fluid value.
//
// The three iteration functions return the reference's (average, max) error
// pair in device memory: `result` holds 4 floats (16 bytes, 8-byte aligned);
// result[0] receives the average, result[1] the maximum, result[2..3] are
// working storage. The average is the reference's: the sum over particles of
// uint64(error * 1000) divided, in double, by 1000 * n.
#include <cmath>
#include <cstdint>

#include "../../include/emerald_sph.h"
#include "engine_types.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr int kRow = kMaxNeighbors;  // entries per particle in the reference layout
constexpr int kThreads = 256;

__host__ __device__ inline unsigned blocks_for(size_t n) {
    return static_cast<unsigned>((n + kThreads - 1) / kThreads);
}

__device__ __forceinline__ float2 ld2(float const* p, size_t i) {
    return make_float2(p[2 * i], p[2 * i + 1]);
}
__device__ __forceinline__ void st2(float* p, size_t i, float2 v) {
    p[2 * i] = v.x;
    p[2 * i + 1] = v.y;
}
__device__ __forceinline__ int count_of(emerald_neighborhood const& nb, size_t i) {
    return nb.counts ? nb.counts[i] : 0;
}
__device__ __forceinline__ float2 zero2() { return make_float2(0.0f, 0.0f); }

// static_cast<uint64_t>(float) of a non-negative, non-NaN value as x86-64
// code computes it (cvttss2si below 2^63, the biased form above, and 0 from
// 2^64 and infinity on).
__device__ __forceinline__ uint64_t to_uint64_x86(float f) {
    if (f < 9.2233720368547758e18f) return static_cast<uint64_t>(static_cast<int64_t>(f));
    if (f < 1.8446744073709552e19f) return static_cast<uint64_t>(f);
    return 0ull;
}

// The error accumulation of the iteration functions: the uint64 sum of
// error * 1000 and update_atomic_max from 0 (emerald/sph_common/common.h:202-207).
// Errors are >= 0 and not NaN, so their bit patterns order as their values.
struct ErrorSink {
    unsigned long long* sum;
    unsigned int* max_bits;
};

__device__ void add_errors(ErrorSink sink, bool counted, float error) {
    unsigned long long s = counted ? to_uint64_x86(error * 1000.0f) : 0ull;
    unsigned int m = counted ? __float_as_uint(error) : 0u;
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    __shared__ unsigned long long ws[kThreads / 32];
    __shared__ unsigned int wm[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5] = s;
        wm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        unsigned int tm = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            t += ws[w];
            tm = max(tm, wm[w]);
        }
        if (t) atomicAdd(sink.sum, t);
        if (tm) atomicMax(sink.max_bits, tm);
    }
}

ErrorSink sink_of(float* result) {
    return ErrorSink{reinterpret_cast<unsigned long long*>(result),
                     reinterpret_cast<unsigned int*>(result + 2)};
}

// Average and maximum from the sums: {double(sum) / double(1000 n), max}.
__global__ void k_finish_errors(size_t n, float* result) {
    unsigned long long const s = *reinterpret_cast<unsigned long long const*>(result);
    unsigned int const m = *reinterpret_cast<unsigned int const*>(result + 2);
    result[0] = static_cast<float>(static_cast<double>(s) / static_cast<double>(1000 * n));
    result[1] = __uint_as_float(m);
}

// ------------------------------------------------------------------ IISPH

// iisph_compute_diis (emerald/sph2d_box/iisph_ops.cpp:20-85).
__device__ __forceinline__ float2 diis_sum(size_t i, int c, float dt, float rho0, float density,
                                           float const* vol, emerald_neighborhood const& nb) {
    float2 m_grad_sum = zero2();
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        float const mass = rho0 * vol[nb.indices[e]];
        m_grad_sum = add2(m_grad_sum, scl2(mass, ld2(nb.kernel_gradients, e)));
    }
    float2 const numer = scl2(-sqrf(dt), m_grad_sum);
    float const denom = sqrf(density);
    return safe_v(numer, denom) ? div2(numer, denom) : zero2();
}

__global__ void k_iisph_diis(size_t n, float dt, float rho0, float* diis, float const* rho,
                             float const* fvol, emerald_neighborhood f, float const* svol,
                             emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    float2 d = cf ? diis_sum(i, cf, dt, rho0, rho[i], fvol, f) : zero2();
    if (cs) d = add2(d, diis_sum(i, cs, dt, rho0, rho[i], svol, s));
    st2(diis, i, d);
}

// iisph_compute_aiis_and_density_stars (emerald/sph2d_box/iisph_ops.cpp:87-221).
__global__ void k_iisph_aiis_stars(size_t n, float dt, float rho0, float* aiis, float* stars,
                                   float const* diis, float const* rho, float const* fvol,
                                   float const* fvel, emerald_neighborhood f, float const* svol,
                                   float const* svel, emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    if (!cf && !cs) {
        stars[i] = rho[i];
        aiis[i] = 0.0f;
        return;
    }
    float2 const dii = ld2(diis, i);
    float2 const vi = ld2(fvel, i);
    float aii = 0.0f;
    float star = rho[i];
    if (cf) {
        float delta = 0.0f;
        for (int k = 0; k < cf; ++k) {
            size_t const e = i * kRow + k;
            uint64_t const j = f.indices[e];
            float2 const g = ld2(f.kernel_gradients, e);
            float const mass = fvol[j] * rho0;
            float2 const numer = scl2(-sqrf(dt) * mass, g);
            float const denom = sqrf(rho[j]);
            if (safe_v(numer, denom)) {
                float2 const dij = div2(numer, denom);
                aii += mass * dot2(sub2(dii, neg2(dij)), g);
            }
            delta += dt * mass * dot2(sub2(vi, ld2(fvel, j)), g);
        }
        star = star + delta;
    }
    if (cs) {
        float aii_s = 0.0f;
        float delta = 0.0f;
        for (int k = 0; k < cs; ++k) {
            size_t const e = i * kRow + k;
            uint64_t const j = s.indices[e];
            float2 const g = ld2(s.kernel_gradients, e);
            float const mass = svol[j] * rho0;
            aii_s += mass * dot2(dii, g);
            delta += dt * mass * dot2(sub2(vi, ld2(svel, j)), g);
        }
        aii = aii + aii_s;
        star = star + delta;
    }
    aiis[i] = aii;
    stars[i] = star;
}

// iisph_compute_sum_dij_pjs (emerald/sph2d_box/iisph_ops.cpp:223-253).
__global__ void k_iisph_sum_dij_pjs(size_t n, float dt, float rho0, float* out, float const* vol,
                                    float const* rho, float const* p, emerald_neighborhood nb) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = nb.counts[i];
    float2 sum = zero2();
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = nb.indices[e];
        float const mass = vol[j] * rho0;
        float2 const numer = scl2(-sqrf(dt) * mass * p[j], ld2(nb.kernel_gradients, e));
        float const denom = sqrf(rho[j]);
        if (safe_v(numer, denom)) sum = add2(sum, div2(numer, denom));
    }
    st2(out, i, sum);
}

// iisph_compute_betas (emerald/sph2d_box/iisph_ops.cpp:255-350).
__global__ void k_iisph_betas(size_t n, float dt, float rho0, float* betas, float const* rho,
                              float const* p, float const* diis, float const* sdp,
                              float const* fvol, emerald_neighborhood f, float const* svol,
                              emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    float2 const sum_i = (cf || cs) ? ld2(sdp, i) : zero2();
    float beta = 0.0f;
    if (cf) {
        float const pi = p[i];
        for (int k = 0; k < cf; ++k) {
            size_t const e = i * kRow + k;
            uint64_t const j = f.indices[e];
            float2 const g = ld2(f.kernel_gradients, e);
            float const mass = rho0 * fvol[j];
            float2 const numer = scl2(-sqrf(dt) * mass, g);
            float const denom = sqrf(rho[j]);
            float2 const dij = safe_v(numer, denom) ? div2(numer, denom) : zero2();
            float2 const not_i = sub2(ld2(sdp, j), scl2(pi, neg2(dij)));
            beta += mass * dot2(sub2(sub2(sum_i, scl2(p[j], ld2(diis, j))), not_i), g);
        }
    }
    if (cs) {
        float beta_s = 0.0f;
        for (int k = 0; k < cs; ++k) {
            size_t const e = i * kRow + k;
            float const mass = rho0 * svol[s.indices[e]];
            beta_s += mass * dot2(sum_i, ld2(s.kernel_gradients, e));
        }
        beta = beta + beta_s;
    }
    betas[i] = beta;
}

// iisph_compute_new_pressures (emerald/sph2d_box/iisph_ops.cpp:352-423). The
// reference prints a message when the division is unsafe and keeps the old
// pressure; here the old pressure is kept without a message.
__global__ void k_iisph_new_pressures(size_t n, float omega, float rho0, float* io,
                                      float const* old_p, float const* alphas,
                                      float const* stars, ErrorSink sink) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool counted = false;
    float error = 0.0f;
    if (i < n) {
        float const alpha = alphas[i];
        float const old_pressure = old_p[i];
        if (alpha == 0.0f) {
            io[i] = old_pressure;
        } else {
            float const numer = rho0 - stars[i] - io[i];
            if (!safe_f(numer, alpha)) {
                io[i] = old_pressure;
            } else {
                error = max_0x(-(numer - (alpha * old_pressure)) / rho0);
                counted = true;
                io[i] = max_0x(mix1(old_pressure, numer / alpha, omega));
            }
        }
    }
    add_errors(sink, counted, error);
}

// ------------------------------------------------------------------ DFSPH

// dfsph_p_compute_shared_coeffs (emerald/sph2d_box/dfsph_p_ops.cpp:19-81).
__global__ void k_dfsph_shared_coeffs(size_t n, float rho0, float* out, float const* rho,
                                      float const* fvol, emerald_neighborhood f,
                                      float const* svol, emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    if (!(cf + cs)) {
        out[i] = 0.0f;
        return;
    }
    float2 sum = zero2();
    float sum_sq = 0.0f;
    for (int k = 0; k < cf; ++k) {
        size_t const e = i * kRow + k;
        float2 const mg = scl2(fvol[f.indices[e]] * rho0, ld2(f.kernel_gradients, e));
        sum = add2(sum, mg);
        sum_sq += dot2(mg, mg);
    }
    for (int k = 0; k < cs; ++k) {
        size_t const e = i * kRow + k;
        sum = add2(sum, scl2(svol[s.indices[e]] * rho0, ld2(s.kernel_gradients, e)));
    }
    float const numer = sqrf(rho[i]);
    float const denom = dot2(sum, sum) + sum_sq;
    out[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
}

// dfsph_p_compute_density_pseudo_pressures and
// dfsph_p_compute_divergence_pseudo_pressures
// (emerald/sph2d_box/dfsph_p_ops.cpp:83-124): with `offset` = target density
// and `denom` = dt^2 for the first, offset 0 and denom dt for the second.
__global__ void k_dfsph_pseudo_pressures(size_t n, float offset, float denom, float* out,
                                         float const* in, float const* coeffs) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float const delta = in[i] - offset;
    if (delta <= 0.0f) {
        out[i] = 0.0f;
    } else {
        float const numer = delta * coeffs[i];
        out[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
    }
}

// ----------------------------------------------------------------- PCISPH

// pcisph_compute_densities (emerald/sph2d_box/pcisph_ops.cpp:18-37).
__global__ void k_pcisph_densities(size_t n, float mass, float h, float* rho,
                                   uint8_t const* counts, float const* w) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    float sum = kernel_w(0.0f, h);
    for (int k = 0; k < c; ++k) sum += w[i * kRow + k];
    rho[i] = mass * sum;
}

// pcisph_accumulate_density_from_solids (emerald/sph2d_box/pcisph_ops.cpp:39-61).
__global__ void k_pcisph_density_solids(size_t n, float rho0, float* rho, float const* svol,
                                        uint8_t const* counts, uint64_t const* idx,
                                        float const* w) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    if (!c) return;
    float frac = 0.0f;
    for (int k = 0; k < c; ++k) frac += svol[idx[i * kRow + k]] * w[i * kRow + k];
    rho[i] += rho0 * frac;
}

// pcisph_update_pressures (emerald/sph2d_box/pcisph_ops.cpp:63-74).
__global__ void k_pcisph_update_pressures(size_t n, float rho0, float denom, float* p,
                                          float const* rho) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    p[i] += max_x0(rho[i] - rho0) / denom;
}

// pcisph_accumulate_pressure_forces (emerald/sph2d_box/pcisph_ops.cpp:76-138):
// symmetric pressure term plus Monaghan's artificial viscosity (alpha 1,
// beta 2, eta^2 = 0.01 h^2) on approaching pairs.
__global__ void k_pcisph_forces(size_t n, float mass, float h, float viscosity, float* forces,
                                uint8_t const* counts, uint64_t const* idx, float const* dist,
                                float const* vto, float const* gw, float const* vel,
                                float const* p, float const* rho) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    if (!c) return;
    float const N2 = 0.01f * h * h;
    float2 const vi = ld2(vel, i);
    float const density = rho[i];
    float const pors = p[i] / sqrf(density);
    float2 pf = zero2();
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = idx[e];
        float2 const r = ld2(vto, e);
        float2 const g = ld2(gw, e);
        float const rho_j = rho[j];
        pf = add2(pf, scl2(pors + (p[j] / sqrf(rho_j)), g));
        float const dvr = dot2(r, sub2(ld2(vel, j), vi));
        if (dvr < 0.0f) {
            float const mu = h * dvr / (dist[e] + N2);
            float const den = (density + rho_j) / 2.0f;
            pf = add2(pf, scl2(((-1.0f * viscosity * mu) + (2.0f * sqrf(mu))) / den, g));
        }
    }
    st2(forces, i, add2(ld2(forces, i), scl2(-(mass * mass), pf)));
}

// pcisph_accumulate_pressure_forces_from_solids (emerald/sph2d_box/pcisph_ops.cpp:140-176).
__global__ void k_pcisph_forces_solids(size_t n, float mass, float rho0, float* forces,
                                       float const* svol, uint8_t const* counts,
                                       uint64_t const* idx, float const* gw, float const* p,
                                       float const* rho) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    if (!c) return;
    float const pors = p[i] / sqrf(rho[i]);
    float2 vg = zero2();
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        vg = add2(vg, scl2(svol[idx[e]], ld2(gw, e)));
    }
    st2(forces, i, add2(ld2(forces, i), scl2(-mass * rho0 * pors, vg)));
}

// -------------------------------------------------------- IISPH_AP family

// iisph_ap_density_stars_and_diagonals (emerald/sph2d_box/iisph_ap_ops.cpp:19-104)
// with dt2 = dt^2, and iisph_pseudo_ap_density_stars_and_pseudo_diagonals
// (emerald/sph2d_box/iisph_pseudo_ap_ops.cpp:19-121), whose numerator has no
// dt^2 factor (pseudo = true).
template <bool kPseudo>
__global__ void k_ap_stars_diagonals(size_t n, float dt, float rho0, float* stars, float* diag,
                                     float const* rho, float const* fvol, float const* fvel,
                                     emerald_neighborhood f, float const* svol, float const* svel,
                                     emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    if (!(cf + cs)) {
        stars[i] = rho[i];
        diag[i] = 0.0f;
        return;
    }
    float const self_mass = fvol[i] * rho0;
    float const density = rho[i];
    float2 const vi = ld2(fvel, i);
    float2 sum = zero2();
    float sum_sq = 0.0f;
    float divergence = 0.0f;
    for (int k = 0; k < cf; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = f.indices[e];
        float2 const g = ld2(f.kernel_gradients, e);
        float const mass = fvol[j] * rho0;
        sum = add2(sum, scl2(mass, g));
        sum_sq += mass * dot2(g, g);
        divergence += mass * dot2(sub2(vi, ld2(fvel, j)), g);
    }
    for (int k = 0; k < cs; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = s.indices[e];
        float2 const g = ld2(s.kernel_gradients, e);
        float const mass = svol[j] * rho0;
        sum = add2(sum, scl2(mass, g));
        divergence += mass * dot2(sub2(vi, ld2(svel, j)), g);
    }
    float const denom = sqrf(density);
    float const numer = kPseudo ? -(dot2(sum, sum) + self_mass * sum_sq)
                                : -sqrf(dt) * (dot2(sum, sum) + self_mass * sum_sq);
    diag[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
    stars[i] = density + dt * divergence;
}

// Api of iisph_ap_iterate_pressures_in_place (emerald/sph2d_box/iisph_ap_ops.cpp:106-192)
// and iisph_pseudo_ap_iterate_pseudo_pressures_in_place
// (emerald/sph2d_box/iisph_pseudo_ap_ops.cpp:216-311): sum over fluid
// neighbours of m (a_i - a_j).gradW, then over solids of m a_i.gradW.
__device__ __forceinline__ float ap_api(size_t i, int cf, int cs, float rho0, float const* acc,
                                        float const* fvol, emerald_neighborhood const& f,
                                        float const* svol, emerald_neighborhood const& s) {
    float2 const ai = ld2(acc, i);
    float api = 0.0f;
    for (int k = 0; k < cf; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = f.indices[e];
        float const mass = rho0 * fvol[j];
        api += mass * dot2(sub2(ai, ld2(acc, j)), ld2(f.kernel_gradients, e));
    }
    for (int k = 0; k < cs; ++k) {
        size_t const e = i * kRow + k;
        float const mass = rho0 * svol[s.indices[e]];
        api += mass * dot2(ai, ld2(s.kernel_gradients, e));
    }
    return api;
}

__global__ void k_iisph_ap_iterate(size_t n, float dt, float rho0, float omega, float* p,
                                   float const* stars, float const* acc, float const* diag,
                                   float const* fvol, emerald_neighborhood f, float const* svol,
                                   emerald_neighborhood s, ErrorSink sink) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool counted = false;
    float error = 0.0f;
    if (i < n) {
        int const cf = f.counts[i];
        int const cs = count_of(s, i);
        if (!cf && !cs) {
            p[i] = 0.0f;
        } else {
            float api = ap_api(i, cf, cs, rho0, acc, fvol, f, svol, s);
            api *= sqrf(dt);
            float const source = rho0 - stars[i];
            float const d = diag[i];
            float const r = api - source;
            error = max_0x(safe_f(r, rho0) ? r / rho0 : 0.0f);
            counted = true;
            float const numer = omega * (source - api);
            p[i] = max_0x(p[i] + (safe_f(numer, d) ? numer / d : 0.0f));
        }
    }
    add_errors(sink, counted, error);
}

// iisph_pseudo_ap_compute_pseudo_pressure_displacements
// (emerald/sph2d_box/iisph_pseudo_ap_ops.cpp:123-214).
__global__ void k_pseudo_ap_displacements(size_t n, float rho0, float* out, float const* pp,
                                          float const* rho, float const* fvol,
                                          emerald_neighborhood f, float const* svol,
                                          emerald_neighborhood s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const cf = f.counts[i];
    int const cs = count_of(s, i);
    float const qi = (cf || cs) ? p_over_rho2(pp[i], rho[i]) : 0.0f;
    float2 disp = zero2();
    for (int k = 0; k < cf; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = f.indices[e];
        float const mass = rho0 * fvol[j];
        float const coeff = qi + p_over_rho2(pp[j], rho[j]);
        disp = add2(disp, scl2(-mass * coeff, ld2(f.kernel_gradients, e)));
    }
    if (cs) {
        float2 ds = zero2();
        for (int k = 0; k < cs; ++k) {
            size_t const e = i * kRow + k;
            float const mass = rho0 * svol[s.indices[e]];
            ds = add2(ds, scl2(-mass * qi, ld2(s.kernel_gradients, e)));
        }
        disp = add2(disp, ds);
    }
    st2(out, i, disp);
}

__global__ void k_pseudo_ap_iterate(size_t n, float rho0, float omega, float* pp,
                                    float const* stars, float const* disp, float const* diag,
                                    float const* fvol, emerald_neighborhood f, float const* svol,
                                    emerald_neighborhood s, ErrorSink sink) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool counted = false;
    float error = 0.0f;
    if (i < n) {
        int const cf = f.counts[i];
        int const cs = count_of(s, i);
        float const d = (cf || cs) ? diag[i] : 0.0f;
        if (d == 0.0f) {
            pp[i] = 0.0f;
        } else {
            float const api = ap_api(i, cf, cs, rho0, disp, fvol, f, svol, s);
            float const source = rho0 - stars[i];
            float const r = api - source;
            error = max_0x(safe_f(r, rho0) ? r / rho0 : 0.0f);
            counted = true;
            float const numer = omega * (source - api);
            pp[i] = max_0x(pp[i] + (safe_f(numer, d) ? numer / d : 0.0f));
        }
    }
    add_errors(sink, counted, error);
}

// iisph_pseudo_ap_integrate_velocities_and_positions_in_place
// (emerald/sph2d_box/iisph_pseudo_ap_ops.cpp:313-330).
__global__ void k_pseudo_ap_integrate(size_t n, float dt, float* vel, float* pos,
                                      float const* disp) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float2 const v = ld2(vel, i);
    float2 const d = ld2(disp, i);
    st2(pos, i, add2(add2(ld2(pos, i), scl2(dt, v)), d));
    if (safe_v(v, dt)) st2(vel, i, add2(v, div2(d, dt)));
}

bool ok() { return cudaGetLastError() == cudaSuccess; }

cudaStream_t S(void* st) { return static_cast<cudaStream_t>(st); }

bool gw_list(emerald_neighborhood const& nb) {
    return nb.counts && nb.indices && nb.kernel_gradients;
}
// A boundary neighbourhood is either absent (NULL counts) or complete.
bool solid_ok(emerald_neighborhood const& nb, float const* vol) {
    return !nb.counts || (nb.indices && nb.kernel_gradients && vol);
}

bool result_ok(float const* result) {
    return result && (reinterpret_cast<uintptr_t>(result) % 8) == 0;
}

// Clears the sums, runs `launch` (which accumulates into them) and turns
// them into {average, max}; n = 0 leaves {0, 0}.
template <typename Launch>
int with_errors(size_t n, float* result, cudaStream_t st, Launch&& launch) {
    if (cudaMemsetAsync(result, 0, 4 * sizeof(float), st) != cudaSuccess) return EMERALD_ECUDA;
    if (n) {
        launch(sink_of(result));
        k_finish_errors<<<1, 1, 0, st>>>(n, result);
    }
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

}  // namespace

}  // namespace emerald

using namespace emerald;

extern "C" {

int emerald_iisph_compute_diis(size_t n, float dt, float target_density, float* diis,
                               float const* self_densities, float const* fluid_volumes,
                               emerald_neighborhood fluid, float const* solid_volumes,
                               emerald_neighborhood solid, void* stream) {
    if (n && (!diis || !self_densities || !fluid_volumes || !gw_list(fluid) ||
              !solid_ok(solid, solid_volumes))) {
        return EMERALD_EINVAL;
    }
    if (n) k_iisph_diis<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, diis, self_densities, fluid_volumes, fluid, solid_volumes, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_compute_aiis_and_density_stars(
  size_t n, float dt, float target_density, float* aiis, float* density_stars, float const* diis,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream) {
    if (n && (!aiis || !density_stars || !diis || !densities || !fluid_volumes ||
              !fluid_velocities || !gw_list(fluid) || !solid_ok(solid, solid_volumes) ||
              (solid.counts && !solid_velocities))) {
        return EMERALD_EINVAL;
    }
    if (n) k_iisph_aiis_stars<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, aiis, density_stars, diis, densities, fluid_volumes,
      fluid_velocities, fluid, solid_volumes, solid_velocities, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_compute_sum_dij_pjs(size_t n, float dt, float target_density,
                                      float* sum_dij_pjs, float const* volumes,
                                      float const* densities, float const* pressures,
                                      emerald_neighborhood neighborhood, void* stream) {
    if (n && (!sum_dij_pjs || !volumes || !densities || !pressures || !gw_list(neighborhood))) {
        return EMERALD_EINVAL;
    }
    if (n) k_iisph_sum_dij_pjs<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, sum_dij_pjs, volumes, densities, pressures, neighborhood);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_compute_betas(size_t n, float dt, float target_density, float* betas,
                                float const* densities, float const* pressures,
                                float const* diis, float const* sum_dij_pjs,
                                float const* fluid_volumes, emerald_neighborhood fluid,
                                float const* solid_volumes, emerald_neighborhood solid,
                                void* stream) {
    if (n && (!betas || !densities || !pressures || !diis || !sum_dij_pjs || !fluid_volumes ||
              !gw_list(fluid) || !solid_ok(solid, solid_volumes))) {
        return EMERALD_EINVAL;
    }
    if (n) k_iisph_betas<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, betas, densities, pressures, diis, sum_dij_pjs, fluid_volumes, fluid,
      solid_volumes, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_compute_new_pressures(size_t n, float omega, float target_density,
                                        float* betas_in_new_pressures_out,
                                        float const* old_pressures, float const* alphas,
                                        float const* density_stars, float* result,
                                        void* stream) {
    if (!result_ok(result) ||
        (n && (!betas_in_new_pressures_out || !old_pressures || !alphas || !density_stars))) {
        return EMERALD_EINVAL;
    }
    cudaStream_t const st = S(stream);
    return with_errors(n, result, st, [&](ErrorSink sink) {
        k_iisph_new_pressures<<<blocks_for(n), kThreads, 0, st>>>(
          n, omega, target_density, betas_in_new_pressures_out, old_pressures, alphas,
          density_stars, sink);
    });
}

int emerald_dfsph_p_compute_shared_coeffs(size_t n, float target_density, float* shared_coeffs,
                                          float const* densities, float const* fluid_volumes,
                                          emerald_neighborhood fluid, float const* solid_volumes,
                                          emerald_neighborhood solid, void* stream) {
    if (n && (!shared_coeffs || !densities || !fluid_volumes || !gw_list(fluid) ||
              !solid_ok(solid, solid_volumes))) {
        return EMERALD_EINVAL;
    }
    if (n) k_dfsph_shared_coeffs<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, target_density, shared_coeffs, densities, fluid_volumes, fluid, solid_volumes, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_dfsph_p_compute_density_pseudo_pressures(size_t n, float dt, float target_density,
                                                     float* density_pseudo_pressures,
                                                     float const* density_stars,
                                                     float const* shared_coeffs, void* stream) {
    if (n && (!density_pseudo_pressures || !density_stars || !shared_coeffs)) {
        return EMERALD_EINVAL;
    }
    if (n) k_dfsph_pseudo_pressures<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, target_density, sqrf(dt), density_pseudo_pressures, density_stars, shared_coeffs);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_dfsph_p_compute_divergence_pseudo_pressures(size_t n, float dt, float target_density,
                                                        float* divergence_pseudo_pressures,
                                                        float const* divergences,
                                                        float const* shared_coeffs,
                                                        void* stream) {
    (void)target_density;  // unused by the reference too
    if (n && (!divergence_pseudo_pressures || !divergences || !shared_coeffs)) {
        return EMERALD_EINVAL;
    }
    if (n) k_dfsph_pseudo_pressures<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, 0.0f, dt, divergence_pseudo_pressures, divergences, shared_coeffs);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_pcisph_compute_densities(size_t n, float mass_per_particle, float support,
                                     float* densities, uint8_t const* neighbor_counts,
                                     float const* neighbor_kernels, void* stream) {
    if (!(support > 0.0f) || (n && (!densities || !neighbor_counts || !neighbor_kernels))) {
        return EMERALD_EINVAL;
    }
    if (n) k_pcisph_densities<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, mass_per_particle, support, densities, neighbor_counts,
      neighbor_kernels);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_pcisph_accumulate_density_from_solids(size_t n, float target_density,
                                                  float* densities, float const* solid_volumes,
                                                  uint8_t const* solid_neighbor_counts,
                                                  uint64_t const* solid_neighbor_indices,
                                                  float const* solid_neighbor_kernels,
                                                  void* stream) {
    if (n && (!densities || !solid_volumes || !solid_neighbor_counts || !solid_neighbor_indices ||
              !solid_neighbor_kernels)) {
        return EMERALD_EINVAL;
    }
    if (n) k_pcisph_density_solids<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, target_density, densities, solid_volumes, solid_neighbor_counts, solid_neighbor_indices,
      solid_neighbor_kernels);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_pcisph_update_pressures(size_t n, float target_density,
                                    float pressure_correction_denom, float* pressures,
                                    float const* densities, void* stream) {
    if (n && (!pressures || !densities)) return EMERALD_EINVAL;
    if (n) k_pcisph_update_pressures<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, target_density, pressure_correction_denom, pressures, densities);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_pcisph_accumulate_pressure_forces(
  size_t n, float mass_per_particle, float support, float viscosity, float* pressure_forces,
  uint8_t const* neighbor_counts, uint64_t const* neighbor_indices,
  float const* neighbor_distances, float const* neighbor_vectors_to,
  float const* neighbor_kernel_gradients, float const* velocities, float const* pressures,
  float const* densities, void* stream) {
    if (n && (!pressure_forces || !neighbor_counts || !neighbor_indices || !neighbor_distances ||
              !neighbor_vectors_to || !neighbor_kernel_gradients || !velocities || !pressures ||
              !densities)) {
        return EMERALD_EINVAL;
    }
    if (n) k_pcisph_forces<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, mass_per_particle, support, viscosity, pressure_forces, neighbor_counts,
      neighbor_indices, neighbor_distances, neighbor_vectors_to, neighbor_kernel_gradients,
      velocities, pressures, densities);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_pcisph_accumulate_pressure_forces_from_solids(
  size_t n, float mass_per_particle, float target_density, float* pressure_forces,
  float const* solid_volumes, uint8_t const* solid_neighbor_counts,
  uint64_t const* solid_neighbor_indices, float const* solid_neighbor_kernel_gradients,
  float const* pressures, float const* densities, void* stream) {
    if (n && (!pressure_forces || !solid_volumes || !solid_neighbor_counts ||
              !solid_neighbor_indices || !solid_neighbor_kernel_gradients || !pressures ||
              !densities)) {
        return EMERALD_EINVAL;
    }
    if (n) k_pcisph_forces_solids<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, mass_per_particle, target_density, pressure_forces, solid_volumes, solid_neighbor_counts,
      solid_neighbor_indices, solid_neighbor_kernel_gradients, pressures, densities);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_ap_density_stars_and_diagonals(
  size_t n, float dt, float target_density, float* density_stars, float* diagonals,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream) {
    if (n && (!density_stars || !diagonals || !densities || !fluid_volumes ||
              !fluid_velocities || !gw_list(fluid) || !solid_ok(solid, solid_volumes) ||
              (solid.counts && !solid_velocities))) {
        return EMERALD_EINVAL;
    }
    if (n) k_ap_stars_diagonals<false><<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, density_stars, diagonals, densities, fluid_volumes,
      fluid_velocities, fluid, solid_volumes, solid_velocities, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_ap_iterate_pressures_in_place(
  size_t n, float dt, float target_density, float omega, float* pressures,
  float const* density_stars, float const* pressure_accelerations, float const* diagonals,
  float const* fluid_volumes, emerald_neighborhood fluid, float const* solid_volumes,
  emerald_neighborhood solid, float* result, void* stream) {
    if (!result_ok(result) ||
        (n && (!pressures || !density_stars || !pressure_accelerations || !diagonals ||
               !fluid_volumes || !gw_list(fluid) || !solid_ok(solid, solid_volumes)))) {
        return EMERALD_EINVAL;
    }
    cudaStream_t const st = S(stream);
    return with_errors(n, result, st, [&](ErrorSink sink) {
        k_iisph_ap_iterate<<<blocks_for(n), kThreads, 0, st>>>(
          n, dt, target_density, omega, pressures, density_stars, pressure_accelerations,
          diagonals, fluid_volumes, fluid, solid_volumes, solid, sink);
    });
}

int emerald_iisph_pseudo_ap_density_stars_and_pseudo_diagonals(
  size_t n, float dt, float target_density, float* density_stars, float* pseudo_diagonals,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream) {
    if (n && (!density_stars || !pseudo_diagonals || !densities || !fluid_volumes ||
              !fluid_velocities || !gw_list(fluid) || !solid_ok(solid, solid_volumes) ||
              (solid.counts && !solid_velocities))) {
        return EMERALD_EINVAL;
    }
    if (n) k_ap_stars_diagonals<true><<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, density_stars, pseudo_diagonals, densities, fluid_volumes,
      fluid_velocities, fluid, solid_volumes, solid_velocities, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_pseudo_ap_compute_pseudo_pressure_displacements(
  size_t n, float target_density, float* pseudo_pressure_displacements,
  float const* pseudo_pressures, float const* densities, float const* fluid_volumes,
  emerald_neighborhood fluid, float const* solid_volumes, emerald_neighborhood solid,
  void* stream) {
    if (n && (!pseudo_pressure_displacements || !pseudo_pressures || !densities ||
              !fluid_volumes || !gw_list(fluid) || !solid_ok(solid, solid_volumes))) {
        return EMERALD_EINVAL;
    }
    if (n) k_pseudo_ap_displacements<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, target_density, pseudo_pressure_displacements, pseudo_pressures, densities,
      fluid_volumes, fluid, solid_volumes, solid);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_iisph_pseudo_ap_iterate_pseudo_pressures_in_place(
  size_t n, float target_density, float omega, float* pseudo_pressures,
  float const* density_stars, float const* pseudo_pressure_displacements,
  float const* pseudo_diagonals, float const* fluid_volumes, emerald_neighborhood fluid,
  float const* solid_volumes, emerald_neighborhood solid, float* result, void* stream) {
    if (!result_ok(result) ||
        (n && (!pseudo_pressures || !density_stars || !pseudo_pressure_displacements ||
               !pseudo_diagonals || !fluid_volumes || !gw_list(fluid) ||
               !solid_ok(solid, solid_volumes)))) {
        return EMERALD_EINVAL;
    }
    cudaStream_t const st = S(stream);
    return with_errors(n, result, st, [&](ErrorSink sink) {
        k_pseudo_ap_iterate<<<blocks_for(n), kThreads, 0, st>>>(
          n, target_density, omega, pseudo_pressures, density_stars,
          pseudo_pressure_displacements, pseudo_diagonals, fluid_volumes, fluid, solid_volumes,
          solid, sink);
    });
}

int emerald_iisph_pseudo_ap_integrate_velocities_and_positions_in_place(
  size_t n, float dt, float* velocities, float* positions,
  float const* pseudo_pressure_displacements, void* stream) {
    if (n && (!velocities || !positions || !pseudo_pressure_displacements)) return EMERALD_EINVAL;
    if (n) k_pseudo_ap_integrate<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, velocities, positions, pseudo_pressure_displacements);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

}  // extern "C"
