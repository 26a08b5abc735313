// The sph_common free functions on device memory: one CUDA kernel per
// reference function, in the reference's argument order (count first,
// outputs before inputs) and arithmetic order, so that results are
// bit-identical to the reference's for the same inputs. Neighbour lists are
// the reference's Neighborhood_pointers layout (64 entries per particle,
// row-major, 64-bit indices). Every call is asynchronous on the given stream
// (NULL: the legacy default stream) and allocates nothing; the reductions
// run in one block and write their result to device memory.
#include <cmath>
#include <cstdint>

#include "../../include/emerald_sph.h"
#include "engine_types.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr int kRow = kMaxNeighbors;  // entries per particle in the reference layout
constexpr float kLowest = -3.40282346638528859811704183484516925e+38f;  // lowest finite float
constexpr int kThreads = 256;
constexpr int kReduceThreads = 1024;

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

// safe_divide(p, sqr(rho)).value_or(0) (emerald/util/safe_divide.h:20-31).
__device__ __forceinline__ float p_over_rho_sqr(float p, float rho) { return p_over_rho2(p, rho); }

// compute_grid_coords (emerald/sph_common/common.cpp:57-67).
__global__ void k_grid_coords(size_t n, float cell, float2 bmin, int32_t* gc, float const* x) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float2 const q = div2(sub2(ld2(x, i), bmin), cell);
    gc[2 * i] = static_cast<int32_t>(floorf(q.x));
    gc[2 * i + 1] = static_cast<int32_t>(floorf(q.y));
}

// compute_z_indices (emerald/sph_common/common.cpp:69-76).
__global__ void k_z_indices(size_t n, uint64_t* z, int32_t const* gc) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    z[i] = morton2(static_cast<uint32_t>(gc[2 * i]), static_cast<uint32_t>(gc[2 * i + 1]));
}

// compute_neighbor_distances_and_vectors_to
// (emerald/sph_common/neighborhood.cpp:154-176).
__global__ void k_distances_vectors(size_t n, float* dist, float* vec, float const* self_x,
                                    float const* other_x, uint8_t const* counts,
                                    uint64_t const* idx) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float2 const p = ld2(self_x, i);
    int const c = counts[i];
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        float2 const d = sub2(ld2(other_x, idx[e]), p);
        st2(vec, e, d);
        dist[e] = length2f(d);
    }
}

// compute_neighbor_kernels (emerald/sph_common/neighborhood.cpp:178-192).
__global__ void k_neighbor_kernels(size_t n, float h, float* w, uint8_t const* counts,
                                   float const* dist) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    for (int k = 0; k < c; ++k) w[i * kRow + k] = kernel_w(dist[i * kRow + k], h);
}

// compute_neighbor_kernel_gradients (emerald/sph_common/neighborhood.cpp:194-210).
__global__ void k_neighbor_gradients(size_t n, float h, float* gw, uint8_t const* counts,
                                     float const* vec) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = counts[i];
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        st2(gw, e, kernel_grad_w(neg2(ld2(vec, e)), h));
    }
}

// compute_densities_partial (emerald/sph_common/density.cpp:10-45).
__global__ void k_densities(size_t n, bool boundary, float h, float rho0, float* rho,
                            float const* self_vol, float const* nbr_vol, emerald_neighborhood nb) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float const w0 = kernel_w(0.0f, h);
    float d = 0.0f;
    if (!boundary) d = self_vol[i] * rho0 * w0;
    int const c = nb.counts[i];
    if (!c) {
        if (!boundary) rho[i] = d;
        return;
    }
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        float const mass = rho0 * nbr_vol[nb.indices[e]];
        d += nb.kernels[e] * mass;
    }
    if (boundary) {
        rho[i] += d;
    } else {
        rho[i] = d;
    }
}

// compute_divergences_partial (emerald/sph_common/divergence.cpp:5-45).
__global__ void k_divergences(size_t n, bool boundary, float rho0, float* div,
                              float const* self_v, float const* nbr_vol, float const* nbr_v,
                              emerald_neighborhood nb) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = nb.counts[i];
    if (!c) {
        if (!boundary) div[i] = 0.0f;
        return;
    }
    float2 const vi = ld2(self_v, i);
    float d = 0.0f;
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = nb.indices[e];
        float const mass = rho0 * nbr_vol[j];
        d += mass * dot2(sub2(vi, ld2(nbr_v, j)), ld2(nb.kernel_gradients, e));
    }
    if (boundary) {
        div[i] += d;
    } else {
        div[i] = d;
    }
}

// predict_density_stars_from_divergences (emerald/sph_common/density.cpp:75-83).
__global__ void k_density_stars(size_t n, float dt, float* stars, float const* rho,
                                float const* div) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    stars[i] = max_0x(rho[i] + (dt * div[i]));
}

// apply_pressures_in_place_partial (emerald/sph_common/pressure.cpp:9-50).
__global__ void k_apply_pressures(size_t n, bool boundary, float dt, float rho0, float* v,
                                  float const* rho, float const* p, float const* nbr_vol,
                                  emerald_neighborhood nb) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = nb.counts[i];
    if (!c) return;
    float const qi = p_over_rho_sqr(p[i], rho[i]);
    float2 acc = make_float2(0.0f, 0.0f);
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = nb.indices[e];
        float const mass = rho0 * nbr_vol[j];
        float2 const g = ld2(nb.kernel_gradients, e);
        if (boundary) {
            acc = add2(acc, scl2(-mass * qi, g));
        } else {
            acc = add2(acc, scl2(-mass * (qi + p_over_rho_sqr(p[j], rho[j])), g));
        }
    }
    st2(v, i, add2(ld2(v, i), scl2(dt, acc)));
}

// compute_pressure_accelerations_partial (emerald/sph_common/pressure.cpp:83-152).
__global__ void k_pressure_accelerations(size_t n, bool boundary, float rho0, float* a,
                                         float const* p, float const* rho, float const* nbr_vol,
                                         emerald_neighborhood nb) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int const c = nb.counts[i];
    if (!c) {
        if (!boundary) st2(a, i, make_float2(0.0f, 0.0f));
        return;
    }
    float const qi = p_over_rho_sqr(p[i], rho[i]);
    float2 acc = make_float2(0.0f, 0.0f);
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        uint64_t const j = nb.indices[e];
        float const mass = rho0 * nbr_vol[j];
        float const coeff = boundary ? qi : qi + p_over_rho_sqr(p[j], rho[j]);
        acc = add2(acc, scl2(-mass * coeff, ld2(nb.kernel_gradients, e)));
    }
    if (boundary) {
        st2(a, i, add2(ld2(a, i), acc));
    } else {
        st2(a, i, acc);
    }
}

// integrate_velocities_in_place with forces (emerald/sph_common/dynamics.cpp:24-37).
__global__ void k_integrate_forces(size_t n, float dt, float rho0, float* v, float const* vol,
                                   float const* f) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float const denom = rho0 * vol[i];
    float2 const numer = scl2(dt, ld2(f, i));
    if (safe_v(numer, denom)) st2(v, i, add2(ld2(v, i), div2(numer, denom)));
}

// accumulate(count, mult, dst, src) (emerald/sph_common/common.h:76-81): the
// velocity and position integrations of emerald/sph_common/dynamics.cpp:39-51.
__global__ void k_accumulate(size_t n, float dt, float* dst, float const* src) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    st2(dst, i, add2(ld2(dst, i), scl2(dt, ld2(src, i))));
}

// fill_array of compute_constant_volumes (emerald/sph_common/volume.cpp:7-14).
__global__ void k_fill(size_t n, float value, float* out) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = value;
}

// Block-wide maximum of non-negative floats (bit order is value order for
// them); NaN values are dropped, as std::max(running, NaN) keeps running.
__device__ float block_max_nonneg(float v) {
    uint32_t m = (v == v && v > 0.0f) ? __float_as_uint(v) : 0u;
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ uint32_t wm[kReduceThreads / 32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t = max(t, wm[w]);
    __syncthreads();
    return __uint_as_float(t);
}

// max_vector_squared_magnitude (emerald/sph_common/common.cpp:87-92) and
// max_density_error (:78-85): one block.
__global__ void k_max_sq(size_t n, float const* vecs, float* out) {
    float m = 0.0f;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        float2 const v = ld2(vecs, i);
        float const d = v.x * v.x + v.y * v.y;
        m = (m < d) ? d : m;
    }
    float const t = block_max_nonneg(m);
    if (threadIdx.x == 0) *out = t;
}

__global__ void k_max_density_error(size_t n, float rho0, float const* rho, float* out) {
    float m = 0.0f;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        float const e = max_0x(rho[i] - rho0);
        m = (m < e) ? e : m;
    }
    float const t = block_max_nonneg(m);
    if (threadIdx.x == 0) *out = t;
}

__device__ __forceinline__ int64_t to_int64_x86(float f) {
    if (!(f > -9.2233720368547758e18f && f < 9.2233720368547758e18f)) return INT64_MIN;
    return static_cast<int64_t>(f);
}

// cfl_maximum_time_step (emerald/sph_common/cfl.cpp:12-21) with to_flicks
// (emerald/util/flicks.h): flicks of factor * support / max |v|, or of 1 s.
__global__ void k_cfl(size_t n, float support, float factor, float const* vels, int64_t* out) {
    float m = 0.0f;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        float2 const v = ld2(vels, i);
        float const d = v.x * v.x + v.y * v.y;
        m = (m < d) ? d : m;
    }
    float const t = block_max_nonneg(m);
    if (threadIdx.x == 0) {
        double const numer = static_cast<double>(factor * support);
        double const denom = sqrt(static_cast<double>(t));
        double const s = safe_d(numer, denom) ? numer / denom : static_cast<double>(1.0f);
        double const f = s * 705600000.0;
        *out = (f > -9.2233720368547758e18 && f < 9.2233720368547758e18) ? static_cast<int64_t>(f)
                                                                          : INT64_MIN;
    }
}

// compute_scalar_average_and_max (emerald/sph_common/common.h:209-240):
// sum of int64(value * discretization) over 1000 * count, and the maximum
// starting from the lowest float.
__global__ void k_average_max(size_t n, float discretization, float const* vals, float* out) {
    long long s = 0;
    float m = kLowest;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        float const v = vals[i];
        s += to_int64_x86(v * discretization);
        m = (m < v) ? v : m;
    }
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        float const other = __shfl_xor_sync(0xffffffffu, m, o);
        m = (m < other) ? other : m;
    }
    __shared__ long long ws[kReduceThreads / 32];
    __shared__ float wm[kReduceThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5] = s;
        wm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        float tm = kLowest;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            t += ws[w];
            tm = (tm < wm[w]) ? wm[w] : tm;
        }
        if (n == 0) {
            out[0] = 0.0f;
            out[1] = 0.0f;
        } else {
            out[0] = static_cast<float>(static_cast<double>(t) / static_cast<double>(1000 * n));
            out[1] = tm;
        }
    }
}

bool ok() { return cudaGetLastError() == cudaSuccess; }

cudaStream_t S(void* st) { return static_cast<cudaStream_t>(st); }

}  // namespace

}  // namespace emerald

using namespace emerald;

extern "C" {

int emerald_compute_grid_coords(size_t n, float cell_size, float bmin_x, float bmin_y,
                                int32_t* grid_coords, float const* positions, void* stream) {
    if (!(cell_size > 0.0f) || (n && (!grid_coords || !positions))) return EMERALD_EINVAL;
    if (n) k_grid_coords<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, cell_size, make_float2(bmin_x, bmin_y), grid_coords, positions);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_z_indices(size_t n, uint64_t* z, int32_t const* grid_coords, void* stream) {
    if (n && (!z || !grid_coords)) return EMERALD_EINVAL;
    if (n) k_z_indices<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, z, grid_coords);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_neighbor_distances_and_vectors_to(size_t n, float* distances,
                                                      float* vectors_to,
                                                      float const* self_positions,
                                                      float const* other_positions,
                                                      uint8_t const* counts,
                                                      uint64_t const* indices, void* stream) {
    if (n && (!distances || !vectors_to || !self_positions || !other_positions || !counts ||
              !indices)) {
        return EMERALD_EINVAL;
    }
    if (n) k_distances_vectors<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, distances, vectors_to, self_positions, other_positions, counts, indices);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_neighbor_kernels(size_t n, float support, float* kernels,
                                     uint8_t const* counts, float const* distances, void* stream) {
    if (!(support > 0.0f) || (n && (!kernels || !counts || !distances))) return EMERALD_EINVAL;
    if (n) k_neighbor_kernels<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, support, kernels,
                                                                         counts, distances);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_neighbor_kernel_gradients(size_t n, float support, float* kernel_gradients,
                                              uint8_t const* counts, float const* vectors_to,
                                              void* stream) {
    if (!(support > 0.0f) || (n && (!kernel_gradients || !counts || !vectors_to))) {
        return EMERALD_EINVAL;
    }
    if (n) k_neighbor_gradients<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, support, kernel_gradients, counts, vectors_to);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_densities(size_t n, float support, float target_density, float* densities,
                              float const* fluid_volumes, emerald_neighborhood fluid,
                              float const* solid_volumes, emerald_neighborhood solid,
                              void* stream) {
    if (!(support > 0.0f) || (n && (!densities || !fluid_volumes || !fluid.counts ||
                                     !fluid.indices || !fluid.kernels))) {
        return EMERALD_EINVAL;
    }
    if (!n) return EMERALD_OK;
    k_densities<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, false, support, target_density,
                                                           densities, fluid_volumes,
                                                           fluid_volumes, fluid);
    if (solid.counts) {
        if (!solid.indices || !solid.kernels || !solid_volumes) return EMERALD_EINVAL;
        k_densities<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, true, support, target_density,
                                                               densities, fluid_volumes,
                                                               solid_volumes, solid);
    }
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_divergences(size_t n, float target_density, float* divergences,
                                float const* fluid_volumes, float const* fluid_velocities,
                                emerald_neighborhood fluid, float const* solid_volumes,
                                float const* solid_velocities, emerald_neighborhood solid,
                                void* stream) {
    if (n && (!divergences || !fluid_volumes || !fluid_velocities || !fluid.counts ||
              !fluid.indices || !fluid.kernel_gradients)) {
        return EMERALD_EINVAL;
    }
    if (!n) return EMERALD_OK;
    k_divergences<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, false, target_density, divergences,
                                                             fluid_velocities, fluid_volumes,
                                                             fluid_velocities, fluid);
    if (solid.counts) {
        if (!solid.indices || !solid.kernel_gradients || !solid_volumes || !solid_velocities) {
            return EMERALD_EINVAL;
        }
        k_divergences<<<blocks_for(n), kThreads, 0, S(stream)>>>(
          n, true, target_density, divergences, fluid_velocities, solid_volumes, solid_velocities,
          solid);
    }
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_predict_density_stars(size_t n, float dt, float target_density, float* density_stars,
                                  float const* densities, float const* fluid_volumes,
                                  float const* fluid_velocities, emerald_neighborhood fluid,
                                  float const* solid_volumes, float const* solid_velocities,
                                  emerald_neighborhood solid, void* stream) {
    int const rc = emerald_compute_divergences(n, target_density, density_stars, fluid_volumes,
                                               fluid_velocities, fluid, solid_volumes,
                                               solid_velocities, solid, stream);
    if (rc != EMERALD_OK || !n) return rc;
    if (!densities) return EMERALD_EINVAL;
    k_density_stars<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, dt, density_stars, densities,
                                                               density_stars);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_apply_pressures_in_place(size_t n, float dt, float target_density, float* velocities,
                                     float const* densities, float const* pressures,
                                     float const* fluid_volumes, emerald_neighborhood fluid,
                                     float const* solid_volumes, emerald_neighborhood solid,
                                     void* stream) {
    if (n && (!velocities || !densities || !pressures || !fluid_volumes || !fluid.counts ||
              !fluid.indices || !fluid.kernel_gradients)) {
        return EMERALD_EINVAL;
    }
    if (!n) return EMERALD_OK;
    k_apply_pressures<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, false, dt, target_density, velocities, densities, pressures, fluid_volumes, fluid);
    if (solid.counts) {
        if (!solid.indices || !solid.kernel_gradients || !solid_volumes) return EMERALD_EINVAL;
        k_apply_pressures<<<blocks_for(n), kThreads, 0, S(stream)>>>(
          n, true, dt, target_density, velocities, densities, pressures, solid_volumes, solid);
    }
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_pressure_accelerations(size_t n, float target_density,
                                           float* pressure_accelerations, float const* pressures,
                                           float const* densities, float const* fluid_volumes,
                                           emerald_neighborhood fluid, float const* solid_volumes,
                                           emerald_neighborhood solid, void* stream) {
    if (n && (!pressure_accelerations || !pressures || !densities || !fluid_volumes ||
              !fluid.counts || !fluid.indices || !fluid.kernel_gradients)) {
        return EMERALD_EINVAL;
    }
    if (!n) return EMERALD_OK;
    k_pressure_accelerations<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, false, target_density, pressure_accelerations, pressures, densities, fluid_volumes, fluid);
    if (solid.counts) {
        if (!solid.indices || !solid.kernel_gradients || !solid_volumes) return EMERALD_EINVAL;
        k_pressure_accelerations<<<blocks_for(n), kThreads, 0, S(stream)>>>(
          n, true, target_density, pressure_accelerations, pressures, densities, solid_volumes,
          solid);
    }
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_integrate_velocities_with_forces(size_t n, float dt, float target_density,
                                             float* velocities, float const* volumes,
                                             float const* forces, void* stream) {
    if (n && (!velocities || !volumes || !forces)) return EMERALD_EINVAL;
    if (n) k_integrate_forces<<<blocks_for(n), kThreads, 0, S(stream)>>>(
      n, dt, target_density, velocities, volumes, forces);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_integrate_velocities(size_t n, float dt, float* velocities,
                                 float const* accelerations, void* stream) {
    if (n && (!velocities || !accelerations)) return EMERALD_EINVAL;
    if (n) k_accumulate<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, dt, velocities,
                                                                   accelerations);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_integrate_positions(size_t n, float dt, float* positions, float const* velocities,
                                void* stream) {
    if (n && (!positions || !velocities)) return EMERALD_EINVAL;
    if (n) k_accumulate<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, dt, positions, velocities);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_compute_constant_volumes(size_t n, float target_density, float mass_per_particle,
                                     float* volumes, void* stream) {
    if (n && !volumes) return EMERALD_EINVAL;
    if (n) k_fill<<<blocks_for(n), kThreads, 0, S(stream)>>>(n, mass_per_particle / target_density,
                                                             volumes);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_max_vector_squared_magnitude(size_t n, float* result, float const* vectors,
                                         void* stream) {
    if (!result || (n && !vectors)) return EMERALD_EINVAL;
    k_max_sq<<<1, kReduceThreads, 0, S(stream)>>>(n, vectors, result);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_max_density_error(size_t n, float target_density, float* result,
                              float const* densities, void* stream) {
    if (!result || (n && !densities)) return EMERALD_EINVAL;
    k_max_density_error<<<1, kReduceThreads, 0, S(stream)>>>(n, target_density, densities, result);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_cfl_maximum_time_step(size_t n, float support, float factor, int64_t* flicks,
                                  float const* velocities, void* stream) {
    if (!flicks || (n && !velocities)) return EMERALD_EINVAL;
    k_cfl<<<1, kReduceThreads, 0, S(stream)>>>(n, support, factor, velocities, flicks);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

int emerald_scalar_average_and_max(size_t n, float discretization, float* average_and_max,
                                   float const* values, void* stream) {
    if (!average_and_max || (n && !values)) return EMERALD_EINVAL;
    k_average_max<<<1, kReduceThreads, 0, S(stream)>>>(n, discretization, values,
                                                       average_and_max);
    return ok() ? EMERALD_OK : EMERALD_ECUDA;
}

}  // extern "C"
