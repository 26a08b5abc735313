// Spatial storage order of the fluid particles.
//
// Every few sub-steps each scene's particles are re-sorted in device memory
// by the Morton key of their grid cell, so that threads of a warp handle
// nearby particles and the neighbour gathers of every kernel hit the same
// cache lines. The reference keeps particles in their original order; this
// engine keeps each particle's original index (oid) beside it and maps back
// wherever the reference's results depend on that order: the within-cell
// member order, the (distance, index) order of neighbour lists, and every
// accessor. Results are therefore independent of the storage order.
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

// Morton key of the cell, relative to a fixed offset and clamped to 12 bits
// per axis (cells outside keep correct results, only their locality drops).
__device__ __forceinline__ uint32_t local_morton(float2 p, float cell) {
    int32_t gx, gy;
    grid_coord(p, cell, gx, gy);
    int32_t const ox = min(max(gx + 64, 0), 4095);
    int32_t const oy = min(max(gy + 64, 0), 4095);
    return static_cast<uint32_t>(morton2(static_cast<uint32_t>(ox), static_cast<uint32_t>(oy)));
}

__global__ void k_order_keys(Arena a, uint64_t* keys, uint32_t* vals, uint32_t n) {
    uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int32_t const s = a.tile_scene[t / kTile];
    uint64_t key = ~0ull;
    if (s >= 0) {
        SceneParams const& P = a.sp[s];
        if (t - P.fluid_begin < P.fluid_count) {
            key = (static_cast<uint64_t>(P.fluid_begin / kTile) << 24) |
                  local_morton(a.x[t], P.cell_size);
        }
    }
    keys[t] = key;
    vals[t] = t;
}

// Moves every real particle from its old slot to its position in the sorted
// order; scenes keep their ranges (the sort's leading key is the scene's
// first tile, and scene s's particles start at sort_base within the sorted
// list).
__global__ void k_permute(Arena a, uint64_t const* keys, uint32_t const* vals, uint32_t n) {
    uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || keys[p] == ~0ull) return;
    uint32_t const old = vals[p];
    int32_t const s = a.tile_scene[old / kTile];
    SceneParams const& P = a.sp[s];
    uint32_t const dst = P.fluid_begin + (p - P.sort_base);
    a.tx[dst] = a.x[old];
    a.tv[dst] = a.v[old];
    a.tkdiv[dst] = a.kdiv[old];
    a.tkdens[dst] = a.kdens[old];
    a.toid[dst] = a.oid[old];
    a.tx64[dst] = a.x64[old];
}

__global__ void k_commit_order(Arena a, uint32_t n) {
    uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int32_t const s = a.tile_scene[t / kTile];
    if (s < 0) return;
    SceneParams const& P = a.sp[s];
    if (t - P.fluid_begin >= P.fluid_count) return;
    a.x[t] = a.tx[t];
    a.v[t] = a.tv[t];
    a.kdiv[t] = a.tkdiv[t];
    a.kdens[t] = a.tkdens[t];
    a.x64[t] = a.tx64[t];
    uint32_t const o = a.toid[t];
    a.oid[t] = o;
    a.slot_of[P.fluid_begin + o] = t;
}

// Original-order views: out[k] = src[slot_of[begin + k]] (gather) and the
// inverse scatter.
__global__ void k_gather_f(Arena a, uint32_t begin, uint32_t count, float const* src, float* out) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = src[a.slot_of[begin + k]];
}
__global__ void k_gather_f2(Arena a, uint32_t begin, uint32_t count, float2 const* src, float2* out) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = src[a.slot_of[begin + k]];
}
__global__ void k_scatter_f2(Arena a, uint32_t begin, uint32_t count, float2 const* in, float2* dst) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[a.slot_of[begin + k]] = in[k];
}
__global__ void k_scatter_f(Arena a, uint32_t begin, uint32_t count, float const* in, float* dst) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[a.slot_of[begin + k]] = in[k];
}
__global__ void k_gather_d2(Arena a, uint32_t begin, uint32_t count, double2 const* src,
                            double2* out) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = src[a.slot_of[begin + k]];
}
__global__ void k_scatter_d2(Arena a, uint32_t begin, uint32_t count, double2 const* in,
                             double2* dst) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[a.slot_of[begin + k]] = in[k];
}

// Sets *flag when any of the n floats is an infinity or a NaN (exponent bits
// all ones).
__global__ void k_flag_nonfinite(float const* p, size_t n, uint32_t* flag) {
    size_t const k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    bool const bad = k < n && (__float_as_uint(p[k]) & 0x7f800000u) == 0x7f800000u;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// Double positions of a scene's particles from their float positions (at
// creation and whenever the caller sets positions).
__global__ void k_positions_to_double(Arena a, uint32_t begin, uint32_t count) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    float2 const p = a.x[begin + k];
    a.x64[begin + k] = make_double2(double(p.x), double(p.y));
}

__global__ void k_identity_order(Arena a, uint32_t begin, uint32_t count) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    a.oid[begin + k] = k;
    a.slot_of[begin + k] = begin + k;
}

}  // namespace

void launch_reorder(Arena const& a, SortScratch& s, uint32_t n, int key_bits, cudaStream_t st) {
    k_order_keys<<<(n + 255) / 256, 256, 0, st>>>(a, s.keys[0], s.vals[0], n);
    int const cur = launch_radix_sort(s, n, key_bits, st);
    k_permute<<<(n + 255) / 256, 256, 0, st>>>(a, s.keys[cur], s.vals[cur], n);
    k_commit_order<<<(n + 255) / 256, 256, 0, st>>>(a, n);
}

void launch_gather_f(Arena const& a, uint32_t begin, uint32_t count, float const* src, float* out,
                     cudaStream_t st) {
    if (count) k_gather_f<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, src, out);
}
void launch_gather_f2(Arena const& a, uint32_t begin, uint32_t count, float2 const* src, float2* out,
                      cudaStream_t st) {
    if (count) k_gather_f2<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, src, out);
}
void launch_scatter_f2(Arena const& a, uint32_t begin, uint32_t count, float2 const* in, float2* dst,
                       cudaStream_t st) {
    if (count) k_scatter_f2<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, in, dst);
}
void launch_scatter_f(Arena const& a, uint32_t begin, uint32_t count, float const* in, float* dst,
                      cudaStream_t st) {
    if (count) k_scatter_f<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, in, dst);
}
void launch_gather_d2(Arena const& a, uint32_t begin, uint32_t count, double2 const* src,
                      double2* out, cudaStream_t st) {
    if (count) k_gather_d2<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, src, out);
}
void launch_scatter_d2(Arena const& a, uint32_t begin, uint32_t count, double2 const* in,
                       double2* dst, cudaStream_t st) {
    if (count) k_scatter_d2<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count, in, dst);
}
void launch_flag_nonfinite(float const* p, size_t n, uint32_t* flag, cudaStream_t st) {
    if (n) k_flag_nonfinite<<<unsigned((n + 255) / 256), 256, 0, st>>>(p, n, flag);
}
void launch_positions_to_double(Arena const& a, uint32_t begin, uint32_t count, cudaStream_t st) {
    if (count) k_positions_to_double<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count);
}
void launch_identity_order(Arena const& a, uint32_t begin, uint32_t count, cudaStream_t st) {
    if (count) k_identity_order<<<(count + 255) / 256, 256, 0, st>>>(a, begin, count);
}

}  // namespace emerald
