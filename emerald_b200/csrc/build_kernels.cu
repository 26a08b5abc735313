// Neighbour build on the GPU: Morton keys, cell binning, cell ranges and the
// per-particle neighbour lists of emerald/sph_common/neighborhood.{h,cpp}.
//
// The reference sorts (z, index) pairs and keeps a hash map from z to the
// [begin, end) range of each cell (neighborhood.cpp:10-124). Here each scene
// has an open-addressing table keyed by z; binning counts the members of
// every cell, an exclusive scan turns the counts into ranges, and each
// cell's member list is ordered by index, which is exactly the order the
// sorted pairs give inside a cell. The neighbour search then walks the 3x3
// cells in the reference's row-major order, keeps the first 64 accepted
// candidates and orders them by (distance, index) (neighborhood.h:199-282),
// so the lists are bit-identical.
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

__device__ __forceinline__ uint32_t cell_hash(uint64_t z, uint32_t log2cap) {
    return static_cast<uint32_t>((z * 0x9E3779B97F4A7C15ull) >> (64u - log2cap));
}

// Inserts z into the table (capacity 2^log2cap plus one extra slot reserved
// for z == kEmptyKey, the key of cell (-1, -1)). Returns the slot or
// UINT32_MAX when the table is full; the probe loop is bounded.
__device__ uint32_t table_insert(uint64_t* keys, uint32_t log2cap, uint64_t z) {
    uint32_t const cap = 1u << log2cap;
    if (z == kEmptyKey) return cap;
    uint32_t h = cell_hash(z, log2cap);
    for (uint32_t probe = 0; probe < cap; ++probe) {
        unsigned long long const prev = atomicCAS(
          reinterpret_cast<unsigned long long*>(keys + h), kEmptyKey, z);
        if (prev == kEmptyKey || prev == z) return h;
        h = (h + 1u) & (cap - 1u);
    }
    return UINT32_MAX;
}

__device__ __forceinline__ bool table_find(uint64_t const* keys,
                                           uint32_t log2cap,
                                           uint64_t z,
                                           uint32_t& slot) {
    uint32_t const cap = 1u << log2cap;
    if (z == kEmptyKey) {
        slot = cap;
        return true;
    }
    uint32_t h = cell_hash(z, log2cap);
    for (uint32_t probe = 0; probe < cap; ++probe) {
        uint64_t const k = keys[h];
        if (k == z) {
            slot = h;
            return true;
        }
        if (k == kEmptyKey) return false;
        h = (h + 1u) & (cap - 1u);
    }
    return false;
}

struct OtherSet {
    float2 const* x;
    uint64_t const* keys;
    uint32_t const* count;
    uint32_t const* start;
    uint32_t const* members;
    uint32_t log2cap;
    uint32_t begin;
    uint32_t const* oid;      // original index of a stored slot (nullptr: slot - begin)
    uint32_t const* slot_of;  // stored slot of an original index (nullptr: begin + oid)
};

__device__ __forceinline__ uint32_t original_index(OtherSet const& o, uint32_t slot) {
    return o.oid ? o.oid[slot] : slot - o.begin;
}
__device__ __forceinline__ uint32_t stored_slot(OtherSet const& o, uint32_t oid) {
    return o.slot_of ? o.slot_of[o.begin + oid] : o.begin + oid;
}

// The neighbour search of create_neighborhoods
// (emerald/sph_common/neighborhood.h:199-282). Accepted candidates are kept
// in `list` as (distance bits << 32 | scene-local index), sorted ascending,
// which is the reference's (distance, index) order for non-negative
// distances. Returns the count.
__device__ int find_neighbors(float2 pos,
                              uint32_t self,
                              bool same_set,
                              float cell,
                              float max_distance,
                              OtherSet const& o,
                              uint64_t (&list)[kMaxNeighbors]) {
    int32_t gx, gy;
    grid_coord(pos, cell, gx, gy);
    int cnt = 0;
    for (int32_t j = gy - 1; cnt < kMaxNeighbors && j <= gy + 1; ++j) {
        for (int32_t k = gx - 1; cnt < kMaxNeighbors && k <= gx + 1; ++k) {
            uint32_t slot;
            uint64_t const z = morton2(static_cast<uint32_t>(k), static_cast<uint32_t>(j));
            if (!table_find(o.keys, o.log2cap, z, slot)) continue;
            uint32_t const b = o.start[slot];
            uint32_t const e = b + o.count[slot];
            for (uint32_t m = b; cnt < kMaxNeighbors && m != e; ++m) {
                uint32_t const other = o.members[m];
                if (same_set && other == self) continue;
                float2 const vec = sub2(o.x[other], pos);
                float const dist = length2f(vec);
                if (dist >= max_distance) continue;
                uint64_t const key = (static_cast<uint64_t>(__float_as_uint(dist)) << 32) |
                                     static_cast<uint64_t>(original_index(o, other));
                int p = cnt;
                while (p > 0 && list[p - 1] > key) {
                    list[p] = list[p - 1];
                    --p;
                }
                list[p] = key;
                ++cnt;
            }
        }
    }
    return cnt;
}

template <bool SOLID>
__global__ void k_bin(Arena a) {
    int32_t const s = (SOLID ? a.stile_scene : a.tile_scene)[blockIdx.x];
    if (s < 0) return;
    SceneParams const& P = a.sp[s];
    if (!SOLID && !a.ss[s].active) return;
    uint32_t const i = blockIdx.x * kTile + threadIdx.x;
    uint32_t const begin = SOLID ? P.solid_begin : P.fluid_begin;
    uint32_t const count = SOLID ? P.solid_count : P.fluid_count;
    if (i - begin >= count) return;
    float2 const p = SOLID ? a.xs[i] : a.x[i];
    int32_t gx, gy;
    grid_coord(p, P.cell_size, gx, gy);
    uint64_t const z = morton2(static_cast<uint32_t>(gx), static_cast<uint32_t>(gy));
    (SOLID ? a.szkey : a.zkey)[i] = z;
    uint32_t const tb = SOLID ? P.stab_begin : P.ftab_begin;
    uint32_t const lg = SOLID ? P.stab_log2 : P.ftab_log2;
    uint32_t const slot = table_insert((SOLID ? a.skeys : a.fkeys) + tb, lg, z);
    uint32_t* out_slot = SOLID ? a.sslot : a.slot;
    if (slot == UINT32_MAX) {
        atomicOr(&a.ss[s].error, kErrTableFull);
        out_slot[i] = UINT32_MAX;
        return;
    }
    uint32_t const r = atomicAdd((SOLID ? a.scount : a.fcount) + tb + slot, 1u);
    out_slot[i] = tb + slot;
    (SOLID ? a.srank : a.rank)[i] = r;
}

template <bool SOLID>
__global__ void k_scatter(Arena a) {
    int32_t const s = (SOLID ? a.stile_scene : a.tile_scene)[blockIdx.x];
    if (s < 0) return;
    SceneParams const& P = a.sp[s];
    if (!SOLID && !a.ss[s].active) return;
    uint32_t const i = blockIdx.x * kTile + threadIdx.x;
    uint32_t const begin = SOLID ? P.solid_begin : P.fluid_begin;
    uint32_t const count = SOLID ? P.solid_count : P.fluid_count;
    if (i - begin >= count) return;
    uint32_t const slot = (SOLID ? a.sslot : a.slot)[i];
    if (slot == UINT32_MAX) return;
    uint32_t const pos = (SOLID ? a.sstart : a.fstart)[slot] + (SOLID ? a.srank : a.rank)[i];
    (SOLID ? a.smembers : a.members)[pos] = i;
}

// Orders every cell's members by original index (the within-cell order of
// the reference's sorted (z, index) pairs). oid may be nullptr (storage order
// is the original order).
__global__ void k_sort_cells(uint32_t const* count,
                             uint32_t const* start,
                             uint32_t* members,
                             uint32_t const* oid,
                             uint32_t total) {
    uint32_t const e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    uint32_t const c = count[e];
    if (c < 2) return;
    uint32_t* m = members + start[e];
    for (uint32_t q = 1; q < c; ++q) {
        uint32_t const v = m[q];
        uint32_t const kv = oid ? oid[v] : v;
        uint32_t p = q;
        while (p > 0 && (oid ? oid[m[p - 1]] : m[p - 1]) > kv) {
            m[p] = m[p - 1];
            --p;
        }
        m[p] = v;
    }
}

// Registers that hold a particle's sorted list on the common path.
constexpr int kRegList = 16;

// The search of find_neighbors with the sorted list in registers: every
// accepted key bubbles through kRegList registers (min/max exchange, static
// indices, so nothing spills). A candidate is rejected before its square root
// when x*x + y*y >= reject_l2: sqrtf is correctly rounded and monotone, so
// that test equals the reference's length() >= max_distance for every
// non-tiny vector, and tiny vectors (dot < 2*FLT_MIN) are far below it.
// Returns the accepted count; above kRegList the registers overflowed and the
// caller redoes the particle with the 64-entry list.
__device__ __forceinline__ int find_neighbors_reg(float2 pos, uint32_t self, bool same_set,
                                                  float cell, float max_distance, float reject_l2,
                                                  OtherSet const& o, uint64_t (&r)[kRegList]) {
#pragma unroll
    for (int q = 0; q < kRegList; ++q) r[q] = ~0ull;
    int32_t gx, gy;
    grid_coord(pos, cell, gx, gy);
    uint64_t const sx0 = spread_bits(static_cast<uint32_t>(gx - 1));
    uint64_t const sx1 = spread_bits(static_cast<uint32_t>(gx));
    uint64_t const sx2 = spread_bits(static_cast<uint32_t>(gx + 1));
    uint64_t const sy0 = spread_bits(static_cast<uint32_t>(gy - 1)) << 1;
    uint64_t const sy1 = spread_bits(static_cast<uint32_t>(gy)) << 1;
    uint64_t const sy2 = spread_bits(static_cast<uint32_t>(gy + 1)) << 1;
    int cnt = 0;
#pragma unroll 1
    for (int jj = 0; jj < 3 && cnt < kMaxNeighbors; ++jj) {
        uint64_t const zy = jj == 0 ? sy0 : (jj == 1 ? sy1 : sy2);
#pragma unroll 1
        for (int kk = 0; kk < 3 && cnt < kMaxNeighbors; ++kk) {
            uint64_t const zx = kk == 0 ? sx0 : (kk == 1 ? sx1 : sx2);
            uint32_t slot;
            if (!table_find(o.keys, o.log2cap, zx | zy, slot)) continue;
            uint32_t const b = o.start[slot];
            uint32_t const e = b + o.count[slot];
#pragma unroll 1
            for (uint32_t m = b; cnt < kMaxNeighbors && m != e; ++m) {
                uint32_t const other = o.members[m];
                if (same_set && other == self) continue;
                float2 const vec = sub2(o.x[other], pos);
                if (vec.x * vec.x + vec.y * vec.y >= reject_l2) continue;
                float const dist = length2f(vec);
                if (dist >= max_distance) continue;
                uint64_t key = (static_cast<uint64_t>(__float_as_uint(dist)) << 32) |
                               static_cast<uint64_t>(original_index(o, other));
#pragma unroll
                for (int q = 0; q < kRegList; ++q) {
                    uint64_t const lo = r[q] < key ? r[q] : key;
                    key = r[q] < key ? key : r[q];
                    r[q] = lo;
                }
                ++cnt;
            }
        }
    }
    return cnt;
}

// Candidates whose member indices, then positions, the shared-memory search
// loads together before it tests them in order.
constexpr int kNeighborBatch = 4;

// The [begin, end) member ranges of the three cells (zx_k | zy) of one row:
// the three first probes are loaded together, then each is resolved (linear
// probing from there, bounded by the capacity), as table_find does.
__device__ __forceinline__ void row_ranges(OtherSet const& o, uint64_t zx0, uint64_t zx1,
                                           uint64_t zx2, uint64_t zy, uint32_t (&b)[3],
                                           uint32_t (&e)[3]) {
    uint32_t const cap = 1u << o.log2cap;
    uint64_t const z[3] = {zx0 | zy, zx1 | zy, zx2 | zy};
    uint32_t h[3];
    uint64_t k[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) h[q] = cell_hash(z[q], o.log2cap);
#pragma unroll
    for (int q = 0; q < 3; ++q) k[q] = (z[q] == kEmptyKey) ? kEmptyKey : o.keys[h[q]];
    uint32_t slot[3] = {0u, 0u, 0u};
    bool found[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        if (z[q] == kEmptyKey) {
            slot[q] = cap;
            found[q] = true;
        } else if (k[q] == z[q]) {
            slot[q] = h[q];
            found[q] = true;
        } else if (k[q] == kEmptyKey) {
            found[q] = false;
        } else {
            uint32_t hh = h[q];
            found[q] = false;
            for (uint32_t probe = 1; probe < cap; ++probe) {
                hh = (hh + 1u) & (cap - 1u);
                uint64_t const kk = o.keys[hh];
                if (kk == z[q]) {
                    slot[q] = hh;
                    found[q] = true;
                    break;
                }
                if (kk == kEmptyKey) break;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        b[q] = found[q] ? o.start[slot[q]] : 0u;
        e[q] = found[q] ? b[q] + o.count[slot[q]] : 0u;
    }
}

// The search of find_neighbors_reg with the sorted list in shared memory:
// entry k of this thread at list[k * kTile]; an accepted key shifts only the
// entries above it (fewer instructions than the register bubble). The three
// cells of a row are looked up together, and each cell's members are taken
// kNeighborBatch at a time (their indices, then their positions, then the
// tests in member order): the candidates and their order are those of the
// one-at-a-time walk, with fewer dependent loads in a row (measured 20%
// faster on B200). Above kRegList entries the caller redoes the particle
// with the 64-entry list.
__device__ __forceinline__ int find_neighbors_smem(float2 pos, uint32_t self, bool same_set,
                                                   float cell, float max_distance, float reject_l2,
                                                   OtherSet const& o, uint64_t* list) {
    int32_t gx, gy;
    grid_coord(pos, cell, gx, gy);
    uint64_t const sx0 = spread_bits(static_cast<uint32_t>(gx - 1));
    uint64_t const sx1 = spread_bits(static_cast<uint32_t>(gx));
    uint64_t const sx2 = spread_bits(static_cast<uint32_t>(gx + 1));
    int cnt = 0;
#pragma unroll 1
    for (int jj = 0; jj < 3 && cnt < kMaxNeighbors; ++jj) {
        uint64_t const zy = spread_bits(static_cast<uint32_t>(gy - 1 + jj)) << 1;
        uint32_t rb[3], re[3];
        row_ranges(o, sx0, sx1, sx2, zy, rb, re);
#pragma unroll 1
        for (int kk = 0; kk < 3 && cnt < kMaxNeighbors; ++kk) {
            uint32_t const e = re[kk];
#pragma unroll 1
            for (uint32_t m0 = rb[kk]; m0 < e && cnt < kMaxNeighbors; m0 += kNeighborBatch) {
                uint32_t oth[kNeighborBatch];
                float2 xo[kNeighborBatch];
#pragma unroll
                for (int u = 0; u < kNeighborBatch; ++u) {
                    if (m0 + u < e) oth[u] = o.members[m0 + u];
                }
#pragma unroll
                for (int u = 0; u < kNeighborBatch; ++u) {
                    if (m0 + u < e) xo[u] = o.x[oth[u]];
                }
#pragma unroll
                for (int u = 0; u < kNeighborBatch; ++u) {
                    if (m0 + u >= e || cnt >= kMaxNeighbors) break;
                    uint32_t const other = oth[u];
                    if (same_set && other == self) continue;
                    float2 const vec = sub2(xo[u], pos);
                    if (vec.x * vec.x + vec.y * vec.y >= reject_l2) continue;
                    float const dist = length2f(vec);
                    if (dist >= max_distance) continue;
                    uint64_t const key = (static_cast<uint64_t>(__float_as_uint(dist)) << 32) |
                                         static_cast<uint64_t>(original_index(o, other));
                    if (cnt < kRegList) {
                        int p = cnt;
                        while (p > 0) {
                            uint64_t const prev = list[(p - 1) * kTile];
                            if (prev < key) break;
                            list[p * kTile] = prev;
                            --p;
                        }
                        list[p * kTile] = key;
                    }
                    ++cnt;
                }
            }
        }
    }
    return cnt;
}

// Writes list entry k of particle i: index, W and GradW(-vector_to)
// (compute_neighbor_kernels / compute_neighbor_kernel_gradients,
// emerald/sph_common/neighborhood.cpp:178-210), the vector recomputed from
// positions bit for bit and its length taken from the search.
__device__ __forceinline__ void write_entry(uint32_t* idx_out, float* w_out, float2* gw_out,
                                            size_t e, uint32_t j, float dist, float2 pos,
                                            float2 const* xo, float h, bool kernels) {
    idx_out[e] = j;
    if (!kernels) return;
    float w, dw;
    kernel_w_dw(dist, h, w, dw);
    w_out[e] = w;
    float2 const dp = neg2(sub2(xo[j], pos));
    float2 g = mk2(0.0f, 0.0f);
    if (safe_v(dp, dist)) {
        float2 const u = div2(dp, dist);
        g = mk2(u.x * dw, u.y * dw);
    }
    gw_out[e] = g;
}

// Compensated mode: the entry's vector and distance come from the double
// positions (x_i - x_j in double, rounded once), so that the rounding of
// large coordinates does not enter the kernel values.
__device__ __noinline__ void write_entry_precise(uint32_t* idx_out, float* w_out, float2* gw_out,
                                                 size_t e, uint32_t j, double2 pos64,
                                                 double2 const* x64o, float2 const* xo, float h) {
    idx_out[e] = j;
    double2 const xj = x64o ? x64o[j] : make_double2(double(xo[j].x), double(xo[j].y));
    double const ddx = pos64.x - xj.x;
    double const ddy = pos64.y - xj.y;
    float2 const dp = mk2(static_cast<float>(ddx), static_cast<float>(ddy));
    float const dist = static_cast<float>(sqrt(ddx * ddx + ddy * ddy));
    float w, dw;
    kernel_w_dw(dist, h, w, dw);
    w_out[e] = w;
    float2 g = mk2(0.0f, 0.0f);
    if (safe_v(dp, dist)) {
        float2 const u = div2(dp, dist);
        g = mk2(u.x * dw, u.y * dw);
    }
    gw_out[e] = g;
}

template <bool SOLID_OTHER, bool COMP>
__global__ void __launch_bounds__(kTile) k_neighbors(Arena a, int write_kernels) {
    int32_t const s = a.tile_scene[blockIdx.x];
    if (s < 0) return;
    SceneParams const& P = a.sp[s];
    if (!a.ss[s].active) return;
    uint32_t const i = blockIdx.x * kTile + threadIdx.x;
    if (i - P.fluid_begin >= P.fluid_count) return;
    float const h = P.support;
    float const cell = P.cell_size;
    OtherSet o;
    if (SOLID_OTHER) {
        o = OtherSet{a.xs, a.skeys + P.stab_begin, a.scount + P.stab_begin, a.sstart + P.stab_begin,
                     a.smembers, P.stab_log2, P.solid_begin, nullptr, nullptr};
    } else {
        o = OtherSet{a.x, a.fkeys + P.ftab_begin, a.fcount + P.ftab_begin, a.fstart + P.ftab_begin,
                     a.members, P.ftab_log2, P.fluid_begin, a.oid, a.slot_of};
    }
    uint8_t* cnt_out = SOLID_OTHER ? a.ns_cnt : a.nf_cnt;
    uint32_t* idx_out = SOLID_OTHER ? a.ns_idx : a.nf_idx;
    float* w_out = SOLID_OTHER ? a.ns_w : a.nf_w;
    float2* gw_out = SOLID_OTHER ? a.ns_gw : a.nf_gw;
    size_t const stride = a.stride;
    if (SOLID_OTHER && P.solid_count == 0) {
        cnt_out[i] = 0;
        return;
    }
    bool const kernels = write_kernels != 0;
    float2 const pos = a.x[i];
    if (SOLID_OTHER && P.near_w) {
        int32_t gx, gy;
        grid_coord(pos, cell, gx, gy);
        int64_t const ix = int64_t(gx) - P.near_x0;
        int64_t const iy = int64_t(gy) - P.near_y0;
        bool near = false;
        if (ix >= 0 && iy >= 0 && ix < int64_t(P.near_w) && iy < int64_t(P.near_h)) {
            uint64_t const bit = uint64_t(iy) * P.near_w + uint64_t(ix);
            near = (a.near_bits[P.near_begin + (bit >> 5)] >> (bit & 31u)) & 1u;
        }
        if (!near) {
            cnt_out[i] = 0;
            return;
        }
    }
    if (!(COMP && P.precision && kernels)) {
        __shared__ uint64_t s_list[kRegList * kTile];
        uint64_t* const list = s_list + threadIdx.x;
        int const cnt = find_neighbors_smem(pos, i, !SOLID_OTHER, cell, cell, P.reject_l2, o, list);
        cnt_out[i] = static_cast<uint8_t>(cnt);
        if (cnt <= kRegList) {
#pragma unroll 1
            for (int k = 0; k < cnt; ++k) {
                uint64_t const key = list[k * kTile];
                write_entry(idx_out, w_out, gw_out, static_cast<size_t>(k) * stride + i,
                            stored_slot(o, static_cast<uint32_t>(key & 0xffffffffu)),
                            __uint_as_float(static_cast<uint32_t>(key >> 32)), pos, o.x, h,
                            kernels);
            }
            return;
        }
        uint64_t full[kMaxNeighbors];
        int const n64 = find_neighbors(pos, i, !SOLID_OTHER, cell, cell, o, full);
#pragma unroll 1
        for (int k = 0; k < n64; ++k) {
            write_entry(idx_out, w_out, gw_out, static_cast<size_t>(k) * stride + i,
                        stored_slot(o, static_cast<uint32_t>(full[k] & 0xffffffffu)),
                        __uint_as_float(static_cast<uint32_t>(full[k] >> 32)), pos, o.x, h,
                        kernels);
        }
        return;
    }
    // compensated scenes: the register list, with entries from double positions
    uint64_t r[kRegList];
    int const cnt = find_neighbors_reg(pos, i, !SOLID_OTHER, cell, cell, P.reject_l2, o, r);
    cnt_out[i] = static_cast<uint8_t>(cnt);
    if (COMP && P.precision && kernels) {
        double2 const pos64 = a.x64[i];
        double2 const* x64o = SOLID_OTHER ? nullptr : a.x64;
        uint64_t full[kMaxNeighbors];
        int const n64 = cnt <= kRegList ? cnt : find_neighbors(pos, i, !SOLID_OTHER, cell, cell, o, full);
#pragma unroll 1
        for (int k = 0; k < n64; ++k) {
            uint64_t key;
            if (cnt <= kRegList) {
                key = r[0];
#pragma unroll
                for (int q = 0; q + 1 < kRegList; ++q) r[q] = r[q + 1];
            } else {
                key = full[k];
            }
            write_entry_precise(idx_out, w_out, gw_out, static_cast<size_t>(k) * stride + i,
                                stored_slot(o, static_cast<uint32_t>(key & 0xffffffffu)), pos64,
                                x64o, o.x, h);
        }
        return;
    }
    if (cnt <= kRegList) {
        // drain the sorted registers from the front: one copy of the entry
        // code, register moves instead of dynamic indexing
#pragma unroll 1
        for (int k = 0; k < cnt; ++k) {
            uint64_t const key = r[0];
#pragma unroll
            for (int q = 0; q + 1 < kRegList; ++q) r[q] = r[q + 1];
            write_entry(idx_out, w_out, gw_out, static_cast<size_t>(k) * stride + i,
                        stored_slot(o, static_cast<uint32_t>(key & 0xffffffffu)),
                        __uint_as_float(static_cast<uint32_t>(key >> 32)), pos, o.x, h, kernels);
        }
        return;
    }
    // more than kRegList neighbours: the full 64-entry list
    uint64_t full[kMaxNeighbors];
    int const n64 = find_neighbors(pos, i, !SOLID_OTHER, cell, cell, o, full);
#pragma unroll 1
    for (int k = 0; k < n64; ++k) {
        write_entry(idx_out, w_out, gw_out, static_cast<size_t>(k) * stride + i,
                    stored_slot(o, static_cast<uint32_t>(full[k] & 0xffffffffu)),
                    __uint_as_float(static_cast<uint32_t>(full[k] >> 32)), pos, o.x, h, kernels);
    }
}

// compute_volumes (emerald/sph2d_box/solids.cpp:52-74) over the solid-solid
// neighbourhood of compute_neighbor_data_and_volumes (:76-137):
// V = numer / (W(0) + sum W) in list order, 1/W(0) without neighbours.
__global__ void k_solid_volumes(Arena a, float numer, int only_scene) {
    int32_t const s = a.stile_scene[blockIdx.x];
    if (s < 0 || s != only_scene) return;
    SceneParams const& P = a.sp[s];
    uint32_t const i = blockIdx.x * kTile + threadIdx.x;
    if (i - P.solid_begin >= P.solid_count) return;
    OtherSet const o{a.xs, a.skeys + P.stab_begin, a.scount + P.stab_begin, a.sstart + P.stab_begin,
                     a.smembers, P.stab_log2, P.solid_begin, nullptr, nullptr};
    uint64_t list[kMaxNeighbors];
    int const cnt = find_neighbors(a.xs[i], i, true, P.cell_size, P.cell_size, o, list);
    float const w0 = kernel_w(0.0f, P.support);
    if (!cnt) {
        a.vols[i] = 1.0f / w0;
        return;
    }
    float m = w0;
    for (int k = 0; k < cnt; ++k) {
        m += kernel_w(__uint_as_float(static_cast<uint32_t>(list[k] >> 32)), P.support);
    }
    a.vols[i] = numer / m;
}

// Exclusive scan of uint32 counts: per-block sums, a single-block scan of
// the sums, then per-block scans offset by the scanned sums.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    int const lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t const t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& excl) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    uint32_t const incl = warp_inclusive_scan(v);
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0u;
        w = warp_inclusive_scan(w);
        if (lane < kScanThreads / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t const warp_off = warp ? warp_sums[warp - 1] : 0u;
    excl = warp_off + incl - v;
    uint32_t const total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return total;
}

__global__ void k_scan_reduce(uint32_t const* in, uint32_t n, uint32_t* sums) {
    size_t const base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * kScanItems;
    uint32_t t = 0;
    for (int k = 0; k < kScanItems; ++k) {
        size_t const e = base + k;
        if (e < n) t += in[e];
    }
    uint32_t excl;
    uint32_t const total = block_exclusive_scan(t, excl);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* sums, uint32_t nblocks) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nblocks; base += kScanThreads) {
        uint32_t const e = base + threadIdx.x;
        uint32_t const v = e < nblocks ? sums[e] : 0u;
        uint32_t excl;
        uint32_t const total = block_exclusive_scan(v, excl);
        if (e < nblocks) sums[e] = carry + excl;
        carry += total;
    }
}

__global__ void k_scan_apply(uint32_t const* in, uint32_t n, uint32_t const* sums, uint32_t* out) {
    size_t const base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * kScanItems;
    uint32_t vals[kScanItems];
    uint32_t t = 0;
    for (int k = 0; k < kScanItems; ++k) {
        size_t const e = base + k;
        vals[k] = e < n ? in[e] : 0u;
        t += vals[k];
    }
    uint32_t excl;
    block_exclusive_scan(t, excl);
    uint32_t run = sums[blockIdx.x] + excl;
    for (int k = 0; k < kScanItems; ++k) {
        size_t const e = base + k;
        if (e < n) out[e] = run;
        run += vals[k];
    }
}

// Cell ranges in one pass: every block scans its slots' counts and takes its
// range of the members array with one atomic on the cursor count[n], which
// the caller cleared with the counts. Cells land in block order, not slot
// order; each cell's members stay contiguous, which is all the searches and
// the sort products read (start[cell], count[cell]).
__global__ void k_cell_ranges(uint32_t const* count, uint32_t n, uint32_t* start) {
    size_t const base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * kScanItems;
    uint32_t vals[kScanItems];
    uint32_t t = 0;
    for (int k = 0; k < kScanItems; ++k) {
        size_t const e = base + k;
        vals[k] = e < n ? count[e] : 0u;
        t += vals[k];
    }
    uint32_t excl;
    uint32_t const total = block_exclusive_scan(t, excl);
    __shared__ uint32_t block_base;
    if (threadIdx.x == 0) {
        block_base = total ? atomicAdd(const_cast<uint32_t*>(count) + n, total) : 0u;
    }
    __syncthreads();
    uint32_t run = block_base + excl;
    for (int k = 0; k < kScanItems; ++k) {
        size_t const e = base + k;
        if (e < n) start[e] = run;
        run += vals[k];
    }
}

}  // namespace

uint32_t scan_scratch_words(uint32_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

void launch_exclusive_scan(uint32_t const* in, uint32_t n, uint32_t* out, uint32_t* scratch,
                           cudaStream_t st) {
    if (n == 0) return;
    uint32_t const nb = (n + kScanBlock - 1) / kScanBlock;
    k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, n, scratch);
    k_scan_sums<<<1, kScanThreads, 0, st>>>(scratch, nb);
    k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, n, scratch, out);
}

// The count arrays hold one word more than the table: the cursor of
// k_cell_ranges, cleared with the counts.
void launch_build_cells(Arena const& a, bool solid, uint32_t tiles, uint32_t* scan_scratch,
                        cudaStream_t st) {
    (void)scan_scratch;
    if (solid) {
        cudaMemsetAsync(a.skeys, 0xff, sizeof(uint64_t) * a.stab_total, st);
        cudaMemsetAsync(a.scount, 0, sizeof(uint32_t) * (a.stab_total + 1), st);
        k_bin<true><<<tiles, kTile, 0, st>>>(a);
        k_cell_ranges<<<(a.stab_total + kScanBlock - 1) / kScanBlock, kScanThreads, 0, st>>>(
          a.scount, a.stab_total, a.sstart);
        k_scatter<true><<<tiles, kTile, 0, st>>>(a);
        k_sort_cells<<<(a.stab_total + 255) / 256, 256, 0, st>>>(a.scount, a.sstart, a.smembers,
                                                                 nullptr, a.stab_total);
    } else {
        cudaMemsetAsync(a.fkeys, 0xff, sizeof(uint64_t) * a.ftab_total, st);
        cudaMemsetAsync(a.fcount, 0, sizeof(uint32_t) * (a.ftab_total + 1), st);
        k_bin<false><<<tiles, kTile, 0, st>>>(a);
        k_cell_ranges<<<(a.ftab_total + kScanBlock - 1) / kScanBlock, kScanThreads, 0, st>>>(
          a.fcount, a.ftab_total, a.fstart);
        k_scatter<false><<<tiles, kTile, 0, st>>>(a);
        k_sort_cells<<<(a.ftab_total + 255) / 256, 256, 0, st>>>(a.fcount, a.fstart, a.members,
                                                                 a.oid, a.ftab_total);
    }
}

void launch_neighbors(Arena const& a, uint32_t tiles, bool solid_other, bool write_kernels,
                      cudaStream_t st, bool comp) {
    int const wk = write_kernels ? 1 : 0;
    if (solid_other) {
        if (comp) {
            k_neighbors<true, true><<<tiles, kTile, 0, st>>>(a, wk);
        } else {
            k_neighbors<true, false><<<tiles, kTile, 0, st>>>(a, wk);
        }
    } else {
        if (comp) {
            k_neighbors<false, true><<<tiles, kTile, 0, st>>>(a, wk);
        } else {
            k_neighbors<false, false><<<tiles, kTile, 0, st>>>(a, wk);
        }
    }
}

void launch_solid_volumes(Arena const& a, uint32_t solid_tiles, float numer, int scene,
                          cudaStream_t st) {
    k_solid_volumes<<<solid_tiles, kTile, 0, st>>>(a, numer, scene);
}

}  // namespace emerald
