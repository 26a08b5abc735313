// The reference's z-order sort and neighbour search functions on device
// memory (emerald/sph_common/neighborhood.h:41-97, neighborhood.cpp:10-152,
// neighborhood.h:199-282), one call each, in the reference's argument order.
//
// std::pair<uint64_t, size_t> arrays (the index pairs and the blocks) are
// interleaved uint64 pairs, which is the reference's own memory layout on
// LP64, so a caller can hand over its arrays byte for byte. The Block_map
// (a TBB concurrent hash map from z key to block) becomes an opaque device
// hash table, emerald_block_map. Every result equals the reference's for the
// same input bit for bit:
// * the pair sort is a stable LSD radix sort on the index, then on the z key,
//   which is the lexicographic order std::sort gives the pairs;
// * block indices are an exclusive scan of "the next pair's z differs";
// * the neighbour search visits the 3x3 cells in the reference's order
//   (rows j - 1 .. j + 1, columns i - 1 .. i + 1, each block in pair order),
//   stops at the 64th accepted candidate as the reference's loops do, and
//   sorts the accepted ones by (distance, index).
// Calls are asynchronous on `stream`; the sort and the block-index scan take
// a caller-allocated device workspace, and a block map allocates (or grows)
// its table when it is filled, as the reference's rehash does.
#include <algorithm>
#include <cstdint>
#include <new>

#include "../../include/emerald_sph.h"
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {
int set_last_error(int code, char const* msg);
}  // namespace emerald

// The device hash table behind one block map: slots (a power of two) keys
// with kEmptyKey marking a free slot, and their (begin, end) ranges; the
// slot after them holds the block whose z key is kEmptyKey itself (cell
// (-1, -1)), present when *full is set.
struct emerald_block_map {
    void* mem = nullptr;
    uint64_t* keys = nullptr;
    uint64_t* ranges = nullptr;
    uint32_t* full = nullptr;
    size_t slots = 0;     // slots of the current table
    size_t capacity = 0;  // slots the allocation holds
    int shift = 0;        // 64 - log2(slots)
    int device = -1;
};

namespace emerald {

namespace {

constexpr int kThreads = 256;
constexpr int kRow = kMaxNeighbors;

cudaStream_t S(void* st) { return static_cast<cudaStream_t>(st); }
unsigned grid(size_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

int cuda_status() {
    cudaError_t const e = cudaGetLastError();
    if (e == cudaSuccess) return EMERALD_OK;
    return set_last_error(EMERALD_ECUDA, cudaGetErrorString(e));
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// workspace: the radix sort's scratch, then a copy of the pairs
size_t workspace_bytes(size_t n) {
    uint32_t const m = static_cast<uint32_t>(std::max<size_t>(n, 1));
    size_t const sort = align256(sort_scratch_bytes(m)) + align256(16 * size_t(m));
    size_t const scan = align256(4 * size_t(m)) + align256(4 * size_t(scan_scratch_words(m) + 16));
    return std::max(sort, scan);
}

// compute_index_pairs (neighborhood.cpp:10-16).
__global__ void k_index_pairs(size_t n, uint64_t* pairs, uint64_t const* z) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    pairs[2 * i] = z[i];
    pairs[2 * i + 1] = i;
}

// First sort key: the pair's index, carrying the pair's position.
__global__ void k_keys_index(uint32_t n, uint64_t const* pairs, uint64_t* copy, uint64_t* keys,
                             uint32_t* vals) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t const z = pairs[2 * size_t(i)];
    uint64_t const idx = pairs[2 * size_t(i) + 1];
    copy[2 * size_t(i)] = z;
    copy[2 * size_t(i) + 1] = idx;
    keys[i] = idx;
    vals[i] = i;
}

// Second sort key: the z key of the pair at each position of the first
// order (read before the slot is rewritten, so in and out may alias).
__global__ void k_keys_z(uint32_t n, uint64_t const* copy, uint32_t const* perm, uint64_t* keys,
                         uint32_t* vals) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t const p = perm[i];
    keys[i] = copy[2 * size_t(p)];
    vals[i] = p;
}

__global__ void k_gather_pairs(uint32_t n, uint64_t const* copy, uint32_t const* perm,
                               uint64_t* pairs) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t const p = perm[i];
    pairs[2 * size_t(i)] = copy[2 * size_t(p)];
    pairs[2 * size_t(i) + 1] = copy[2 * size_t(p) + 1];
}

// 1 where the next pair starts a new block (the scan's input).
__global__ void k_block_breaks(uint32_t n, uint64_t const* pairs, uint32_t* flags) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i + 1 < n && pairs[2 * size_t(i)] != pairs[2 * size_t(i) + 2]) ? 1u : 0u;
}

// fill_blocks (neighborhood.cpp:66-93): a block starts where its index
// first appears and ends where the next index begins.
__global__ void k_fill_blocks(size_t n, uint64_t* blocks, uint32_t const* bi) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    uint32_t const b = bi[i];
    if (i == 0 || bi[i - 1] != b) blocks[2 * size_t(b)] = i;
    if (i + 1 == n || bi[i + 1] != b) blocks[2 * size_t(b) + 1] = i + 1;
}

__device__ __forceinline__ uint64_t slot_of(uint64_t z, int shift) {
    return (z * 0x9E3779B97F4A7C15ull) >> shift;
}

struct MapView {
    uint64_t const* keys;
    uint64_t const* ranges;
    uint32_t const* full;
    uint64_t mask;
    int shift;
};

// create_block_map (neighborhood.cpp:95-110): z key of each block's first
// pair -> the block. A key already present keeps its first block, as
// emplace does.
__global__ void k_map_insert(size_t nblocks, uint64_t const* blocks, uint64_t const* pairs,
                             uint64_t* keys, uint64_t* ranges, uint32_t* full, uint64_t mask,
                             int shift) {
    size_t const b = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (b >= nblocks) return;
    uint64_t const begin = blocks[2 * b];
    uint64_t const end = blocks[2 * b + 1];
    uint64_t const z = pairs[2 * begin];
    if (z == kEmptyKey) {
        if (atomicCAS(full, 0u, 1u) == 0u) {
            ranges[2 * (mask + 1)] = begin;
            ranges[2 * (mask + 1) + 1] = end;
        }
        return;
    }
    uint64_t s = slot_of(z, shift);
    // at most half the slots are taken, so a free slot is always found
    for (uint64_t probe = 0; probe <= mask; ++probe, s = (s + 1) & mask) {
        unsigned long long const prev = atomicCAS(reinterpret_cast<unsigned long long*>(keys + s),
                                                  static_cast<unsigned long long>(kEmptyKey),
                                                  static_cast<unsigned long long>(z));
        if (prev == kEmptyKey) {
            ranges[2 * s] = begin;
            ranges[2 * s + 1] = end;
            return;
        }
        if (prev == z) return;
    }
}

__device__ __forceinline__ bool map_find(MapView const& m, uint64_t z, uint64_t& begin,
                                         uint64_t& end) {
    if (z == kEmptyKey) {
        if (!*m.full) return false;
        begin = m.ranges[2 * (m.mask + 1)];
        end = m.ranges[2 * (m.mask + 1) + 1];
        return true;
    }
    uint64_t s = slot_of(z, m.shift);
    for (uint64_t probe = 0; probe <= m.mask; ++probe, s = (s + 1) & m.mask) {
        uint64_t const k = m.keys[s];
        if (k == z) {
            begin = m.ranges[2 * s];
            end = m.ranges[2 * s + 1];
            return true;
        }
        if (k == kEmptyKey) return false;
    }
    return false;
}

// create_neighborhoods with the accept-all condition
// (neighborhood.cpp:112-136, neighborhood.h:199-282): the accepted
// candidates in visiting order, at most 64, then sorted by (distance,
// index). Entries past a particle's count are left as they were.
__global__ void __launch_bounds__(128)
  k_regular_neighborhoods(size_t n, float max_distance, uint8_t* counts, uint64_t* idx,
                          float* dist, float* vec, float const* self_x, int32_t const* self_gc,
                          float const* other_x, uint64_t const* pairs, MapView map, int same) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float2 const pos = make_float2(self_x[2 * i], self_x[2 * i + 1]);
    int64_t const gx = self_gc[2 * i];
    int64_t const gy = self_gc[2 * i + 1];
    uint64_t ci[kRow];
    float cd[kRow];
    float2 cv[kRow];
    int c = 0;
    for (int64_t j = gy - 1; c < kRow && j <= gy + 1; ++j) {
        for (int64_t k = gx - 1; c < kRow && k <= gx + 1; ++k) {
            uint64_t begin, end;
            if (!map_find(map, morton2(static_cast<uint32_t>(k), static_cast<uint32_t>(j)), begin,
                          end)) {
                continue;
            }
            for (uint64_t sip = begin; c < kRow && sip != end; ++sip) {
                uint64_t const o = pairs[2 * sip + 1];
                if (same && o == i) continue;
                float2 const d = sub2(make_float2(other_x[2 * o], other_x[2 * o + 1]), pos);
                float const r = length2f(d);
                if (r >= max_distance) continue;
                ci[c] = o;
                cd[c] = r;
                cv[c] = d;
                ++c;
            }
        }
    }
    // insertion sort by neighbor_order (neighborhood.h:172-180)
    for (int a = 1; a < c; ++a) {
        uint64_t const ti = ci[a];
        float const td = cd[a];
        float2 const tv = cv[a];
        int b = a - 1;
        while (b >= 0 && (td < cd[b] || (!(td > cd[b]) && ti < ci[b]))) {
            ci[b + 1] = ci[b];
            cd[b + 1] = cd[b];
            cv[b + 1] = cv[b];
            --b;
        }
        ci[b + 1] = ti;
        cd[b + 1] = td;
        cv[b + 1] = tv;
    }
    counts[i] = static_cast<uint8_t>(c);
    for (int k = 0; k < c; ++k) {
        size_t const e = i * kRow + k;
        idx[e] = ci[k];
        dist[e] = cd[k];
        vec[2 * e] = cv[k].x;
        vec[2 * e + 1] = cv[k].y;
    }
}

}  // namespace

}  // namespace emerald

using namespace emerald;

extern "C" {

int emerald_compute_index_pairs(size_t n, uint64_t* index_pairs, uint64_t const* z_indices,
                                void* stream) {
    if (n && (!index_pairs || !z_indices)) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (n) k_index_pairs<<<grid(n), kThreads, 0, S(stream)>>>(n, index_pairs, z_indices);
    return cuda_status();
}

int emerald_index_pairs_workspace(size_t n, size_t* bytes) {
    if (!bytes) return set_last_error(EMERALD_EINVAL, "bytes is NULL");
    if (n >= UINT32_MAX) return set_last_error(EMERALD_EINVAL, "n must be below 2^32 - 1");
    *bytes = workspace_bytes(n);
    return EMERALD_OK;
}

int emerald_sort_index_pairs(size_t n, uint64_t* index_pairs, void* workspace,
                             size_t workspace_size, void* stream) {
    if (n <= 1) return EMERALD_OK;  // neighborhood.cpp:20
    if (n >= UINT32_MAX) return set_last_error(EMERALD_EINVAL, "n must be below 2^32 - 1");
    if (!index_pairs || !workspace) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (workspace_size < workspace_bytes(n)) {
        return set_last_error(EMERALD_EINVAL, "workspace is smaller than emerald_index_pairs_workspace");
    }
    if (reinterpret_cast<uintptr_t>(workspace) % 256 || reinterpret_cast<uintptr_t>(index_pairs) % 8) {
        return set_last_error(EMERALD_EINVAL, "workspace must be 256-byte aligned, pairs 8-byte");
    }
    uint32_t const m = static_cast<uint32_t>(n);
    char* base = static_cast<char*>(workspace);
    SortScratch s;
    sort_scratch_carve(base, m, s);
    uint64_t* copy = reinterpret_cast<uint64_t*>(base + align256(sort_scratch_bytes(m)));
    cudaStream_t const st = S(stream);
    unsigned const g = grid(n);
    k_keys_index<<<g, kThreads, 0, st>>>(m, index_pairs, copy, s.keys[0], s.vals[0]);
    int const a = launch_radix_sort(s, m, 64, st);
    k_keys_z<<<g, kThreads, 0, st>>>(m, copy, s.vals[a], s.keys[0], s.vals[0]);
    int const b = launch_radix_sort(s, m, 64, st);
    k_gather_pairs<<<g, kThreads, 0, st>>>(m, copy, s.vals[b], index_pairs);
    return cuda_status();
}

int emerald_compute_block_indices(size_t n, uint32_t* block_indices,
                                  uint64_t const* sorted_index_pairs, void* workspace,
                                  size_t workspace_size, void* stream) {
    if (n < 1) return EMERALD_OK;  // neighborhood.cpp:33
    if (n >= UINT32_MAX) return set_last_error(EMERALD_EINVAL, "n must be below 2^32 - 1");
    if (!block_indices || !sorted_index_pairs || !workspace) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (workspace_size < workspace_bytes(n)) {
        return set_last_error(EMERALD_EINVAL, "workspace is smaller than emerald_index_pairs_workspace");
    }
    if (reinterpret_cast<uintptr_t>(workspace) % 256) {
        return set_last_error(EMERALD_EINVAL, "workspace must be 256-byte aligned");
    }
    uint32_t const m = static_cast<uint32_t>(n);
    char* base = static_cast<char*>(workspace);
    uint32_t* flags = reinterpret_cast<uint32_t*>(base);
    uint32_t* scratch = reinterpret_cast<uint32_t*>(base + align256(4 * size_t(m)));
    k_block_breaks<<<grid(n), kThreads, 0, S(stream)>>>(m, sorted_index_pairs, flags);
    launch_exclusive_scan(flags, m, block_indices, scratch, S(stream));
    return cuda_status();
}

int emerald_fill_blocks(size_t n, uint64_t* blocks, uint32_t const* block_indices, void* stream) {
    if (n && (!blocks || !block_indices)) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (n) k_fill_blocks<<<grid(n), kThreads, 0, S(stream)>>>(n, blocks, block_indices);
    return cuda_status();
}

int emerald_block_map_create(emerald_block_map** map) {
    if (!map) return set_last_error(EMERALD_EINVAL, "map is NULL");
    *map = new (std::nothrow) emerald_block_map();
    return *map ? EMERALD_OK : set_last_error(EMERALD_ENOMEM, "block map");
}

int emerald_block_map_destroy(emerald_block_map* map) {
    if (!map) return EMERALD_OK;
    if (map->mem) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(map->device);
        cudaFree(map->mem);
        cudaSetDevice(cur);
    }
    delete map;
    return EMERALD_OK;
}

int emerald_create_block_map(size_t block_count, emerald_block_map* into, uint64_t const* blocks,
                             uint64_t const* sorted_index_pairs, void* stream) {
    if (!into) return set_last_error(EMERALD_EINVAL, "map is NULL");
    if (block_count && (!blocks || !sorted_index_pairs)) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (block_count > (size_t(1) << 40)) return set_last_error(EMERALD_EINVAL, "too many blocks");
    int dev = 0;
    cudaGetDevice(&dev);
    // rehash(2 * block_count) (neighborhood.cpp:100): a power of two of at
    // least twice the blocks, so probes always meet a free slot
    size_t slots = 16;
    int log2 = 4;
    while (slots < 2 * block_count) {
        slots <<= 1;
        ++log2;
    }
    cudaStream_t const st = S(stream);
    if (slots > into->capacity || (into->mem && into->device != dev)) {
        if (into->mem) {
            // the old table may still be read by work queued on `stream`
            cudaStreamSynchronize(st);
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(into->device);
            cudaFree(into->mem);
            cudaSetDevice(cur);
            into->mem = nullptr;
        }
        size_t const bytes = 8 * (slots + 1) + 16 * (slots + 1) + 256;
        if (cudaMalloc(&into->mem, bytes) != cudaSuccess) {
            cudaGetLastError();
            into->mem = nullptr;
            into->capacity = 0;
            return set_last_error(EMERALD_ENOMEM, "block map table");
        }
        into->capacity = slots;
        into->device = dev;
    }
    char* base = static_cast<char*>(into->mem);
    into->keys = reinterpret_cast<uint64_t*>(base);
    into->ranges = reinterpret_cast<uint64_t*>(base + 8 * (into->capacity + 1));
    into->full = reinterpret_cast<uint32_t*>(base + 24 * (into->capacity + 1));
    into->slots = slots;
    into->shift = 64 - log2;
    cudaMemsetAsync(into->keys, 0xff, 8 * slots, st);
    cudaMemsetAsync(into->full, 0, sizeof(uint32_t), st);
    if (block_count) {
        k_map_insert<<<grid(block_count), kThreads, 0, st>>>(
          block_count, blocks, sorted_index_pairs, into->keys, into->ranges, into->full,
          uint64_t(slots - 1), into->shift);
    }
    return cuda_status();
}

int emerald_create_regular_neighborhoods(size_t n, float max_distance, uint8_t* counts,
                                         uint64_t* indices, float* distances, float* vectors_to,
                                         float const* self_positions,
                                         int32_t const* self_grid_coords,
                                         float const* other_positions,
                                         uint64_t const* other_sorted_index_pairs,
                                         emerald_block_map const* other_block_map, void* stream) {
    if (!n) return EMERALD_OK;
    if (!counts || !indices || !distances || !vectors_to || !self_positions ||
        !self_grid_coords || !other_positions || !other_sorted_index_pairs) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    if (!other_block_map || !other_block_map->mem) {
        return set_last_error(EMERALD_EINVAL, "the block map was not filled");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (other_block_map->device != dev) {
        return set_last_error(EMERALD_EINVAL, "the block map lives on another device");
    }
    MapView const mv{other_block_map->keys, other_block_map->ranges, other_block_map->full,
                     uint64_t(other_block_map->slots - 1), other_block_map->shift};
    int const same = other_positions == self_positions ? 1 : 0;
    k_regular_neighborhoods<<<static_cast<unsigned>((n + 127) / 128), 128, 0, S(stream)>>>(
      n, max_distance, counts, indices, distances, vectors_to, self_positions, self_grid_coords,
      other_positions, other_sorted_index_pairs, mv, same);
    return cuda_status();
}

}  // extern "C"
