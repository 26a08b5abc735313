// Stable LSD radix sort of (u64 key, u32 value) pairs and the reference's
// z-order sort products (emerald/sph_common/neighborhood.cpp:10-106).
//
// The step itself never needs a global z-sorted order: cells are found
// through the per-scene hash tables. The sorted (z, index) pairs, block
// indices and block ranges are produced here when a caller asks for them,
// by sorting the occupied cells by z and expanding each cell's (already
// index-ordered) member list.
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr int kThreads = 256;
constexpr int kRounds = 8;
constexpr int kItems = kThreads * kRounds;  // keys per block and pass
constexpr int kDigits = 256;

__global__ void k_hist(uint64_t const* keys, uint32_t n, int shift, uint32_t* hist, uint32_t nblocks) {
    __shared__ uint32_t cnt[kDigits];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    size_t const base = static_cast<size_t>(blockIdx.x) * kItems;
    for (int r = 0; r < kRounds; ++r) {
        size_t const e = base + static_cast<size_t>(r) * kThreads + threadIdx.x;
        if (e < n) atomicAdd(&cnt[(keys[e] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[static_cast<size_t>(threadIdx.x) * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void k_rank_scatter(uint64_t const* kin, uint32_t const* vin, uint64_t* kout,
                               uint32_t* vout, uint32_t n, int shift, uint32_t const* offsets,
                               uint32_t nblocks) {
    __shared__ uint32_t base[kDigits];
    __shared__ uint32_t wcnt[kThreads / 32][kDigits];
    base[threadIdx.x] = offsets[static_cast<size_t>(threadIdx.x) * nblocks + blockIdx.x];
    int const lane = threadIdx.x & 31;
    int const warp = threadIdx.x >> 5;
    uint32_t const lt = (1u << lane) - 1u;
    size_t const blk = static_cast<size_t>(blockIdx.x) * kItems;
    for (int r = 0; r < kRounds; ++r) {
        for (int w = 0; w < kThreads / 32; ++w) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        size_t const e = blk + static_cast<size_t>(r) * kThreads + threadIdx.x;
        bool const live = e < n;
        uint64_t const key = live ? kin[e] : 0ull;
        uint32_t const dg = live ? static_cast<uint32_t>((key >> shift) & 0xffu) : 0xffffffffu;
        uint32_t const peers = __match_any_sync(0xffffffffu, dg);
        uint32_t const rank = __popc(peers & lt);
        if (live && rank == 0) wcnt[warp][dg] = __popc(peers);
        __syncthreads();
        uint32_t run = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            uint32_t const t = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = base[threadIdx.x] + run;
            run += t;
        }
        base[threadIdx.x] += run;
        __syncthreads();
        if (live) {
            uint32_t const pos = wcnt[warp][dg] + rank;
            kout[pos] = key;
            vout[pos] = vin[e];
        }
        __syncthreads();
    }
}

__global__ void k_occupied_flags(uint32_t const* count, uint32_t total, uint32_t* flags) {
    uint32_t const e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < total) flags[e] = count[e] ? 1u : 0u;
}

__global__ void k_compact_cells(uint64_t const* keys, uint32_t const* count, uint32_t const* flags,
                                uint32_t const* offsets, uint32_t total, uint32_t cap,
                                uint64_t* kout, uint32_t* vout, uint32_t* ncells) {
    uint32_t const e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    if (flags[e]) {
        uint32_t const o = offsets[e];
        kout[o] = (e == cap) ? kEmptyKey : keys[e];
        vout[o] = e;
    }
    if (e == total - 1) *ncells = offsets[e] + flags[e];
}

__global__ void k_fill_tail(uint64_t* keys, uint32_t* vals, uint32_t const* ncells, uint32_t limit) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= limit || k < *ncells) return;
    keys[k] = kEmptyKey;
    vals[k] = UINT32_MAX;
}

__global__ void k_cell_counts(uint32_t const* sorted_slots, uint32_t const* count,
                              uint32_t const* ncells, uint32_t limit, uint32_t* cell_count) {
    uint32_t const c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= limit) return;
    cell_count[c] = c < *ncells ? count[sorted_slots[c]] : 0u;
}

__global__ void k_expand_pairs(uint64_t const* sorted_z, uint32_t const* sorted_slots,
                               uint32_t const* cell_start, uint32_t const* count,
                               uint32_t const* start, uint32_t const* members,
                               uint32_t const* oid, uint32_t const* ncells, uint32_t limit,
                               uint32_t first, uint64_t* pair_z, uint32_t* pair_index,
                               uint32_t* block_indices, uint32_t* blocks) {
    uint32_t const c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= limit || c >= *ncells) return;
    uint32_t const slot = sorted_slots[c];
    uint32_t const n = count[slot];
    uint32_t const b = cell_start[c];
    uint32_t const* m = members + start[slot];
    for (uint32_t k = 0; k < n; ++k) {
        pair_z[b + k] = sorted_z[c];
        pair_index[b + k] = oid ? oid[m[k]] : m[k] - first;
        block_indices[b + k] = c;
    }
    blocks[2 * c] = b;
    blocks[2 * c + 1] = b + n;
}

__device__ __forceinline__ uint32_t compact_bits(uint64_t x) {
    x &= 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
    return static_cast<uint32_t>(x);
}

// Grid coords and z keys of the last build per original index, recovered
// from the stored keys.
__global__ void k_keys_of(uint64_t const* zkey, uint32_t const* slot_of, uint32_t begin,
                          uint32_t count, int2* gc, uint64_t* z) {
    uint32_t const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    uint64_t const key = zkey[slot_of ? slot_of[begin + k] : begin + k];
    gc[k] = make_int2(static_cast<int32_t>(compact_bits(key)),
                      static_cast<int32_t>(compact_bits(key >> 1)));
    z[k] = key;
}

}  // namespace

// Lays out the scratch regions for n keys; with base == nullptr it only
// measures. Sizing and placement share this code so they cannot disagree.
static size_t carve(char* base, uint32_t n, SortScratch* s) {
    size_t const nb = (n + kItems - 1) / kItems + 1;
    size_t const words = static_cast<size_t>(n) + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* r = base ? base + off : nullptr;
        off += (bytes + 255) & ~size_t(255);
        return r;
    };
    char* k0 = take(words * 8);
    char* k1 = take(words * 8);
    char* v0 = take(words * 4);
    char* v1 = take(words * 4);
    char* fl = take(words * 4);
    char* of = take(words * 4);
    char* hi = take(kDigits * nb * 8);
    char* sc = take((scan_scratch_words(static_cast<uint32_t>(kDigits * nb + words)) + 16) * 4);
    if (s) {
        s->keys[0] = reinterpret_cast<uint64_t*>(k0);
        s->keys[1] = reinterpret_cast<uint64_t*>(k1);
        s->vals[0] = reinterpret_cast<uint32_t*>(v0);
        s->vals[1] = reinterpret_cast<uint32_t*>(v1);
        s->flags = reinterpret_cast<uint32_t*>(fl);
        s->offsets = reinterpret_cast<uint32_t*>(of);
        s->hist = reinterpret_cast<uint32_t*>(hi);
        s->scan = reinterpret_cast<uint32_t*>(sc);
        s->capacity = n;
    }
    return off;
}

size_t sort_scratch_bytes(uint32_t n) { return carve(nullptr, n, nullptr); }

void sort_scratch_carve(void* base, uint32_t n, SortScratch& s) {
    carve(static_cast<char*>(base), n, &s);
}

int launch_radix_sort(SortScratch& s, uint32_t n, int bits, cudaStream_t st) {
    int cur = 0;
    if (n <= 1) return cur;
    uint32_t const nb = (n + kItems - 1) / kItems;
    uint32_t* offsets = s.hist + static_cast<size_t>(kDigits) * nb;
    for (int shift = 0; shift < bits; shift += 8) {
        k_hist<<<nb, kThreads, 0, st>>>(s.keys[cur], n, shift, s.hist, nb);
        launch_exclusive_scan(s.hist, kDigits * nb, offsets, s.scan, st);
        k_rank_scatter<<<nb, kThreads, 0, st>>>(s.keys[cur], s.vals[cur], s.keys[cur ^ 1],
                                                s.vals[cur ^ 1], n, shift, offsets, nb);
        cur ^= 1;
    }
    return cur;
}

void launch_sort_products(Arena const& a, bool solid, int scene, uint32_t begin, uint32_t count,
                          uint32_t tab_begin, uint32_t tab_size, float cell, SortScratch& s,
                          int2* grid_coords, uint64_t* z, uint64_t* pair_z, uint32_t* pair_index,
                          uint32_t* block_indices, uint32_t* blocks, uint32_t* nblocks,
                          cudaStream_t st) {
    (void)scene;
    uint32_t const* cnt = (solid ? a.scount : a.fcount) + tab_begin;
    uint32_t const* start = (solid ? a.sstart : a.fstart) + tab_begin;
    uint64_t const* keys = (solid ? a.skeys : a.fkeys) + tab_begin;
    uint32_t const* members = solid ? a.smembers : a.members;
    (void)cell;
    if (count) {
        k_keys_of<<<(count + 255) / 256, 256, 0, st>>>(solid ? a.szkey : a.zkey,
                                                      solid ? nullptr : a.slot_of, begin, count,
                                                      grid_coords, z);
    }
    uint32_t const total = tab_size;
    k_occupied_flags<<<(total + 255) / 256, 256, 0, st>>>(cnt, total, s.flags);
    launch_exclusive_scan(s.flags, total, s.offsets, s.scan, st);
    k_compact_cells<<<(total + 255) / 256, 256, 0, st>>>(keys, cnt, s.flags, s.offsets, total,
                                                        total - 1, s.keys[0], s.vals[0], nblocks);
    // Every occupied cell holds at least one particle, so count bounds the
    // number of cells; unused tail keys sort last.
    uint32_t const limit = count;
    // The tail [ncells, limit) gets the largest key; the stable sort keeps it
    // behind every real cell, including a real cell with that key.
    k_fill_tail<<<(limit + 255) / 256, 256, 0, st>>>(s.keys[0], s.vals[0], nblocks, limit);
    int const cur = launch_radix_sort(s, limit, 64, st);
    uint32_t* cell_count = s.flags;
    uint32_t* cell_start = s.offsets;
    k_cell_counts<<<(limit + 255) / 256, 256, 0, st>>>(s.vals[cur], cnt, nblocks, limit, cell_count);
    launch_exclusive_scan(cell_count, limit, cell_start, s.scan, st);
    k_expand_pairs<<<(limit + 255) / 256, 256, 0, st>>>(s.keys[cur], s.vals[cur], cell_start, cnt,
                                                       start, members, solid ? nullptr : a.oid,
                                                       nblocks, limit, begin, pair_z, pair_index,
                                                       block_indices, blocks);
}

}  // namespace emerald
