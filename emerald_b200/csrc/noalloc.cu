// emerald_neighbors_static: the neighbour build of one point set against
// itself with every scratch buffer in a file-scope device array, for callers
// that cannot allocate device memory themselves. Some hosts own all device
// memory through their own allocator and do not allow a library to call
// cudaMalloc behind their back; others run the build inside a per-frame loop
// where cudaMalloc and cudaFree, which synchronise the device, would stall
// the pipeline. This entry point allocates nothing: the caller passes the
// positions and the output lists, and the cell table, particle slots, member
// lists and scan scratch live in g_static_scratch below, sized for
// EMERALD_STATIC_MAX_POINTS points (about 3.4 MB held by every device that
// loads the library, until the process exits).
#include <cstdint>

#include "../../include/emerald_sph.h"
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr uint32_t kMaxPoints = EMERALD_STATIC_MAX_POINTS;
constexpr uint32_t kTableLog2 = 17;  // 2^17 slots >= 2 * kMaxPoints
constexpr uint32_t kTableSize = (1u << kTableLog2) + 1;
// Linear probing over the whole table finds a free slot while one is left;
// kMaxPoints points make at most kMaxPoints cells, under half the slots, so
// the build never flags a full table.
static_assert((1u << kTableLog2) >= 2u * kMaxPoints, "cell table must hold twice the points");
static_assert(kMaxNeighbors == EMERALD_MAX_NEIGHBORS, "list slots differ from the header's");
constexpr uint32_t kMaxTiles = kMaxPoints / kTile;
constexpr uint32_t kScanWords = (kTableSize + 2047) / 2048 + 64;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Byte offsets of the regions inside the static array.
constexpr size_t kOffParams = 0;
constexpr size_t kOffState = align256(kOffParams + sizeof(SceneParams));
constexpr size_t kOffLoops = align256(kOffState + sizeof(SceneState));
constexpr size_t kOffTiles = align256(kOffLoops + 4 * sizeof(unsigned long long));
constexpr size_t kOffKeys = align256(kOffTiles + kMaxTiles * sizeof(int32_t));
constexpr size_t kOffCount = align256(kOffKeys + size_t(kTableSize) * 8);
constexpr size_t kOffStart = align256(kOffCount + size_t(kTableSize) * 4);
constexpr size_t kOffSlot = align256(kOffStart + size_t(kTableSize) * 4);
constexpr size_t kOffRank = align256(kOffSlot + size_t(kMaxPoints) * 4);
constexpr size_t kOffMembers = align256(kOffRank + size_t(kMaxPoints) * 4);
constexpr size_t kOffZkey = align256(kOffMembers + size_t(kMaxPoints) * 4);
constexpr size_t kOffScan = align256(kOffZkey + size_t(kMaxPoints) * 8);
constexpr size_t kScratchBytes = align256(kOffScan + size_t(kScanWords) * 4);

// The cell build keeps a cursor one word past the counts.
static_assert(kOffStart >= kOffCount + (size_t(kTableSize) + 1) * 4, "count cursor overlaps starts");

static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

// Writes the one-scene description the build kernels read.
__global__ void k_static_setup(Arena a, uint32_t n, float support, float reject_l2) {
    uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kMaxTiles) {
        const_cast<int32_t*>(a.tile_scene)[t] = (t * kTile < n) ? 0 : -1;
    }
    if (t == 0) {
        SceneParams p{};
        p.fluid_begin = 0;
        p.fluid_count = n;
        p.ftab_begin = 0;
        p.ftab_log2 = kTableLog2;
        p.support = support;
        p.cell_size = support * 2.0f;
        p.reject_l2 = reject_l2;
        *const_cast<SceneParams*>(a.sp) = p;
        SceneState s{};
        s.active = 1;
        *a.ss = s;
    }
}

}  // namespace

int set_last_error(int code, char const* msg);

}  // namespace emerald

using namespace emerald;

extern "C" int emerald_neighbors_static(void const* d_xy, uint32_t n, float support,
                                        uint8_t* d_counts, uint32_t* d_idx, float* d_w,
                                        void* d_gw, uint32_t stride, void* stream) {
    if (n > kMaxPoints) {
        return set_last_error(EMERALD_EINVAL, "more points than EMERALD_STATIC_MAX_POINTS");
    }
    if (!(support > 0.0f)) return set_last_error(EMERALD_EINVAL, "support must be positive");
    if (stride < n) return set_last_error(EMERALD_EINVAL, "stride is smaller than n");
    if (n == 0) return EMERALD_OK;
    if (!d_xy || !d_counts || !d_idx || !d_w || !d_gw) {
        return set_last_error(EMERALD_EINVAL, "a device pointer is NULL");
    }
    // Positions and gradients are read and written as float2, index and
    // kernel-value lists as 32-bit words.
    if ((reinterpret_cast<uintptr_t>(d_xy) | reinterpret_cast<uintptr_t>(d_gw)) % 8 != 0) {
        return set_last_error(EMERALD_EINVAL, "d_xy and d_gw must be 8-byte aligned");
    }
    if ((reinterpret_cast<uintptr_t>(d_idx) | reinterpret_cast<uintptr_t>(d_w)) % 4 != 0) {
        return set_last_error(EMERALD_EINVAL, "d_idx and d_w must be 4-byte aligned");
    }
    // The array's device address, looked up on every call with the caller's
    // device current: each device (and each context a device gets after
    // cudaDeviceReset) has its own copy of g_static_scratch, and the host
    // symbol itself is not a device address.
    void* ptr = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        return set_last_error(EMERALD_ECUDA, e != cudaSuccess ? cudaGetErrorString(e)
                                                              : "no device address for the scratch");
    }
    unsigned char* const base = static_cast<unsigned char*>(ptr);
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    Arena a{};
    a.sp = reinterpret_cast<SceneParams const*>(base + kOffParams);
    a.ss = reinterpret_cast<SceneState*>(base + kOffState);
    a.loop_iterations = reinterpret_cast<unsigned long long*>(base + kOffLoops);
    a.loop_scene = nullptr;  // the neighbour build runs no solver loop
    a.loop_wt0 = nullptr;
    a.loop_n = nullptr;
    a.batch = 0;
    a.tile_scene = reinterpret_cast<int32_t const*>(base + kOffTiles);
    a.stride = stride;
    a.x = const_cast<float2*>(static_cast<float2 const*>(d_xy));
    a.nf_cnt = d_counts;
    a.nf_idx = d_idx;
    a.nf_w = d_w;
    a.nf_gw = static_cast<float2*>(d_gw);
    a.fkeys = reinterpret_cast<uint64_t*>(base + kOffKeys);
    a.fcount = reinterpret_cast<uint32_t*>(base + kOffCount);
    a.fstart = reinterpret_cast<uint32_t*>(base + kOffStart);
    a.slot = reinterpret_cast<uint32_t*>(base + kOffSlot);
    a.rank = reinterpret_cast<uint32_t*>(base + kOffRank);
    a.members = reinterpret_cast<uint32_t*>(base + kOffMembers);
    a.zkey = reinterpret_cast<uint64_t*>(base + kOffZkey);
    a.ftab_total = kTableSize;
    uint32_t const tiles = (n + kTile - 1) / kTile;
    k_static_setup<<<(kMaxTiles + 127) / 128, 128, 0, st>>>(a, n, support,
                                                             reject_threshold(support * 2.0f));
    // The table is cleared by the build itself (keys to empty, counts to zero).
    launch_build_cells(a, false, tiles, reinterpret_cast<uint32_t*>(base + kOffScan), st);
    launch_neighbors(a, tiles, false, true, st);
    cudaError_t const le = cudaGetLastError();
    if (le != cudaSuccess) return set_last_error(EMERALD_ECUDA, cudaGetErrorString(le));
    return EMERALD_OK;
}
