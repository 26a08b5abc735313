// Host-side launchers of the engine's kernels (all stream ordered).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "engine_types.cuh"

namespace emerald {

// neighbour build (build_kernels.cu)
uint32_t scan_scratch_words(uint32_t n);
void launch_exclusive_scan(uint32_t const* in, uint32_t n, uint32_t* out, uint32_t* scratch,
                           cudaStream_t st);
void launch_build_cells(Arena const& a, bool solid, uint32_t tiles, uint32_t* scan_scratch,
                        cudaStream_t st);
void launch_neighbors(Arena const& a, uint32_t tiles, bool solid_other, bool write_kernels,
                      cudaStream_t st, bool comp = false);
void launch_solid_volumes(Arena const& a, uint32_t solid_tiles, float numer, int scene,
                          cudaStream_t st);

// z-order sort products on request (sort_kernels.cu)
struct SortScratch {
    uint64_t* keys[2];
    uint32_t* vals[2];
    uint32_t* flags;
    uint32_t* offsets;
    uint32_t* hist;
    uint32_t* scan;
    uint32_t capacity;
};
size_t sort_scratch_bytes(uint32_t n);
void sort_scratch_carve(void* base, uint32_t n, SortScratch& s);
// Stable LSD radix sort of (key, value) pairs on the low `bits` key bits;
// returns the buffer index (0 or 1) holding the result.
int launch_radix_sort(SortScratch& s, uint32_t n, int bits, cudaStream_t st);
// Reference sort products of one scene's fluid (solid=false) or boundary set:
// per particle grid coords (int2) and z keys, the sorted (z, index) pairs
// with scene-local indices, block indices and the [begin, end) block ranges.
// Returns the number of blocks through *nblocks (device word).
void launch_sort_products(Arena const& a, bool solid, int scene, uint32_t begin, uint32_t count,
                          uint32_t tab_begin, uint32_t tab_size, float cell, SortScratch& s,
                          int2* grid_coords, uint64_t* z, uint64_t* pair_z, uint32_t* pair_index,
                          uint32_t* block_indices, uint32_t* blocks, uint32_t* nblocks,
                          cudaStream_t st);

// storage order (reorder_kernels.cu)
void launch_reorder(Arena const& a, SortScratch& s, uint32_t n, int key_bits, cudaStream_t st);
void launch_gather_f(Arena const& a, uint32_t begin, uint32_t count, float const* src, float* out,
                     cudaStream_t st);
void launch_gather_f2(Arena const& a, uint32_t begin, uint32_t count, float2 const* src, float2* out,
                      cudaStream_t st);
void launch_scatter_f2(Arena const& a, uint32_t begin, uint32_t count, float2 const* in, float2* dst,
                       cudaStream_t st);
void launch_scatter_f(Arena const& a, uint32_t begin, uint32_t count, float const* in, float* dst,
                      cudaStream_t st);
void launch_gather_d2(Arena const& a, uint32_t begin, uint32_t count, double2 const* src,
                      double2* out, cudaStream_t st);
void launch_scatter_d2(Arena const& a, uint32_t begin, uint32_t count, double2 const* in,
                       double2* dst, cudaStream_t st);
// *flag |= 1 when p[0, n) holds an infinity or a NaN.
void launch_flag_nonfinite(float const* p, size_t n, uint32_t* flag, cudaStream_t st);
void launch_positions_to_double(Arena const& a, uint32_t begin, uint32_t count, cudaStream_t st);
void launch_identity_order(Arena const& a, uint32_t begin, uint32_t count, cudaStream_t st);

// solver (solve_kernels.cu)
void launch_max_v2(Arena const& a, uint32_t tiles, cudaStream_t st);
// frame graphs: zero the per-launch sub-step counts; after each sub-step,
// count it and set `cond` while an active scene's frame has sub-steps left
void launch_frame_begin(Arena const& a, int nscenes, cudaStream_t st);
void launch_frame_check(Arena const& a, int nscenes, int method, cudaGraphConditionalHandle cond,
                        cudaStream_t st);
void launch_begin_substep(Arena const& a, int nscenes, cudaStream_t st);
void launch_zero_kappas(Arena const& a, uint32_t tiles, cudaStream_t st);
// use_cond: also set `cond` (the loop's while condition) to 1
void launch_iter_reset(Arena const& a, int nscenes, int kind, cudaStream_t st,
                       cudaGraphConditionalHandle cond = 0, int use_cond = 0);
void launch_iter_check(Arena const& a, int nscenes, int kind, int* running,
                       cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st);
// comp: some resident scene is in compensated mode (selects the kernel variant)
// mode: the divergence family's tuning value; with kPersistentWarps the
// persistent-warp variant (same bits)
void launch_dfsph_density_alpha(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st,
                                int mode = 0);
// chunk: neighbour entries loaded together in the gather sums (1, 4 or 8;
// every choice gives the same bits), plus kPrefetchLists to have each warp
// ask L2 for its list rows before the sums
constexpr int kPrefetchLists = 16;
// kPersistentWarps selects the persistent-warp kernels of a gather family:
// a grid of resident blocks whose warps walk their tiles with the next
// tile's lists already requested into L2 (same bits; kPrefetchLists is
// implied)
constexpr int kPersistentWarps = 32;
// with kPersistentWarps: blocks of 256 threads instead of 128
constexpr int kPersistentBlocks256 = 64;
// with kPersistentWarps, on a solver loop's final kernel (DFSPH apply,
// IISPH beta): the iteration's exit test runs in that kernel's last block
constexpr int kFusedExitTest = 128;
constexpr int kChunkMask = 15;
// An iteration's exit test fused into the last block of its final
// persistent-warp kernel (counter != nullptr; needs kPersistentWarps): the
// loop kind, the scenes, the host-visible running flag, the loop's while
// condition and a device counter of finished blocks (zero between launches).
struct LoopCheck {
    unsigned int* counter;
    int* running;
    cudaGraphConditionalHandle cond;
    int nscenes, kind, use_cond;
};
void launch_apply_pressures(Arena const& a, uint32_t tiles, int which_q, int external,
                            int skip_done, bool comp, cudaStream_t st, int chunk = 4,
                            LoopCheck lc = LoopCheck{nullptr, nullptr, 0, 0, 0, 0});
void launch_dfsph_divergence(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st,
                             int chunk = 8);
void launch_dfsph_density(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st,
                          int chunk = 8);
void launch_integrate_positions(Arena const& a, uint32_t tiles, bool comp, cudaStream_t st);
// comp (the IISPH, IISPH_AP, IISPH_PSEUDO_AP and PCISPH kernels below): some
// resident scene is in compensated mode; its neighbour sums are then
// Kahan-compensated
void launch_iisph_density_dii(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_iisph_aii(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_iisph_sum_dij(Arena const& a, uint32_t tiles, cudaStream_t st, int chunk, bool comp);
void launch_iisph_beta_pressure(Arena const& a, uint32_t tiles, cudaStream_t st, int chunk,
                                bool comp, LoopCheck lc = LoopCheck{nullptr, nullptr, 0, 0, 0, 0});
void launch_make_q(Arena const& a, uint32_t tiles, cudaStream_t st);
void launch_apply_integrate(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_ap_density(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_ap_diag(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp);
void launch_pressure_accel(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_ap_iterate(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp);
void launch_ap_finish(Arena const& a, uint32_t tiles, int pseudo, cudaStream_t st, bool comp);
void launch_pc_init(Arena const& a, uint32_t tiles, cudaStream_t st);
void launch_pc_predict(Arena const& a, uint32_t tiles, cudaStream_t st);
void launch_pc_density(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_pc_forces(Arena const& a, uint32_t tiles, cudaStream_t st, bool comp);
void launch_pc_final(Arena const& a, uint32_t tiles, cudaStream_t st);

}  // namespace emerald
