// Engine: device arena management and the per-method launch sequence of one
// sub-step (emerald/sph2d_box/{iisph,iisph_ap,iisph_pseudo_ap,dfsph_p,pcisph}.cpp).
#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace emerald {

namespace {

std::atomic<int64_t> g_launches{0};

uint32_t ceil_log2(uint64_t v) {
    uint32_t l = 0;
    while ((uint64_t(1) << l) < v) ++l;
    return l;
}

uint32_t tiles_for(uint32_t n) { return (n + kTile - 1) / kTile; }

}  // namespace

int64_t kernel_launch_count() { return g_launches.load(); }

// ------------------------------------------------------------ allocator

RangeAllocator::RangeAllocator(uint32_t capacity) : capacity_(capacity) {
    if (capacity) free_[0] = capacity;
}

bool RangeAllocator::alloc(uint32_t size, uint32_t& begin) {
    if (size == 0) {
        begin = 0;
        return true;
    }
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second >= size) {
            begin = it->first;
            uint32_t const rest = it->second - size;
            free_.erase(it);
            if (rest) free_[begin + size] = rest;
            return true;
        }
    }
    return false;
}

void RangeAllocator::release(uint32_t begin, uint32_t size) {
    if (!size) return;
    auto it = free_.emplace(begin, size).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
        it->second += next->second;
        free_.erase(next);
    }
    if (it != free_.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            free_.erase(it);
        }
    }
}

uint32_t RangeAllocator::largest_free() const {
    uint32_t best = 0;
    for (auto const& kv : free_) best = std::max(best, kv.second);
    return best;
}

// --------------------------------------------------------------- engine

void Engine::check(char const* what) {
    cudaError_t const e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

Engine::Room Engine::room() const {
    return Room{fluid_tiles_.largest_free(), solid_tiles_.largest_free(), ftab_.largest_free(),
                stab_.largest_free(), free_scene_slots()};
}

// The same sizes add_scene allocates.
bool Engine::Room::fits(uint32_t n_fluid, uint32_t n_solid) const {
    uint32_t const flog = std::max<uint32_t>(6, ceil_log2(2ull * std::max<uint32_t>(n_fluid, 1)));
    uint32_t const slog = std::max<uint32_t>(6, ceil_log2(2ull * std::max<uint32_t>(n_solid, 1)));
    return scene_slots > 0 && tiles_for(n_fluid) <= fluid_tiles &&
           tiles_for(n_solid) <= solid_tiles && (1u << flog) + 1 <= fluid_table &&
           (1u << slog) + 1 <= solid_table;
}

// The sum of the constructor's allocations below, region by region.
size_t Engine::footprint(uint32_t fluid_capacity, uint32_t solid_capacity, int max_scenes) {
    size_t const N = size_t(tiles_for(std::max<uint32_t>(fluid_capacity, 1))) * kTile;
    size_t const S = size_t(tiles_for(std::max<uint32_t>(solid_capacity, 1))) * kTile;
    size_t const M = size_t(std::max(max_scenes, 1));
    size_t const E = N * kMaxNeighbors;
    size_t const ftab = 4 * N + 72 * M;
    size_t const stab = 4 * S + 72 * M;
    auto r = [](size_t b) { return std::max<size_t>(b, 16); };
    size_t bytes = r(sizeof(SceneParams) * M) + r(sizeof(SceneState) * M) + r(4 * (N / kTile)) +
                   r(4 * (S / kTile));
    bytes += 13 * r(8 * N) + 18 * r(4 * N) + 2 * r(N);   // per-particle state and scratch
    bytes += 2 * r(16 * N);                                 // double positions and their staging
    bytes += r(4 * (N / 4 + 64 * M));                       // boundary-proximity maps
    bytes += r(sort_scratch_bytes(uint32_t(N)));            // storage-order sort
    bytes += 2 * (2 * r(4 * E) + r(8 * E));                 // fluid and solid neighbour lists
    bytes += r(8 * ftab) + r(4 * (ftab + 1)) + r(4 * ftab); // fluid cell table
    bytes += 3 * r(8 * S) + 4 * r(4 * S);                   // solid particles
    bytes += r(8 * stab) + r(4 * (stab + 1)) + r(4 * stab); // solid cell table
    size_t const scan_words = std::max(scan_scratch_words(uint32_t(ftab)),
                                       scan_scratch_words(uint32_t(stab))) + 64;
    bytes += r(4 * scan_words) + r(sizeof(int)) + 2 * r(sizeof(uint32_t)) +
             r(sizeof(unsigned long long) * kLoopSlots);
    bytes += r(4 * M) + r(4 * (M + 1)) + r(4);              // solver-loop work list
    return bytes;
}

Engine::Engine(uint32_t fluid_capacity, uint32_t solid_capacity, int max_scenes)
  : fluid_cap_(tiles_for(std::max<uint32_t>(fluid_capacity, 1)) * kTile),
    solid_cap_(tiles_for(std::max<uint32_t>(solid_capacity, 1)) * kTile),
    max_scenes_(std::max(max_scenes, 1)),
    fluid_tiles_(fluid_cap_ / kTile),
    solid_tiles_(solid_cap_ / kTile) {
    // Cell tables: a scene of n particles takes 2^ceil_log2(max(64, 2n)) + 1
    // slots, below 4n + 65.
    uint64_t const ftab = 4ull * fluid_cap_ + 72ull * max_scenes_;
    uint64_t const stab = 4ull * solid_cap_ + 72ull * max_scenes_;
    if (ftab > 0xffffffffull || stab > 0xffffffffull) throw std::runtime_error("arena too large");
    ftab_ = RangeAllocator(uint32_t(ftab));
    stab_ = RangeAllocator(uint32_t(stab));
    near_words_ = RangeAllocator(uint32_t(fluid_cap_ / 4 + 64ull * max_scenes_));

    auto dev = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            throw std::bad_alloc();
        }
        allocations_.push_back(p);
        device_bytes_ += std::max<size_t>(bytes, 16);
        return p;
    };
    size_t const N = fluid_cap_;
    size_t const S = solid_cap_;
    size_t const E = N * kMaxNeighbors;
    d_sp_ = static_cast<SceneParams*>(dev(sizeof(SceneParams) * max_scenes_));
    d_ss_ = static_cast<SceneState*>(dev(sizeof(SceneState) * max_scenes_));
    d_tile_scene_ = static_cast<int32_t*>(dev(sizeof(int32_t) * (N / kTile)));
    d_stile_scene_ = static_cast<int32_t*>(dev(sizeof(int32_t) * (S / kTile)));
    a_.sp = d_sp_;
    a_.ss = d_ss_;
    a_.tile_scene = d_tile_scene_;
    a_.stile_scene = d_stile_scene_;
    a_.stride = uint32_t(N);
    a_.sstride = uint32_t(S);
    a_.x = static_cast<float2*>(dev(8 * N));
    a_.v = static_cast<float2*>(dev(8 * N));
    a_.rho = static_cast<float*>(dev(4 * N));
    a_.rho_star = static_cast<float*>(dev(4 * N));
    a_.pbuf0 = static_cast<float*>(dev(4 * N));
    a_.pbuf1 = static_cast<float*>(dev(4 * N));
    a_.alpha = static_cast<float*>(dev(4 * N));
    a_.kdiv = static_cast<float*>(dev(4 * N));
    a_.kdens = static_cast<float*>(dev(4 * N));
    a_.qdiv = static_cast<float*>(dev(4 * N));
    a_.qdens = static_cast<float*>(dev(4 * N));
    a_.aii = static_cast<float*>(dev(4 * N));
    a_.dii = static_cast<float2*>(dev(8 * N));
    a_.sdp = static_cast<float2*>(dev(8 * N));
    a_.acc = static_cast<float2*>(dev(8 * N));
    a_.vext = static_cast<float2*>(dev(8 * N));
    a_.xstar = static_cast<float2*>(dev(8 * N));
    a_.vstar = static_cast<float2*>(dev(8 * N));
    a_.fp = static_cast<float2*>(dev(8 * N));
    a_.ext_f = static_cast<float2*>(dev(8 * N));
    a_.oid = static_cast<uint32_t*>(dev(4 * N));
    a_.slot_of = static_cast<uint32_t*>(dev(4 * N));
    a_.tx = static_cast<float2*>(dev(8 * N));
    a_.tv = static_cast<float2*>(dev(8 * N));
    a_.tkdiv = static_cast<float*>(dev(4 * N));
    a_.tkdens = static_cast<float*>(dev(4 * N));
    a_.toid = static_cast<uint32_t*>(dev(4 * N));
    d_near_ = static_cast<uint32_t*>(dev(4ull * near_words_.capacity()));
    a_.near_bits = d_near_;
    a_.x64 = static_cast<double2*>(dev(16 * N));
    a_.tx64 = static_cast<double2*>(dev(16 * N));
    order_buf_ = dev(sort_scratch_bytes(uint32_t(N)));
    sort_scratch_carve(order_buf_, uint32_t(N), order_sort_);
    a_.nf_cnt = static_cast<uint8_t*>(dev(N));
    a_.nf_idx = static_cast<uint32_t*>(dev(4 * E));
    a_.nf_w = static_cast<float*>(dev(4 * E));
    a_.nf_gw = static_cast<float2*>(dev(8 * E));
    a_.ns_cnt = static_cast<uint8_t*>(dev(N));
    a_.ns_idx = static_cast<uint32_t*>(dev(4 * E));
    a_.ns_w = static_cast<float*>(dev(4 * E));
    a_.ns_gw = static_cast<float2*>(dev(8 * E));
    a_.slot = static_cast<uint32_t*>(dev(4 * N));
    a_.rank = static_cast<uint32_t*>(dev(4 * N));
    a_.members = static_cast<uint32_t*>(dev(4 * N));
    a_.zkey = static_cast<uint64_t*>(dev(8 * N));
    a_.ftab_total = ftab_.capacity();
    a_.fkeys = static_cast<uint64_t*>(dev(8ull * a_.ftab_total));
    a_.fcount = static_cast<uint32_t*>(dev(4ull * (a_.ftab_total + 1)));  // + range cursor
    a_.fstart = static_cast<uint32_t*>(dev(4ull * a_.ftab_total));
    a_.xs = static_cast<float2*>(dev(8 * S));
    a_.vs = static_cast<float2*>(dev(8 * S));
    a_.vols = static_cast<float*>(dev(4 * S));
    a_.sslot = static_cast<uint32_t*>(dev(4 * S));
    a_.srank = static_cast<uint32_t*>(dev(4 * S));
    a_.smembers = static_cast<uint32_t*>(dev(4 * S));
    a_.szkey = static_cast<uint64_t*>(dev(8 * S));
    a_.stab_total = stab_.capacity();
    a_.skeys = static_cast<uint64_t*>(dev(8ull * a_.stab_total));
    a_.scount = static_cast<uint32_t*>(dev(4ull * (a_.stab_total + 1)));
    a_.sstart = static_cast<uint32_t*>(dev(4ull * a_.stab_total));
    uint32_t const scan_words =
      std::max(scan_scratch_words(a_.ftab_total), scan_scratch_words(a_.stab_total)) + 64;
    d_scan_ = static_cast<uint32_t*>(dev(4ull * scan_words));
    d_running_ = static_cast<int*>(dev(sizeof(int)));
    d_flag_ = static_cast<uint32_t*>(dev(sizeof(uint32_t)));
    d_check_counter_ = static_cast<unsigned int*>(dev(sizeof(unsigned int)));
    cudaMemset(d_check_counter_, 0, sizeof(unsigned int));
    d_loop_iters_ = static_cast<unsigned long long*>(dev(sizeof(unsigned long long) * kLoopSlots));
    a_.loop_iterations = d_loop_iters_;
    cudaMemset(d_loop_iters_, 0, sizeof(unsigned long long) * kLoopSlots);
    a_.loop_scene = static_cast<int32_t*>(dev(4ull * max_scenes_));
    a_.loop_wt0 = static_cast<uint32_t*>(dev(4ull * (max_scenes_ + 1)));
    a_.loop_n = static_cast<uint32_t*>(dev(4));
    cudaMemset(a_.loop_n, 0, 4);
    cudaMemset(a_.loop_wt0, 0, 4);
    a_.batch = max_scenes_ > 1 ? 1 : 0;
    if (cudaStreamCreateWithFlags(&cap_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&body_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&frame_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&side_st_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming) != cudaSuccess) {
        throw std::runtime_error("stream creation failed");
    }
    if (cudaMallocHost(reinterpret_cast<void**>(&h_running_), sizeof(int)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&h_flag_), sizeof(uint32_t)) != cudaSuccess) {
        throw std::bad_alloc();
    }
    cudaMemset(d_ss_, 0, sizeof(SceneState) * max_scenes_);
    cudaMemset(a_.vs, 0, 8 * S);
    cudaMemset(a_.nf_cnt, 0, N);
    cudaMemset(a_.ns_cnt, 0, N);
    cudaMemset(a_.kdiv, 0, 4 * N);
    cudaMemset(a_.kdens, 0, 4 * N);
    scenes_.resize(max_scenes_);
    tile_scene_.assign(N / kTile, -1);
    stile_scene_.assign(S / kTile, -1);
    upload_tiles();
    update_extent();
    check("engine allocation");
}

void Engine::destroy_graphs() {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_fixed_kernels_.clear();
    for (auto& kv : frame_graphs_) cudaGraphExecDestroy(kv.second);
    frame_graphs_.clear();
    frame_fixed_kernels_.clear();
}

Engine::~Engine() {
    destroy_graphs();
    if (cap_st_) cudaStreamDestroy(cap_st_);
    if (body_st_) cudaStreamDestroy(body_st_);
    if (frame_st_) cudaStreamDestroy(frame_st_);
    if (side_st_) cudaStreamDestroy(side_st_);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    for (auto& p : pending_) {
        cudaEventDestroy(p.start);
        cudaEventDestroy(p.stop);
    }
    for (auto e : event_pool_) cudaEventDestroy(e);
    if (sort_buf_) cudaFree(sort_buf_);
    for (void* p : allocations_) cudaFree(p);
    if (h_running_) cudaFreeHost(h_running_);
    if (h_flag_) cudaFreeHost(h_flag_);
}

template <class F>
void Engine::launch(char const* name, F&& f, int kernels) {
    if (count_host_) {
        if (capturing_) {
            capture_kernels_ += kernels;
        } else {
            g_launches.fetch_add(kernels, std::memory_order_relaxed);
            host_launches_ += kernels;
        }
    }
    if (!timing_ || capturing_) {
        f();
        return;
    }
    auto take = [&]() {
        cudaEvent_t e;
        if (!event_pool_.empty()) {
            e = event_pool_.back();
            event_pool_.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    };
    Pending p{name, take(), take()};
    cudaEventRecord(p.start, st_);
    f();
    cudaEventRecord(p.stop, st_);
    pending_.push_back(p);
}

void Engine::enable_timing(bool on) { timing_ = on; }

void Engine::reset_timing() {
    kernel_times();
    times_ = KernelTimes{};
}

KernelTimes const& Engine::kernel_times() {
    if (!pending_.empty()) {
        host_wait(st_);
        for (auto& p : pending_) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, p.start, p.stop);
            times_.ms[p.name] += ms;
            times_.launches[p.name] += 1;
            event_pool_.push_back(p.start);
            event_pool_.push_back(p.stop);
        }
        pending_.clear();
    }
    return times_;
}

// Leading key of the storage-order sort: the scene's first tile above a
// 24-bit cell key (see reorder_kernels.cu), rounded up to whole 8-bit passes.
int Engine::order_key_bits() const {
    int bits = 24;
    if (max_scenes_ > 1) bits += int(ceil_log2(uint64_t(fluid_cap_ / kTile) + 1));
    return (bits + 7) / 8 * 8;
}

// sort_base of each scene: the real particles of all scenes stored before it.
void Engine::update_sort_bases() {
    std::vector<std::pair<uint32_t, int>> order;
    for (int id = 0; id < max_scenes_; ++id) {
        if (scenes_[id].used) order.push_back({scenes_[id].p.fluid_begin, id});
    }
    std::sort(order.begin(), order.end());
    uint32_t base = 0;
    for (auto const& kv : order) {
        Scene& sc = scenes_[kv.second];
        if (sc.p.sort_base != base) {
            sc.p.sort_base = base;
            upload_params(kv.second);
        }
        base += sc.p.fluid_count;
    }
}

void Engine::upload_tiles() {
    cudaMemcpyAsync(d_tile_scene_, tile_scene_.data(), sizeof(int32_t) * tile_scene_.size(),
                    cudaMemcpyHostToDevice, st_);
    cudaMemcpyAsync(d_stile_scene_, stile_scene_.data(), sizeof(int32_t) * stile_scene_.size(),
                    cudaMemcpyHostToDevice, st_);
    tiles_dirty_ = false;
}

void Engine::upload_params(int id) {
    cudaMemcpyAsync(d_sp_ + id, &scenes_[id].p, sizeof(SceneParams), cudaMemcpyHostToDevice, st_);
}

int Engine::add_scene(SceneSpec const& spec) {
    int id = -1;
    for (int k = 0; k < max_scenes_; ++k) {
        if (!scenes_[k].used) {
            id = k;
            break;
        }
    }
    if (id < 0) return -1;
    Scene sc;
    sc.ftile_count = tiles_for(spec.n_fluid);
    sc.stile_count = tiles_for(spec.n_solid);
    uint32_t const flog = std::max<uint32_t>(6, ceil_log2(2ull * std::max<uint32_t>(spec.n_fluid, 1)));
    uint32_t const slog = std::max<uint32_t>(6, ceil_log2(2ull * std::max<uint32_t>(spec.n_solid, 1)));
    sc.ftab_size = (1u << flog) + 1;
    sc.stab_size = (1u << slog) + 1;
    uint32_t ft = 0, stl = 0, fb = 0, sb = 0;
    if (!fluid_tiles_.alloc(sc.ftile_count, ft)) return -1;
    if (!solid_tiles_.alloc(sc.stile_count, stl)) {
        fluid_tiles_.release(ft, sc.ftile_count);
        return -1;
    }
    if (!ftab_.alloc(sc.ftab_size, fb)) {
        fluid_tiles_.release(ft, sc.ftile_count);
        solid_tiles_.release(stl, sc.stile_count);
        return -1;
    }
    if (!stab_.alloc(sc.stab_size, sb)) {
        fluid_tiles_.release(ft, sc.ftile_count);
        solid_tiles_.release(stl, sc.stile_count);
        ftab_.release(fb, sc.ftab_size);
        return -1;
    }
    sc.ftile_begin = ft;
    sc.stile_begin = stl;
    sc.used = true;
    sc.active = false;

    emerald_params const& ep = spec.params;
    DerivedConfig const cfg = derive_config(ep);
    SceneParams& P = sc.p;
    P.fluid_begin = ft * kTile;
    P.fluid_count = spec.n_fluid;
    P.solid_begin = stl * kTile;
    P.solid_count = spec.n_solid;
    P.ftab_begin = fb;
    P.ftab_log2 = flog;
    P.stab_begin = sb;
    P.stab_log2 = slog;
    P.support = ep.support;
    P.cell_size = ep.support * 2.0f;
    P.rho0 = ep.target_density;
    P.mass = cfg.mass_per_particle;
    P.fluid_volume = cfg.mass_per_particle / ep.target_density;
    P.gravity = ep.gravity;
    P.viscosity = ep.viscosity;
    P.w0 = kernel_w(0.0f, ep.support);
    P.iisph_omega = ep.iisph_omega;
    P.iisph_err_avg = ep.iisph_error_average_threshold;
    P.iisph_err_max = ep.iisph_error_max_threshold;
    P.iisph_max_iter = ep.iisph_max_pressure_iterations;
    P.dfsph_max_iter = ep.dfsph_max_correction_iterations;
    P.dfsph_dens_avg = ep.dfsph_density_error_average_threshold;
    P.dfsph_dens_max = ep.dfsph_density_error_max_threshold;
    P.dfsph_div_avg = ep.dfsph_divergence_error_average_threshold;
    P.dfsph_div_max = ep.dfsph_divergence_error_max_threshold;
    P.pcisph_denom = cfg.pressure_correction_denom;
    P.method = spec.method;
    P.mode = spec.mode;
    P.time_per_step = ep.time_per_step_flicks;
    P.sub_steps = ep.sub_steps;
    P.min_denom = 60;
    P.max_denom = spec.method == kIisph ? 6 : 4;
    P.cfl_factor = spec.method == kIisph ? 0.2f : 0.4f;
    P.seconds_per_sub_step = cfg.seconds_per_sub_step;
    P.fixed_dt = spec.fixed_dt;
    P.sort_base = 0;
    P.reject_l2 = reject_threshold(P.cell_size);
    P.precision = ep.precision;
    // default_gravity_forces(params.gravity) (emerald/sph2d_box/forces.cpp:73-83)
    P.force_count = 1;
    P.force_array = 0;
    P.force_terms[0] = ForceTerm{kForceGravity, ep.gravity, 0.0f, 0.0f};
    P.fixed_t = 0.0f;
    sc.draw_radius = cfg.draw_radius;
    build_near_map(sc, spec.solid_xy, spec.n_solid);
    scenes_[id] = sc;

    for (uint32_t t = 0; t < sc.ftile_count; ++t) tile_scene_[ft + t] = id;
    for (uint32_t t = 0; t < sc.stile_count; ++t) stile_scene_[stl + t] = id;
    upload_tiles();
    upload_params(id);
    SceneState s0{};
    cudaMemcpyAsync(d_ss_ + id, &s0, sizeof(SceneState), cudaMemcpyHostToDevice, st_);
    if (spec.n_fluid) {
        cudaMemcpyAsync(a_.x + P.fluid_begin, spec.fluid_xy, 8ull * spec.n_fluid,
                        cudaMemcpyHostToDevice, st_);
        if (spec.fluid_v) {
            cudaMemcpyAsync(a_.v + P.fluid_begin, spec.fluid_v, 8ull * spec.n_fluid,
                            cudaMemcpyHostToDevice, st_);
        } else {
            cudaMemsetAsync(a_.v + P.fluid_begin, 0, 8ull * spec.n_fluid, st_);
        }
        cudaMemsetAsync(a_.kdiv + P.fluid_begin, 0, 4ull * spec.n_fluid, st_);
        cudaMemsetAsync(a_.kdens + P.fluid_begin, 0, 4ull * spec.n_fluid, st_);
        cudaMemsetAsync(a_.nf_cnt + P.fluid_begin, 0, spec.n_fluid, st_);
        launch_identity_order(a_, P.fluid_begin, spec.n_fluid, st_);
        launch_positions_to_double(a_, P.fluid_begin, spec.n_fluid, st_);
        cudaMemsetAsync(a_.ns_cnt + P.fluid_begin, 0, spec.n_fluid, st_);
    }
    if (spec.n_solid) {
        cudaMemcpyAsync(a_.xs + P.solid_begin, spec.solid_xy, 8ull * spec.n_solid,
                        cudaMemcpyHostToDevice, st_);
        cudaMemsetAsync(a_.vs + P.solid_begin, 0, 8ull * spec.n_solid, st_);
    }
    update_sort_bases();
    update_extent();
    rebuild_solids();
    if (spec.n_solid) {
        if (spec.solid_volumes) {
            cudaMemcpyAsync(a_.vols + P.solid_begin, spec.solid_volumes, 4ull * spec.n_solid,
                            cudaMemcpyHostToDevice, st_);
        } else {
            launch("solid_volumes", [&] {
                launch_solid_volumes(a_, ext_stiles_, 1.7f, id, st_);
            });
        }
    }
    check("add_scene");
    return id;
}

// Marks the 3x3 cell block around every boundary particle's cell (the cells
// whose particles can have that boundary particle within the search radius,
// emerald/sph_common/neighborhood.h:199-282), with the same float cell
// arithmetic as the kernels. No map when the boundary is empty, its cell box
// is above 2^26 cells, or the map arena is full.
void Engine::build_near_map(Scene& sc, float const* solid_xy, uint32_t n_solid) {
    SceneParams& P = sc.p;
    P.near_w = P.near_h = 0;
    P.near_begin = 0;
    P.near_x0 = P.near_y0 = 0;
    sc.near_words = 0;
    if (!n_solid || !solid_xy) return;
    std::vector<int32_t> cx(n_solid), cy(n_solid);
    int64_t x0 = INT64_MAX, y0 = INT64_MAX, x1 = INT64_MIN, y1 = INT64_MIN;
    for (uint32_t k = 0; k < n_solid; ++k) {
        grid_coord(mk2(solid_xy[2 * k], solid_xy[2 * k + 1]), P.cell_size, cx[k], cy[k]);
        x0 = std::min<int64_t>(x0, cx[k]);
        y0 = std::min<int64_t>(y0, cy[k]);
        x1 = std::max<int64_t>(x1, cx[k]);
        y1 = std::max<int64_t>(y1, cy[k]);
    }
    int64_t const w = x1 - x0 + 3, h = y1 - y0 + 3;
    if (w * h > (int64_t(1) << 26)) return;
    uint64_t const words = (uint64_t(w) * uint64_t(h) + 31) / 32;
    uint32_t begin = 0;
    if (!near_words_.alloc(uint32_t(words), begin)) return;
    std::vector<uint32_t> bits(words, 0u);
    for (uint32_t k = 0; k < n_solid; ++k) {
        for (int dy = 0; dy < 3; ++dy) {
            for (int dx = 0; dx < 3; ++dx) {
                uint64_t const b =
                  uint64_t(cy[k] - y0 + dy) * uint64_t(w) + uint64_t(cx[k] - x0 + dx);
                bits[b >> 5] |= 1u << (b & 31u);
            }
        }
    }
    if (cudaMemcpy(d_near_ + begin, bits.data(), 4 * words, cudaMemcpyHostToDevice) != cudaSuccess) {
        near_words_.release(begin, uint32_t(words));
        check("near map upload");
        return;
    }
    P.near_begin = begin;
    P.near_w = uint32_t(w);
    P.near_h = uint32_t(h);
    P.near_x0 = int32_t(x0 - 1);
    P.near_y0 = int32_t(y0 - 1);
    sc.near_words = uint32_t(words);
}

void Engine::rebuild_solids() {
    Arena const e = extent_arena();
    launch("build_cells_solid", [&] { launch_build_cells(e, true, ext_stiles_, d_scan_, st_); }, 4);
}

// Launch extents grow and shrink in steps of 1/EMERALD_EXTENT_DIV of the
// arena (at least min_quantum): a change re-captures the sub-step graphs.
#ifndef EMERALD_EXTENT_DIV
#define EMERALD_EXTENT_DIV 32
#endif
namespace {
uint32_t round_extent(uint64_t used, uint32_t capacity, uint32_t min_quantum) {
    uint64_t const q = std::max<uint64_t>(min_quantum, capacity / EMERALD_EXTENT_DIV);
    uint64_t const r = (used + q - 1) / q * q;
    return uint32_t(std::min<uint64_t>(std::max<uint64_t>(r, 1), capacity));
}
}  // namespace

void Engine::update_extent() {
    uint64_t t = 0, st = 0, ft = 0, sb = 0;
    for (auto const& sc : scenes_) {
        if (!sc.used) continue;
        t = std::max<uint64_t>(t, sc.ftile_begin + sc.ftile_count);
        st = std::max<uint64_t>(st, sc.stile_begin + sc.stile_count);
        ft = std::max<uint64_t>(ft, uint64_t(sc.p.ftab_begin) + sc.ftab_size);
        sb = std::max<uint64_t>(sb, uint64_t(sc.p.stab_begin) + sc.stab_size);
    }
    uint32_t const nt = round_extent(t, fluid_cap_ / kTile, 16);
    uint32_t const ns = round_extent(st, solid_cap_ / kTile, 16);
    uint32_t const nf = round_extent(ft, ftab_.capacity(), 8192);
    uint32_t const nsb = round_extent(sb, stab_.capacity(), 8192);
    bool comp = false;
    for (auto const& sc : scenes_) comp = comp || (sc.used && sc.p.precision != 0);
    if (nt != ext_tiles_ || nf != ext_ftab_ || comp != compensated_) destroy_graphs();
    compensated_ = comp;
    ext_tiles_ = nt;
    ext_stiles_ = ns;
    ext_ftab_ = nf;
    ext_stab_ = nsb;
}

Arena Engine::extent_arena() const {
    Arena e = a_;
    e.ftab_total = ext_ftab_;
    e.stab_total = ext_stab_;
    return e;
}

void Engine::remove_scene(int id) {
    if (!scene_used(id)) return;
    Scene& sc = scenes_[id];
    SceneState s0{};
    cudaMemcpyAsync(d_ss_ + id, &s0, sizeof(SceneState), cudaMemcpyHostToDevice, st_);
    for (uint32_t t = 0; t < sc.ftile_count; ++t) tile_scene_[sc.ftile_begin + t] = -1;
    for (uint32_t t = 0; t < sc.stile_count; ++t) stile_scene_[sc.stile_begin + t] = -1;
    upload_tiles();
    fluid_tiles_.release(sc.ftile_begin, sc.ftile_count);
    solid_tiles_.release(sc.stile_begin, sc.stile_count);
    ftab_.release(sc.p.ftab_begin, sc.ftab_size);
    stab_.release(sc.p.stab_begin, sc.stab_size);
    if (sc.near_words) near_words_.release(sc.p.near_begin, sc.near_words);
    sc = Scene{};
    update_sort_bases();
    update_extent();
    rebuild_solids();
}

void Engine::set_active(int id, bool active) {
    if (!scene_used(id)) return;
    scenes_[id].active = active;
    int32_t const v = active ? 1 : 0;
    cudaMemcpyAsync(reinterpret_cast<char*>(d_ss_ + id) + offsetof(SceneState, active), &v,
                    sizeof(int32_t), cudaMemcpyHostToDevice, st_);
    host_wait(st_);
}

void Engine::set_mode(int id, int32_t mode, float fixed_dt, float fixed_t) {
    if (!scene_used(id)) return;
    SceneParams& P = scenes_[id].p;
    if (P.mode != mode || P.fixed_dt != fixed_dt ||
        (mode == kFixedDt && !(P.fixed_t == fixed_t))) {
        P.mode = mode;
        P.fixed_dt = fixed_dt;
        P.fixed_t = fixed_t;
        upload_params(id);
    }
}

void Engine::set_forces(int id, ForceTerm const* terms, int count) {
    if (!scene_used(id)) throw std::invalid_argument("no such scene");
    if (count < 0 || count > kMaxForceTerms || (count && !terms)) {
        throw std::invalid_argument("between 0 and 4 force terms");
    }
    SceneParams& P = scenes_[id].p;
    P.force_count = count;
    for (int k = 0; k < kMaxForceTerms; ++k) {
        P.force_terms[k] = k < count ? terms[k] : ForceTerm{0, 0.0f, 0.0f, 0.0f};
    }
    upload_params(id);
}

void Engine::set_force_callback(int id, ForceCallback fn, void* user) {
    if (!scene_used(id)) throw std::invalid_argument("no such scene");
    Scene& sc = scenes_[id];
    sc.force_fn = fn;
    sc.force_user = user;
    sc.p.force_array = fn ? 1 : 0;
    upload_params(id);
}

bool Engine::has_force_callbacks() const {
    for (auto const& sc : scenes_) {
        if (sc.used && sc.active && sc.force_fn) return true;
    }
    return false;
}

// compute_all_external_forces with the scenes' host callbacks: the state at
// this point of the sub-step goes to the host in original order, the
// callback fills the zeroed forces, and they come back in storage order.
// The time is the sub-step's, plus dt under DFSPH_P, whose force point
// comes after the divergence solve (emerald/sph2d_box/dfsph_p.cpp:350).
void Engine::host_forces(int32_t method) {
    for (int id = 0; id < max_scenes_; ++id) {
        Scene& sc = scenes_[id];
        if (!sc.used || !sc.active || !sc.force_fn) continue;
        uint32_t const b = sc.p.fluid_begin, n = sc.p.fluid_count;
        SceneState const s = scene_state(id);
        hx_.resize(2ull * n);
        hv_.resize(2ull * n);
        hf_.assign(2ull * n, 0.0f);
        get_state(id, hx_.data(), hv_.data(), true);
        float const time = method == kDfsph ? s.t + s.dt : s.t;
        sc.force_fn(sc.force_user, n, time, s.dt, sc.p.mass, sc.draw_radius, hf_.data(),
                    hx_.data(), hv_.data());
        cudaMemcpyAsync(a_.tx + b, hf_.data(), 8ull * n, cudaMemcpyHostToDevice, st_);
        launch_scatter_f2(a_, b, n, a_.tx + b, a_.ext_f, st_);
        host_wait(st_);
        check("host forces");
    }
}

int Engine::active_scenes() const {
    int n = 0;
    for (auto const& s : scenes_) n += (s.used && s.active) ? 1 : 0;
    return n;
}

void Engine::begin_frame(int32_t method) {
    if (method == kDfsph) {
        launch("zero_kappas", [&] { launch_zero_kappas(a_, ext_tiles_, st_); });
    }
}

int Engine::max_iterations(int kind) const {
    int m = 0;
    for (auto const& s : scenes_) {
        if (!s.used || !s.active) continue;
        int const v = (kind == 0) ? s.p.iisph_max_iter : (kind == 3 ? 6 : s.p.dfsph_max_iter);
        m = std::max(m, v);
    }
    return m;
}

// Solver iteration kernels of one loop kind (launched on cur_).
void Engine::emit_loop_body(int kind, int32_t method, cudaGraphConditionalHandle cond,
                            bool use_cond) {
    uint32_t const tiles = ext_tiles_;
    cudaStream_t const st = cur_;
    // loop kernels are counted on the device, once per executed iteration
    bool const was_counting = count_host_;
    count_host_ = false;
    // the exit test in the last block of the iteration's final kernel, when
    // that kernel is a persistent-warp one tuned to carry it
    auto fused = [&](int v) {
        return (v & kPersistentWarps) && (v & kFusedExitTest) && !timing_;
    };
    LoopCheck const lc{d_check_counter_, d_running_, cond, max_scenes_, kind, use_cond ? 1 : 0};
    LoopCheck const none{nullptr, nullptr, 0, 0, 0, 0};
    bool carried = false;
    switch (method) {
    case kDfsph:
        carried = fused(tuning_.apply);
        if (kind == 2) {
            launch("dfsph_divergence", [&] { launch_dfsph_divergence(a_, tiles, compensated_, st, tuning_.divergence); });
            launch("apply_pressures", [&] { launch_apply_pressures(a_, tiles, 0, 0, 1, compensated_, st, tuning_.apply, carried ? lc : none); });
        } else {
            launch("dfsph_density", [&] { launch_dfsph_density(a_, tiles, compensated_, st, tuning_.divergence); });
            launch("apply_pressures", [&] { launch_apply_pressures(a_, tiles, 1, 0, 1, compensated_, st, tuning_.apply, carried ? lc : none); });
        }
        break;
    case kIisph:
        carried = fused(tuning_.iisph_beta);
        launch("iisph_sum_dij", [&] { launch_iisph_sum_dij(a_, tiles, st, tuning_.iisph_sum, compensated_); });
        launch("iisph_beta_pressure", [&] { launch_iisph_beta_pressure(a_, tiles, st, tuning_.iisph_beta, compensated_, carried ? lc : none); });
        break;
    case kIisphAp:
    case kIisphPseudoAp: {
        int const pseudo = method == kIisphPseudoAp ? 1 : 0;
        launch("pressure_accel", [&] { launch_pressure_accel(a_, tiles, st, compensated_); });
        launch("ap_iterate", [&] { launch_ap_iterate(a_, tiles, pseudo, st, compensated_); });
        break;
    }
    case kPcisph:
        launch("pc_predict", [&] { launch_pc_predict(a_, tiles, st); });
        launch("pc_density", [&] { launch_pc_density(a_, tiles, st, compensated_); });
        launch("pc_forces", [&] { launch_pc_forces(a_, tiles, st, compensated_); });
        break;
    default: break;
    }
    if (!carried) {
        launch("iter_check", [&] {
            launch_iter_check(a_, max_scenes_, kind, d_running_, cond, use_cond ? 1 : 0, st);
        });
    }
    // kernels per executed iteration of this loop kind (body + check)
    loop_kernels_[kind] = (kind == 3 ? 4 : 3) - (carried ? 1 : 0);
    count_host_ = was_counting;
}

int64_t Engine::kernel_launches() {
    unsigned long long it[kLoopSlots] = {};
    cudaMemcpyAsync(it, d_loop_iters_, sizeof(it), cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    int64_t n = host_launches_;
    for (int k = 0; k < 4; ++k) n += int64_t(it[k]) * loop_kernels_[k];
    for (int m = 0; m < 5; ++m) n += int64_t(it[4 + m]) * frame_body_kernels_[m];
    return n;
}

void Engine::run_loop(int kind, int max_iter, int32_t method) {
    if (!capturing_) {
        launch("iter_reset", [&] { launch_iter_reset(a_, max_scenes_, kind, cur_); });
    }
    if (capturing_) {
        // while (any scene iterates) { body; check } as a conditional node,
        // opened by the reset kernel every time the loop is reached
        cudaStreamCaptureStatus status;
        cudaGraph_t g = nullptr;
        cudaGraphNode_t const* deps = nullptr;
        size_t ndeps = 0;
        if (cudaStreamGetCaptureInfo(cur_, &status, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
            status != cudaStreamCaptureStatusActive) {
            throw std::runtime_error("graph capture: no active capture");
        }
        cudaGraphConditionalHandle cond;
        if (cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            throw std::runtime_error("graph capture: conditional handle");
        }
        launch("iter_reset", [&] { launch_iter_reset(a_, max_scenes_, kind, cur_, cond, 1); });
        if (cudaStreamGetCaptureInfo(cur_, &status, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
            status != cudaStreamCaptureStatusActive) {
            throw std::runtime_error("graph capture: no active capture");
        }
        cudaGraphNodeParams params{};
        params.type = cudaGraphNodeTypeConditional;
        params.conditional.handle = cond;
        params.conditional.type = cudaGraphCondTypeWhile;
        params.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g, deps, ndeps, &params) != cudaSuccess) {
            throw std::runtime_error("graph capture: conditional node");
        }
        if (cudaStreamUpdateCaptureDependencies(cur_, &node, 1, cudaStreamSetCaptureDependencies) !=
            cudaSuccess) {
            throw std::runtime_error("graph capture: dependencies");
        }
        cudaGraph_t body = params.conditional.phGraph_out[0];
        cudaStream_t const outer = cur_;
        if (cudaStreamBeginCaptureToGraph(body_st_, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            throw std::runtime_error("graph capture: body");
        }
        cur_ = body_st_;
        // Several iterations per body launch: every body kernel returns at
        // once for scenes that have converged and the last exit test sets
        // the loop condition, so the results are those of one iteration per
        // body, with fewer body launches.
        for (int u = 0; u < loop_unroll_; ++u) emit_loop_body(kind, method, cond, true);
        cur_ = outer;
        if (cudaStreamEndCapture(body_st_, &body) != cudaSuccess) {
            throw std::runtime_error("graph capture: body end");
        }
        return;
    }
    for (int it = 0; it < max_iter; ++it) {
        emit_loop_body(kind, method, 0, false);
        if (!unrolled_) {
            cudaMemcpyAsync(h_running_, d_running_, sizeof(int), cudaMemcpyDeviceToHost, cur_);
            host_wait(cur_);
            if (!*h_running_) break;
        }
    }
}

void Engine::emit_substep(int32_t method, bool reorder) {
    uint32_t const tiles = ext_tiles_;
    cudaStream_t const st = cur_;
    if (reorder) {
        // keys, three to five radix passes of three kernels, permute, commit
        int const bits = order_key_bits();
        launch("reorder", [&] { launch_reorder(a_, order_sort_, tiles * kTile, bits, st); },
               3 + 3 * (bits / 8));
    }
    launch("max_v2", [&] { launch_max_v2(a_, tiles, st); });
    launch("begin_substep", [&] { launch_begin_substep(a_, max_scenes_, st); });
    // binning, cell ranges, scatter, per-cell ordering
    Arena const ext = extent_arena();
    bool const kernels = method != kPcisph;
    // The boundary lists read only positions and the static boundary tables,
    // so they are built on a side stream (a parallel branch of the graph)
    // while the fluid cells and fluid lists are built; the per-kernel timing
    // mode keeps everything on one stream.
    bool const fork = !timing_;
    if (fork) {
        cudaEventRecord(ev_fork_, st);
        cudaStreamWaitEvent(side_st_, ev_fork_, 0);
        launch("neighbors_solid",
               [&] { launch_neighbors(a_, tiles, true, kernels, side_st_, compensated_); });
        cudaEventRecord(ev_join_, side_st_);
    }
    launch("build_cells", [&] { launch_build_cells(ext, false, tiles, d_scan_, st); }, 4);
    launch("neighbors_fluid", [&] { launch_neighbors(a_, tiles, false, kernels, st, compensated_); });
    if (fork) {
        cudaStreamWaitEvent(st, ev_join_, 0);
    } else {
        launch("neighbors_solid",
               [&] { launch_neighbors(a_, tiles, true, kernels, st, compensated_); });
    }
    switch (method) {
    case kDfsph:
        launch("dfsph_density_alpha", [&] {
            launch_dfsph_density_alpha(a_, tiles, compensated_, st, tuning_.divergence);
        });
        launch("apply_pressures", [&] { launch_apply_pressures(a_, tiles, 0, 0, 0, compensated_, st, tuning_.apply); });
        run_loop(2, max_iterations(2), method);
        if (!capturing_ && has_force_callbacks()) host_forces(method);
        launch("apply_pressures_ext", [&] { launch_apply_pressures(a_, tiles, 1, 1, 0, compensated_, st, tuning_.apply); });
        run_loop(1, max_iterations(1), method);
        launch("integrate_positions", [&] { launch_integrate_positions(a_, tiles, compensated_, st); });
        break;
    case kIisph:
        if (!capturing_ && has_force_callbacks()) host_forces(method);
        launch("iisph_density_dii", [&] { launch_iisph_density_dii(a_, tiles, st, compensated_); });
        launch("iisph_aii", [&] { launch_iisph_aii(a_, tiles, st, compensated_); });
        run_loop(0, max_iterations(0), method);
        launch("make_q", [&] { launch_make_q(a_, tiles, st); });
        launch("apply_integrate", [&] { launch_apply_integrate(a_, tiles, st, compensated_); });
        break;
    case kIisphAp:
    case kIisphPseudoAp: {
        int const pseudo = method == kIisphPseudoAp ? 1 : 0;
        if (!capturing_ && has_force_callbacks()) host_forces(method);
        launch("ap_density", [&] { launch_ap_density(a_, tiles, st, compensated_); });
        launch("ap_diag", [&] { launch_ap_diag(a_, tiles, pseudo, st, compensated_); });
        run_loop(0, max_iterations(0), method);
        launch("ap_finish", [&] { launch_ap_finish(a_, tiles, pseudo, st, compensated_); });
        break;
    }
    case kPcisph:
        if (!capturing_ && has_force_callbacks()) host_forces(method);
        launch("pc_init", [&] { launch_pc_init(a_, tiles, st); });
        run_loop(3, 6, method);
        launch("pc_final", [&] { launch_pc_final(a_, tiles, st); });
        break;
    default: throw std::runtime_error("unknown method");
    }
}

// Records one sub-step of `method` into a graph. Kernel arguments are the
// arena pointers and the tile count, which never change for an engine, and
// every kernel reads scene membership and parameters from device memory, so
// the graph stays valid as scenes are added, removed or (de)activated.
void Engine::capture_substep(int32_t method, bool reorder) {
    host_wait(st_);
    if (cudaStreamBeginCapture(cap_st_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        throw std::runtime_error("graph capture: begin");
    }
    capturing_ = true;
    capture_kernels_ = 0;
    cur_ = cap_st_;
    try {
        emit_substep(method, reorder);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cap_st_, &g);
        if (g) cudaGraphDestroy(g);
        capturing_ = false;
        cur_ = st_;
        throw;
    }
    capturing_ = false;
    cur_ = st_;
    cudaGraph_t g = nullptr;
    if (cudaStreamEndCapture(cap_st_, &g) != cudaSuccess) {
        throw std::runtime_error("graph capture: end");
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t const e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    graphs_[method * 2 + (reorder ? 1 : 0)] = exec;
    graph_fixed_kernels_[method * 2 + (reorder ? 1 : 0)] = capture_kernels_;
}

// Records one frame of `method` into a graph: the storage-order re-sort
// (when due), then a conditional while node whose body is one sub-step
// followed by k_frame_check, which continues the loop while an active
// scene's frame has sub-steps left. The solver loops inside the sub-step
// are conditional nodes nested in that body.
void Engine::capture_frame(int32_t method, bool reorder) {
    host_wait(st_);
    if (cudaStreamBeginCapture(cap_st_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        throw std::runtime_error("frame capture: begin");
    }
    capturing_ = true;
    capture_kernels_ = 0;
    cur_ = cap_st_;
    cudaGraph_t g = nullptr;
    auto abort = [&] {
        for (cudaStream_t sst : {body_st_, frame_st_, cap_st_}) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(sst, &cs) == cudaSuccess &&
                cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t dead = nullptr;
                cudaStreamEndCapture(sst, &dead);
                if (dead) cudaGraphDestroy(dead);
            }
        }
        cudaGetLastError();
        capturing_ = false;
        cur_ = st_;
    };
    try {
        launch("frame_begin", [&] { launch_frame_begin(a_, max_scenes_, cap_st_); });
        if (reorder) {
            int const bits = order_key_bits();
            launch("reorder",
                   [&] { launch_reorder(a_, order_sort_, ext_tiles_ * kTile, bits, cap_st_); },
                   3 + 3 * (bits / 8));
        }
        cudaStreamCaptureStatus status;
        cudaGraph_t outer = nullptr;
        cudaGraphNode_t const* deps = nullptr;
        size_t ndeps = 0;
        if (cudaStreamGetCaptureInfo(cap_st_, &status, nullptr, &outer, &deps, &ndeps) !=
              cudaSuccess ||
            status != cudaStreamCaptureStatusActive) {
            throw std::runtime_error("frame capture: no active capture");
        }
        cudaGraphConditionalHandle cond;
        if (cudaGraphConditionalHandleCreate(&cond, outer, 1, cudaGraphCondAssignDefault) !=
            cudaSuccess) {
            throw std::runtime_error("frame capture: conditional handle");
        }
        cudaGraphNodeParams params{};
        params.type = cudaGraphNodeTypeConditional;
        params.conditional.handle = cond;
        params.conditional.type = cudaGraphCondTypeWhile;
        params.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, outer, deps, ndeps, &params) != cudaSuccess ||
            cudaStreamUpdateCaptureDependencies(cap_st_, &node, 1,
                                                cudaStreamSetCaptureDependencies) != cudaSuccess) {
            throw std::runtime_error("frame capture: conditional node");
        }
        cudaGraph_t body = params.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(frame_st_, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            throw std::runtime_error("frame capture: body");
        }
        int64_t const outside = capture_kernels_;
        cur_ = frame_st_;
        emit_substep(method, false);
        launch("frame_check",
               [&] { launch_frame_check(a_, max_scenes_, method, cond, frame_st_); });
        frame_body_kernels_[method] = capture_kernels_ - outside;
        capture_kernels_ = outside;
        if (cudaStreamEndCapture(frame_st_, &body) != cudaSuccess) {
            throw std::runtime_error("frame capture: body end");
        }
        cur_ = cap_st_;
    } catch (...) {
        abort();
        throw;
    }
    capturing_ = false;
    cur_ = st_;
    if (cudaStreamEndCapture(cap_st_, &g) != cudaSuccess) {
        throw std::runtime_error("frame capture: end");
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t const e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("frame graph instantiate: ") + cudaGetErrorString(e));
    }
    frame_graphs_[method * 2 + (reorder ? 1 : 0)] = exec;
    frame_fixed_kernels_[method * 2 + (reorder ? 1 : 0)] = capture_kernels_;
}

int Engine::frame(int id, int32_t method, SceneState& out) {
    if (!use_graphs_ || timing_ || has_force_callbacks() || active_scenes() != 1 ||
        !scenes_[id].active || !frame_graphs_ok_) {
        // host loop: one sub-step at a time, the frame's end read after each
        int n = 0;
        do {
            substep(method);
            ++n;
            out = scene_state(id);
        } while (out.remaining > 0 && n < 100000);
        return n;
    }
    prepare_substep(method);
    bool const reorder = reorder_every_ > 0 && (frames_launched_ % 2) == 0;
    ++frames_launched_;
    int const key = method * 2 + (reorder ? 1 : 0);
    auto it = frame_graphs_.find(key);
    if (it == frame_graphs_.end()) {
        try {
            capture_frame(method, reorder);
        } catch (std::runtime_error const&) {
            // a device or driver without the frame graph's nested
            // conditional nodes: frames keep the host loop from now on
            frame_graphs_ok_ = false;
            --frames_launched_;
            return frame(id, method, out);
        }
        it = frame_graphs_.find(key);
    }
    if (cudaGraphLaunch(it->second, st_) != cudaSuccess) {
        check("frame graph launch");
        throw std::runtime_error("frame graph launch failed");
    }
    int64_t const fixed = frame_fixed_kernels_[key];
    host_launches_ += fixed;
    g_launches.fetch_add(fixed, std::memory_order_relaxed);
    out = scene_state(id);
    substeps_launched_ += out.call_substeps;
    return out.call_substeps;
}

// Tunings chosen by autotune, per (method, log2 of the active particle
// count); engines of the same size class start from them.
namespace {
std::mutex g_tuning_mutex;
std::map<uint64_t, Engine::Tuning> g_tuning_cache;
}  // namespace

uint64_t Engine::tuning_key(int32_t method) const {
    uint64_t n = 0;
    for (auto const& sc : scenes_) {
        if (sc.used && sc.active) n += sc.p.fluid_count;
    }
    // batches and single scenes keep separate tunings
    return uint64_t(method) * 128u + (max_scenes_ > 1 ? 64u : 0u) +
           ceil_log2(std::max<uint64_t>(n, 1));
}

// Tuning cache lookup and per-scene method parameters before a sub-step or
// frame of `method`.
void Engine::prepare_substep(int32_t method) {
    if (!tuning_locked_ && !tuning_pinned_) {
        std::lock_guard<std::mutex> lock(g_tuning_mutex);
        auto const it = g_tuning_cache.find(tuning_key(method));
        if (it != g_tuning_cache.end() && !(it->second == tuning_)) {
            tuning_ = it->second;
            destroy_graphs();
        }
    }
    last_method_ = method;
    for (int id = 0; id < max_scenes_; ++id) {
        Scene& sc = scenes_[id];
        if (!sc.used || !sc.active) continue;
        if (sc.p.method != method) {
            sc.p.method = method;
            sc.p.max_denom = method == kIisph ? 6 : 4;
            sc.p.cfl_factor = method == kIisph ? 0.2f : 0.4f;
            upload_params(id);
        }
    }
}

void Engine::substep(int32_t method) {
    if (active_scenes() == 0) return;
    prepare_substep(method);
    bool const reorder = reorder_every_ > 0 && (substeps_launched_ % reorder_every_) == 0;
    ++substeps_launched_;
    if (use_graphs_ && !timing_ && !has_force_callbacks()) {
        int const key = method * 2 + (reorder ? 1 : 0);
        auto it = graphs_.find(key);
        if (it == graphs_.end()) {
            capture_substep(method, reorder);
            it = graphs_.find(key);
        }
        if (cudaGraphLaunch(it->second, st_) != cudaSuccess) {
            check("graph launch");
            throw std::runtime_error("graph launch failed");
        }
        int64_t const fixed = graph_fixed_kernels_[key];
        host_launches_ += fixed;
        g_launches.fetch_add(fixed, std::memory_order_relaxed);
        check("substep graph");
        return;
    }
    cur_ = st_;
    emit_substep(method, reorder);
    check("substep");
}

// Times whole sub-steps of `method` with each candidate tuning, every
// candidate from the same state (positions, velocities, kappas, storage
// order, frame clocks and launch counters are snapshotted and restored), and
// keeps the fastest. The candidates give the same bits, so the choice
// changes speed only.
Engine::TuneReport Engine::autotune(int32_t method, int substeps) {
    if (last_method_ != method) {
        throw std::invalid_argument("autotune: run a sub-step of this method first");
    }
    if (method != kDfsph && method != kIisph) {
        throw std::invalid_argument("autotune: DFSPH_P and IISPH have tunable kernels");
    }
    size_t const N = fluid_cap_;
    struct Region {
        void* dev;
        size_t size;
    };
    Region const regions[] = {{a_.x, 8 * N},      {a_.v, 8 * N},         {a_.kdiv, 4 * N},
                              {a_.kdens, 4 * N},  {a_.x64, 16 * N},      {a_.oid, 4 * N},
                              {a_.slot_of, 4 * N}, {d_ss_, sizeof(SceneState) * size_t(max_scenes_)},
                              {d_loop_iters_, sizeof(unsigned long long) * kLoopSlots}};
    size_t bytes = 0;
    for (auto const& r : regions) bytes += r.size;
    char* snap = nullptr;
    if (cudaMalloc(&snap, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw std::bad_alloc();
    }
    auto copy = [&](bool save) {
        size_t off = 0;
        for (auto const& r : regions) {
            if (save) {
                cudaMemcpyAsync(snap + off, r.dev, r.size, cudaMemcpyDeviceToDevice, st_);
            } else {
                cudaMemcpyAsync(r.dev, snap + off, r.size, cudaMemcpyDeviceToDevice, st_);
            }
            off += r.size;
        }
    };
    copy(true);
    int64_t const launched0 = substeps_launched_;
    int64_t const host0 = host_launches_;
    int64_t const global0 = g_launches.load();
    std::vector<Tuning> cand;
    if (method == kDfsph) {
        // chunks, with kPrefetchLists (P) where the warps first ask L2 for
        // their list rows: it pays when the lists do not stay in L2
        // and with kPersistentWarps (W), the persistent-warp kernels
        int const P = kPrefetchLists;
        int const W = kPersistentWarps;
        // (W2: the same in blocks of 256 threads)
        int const W2 = kPersistentWarps | kPersistentBlocks256;
        // (F: the loop's exit test fused into the apply kernel's last block)
        int const F = kFusedExitTest;
        int const opts[][2] = {{4, 8}, {1, 4}, {4, 4}, {1, 8}, {8, 8},
                               {1 | P, 4 | P}, {4 | P, 8 | P}, {1 | P, 4},
                               {1 | W, 4 | W}, {4 | W, 4 | W}, {1 | W, 1 | W}, {4 | W, 8 | W},
                               {1 | W2, 4 | W2}, {4 | W2, 4 | W2},
                               {1 | W | F, 4 | W}, {1 | W2 | F, 4 | W2}};
        for (auto const& o : opts) {
            Tuning t = tuning_;
            t.apply = o[0];
            t.divergence = o[1];
            cand.push_back(t);
        }
    } else {
        int const P = kPrefetchLists;
        int const W = kPersistentWarps;
        int const W2 = kPersistentWarps | kPersistentBlocks256;
        int const F = kFusedExitTest;
        int const opts[][2] = {{4, 4}, {1, 1}, {1, 4}, {4, 1}, {8, 4},
                               {4 | P, 4 | P}, {1 | P, 1 | P}, {4 | P, 1 | P},
                               {4 | W, 4 | W}, {1 | W, 1 | W}, {1 | W, 4 | W}, {4 | W2, 4 | W2},
                               {4 | W, 4 | W | F}, {4 | W2, 4 | W2 | F}};
        for (auto const& o : opts) {
            Tuning t = tuning_;
            t.iisph_sum = o[0];
            t.iisph_beta = o[1];
            cand.push_back(t);
        }
    }
    if (max_scenes_ > 1) {
        // A batch's loops run as long as its slowest scene's; only the
        // persistent-warp kernels walk just the scenes still iterating, so a
        // batch chooses among them (a few sub-steps after the start, where
        // the tuner times them, do not yet show the slow scenes' long loops)
        bool const dfsph = method == kDfsph;
        cand.erase(std::remove_if(cand.begin(), cand.end(),
                                  [&](Tuning const& t) {
                                      int const x = dfsph ? t.apply : t.iisph_sum;
                                      int const y = dfsph ? t.divergence : t.iisph_beta;
                                      return !((x & kPersistentWarps) && (y & kPersistentWarps));
                                  }),
                   cand.end());
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    TuneReport rep{};
    tuning_locked_ = true;
    float best = 0.0f;
    Tuning best_t = cand[0];
    try {
        for (size_t k = 0; k < cand.size(); ++k) {
            tuning_ = cand[k];
            destroy_graphs();
            // the same sub-steps once untimed: captures every graph they use
            for (int q = 0; q < substeps; ++q) substep(method);
            copy(false);
            substeps_launched_ = launched0;
            cudaEventRecord(e0, st_);
            for (int q = 0; q < substeps; ++q) substep(method);
            cudaEventRecord(e1, st_);
            ++host_waits_;
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            rep.candidates[k] = cand[k];
            rep.ms[k] = ms / float(substeps);
            if (k == 0 || rep.ms[k] < best) {
                best = rep.ms[k];
                best_t = cand[k];
            }
            copy(false);
            substeps_launched_ = launched0;
        }
    } catch (...) {
        tuning_locked_ = false;
        cudaFree(snap);
        throw;
    }
    rep.count = int(cand.size());
    tuning_locked_ = false;
    host_wait(st_);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(snap);
    host_launches_ = host0;
    g_launches.fetch_sub(g_launches.load() - global0);
    check("autotune");
    tuning_ = best_t;
    destroy_graphs();
    {
        std::lock_guard<std::mutex> lock(g_tuning_mutex);
        g_tuning_cache[tuning_key(method)] = tuning_;
    }
    rep.chosen = tuning_;
    return rep;
}

void Engine::set_tuning(Tuning const* t) {
    tuning_pinned_ = t != nullptr;
    if (t && !(*t == tuning_)) {
        tuning_ = *t;
        destroy_graphs();
    }
}

// ------------------------------------------------------------ accessors

SceneState Engine::scene_state(int id) {
    SceneState s{};
    cudaMemcpyAsync(&s, d_ss_ + id, sizeof(SceneState), cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    check("scene_state");
    return s;
}

std::vector<SceneState> Engine::all_states() {
    std::vector<SceneState> s(max_scenes_);
    cudaMemcpyAsync(s.data(), d_ss_, sizeof(SceneState) * max_scenes_, cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    check("all_states");
    return s;
}

// Positions and velocities in original particle order: gathered through
// slot_of into the reorder staging buffers, then copied out.
void Engine::get_state(int id, float* x, float* v, bool sync) {
    SceneParams const& P = scenes_[id].p;
    uint32_t const b = P.fluid_begin, n = P.fluid_count;
    if (x) {
        launch_gather_f2(a_, b, n, a_.x, a_.tx + b, st_);
        cudaMemcpyAsync(x, a_.tx + b, 8ull * n, cudaMemcpyDeviceToHost, st_);
    }
    if (v) {
        launch_gather_f2(a_, b, n, a_.v, a_.tv + b, st_);
        cudaMemcpyAsync(v, a_.tv + b, 8ull * n, cudaMemcpyDeviceToHost, st_);
    }
    if (sync) host_wait(st_);
    check("get_state");
}

bool Engine::set_state(int id, float const* x, float const* v, bool sync) {
    SceneParams const& P = scenes_[id].p;
    uint32_t const b = P.fluid_begin, n = P.fluid_count;
    if (!x && !v) return true;
    // the new values are staged and checked on the device before any of
    // them replaces the scene's state
    cudaMemsetAsync(d_flag_, 0, sizeof(uint32_t), st_);
    if (x) {
        cudaMemcpyAsync(a_.tx + b, x, 8ull * n, cudaMemcpyHostToDevice, st_);
        launch_flag_nonfinite(reinterpret_cast<float const*>(a_.tx + b), 2ull * n, d_flag_, st_);
    }
    if (v) {
        cudaMemcpyAsync(a_.tv + b, v, 8ull * n, cudaMemcpyHostToDevice, st_);
        launch_flag_nonfinite(reinterpret_cast<float const*>(a_.tv + b), 2ull * n, d_flag_, st_);
    }
    cudaMemcpyAsync(h_flag_, d_flag_, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    check("set_state");
    if (*h_flag_) return false;
    if (x) {
        launch_scatter_f2(a_, b, n, a_.tx + b, a_.x, st_);
        launch_positions_to_double(a_, b, n, st_);
    }
    if (v) launch_scatter_f2(a_, b, n, a_.tv + b, a_.v, st_);
    if (sync) host_wait(st_);
    check("set_state");
    return true;
}

namespace {
struct SnapshotHeader {
    char magic[8];
    uint32_t version;
    uint32_t n_fluid, n_solid;
    int32_t precision;
    uint64_t bytes;
};
constexpr char kSnapshotMagic[8] = {'E', 'M', 'S', 'N', 'A', 'P', '0', '1'};

size_t snapshot_bytes(uint32_t n, uint32_t ns, bool x64) {
    return sizeof(SnapshotHeader) + sizeof(SceneState) + 16ull * n + 8ull * n +
           (x64 ? 16ull * n : 0) + 20ull * ns;
}
}  // namespace

size_t Engine::snapshot_size(int id) const {
    SceneParams const& P = scenes_[id].p;
    return snapshot_bytes(P.fluid_count, P.solid_count, P.precision != 0);
}

// Layout: header, SceneState, positions and velocities (float pairs), the
// DFSPH divergence and density kappas, in compensated mode the FP64
// positions (all in original particle order), then the boundary positions,
// velocities and volumes.
void Engine::snapshot(int id, void* out) {
    SceneParams const& P = scenes_[id].p;
    uint32_t const b = P.fluid_begin, n = P.fluid_count, ns = P.solid_count;
    bool const x64 = P.precision != 0;
    auto* p = static_cast<unsigned char*>(out);
    SnapshotHeader h{};
    std::memcpy(h.magic, kSnapshotMagic, 8);
    h.version = 1;
    h.n_fluid = n;
    h.n_solid = ns;
    h.precision = P.precision;
    h.bytes = snapshot_bytes(n, ns, x64);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    SceneState const s = scene_state(id);
    std::memcpy(p, &s, sizeof(s));
    p += sizeof(s);
    get_state(id, reinterpret_cast<float*>(p), reinterpret_cast<float*>(p + 8ull * n), true);
    p += 16ull * n;
    launch_gather_f(a_, b, n, a_.kdiv, a_.tkdiv + b, st_);
    cudaMemcpyAsync(p, a_.tkdiv + b, 4ull * n, cudaMemcpyDeviceToHost, st_);
    launch_gather_f(a_, b, n, a_.kdens, a_.tkdens + b, st_);
    cudaMemcpyAsync(p + 4ull * n, a_.tkdens + b, 4ull * n, cudaMemcpyDeviceToHost, st_);
    p += 8ull * n;
    if (x64) {
        launch_gather_d2(a_, b, n, a_.x64, a_.tx64 + b, st_);
        cudaMemcpyAsync(p, a_.tx64 + b, 16ull * n, cudaMemcpyDeviceToHost, st_);
        p += 16ull * n;
    }
    cudaMemcpyAsync(p, a_.xs + P.solid_begin, 8ull * ns, cudaMemcpyDeviceToHost, st_);
    cudaMemcpyAsync(p + 8ull * ns, a_.vs + P.solid_begin, 8ull * ns, cudaMemcpyDeviceToHost, st_);
    cudaMemcpyAsync(p + 16ull * ns, a_.vols + P.solid_begin, 4ull * ns, cudaMemcpyDeviceToHost,
                    st_);
    host_wait(st_);
    check("snapshot");
}

void Engine::restore(int id, void const* data, size_t bytes) {
    SceneParams const& P = scenes_[id].p;
    uint32_t const b = P.fluid_begin, n = P.fluid_count, ns = P.solid_count;
    bool const x64 = P.precision != 0;
    auto const* p = static_cast<unsigned char const*>(data);
    SnapshotHeader h{};
    if (bytes < sizeof(h)) throw std::invalid_argument("snapshot too short");
    std::memcpy(&h, p, sizeof(h));
    if (std::memcmp(h.magic, kSnapshotMagic, 8) != 0 || h.version != 1) {
        throw std::invalid_argument("not a snapshot of this library");
    }
    if (h.n_fluid != n || h.n_solid != ns || h.precision != P.precision) {
        throw std::invalid_argument("snapshot of a scene with other particle counts or precision");
    }
    if (h.bytes != bytes || bytes != snapshot_bytes(n, ns, x64)) {
        throw std::invalid_argument("snapshot size does not match");
    }
    p += sizeof(h);
    SceneState s{};
    std::memcpy(&s, p, sizeof(s));
    p += sizeof(s);
    float const* xv = reinterpret_cast<float const*>(p);
    if (!set_state(id, xv, xv + 2ull * n, false)) {
        throw std::invalid_argument("snapshot holds non-finite positions or velocities");
    }
    p += 16ull * n;
    cudaMemcpyAsync(a_.tkdiv + b, p, 4ull * n, cudaMemcpyHostToDevice, st_);
    launch_scatter_f(a_, b, n, a_.tkdiv + b, a_.kdiv, st_);
    cudaMemcpyAsync(a_.tkdens + b, p + 4ull * n, 4ull * n, cudaMemcpyHostToDevice, st_);
    launch_scatter_f(a_, b, n, a_.tkdens + b, a_.kdens, st_);
    p += 8ull * n;
    if (x64) {
        cudaMemcpyAsync(a_.tx64 + b, p, 16ull * n, cudaMemcpyHostToDevice, st_);
        launch_scatter_d2(a_, b, n, a_.tx64 + b, a_.x64, st_);
        p += 16ull * n;
    }
    host_wait(st_);
    check("restore");
    float const* sxy = reinterpret_cast<float const*>(p);
    set_solid(id, sxy, sxy + 2ull * ns, sxy + 4ull * ns);
    // the frame clock, counters and last statistics; the scene stays as
    // active as it is now
    int32_t const active = scenes_[id].active ? 1 : 0;
    s.active = active;
    cudaMemcpyAsync(d_ss_ + id, &s, sizeof(s), cudaMemcpyHostToDevice, st_);
    host_wait(st_);
    check("restore");
}

void Engine::get_solid(int id, float* xy, float* volumes) {
    SceneParams const& P = scenes_[id].p;
    if (xy) cudaMemcpyAsync(xy, a_.xs + P.solid_begin, 8ull * P.solid_count, cudaMemcpyDeviceToHost, st_);
    if (volumes) {
        cudaMemcpyAsync(volumes, a_.vols + P.solid_begin, 4ull * P.solid_count,
                        cudaMemcpyDeviceToHost, st_);
    }
    host_wait(st_);
    check("get_solid");
}

void Engine::set_solid(int id, float const* xy, float const* v, float const* volumes) {
    Scene& sc = scenes_[id];
    SceneParams& P = sc.p;
    uint32_t const b = P.solid_begin, n = P.solid_count;
    if (!n) return;
    if (xy) {
        cudaMemcpyAsync(a_.xs + b, xy, 8ull * n, cudaMemcpyHostToDevice, st_);
        host_wait(st_);
        if (sc.near_words) near_words_.release(P.near_begin, sc.near_words);
        build_near_map(sc, xy, n);
        upload_params(id);
        rebuild_solids();
    }
    if (v) cudaMemcpyAsync(a_.vs + b, v, 8ull * n, cudaMemcpyHostToDevice, st_);
    if (volumes) {
        cudaMemcpyAsync(a_.vols + b, volumes, 4ull * n, cudaMemcpyHostToDevice, st_);
    } else if (xy) {
        launch("solid_volumes", [&] { launch_solid_volumes(a_, ext_stiles_, 1.7f, id, st_); });
    }
    host_wait(st_);
    check("set_solid");
}

bool Engine::get_array(int id, std::string const& name, float* out, int& width) {
    SceneParams const& P = scenes_[id].p;
    void const* src = nullptr;
    width = 1;
    if (name == "densities") {
        src = a_.rho;
    } else if (name == "pressures") {
        if (P.method == kIisph) {
            SceneState const s = scene_state(id);
            src = (s.iter & 1) ? a_.pbuf1 : a_.pbuf0;
        } else if (P.method == kDfsph) {
            return false;
        } else {
            src = a_.pbuf0;
        }
    } else if (name == "density_stars") {
        src = a_.rho_star;
    } else if (name == "aiis") {
        src = a_.aii;
    } else if (name == "alphas") {
        src = a_.alpha;
    } else if (name == "divergence_kappas") {
        src = a_.kdiv;
    } else if (name == "density_kappas") {
        src = a_.kdens;
    } else if (name == "diis") {
        src = a_.dii;
        width = 2;
    } else if (name == "sum_dij_pjs") {
        src = a_.sdp;
        width = 2;
    } else if (name == "pressure_forces") {
        src = a_.fp;
        width = 2;
    } else if (name == "pressure_accelerations") {
        src = a_.acc;
        width = 2;
    } else if (name == "velocity_external_forces") {
        src = a_.vext;
        width = 2;
    } else if (name == "position_stars") {
        src = a_.xstar;
        width = 2;
    } else if (name == "velocity_stars") {
        src = a_.vstar;
        width = 2;
    } else {
        return false;
    }
    if (out) {
        uint32_t const b = P.fluid_begin, n = P.fluid_count;
        if (width == 2) {
            launch_gather_f2(a_, b, n, static_cast<float2 const*>(src), a_.tx + b, st_);
            cudaMemcpyAsync(out, a_.tx + b, 8ull * n, cudaMemcpyDeviceToHost, st_);
        } else {
            launch_gather_f(a_, b, n, static_cast<float const*>(src), a_.tkdiv + b, st_);
            cudaMemcpyAsync(out, a_.tkdiv + b, 4ull * n, cudaMemcpyDeviceToHost, st_);
        }
        host_wait(st_);
        check("get_array");
    }
    return true;
}

void Engine::get_neighbors(int id, bool solid, uint8_t* counts, uint32_t* idx, float* w,
                           float* gw) {
    SceneParams const& P = scenes_[id].p;
    uint32_t const n = P.fluid_count;
    size_t const stride = a_.stride;
    std::vector<uint8_t> cnt(n);
    cudaMemcpyAsync(cnt.data(), (solid ? a_.ns_cnt : a_.nf_cnt) + P.fluid_begin, n,
                    cudaMemcpyDeviceToHost, st_);
    std::vector<uint32_t> ri(size_t(n) * kMaxNeighbors);
    std::vector<float> rw(size_t(n) * kMaxNeighbors);
    std::vector<float2> rg(size_t(n) * kMaxNeighbors);
    for (int k = 0; k < kMaxNeighbors; ++k) {
        size_t const off = size_t(k) * stride + P.fluid_begin;
        if (idx) {
            cudaMemcpyAsync(ri.data() + size_t(k) * n, (solid ? a_.ns_idx : a_.nf_idx) + off, 4ull * n,
                            cudaMemcpyDeviceToHost, st_);
        }
        if (w) {
            cudaMemcpyAsync(rw.data() + size_t(k) * n, (solid ? a_.ns_w : a_.nf_w) + off, 4ull * n,
                            cudaMemcpyDeviceToHost, st_);
        }
        if (gw) {
            cudaMemcpyAsync(rg.data() + size_t(k) * n, (solid ? a_.ns_gw : a_.nf_gw) + off, 8ull * n,
                            cudaMemcpyDeviceToHost, st_);
        }
    }
    std::vector<uint32_t> oid(n), slot_of(n);
    cudaMemcpyAsync(oid.data(), a_.oid + P.fluid_begin, 4ull * n, cudaMemcpyDeviceToHost, st_);
    cudaMemcpyAsync(slot_of.data(), a_.slot_of + P.fluid_begin, 4ull * n, cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    check("get_neighbors");
    uint32_t const base = solid ? P.solid_begin : P.fluid_begin;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t const row = slot_of[i] - P.fluid_begin;  // storage column of particle i
        if (counts) counts[i] = cnt[row];
        for (int k = 0; k < kMaxNeighbors; ++k) {
            size_t const o = size_t(i) * kMaxNeighbors + k;
            size_t const r = size_t(k) * n + row;
            bool const live = k < cnt[row];
            uint32_t const j = live ? ri[r] - base : 0u;
            if (idx) idx[o] = live ? (solid ? j : oid[j]) : 0u;
            if (w) w[o] = live ? rw[r] : 0.0f;
            if (gw) {
                gw[2 * o] = live ? rg[r].x : 0.0f;
                gw[2 * o + 1] = live ? rg[r].y : 0.0f;
            }
        }
    }
}

void Engine::ensure_sort_scratch(uint32_t n) {
    if (sort_buf_ && sort_cap_ >= n) return;
    if (sort_buf_) cudaFree(sort_buf_);
    sort_buf_ = nullptr;
    size_t const bytes = sort_scratch_bytes(n);
    if (cudaMalloc(&sort_buf_, bytes) != cudaSuccess) {
        cudaGetLastError();
        sort_buf_ = nullptr;
        throw std::bad_alloc();
    }
    sort_cap_ = n;
    sort_scratch_carve(sort_buf_, n, sort_);
}

size_t Engine::get_sort(int id, bool solid, int32_t* gc, uint64_t* z, uint64_t* pair_z,
                        uint64_t* pair_index, uint32_t* block_indices, uint64_t* blocks) {
    SceneParams const& P = scenes_[id].p;
    Scene const& sc = scenes_[id];
    uint32_t const n = solid ? P.solid_count : P.fluid_count;
    if (n == 0) return 0;
    ensure_sort_scratch(std::max(n, solid ? sc.stab_size : sc.ftab_size));
    size_t const words = size_t(n);
    void* out = nullptr;
    size_t const bytes = words * (8 + 8 + 8 + 4 + 4 + 8) + 64;
    if (cudaMalloc(&out, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw std::bad_alloc();
    }
    char* p = static_cast<char*>(out);
    int2* d_gc = reinterpret_cast<int2*>(p);
    p += 8 * words;
    uint64_t* d_z = reinterpret_cast<uint64_t*>(p);
    p += 8 * words;
    uint64_t* d_pz = reinterpret_cast<uint64_t*>(p);
    p += 8 * words;
    uint32_t* d_pi = reinterpret_cast<uint32_t*>(p);
    p += 4 * words;
    uint32_t* d_bi = reinterpret_cast<uint32_t*>(p);
    p += 4 * words;
    uint32_t* d_bl = reinterpret_cast<uint32_t*>(p);
    p += 8 * words;
    uint32_t* d_nb = reinterpret_cast<uint32_t*>(p);
    launch("sort_products", [&] {
        launch_sort_products(a_, solid, id, solid ? P.solid_begin : P.fluid_begin, n,
                             solid ? P.stab_begin : P.ftab_begin, solid ? sc.stab_size : sc.ftab_size,
                             P.cell_size, sort_, d_gc, d_z, d_pz, d_pi, d_bi, d_bl, d_nb, st_);
    });
    uint32_t nb = 0;
    std::vector<uint32_t> hpi(n), hbl(2 * size_t(n));
    cudaMemcpyAsync(&nb, d_nb, 4, cudaMemcpyDeviceToHost, st_);
    if (gc) cudaMemcpyAsync(gc, d_gc, 8 * words, cudaMemcpyDeviceToHost, st_);
    if (z) cudaMemcpyAsync(z, d_z, 8 * words, cudaMemcpyDeviceToHost, st_);
    if (pair_z) cudaMemcpyAsync(pair_z, d_pz, 8 * words, cudaMemcpyDeviceToHost, st_);
    cudaMemcpyAsync(hpi.data(), d_pi, 4 * words, cudaMemcpyDeviceToHost, st_);
    if (block_indices) cudaMemcpyAsync(block_indices, d_bi, 4 * words, cudaMemcpyDeviceToHost, st_);
    cudaMemcpyAsync(hbl.data(), d_bl, 8 * words, cudaMemcpyDeviceToHost, st_);
    host_wait(st_);
    cudaFree(out);
    check("get_sort");
    if (pair_index) {
        for (uint32_t k = 0; k < n; ++k) pair_index[k] = hpi[k];
    }
    if (blocks) {
        for (uint32_t b = 0; b < nb; ++b) {
            blocks[2 * b] = hbl[2 * b];
            blocks[2 * b + 1] = hbl[2 * b + 1];
        }
    }
    return nb;
}

}  // namespace emerald
