// Host-side engine: owns a device arena of scenes and launches the kernel
// sequence of one solver sub-step for every active scene.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/emerald_sph.h"
#include "engine_types.cuh"
#include "kernels.cuh"
#include "sph_math.cuh"

namespace emerald {

// First-fit allocator of [begin, begin + size) ranges in [0, capacity).
class RangeAllocator {
public:
    explicit RangeAllocator(uint32_t capacity = 0);
    bool alloc(uint32_t size, uint32_t& begin);
    void release(uint32_t begin, uint32_t size);
    uint32_t capacity() const { return capacity_; }
    uint32_t largest_free() const;

private:
    uint32_t capacity_;
    std::map<uint32_t, uint32_t> free_;  // begin -> size
};

struct SceneSpec {
    emerald_params params;
    int32_t method = kDfsph;
    int32_t mode = kFrame;
    float fixed_dt = 0.0f;
    float const* solid_xy = nullptr;
    float const* solid_volumes = nullptr;  // NULL: compute_volumes with numer 1.7
    uint32_t n_solid = 0;
    float const* fluid_xy = nullptr;
    float const* fluid_v = nullptr;
    uint32_t n_fluid = 0;
};

// Simulation_config derived from Parameters (emerald/sph2d_box/config.cpp:16-132).
struct DerivedConfig {
    float seconds_per_sub_step;
    float mass_per_particle;
    float draw_radius;
    float pressure_correction_denom;
};
DerivedConfig derive_config(emerald_params const& p);
void default_params(emerald_params& p);

struct KernelTimes {
    std::map<std::string, double> ms;
    std::map<std::string, int> launches;
};

class Engine {
public:
    // Neighbour entries loaded together by each gather-sum kernel (1, 4 or
    // 8); every choice gives the same bits. The DFSPH defaults are the
    // autotuner's usual pick for the dam break (measured on B200 from the same
    // state: 2.13 against 2.24 ms per sub-step at 262,144 particles, 6.85
    // against 7.67 ms at 1,048,576, over (4, 8)); engines that are not tuned
    // (request-loop lanes, size classes without a tuned entry) start there.
    struct Tuning {
        int apply = 1, divergence = 4, iisph_sum = 4, iisph_beta = 4;
        bool operator==(Tuning const& o) const {
            return apply == o.apply && divergence == o.divergence && iisph_sum == o.iisph_sum &&
                   iisph_beta == o.iisph_beta;
        }
    };
    struct TuneReport {
        Tuning chosen;
        int count;               // candidates timed
        Tuning candidates[16];
        float ms[16];            // mean sub-step time of each candidate
    };
    Engine(uint32_t fluid_capacity, uint32_t solid_capacity, int max_scenes);
    ~Engine();
    // Device bytes the constructor allocates for these capacities.
    static size_t footprint(uint32_t fluid_capacity, uint32_t solid_capacity, int max_scenes);
    size_t device_bytes() const { return device_bytes_; }
    uint32_t fluid_capacity() const { return fluid_cap_; }
    uint32_t solid_capacity() const { return solid_cap_; }
    Engine(Engine const&) = delete;
    Engine& operator=(Engine const&) = delete;

    // Returns the scene id, or -1 when the arena has no room.
    int add_scene(SceneSpec const& spec);
    void remove_scene(int id);
    void set_active(int id, bool active);
    // Frame mode, or fixed-dt mode with the caller's sub-step time t and dt.
    void set_mode(int id, int32_t mode, float fixed_dt, float fixed_t = 0.0f);
    // External forces of a scene (compute_all_external_forces,
    // emerald/sph2d_box/forces.cpp:11-33): `count` terms (at most
    // kMaxForceTerms; 0: none) evaluated on the device where the solver
    // computes its forces. A new scene has one gravity term with the
    // parameters' gravity, as default_gravity_forces gives.
    void set_forces(int id, ForceTerm const* terms, int count);
    // A host function standing for the reference's User_forces_function
    // (emerald/sph2d_box/forces.h:13-21): once per sub-step, at the point of
    // the sub-step where the solver computes its external forces, it gets
    // the scene's positions and velocities at that point (original particle
    // order), the sub-step's time and dt, the mass and draw radius, and
    // fills the forces (zeroed first). Sub-steps of an engine with a
    // callback run without graphs (the call needs the state on the host).
    // NULL removes it; the force terms apply again.
    using ForceCallback = void (*)(void* user, size_t count, float time, float dt, float mass,
                                   float radius, float* forces, float const* positions,
                                   float const* velocities);
    void set_force_callback(int id, ForceCallback fn, void* user);
    bool scene_used(int id) const { return id >= 0 && id < (int)scenes_.size() && scenes_[id].used; }

    void set_stream(cudaStream_t st) { st_ = st; }
    cudaStream_t stream() const { return st_; }

    // Zeroes the per-frame temporaries of the active scenes (fixed-dt runs).
    void begin_frame(int32_t method);
    // One sub-step of `method` for every active scene.
    void substep(int32_t method);

    // Synchronous accessors of one scene (original particle order).
    // sync = false leaves the copies queued on the engine's stream (the
    // caller synchronizes before it touches the host buffers).
    void get_state(int id, float* x, float* v, bool sync = true);
    // Returns false, and leaves the scene as it was, when x or v holds an
    // infinity or a NaN (checked on the device before anything is replaced;
    // one stream synchronisation).
    bool set_state(int id, float const* x, float const* v, bool sync = true);
    // Checkpoint of one scene between sub-steps: its frame clock and
    // counters (SceneState), positions, velocities and DFSPH kappas in
    // original order, the FP64 positions of a compensated scene, and its
    // boundary. restore() takes a snapshot of a scene with the same particle
    // counts and precision mode; the sub-steps after it equal those after
    // the snapshot was taken, bit for bit.
    size_t snapshot_size(int id) const;
    void snapshot(int id, void* out);
    void restore(int id, void const* data, size_t bytes);
    void get_solid(int id, float* xy, float* volumes);
    // Replaces a scene's boundary particles between sub-steps (count kept):
    // positions (NULL keeps them; new ones rebuild the boundary cell tables
    // and proximity map), velocities (NULL keeps them) and volumes (NULL:
    // recomputed from new positions, kept otherwise).
    void set_solid(int id, float const* xy, float const* v, float const* volumes);
    bool get_array(int id, std::string const& name, float* out, int& width);
    void get_neighbors(int id, bool solid, uint8_t* counts, uint32_t* idx, float* w, float* gw);
    size_t get_sort(int id, bool solid, int32_t* gc, uint64_t* z, uint64_t* pair_z,
                    uint64_t* pair_index, uint32_t* block_indices, uint64_t* blocks);
    SceneState scene_state(int id);
    SceneParams const& scene_params(int id) const { return scenes_[id].p; }
    std::vector<SceneState> all_states();
    uint32_t fluid_count(int id) const { return scenes_[id].p.fluid_count; }
    uint32_t solid_count(int id) const { return scenes_[id].p.solid_count; }
    float2* device_x(int id) { return a_.x + scenes_[id].p.fluid_begin; }
    float2* device_v(int id) { return a_.v + scenes_[id].p.fluid_begin; }
    int active_scenes() const;
    size_t free_fluid() const { return size_t(fluid_tiles_.largest_free()) * kTile; }
    // Largest free runs of each arena region, for admission decisions made
    // away from the thread that owns the engine.
    struct Room {
        uint32_t fluid_tiles, solid_tiles, fluid_table, solid_table;
        int scene_slots;
        bool fits(uint32_t n_fluid, uint32_t n_solid) const;
    };
    Room room() const;
    int free_scene_slots() const {
        int n = 0;
        for (auto const& s : scenes_) n += s.used ? 0 : 1;
        return n;
    }

    void enable_timing(bool on);
    KernelTimes const& kernel_times();
    void reset_timing();
    // Loop control: false runs the exit test on the host after each solver
    // iteration (one stream synchronisation per iteration, like the
    // reference); true launches every iteration up to the cap and lets
    // finished scenes' kernels return at once (no host round trips).
    void set_unrolled_loops(bool on) { unrolled_ = on; }
    // Graph mode (default): each sub-step is one CUDA graph launch, with the
    // solver loops as conditional while nodes (no host round trips).
    void set_graphs(bool on) { use_graphs_ = on; }
    // Sub-steps between re-sorts of the particle storage order (0: never).
    void set_reorder_every(int k) { reorder_every_ = k; }
    // Kernels this engine launched (graph nodes included, loop bodies
    // counted per executed iteration).
    int64_t kernel_launches();
    // Times this engine waited on the host for the device.
    int64_t host_waits() const { return host_waits_; }
    // One frame of the single resident scene (emerald_sim_frame): with
    // graphs, one graph launch (re-sort, then a conditional while node
    // around the sub-step while the frame has sub-steps left) and one host
    // wait; returns the sub-steps run and the scene's state after them.
    int frame(int id, int32_t method, SceneState& out);

    void check(char const* what);

    // Picks the fastest chunk settings of `method`'s gather kernels by timing
    // whole sub-steps on the resident scenes (after at least one sub-step of
    // it), restoring the state after each; the choice is kept for engines of
    // the same method and size class.
    TuneReport autotune(int32_t method, int substeps = 4);
    Tuning const& tuning() const { return tuning_; }
    // Pins the gather kernels' settings (no cache lookups until unpinned);
    // nullptr unpins.
    void set_tuning(Tuning const* t);

private:
    uint64_t tuning_key(int32_t method) const;
    Tuning tuning_{};
    bool tuning_locked_ = false;
    bool tuning_pinned_ = false;
    int32_t last_method_ = -1;
    struct Scene {
        bool used = false;
        SceneParams p{};
        uint32_t ftile_begin = 0, ftile_count = 0, stile_begin = 0, stile_count = 0;
        uint32_t ftab_size = 0, stab_size = 0;
        uint32_t near_words = 0;
        bool active = false;
        float draw_radius = 0.0f;
        ForceCallback force_fn = nullptr;
        void* force_user = nullptr;
    };
    bool has_force_callbacks() const;
    // Calls the force callbacks of the active scenes and uploads their forces.
    void host_forces(int32_t method);
    std::vector<float> hx_, hv_, hf_;

    template <class F>
    void launch(char const* name, F&& f, int kernels = 1);
    void upload_params(int id);
    void upload_tiles();
    void run_loop(int kind, int max_iter, int32_t method);
    void emit_substep(int32_t method, bool reorder);
    void emit_loop_body(int kind, int32_t method, cudaGraphConditionalHandle cond, bool use_cond);
    void capture_substep(int32_t method, bool reorder);
    void update_sort_bases();
    int order_key_bits() const;
    void destroy_graphs();
    void capture_frame(int32_t method, bool reorder);
    void prepare_substep(int32_t method);
    int64_t frames_launched_ = 0;
    bool frame_graphs_ok_ = true;
    void host_wait(cudaStream_t s) {
        ++host_waits_;
        cudaStreamSynchronize(s);
    }
    int64_t host_waits_ = 0;
    cudaStream_t frame_st_ = nullptr;                  // frame-loop body capture
    std::map<int32_t, cudaGraphExec_t> frame_graphs_;  // key: method * 2 + reorder
    std::map<int32_t, int64_t> frame_fixed_kernels_;   // per graph, outside the loop
    int64_t frame_body_kernels_[5] = {0, 0, 0, 0, 0};  // per method, one frame iteration
    int max_iterations(int kind) const;
    void rebuild_solids();
    // Boundary-proximity map of a scene from its boundary positions.
    void build_near_map(Scene& sc, float const* solid_xy, uint32_t n_solid);
    // Extent of the arena the per-sub-step launches cover: the highest tile
    // and cell-table slot any resident scene uses, rounded up to 1/32 of the
    // capacity so that graphs are re-captured only when it moves by that much.
    void update_extent();
    Arena extent_arena() const;
    void ensure_sort_scratch(uint32_t n);

    cudaStream_t st_ = nullptr;
    uint32_t fluid_cap_, solid_cap_;
    int max_scenes_;
    Arena a_{};
    std::vector<void*> allocations_;
    size_t device_bytes_ = 0;
    uint32_t ext_tiles_ = 0, ext_stiles_ = 0, ext_ftab_ = 0, ext_stab_ = 0;
    bool compensated_ = false;  // some resident scene is in compensated mode
    SceneParams* d_sp_ = nullptr;
    SceneState* d_ss_ = nullptr;
    int32_t* d_tile_scene_ = nullptr;
    int32_t* d_stile_scene_ = nullptr;
    uint32_t* d_scan_ = nullptr;
    int* d_running_ = nullptr;
    int* h_running_ = nullptr;
    uint32_t* d_flag_ = nullptr;
    uint32_t* h_flag_ = nullptr;
    unsigned int* d_check_counter_ = nullptr;  // finished blocks of a fused exit test
    int loop_kernels_[4] = {3, 3, 3, 4};        // kernels per iteration of each loop kind
    std::vector<Scene> scenes_;
    std::vector<int32_t> tile_scene_, stile_scene_;
    RangeAllocator fluid_tiles_, solid_tiles_, ftab_, stab_, near_words_;
    uint32_t* d_near_ = nullptr;
    bool tiles_dirty_ = true;
    bool unrolled_ = false;
    bool use_graphs_ = true;
    bool capturing_ = false;
    cudaStream_t cur_ = nullptr;  // stream the emitted work goes to
    cudaStream_t cap_st_ = nullptr;
    cudaStream_t body_st_ = nullptr;
    cudaStream_t side_st_ = nullptr;  // parallel branch of a sub-step
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    std::map<int32_t, cudaGraphExec_t> graphs_;        // key: method * 2 + reorder
    std::map<int32_t, int64_t> graph_fixed_kernels_;
#ifndef EMERALD_REORDER_EVERY
#define EMERALD_REORDER_EVERY 16
#endif
    int reorder_every_ = EMERALD_REORDER_EVERY;
#ifndef EMERALD_LOOP_UNROLL
#define EMERALD_LOOP_UNROLL 3
#endif
    int loop_unroll_ = EMERALD_LOOP_UNROLL;  // solver iterations per conditional-loop body
    int64_t substeps_launched_ = 0;
    void* order_buf_ = nullptr;
    SortScratch order_sort_{};
    int64_t host_launches_ = 0;
    int64_t capture_kernels_ = 0;
    bool count_host_ = true;
    unsigned long long* d_loop_iters_ = nullptr;

    void* sort_buf_ = nullptr;
    uint32_t sort_cap_ = 0;
    SortScratch sort_{};

    bool timing_ = false;
    struct Pending {
        std::string name;
        cudaEvent_t start, stop;
    };
    std::vector<Pending> pending_;
    std::vector<cudaEvent_t> event_pool_;
    KernelTimes times_;
};

int64_t kernel_launch_count();

}  // namespace emerald
