// Device-side data layout of the SPH engine.
//
// Every simulation is a batch of scenes. A scene's fluid particles occupy a
// contiguous range of the fluid arena that starts on a tile boundary (tiles
// of kTile particles, one thread block per tile), so each block belongs to
// exactly one scene and reads that scene's constants once. Boundary
// (solid) particles live in a second arena laid out the same way.
// Particles keep their original order inside a scene, as the reference's
// State vectors do (emerald/sph2d_box/state.h:13-17).
//
// Neighbour lists are fixed-capacity (64, NEIGHBORHOOD_MAX_COUNT in
// emerald/sph_common/neighborhood.h:38) and stored slot-major over the whole
// arena: entry k of particle i lives at [k * stride + i], so the threads of a
// warp (consecutive particles) read entry k of their lists in one coalesced
// transaction. Indices are arena-global.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace emerald {

constexpr int kTile = 128;
constexpr int kMaxNeighbors = 64;
constexpr uint64_t kEmptyKey = ~0ull;
constexpr int kLoopSlots = 9;  // Arena::loop_iterations entries

enum Method : int { kPcisph = 0, kIisph = 1, kIisphAp = 2, kIisphPseudoAp = 3, kDfsph = 4 };

enum StepMode : int { kFixedDt = 0, kFrame = 1 };

// Error bits reported through SceneState::error.
enum ErrorBits : int { kErrTableFull = 1, kErrNonFinite = 2 };

// External force terms, the reference's force functions
// (emerald/sph2d_box/forces.cpp): gravity (accumulate_gravity_forces,
// :63-71, a = g), pole attraction with swirl
// (accumulate_constant_pole_attraction_forces, :85-101, a = magnitude,
// (b, c) = pole) and drag (accumulate_simple_drag_forces, :104-111,
// a = magnitude, b = particle diameter). Numbered as EMERALD_FORCE_*.
enum ForceKind : int32_t { kForceGravity = 1, kForcePole = 2, kForceDrag = 3 };
constexpr int kMaxForceTerms = 4;
struct ForceTerm {
    int32_t kind;
    float a, b, c;
};

// Constants of one scene (mirrors Parameters + Simulation_config,
// emerald/sph2d_box/parameters.h:12-41, config.h:7-18).
struct SceneParams {
    uint32_t fluid_begin, fluid_count;
    uint32_t solid_begin, solid_count;
    uint32_t ftab_begin, ftab_log2;  // fluid cell table region (size 2^log2 + 1)
    uint32_t stab_begin, stab_log2;  // solid cell table region
    float support, cell_size, rho0, mass, fluid_volume, gravity, viscosity, w0;
    float iisph_omega, iisph_err_avg, iisph_err_max;
    int32_t iisph_max_iter;
    int32_t dfsph_max_iter;
    float dfsph_dens_avg, dfsph_dens_max, dfsph_div_avg, dfsph_div_max;
    float pcisph_denom;
    int32_t method;
    int32_t mode;
    int64_t time_per_step;  // flicks
    int32_t sub_steps;      // PCISPH sub-steps per frame
    int32_t min_denom, max_denom;
    float cfl_factor;
    float seconds_per_sub_step;
    float fixed_dt;
    uint32_t sort_base;  // real particles of scenes stored before this one
    float reject_l2;     // smallest float whose sqrtf is >= cell_size
    int32_t precision;   // 0: the reference's FP32 arithmetic; 1: FP64 positions (+ Kahan sums under DFSPH_P)
    // Cells within one cell of a boundary particle's cell: bit
    // (y - near_y0) * near_w + (x - near_x0) of the words from near_begin.
    // A fluid particle whose cell is clear has no boundary neighbours.
    // near_w == 0: no map (every particle searches).
    uint32_t near_begin, near_w, near_h;
    int32_t near_x0, near_y0;
    // External forces where the solver computes them
    // (compute_all_external_forces, emerald/sph2d_box/forces.cpp:11-33):
    // zero, then each of the force_count terms in order; with force_array
    // the host callback's forces in Arena::ext_f instead.
    int32_t force_count;
    int32_t force_array;
    ForceTerm force_terms[kMaxForceTerms];
    float fixed_t;  // the caller's sub-step time (fixed-dt mode)
};

// Mutable per-scene state, device resident.
struct SceneState {
    int64_t frame_time;  // flicks at the start of the current frame
    int64_t elapsed;     // flicks into the current frame
    int32_t remaining;   // frame sub-step units left; 0: a new frame starts next
    int32_t frame_substeps;
    float dt, t;
    int32_t active;
    int32_t new_frame;
    int32_t iter, done;
    unsigned long long err_sum;
    uint32_t err_max;  // bits of a non-negative float
    uint32_t max_v2;   // bits of a non-negative float
    float stat_avg, stat_max;
    int32_t stat_iters;
    float stat_div_avg, stat_div_max;
    int32_t stat_div_iters;
    int32_t error;
    int32_t substeps_total;
    int32_t call_substeps;  // sub-steps run by the current frame-graph launch
    double err_sum_d;  // exact sum of the errors (DFSPH loops)
    double stat_avg_exact, stat_div_avg_exact;
};

// Raw device pointers of an arena, passed by value to every kernel.
struct Arena {
    SceneParams const* sp;
    SceneState* ss;
    // executed solver iterations per loop kind (0-3), then sub-steps run by
    // frame graphs per method (4 + method)
    unsigned long long* loop_iterations;
    // Solver-loop work list of the persistent-warp loop kernels: the scenes
    // whose loop still runs (loop_scene[0, *loop_n)) and the exclusive prefix
    // of their warp tiles (loop_wt0, *loop_n + 1 entries), rebuilt by every
    // loop reset and exit test.
    int32_t* loop_scene;
    uint32_t* loop_wt0;
    uint32_t* loop_n;
    int32_t batch;  // the arena holds more than one scene slot (loop kernels walk the work list)
    int32_t const* tile_scene;   // fluid tile -> scene (-1: free)
    int32_t const* stile_scene;  // solid tile -> scene
    uint32_t stride;             // fluid arena capacity (multiple of kTile)
    uint32_t sstride;            // solid arena capacity

    // fluid state and solver temporaries (emerald/sph2d_box/state.h:34-69)
    float2* x;
    float2* v;
    float* rho;
    float* rho_star;
    float* pbuf0;   // pressures / pseudo pressures (ping)
    float* pbuf1;   // (pong)
    float* alpha;
    float* kdiv;
    float* kdens;
    float* qdiv;    // cached kdiv / rho^2
    float* qdens;   // cached kdens / rho^2, also p / rho^2 for the AP solvers
    float* aii;
    float2* dii;
    float2* sdp;    // sum_j d_ij p_j
    float2* acc;    // pressure accelerations / displacements
    float2* vext;
    float2* xstar;
    float2* vstar;
    float2* fp;     // PCISPH pressure forces
    float2* ext_f;  // external forces from a host callback (storage order)

    // storage order: oid[slot] = original (scene-local) index of the particle
    // stored at `slot`; slot_of[fluid_begin + oid] = its slot. nullptr means
    // storage order is the original order.
    uint32_t* oid;
    uint32_t* slot_of;
    float2* tx;  // reorder staging
    float2* tv;
    float* tkdiv;
    float* tkdens;
    uint32_t* toid;
    uint32_t const* near_bits;  // boundary-proximity maps of the scenes
    double2* x64;   // positions accumulated in double (compensated mode)
    double2* tx64;

    // neighbour lists, slot-major
    uint8_t* nf_cnt;
    uint32_t* nf_idx;
    float* nf_w;
    float2* nf_gw;
    uint8_t* ns_cnt;
    uint32_t* ns_idx;
    float* ns_w;
    float2* ns_gw;

    // neighbour build scratch
    uint32_t* slot;
    uint32_t* rank;
    uint64_t* zkey;   // z key of each particle at the last build
    uint32_t* members;
    uint64_t* fkeys;
    uint32_t* fcount;
    uint32_t* fstart;
    uint32_t ftab_total;

    // boundary particles (static)
    float2* xs;
    float2* vs;
    float* vols;
    uint32_t* sslot;
    uint32_t* srank;
    uint64_t* szkey;
    uint32_t* smembers;
    uint64_t* skeys;
    uint32_t* scount;
    uint32_t* sstart;
    uint32_t stab_total;
};

}  // namespace emerald
