/*
 * emerald-b200: C ABI of the B200 implementation of the emerald 2D SPH step
 * (emerald/sph2d_box + emerald/sph_common + emerald/z_index).
 *
 * The reference exposes C++ free functions and the EZ_EXAMPLE_SIM driver
 * (emerald/sph2d_box/simulation.h:24-44); it has no C ABI. These entry points
 * are the flat equivalents a foreign-function caller binds. Every function
 * returns an emerald status code; buffers are caller-owned host arrays of
 * interleaved (x, y) floats unless stated otherwise; particle indices are
 * the caller's original order, as in the reference's State vectors.
 */
#ifndef EMERALD_SPH_H
#define EMERALD_SPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference aborts through EMLD_ASSERT/EMLD_FAIL
 * (emerald/util/assert.h:14-26); here each failure is a return value and a
 * message retrievable with emerald_last_error(). */
#define EMERALD_OK 0
#define EMERALD_EINVAL 22
#define EMERALD_ENOMEM 12
#define EMERALD_ENOSPC 28
#define EMERALD_ENOTFOUND 2
#define EMERALD_ETIMEOUT 110
#define EMERALD_ECUDA 1000
#define EMERALD_ESOLVER 1001
#define EMERALD_ECANCELED 125

/* Neighbour slots per particle, NEIGHBORHOOD_MAX_COUNT
 * (emerald/sph_common/neighborhood.h:38). Every list buffer of this API has
 * this many slots per particle. */
#define EMERALD_MAX_NEIGHBORS 64

/* Solver methods, numbered as EZ_EXAMPLE_SIM::Method
 * (emerald/sph2d_box/simulation.h:25). */
#define EMERALD_PCISPH 0
#define EMERALD_IISPH 1
#define EMERALD_IISPH_AP 2
#define EMERALD_IISPH_PSEUDO_AP 3
#define EMERALD_DFSPH_P 4

/* Parameters (emerald/sph2d_box/parameters.h:12-41) plus the two derived
 * Simulation_config values (emerald/sph2d_box/config.h:7-18). A zero
 * mass_per_particle or pressure_correction_denom is derived from the
 * reference's hex template (config.cpp:16-132). */
typedef struct emerald_params {
    uint64_t seed;
    int64_t time_per_step_flicks;
    int32_t sub_steps;
    float length;
    float support;
    float gravity;
    float viscosity;
    float target_density;
    int32_t iisph_max_pressure_iterations;
    float iisph_error_average_threshold;
    float iisph_error_max_threshold;
    float iisph_omega;
    int32_t dfsph_max_correction_iterations;
    float dfsph_density_error_average_threshold;
    float dfsph_density_error_max_threshold;
    float dfsph_divergence_error_average_threshold;
    float dfsph_divergence_error_max_threshold;
    float mass_per_particle;
    float pressure_correction_denom;
    int32_t precision; /* EMERALD_PRECISION_*; not in the reference */
} emerald_params;

/* Arithmetic of a scene. REFERENCE (default): the reference's FP32
 * operations in its order, bit-identical results. COMPENSATED: positions
 * accumulated in FP64 and the neighbour vectors x_i - x_j taken from them
 * (every method); under DFSPH_P also the neighbour sums in FP32 with Kahan
 * compensation (the other methods keep the reference's sums). The solver's
 * exit test is the reference's in both modes (an exact int64 sum and an
 * FP64 division); the exact FP64 mean of the errors is reported in
 * emerald_step_stats. */
#define EMERALD_PRECISION_REFERENCE 0
#define EMERALD_PRECISION_COMPENSATED 1

/* Statistics of the last sub-step (or of the last sub-step of a frame). The
 * reference keeps these in local variables; they are returned here. */
typedef struct emerald_step_stats {
    int32_t sub_steps;
    int32_t pressure_iterations;
    float error_average;
    float error_max;
    int32_t divergence_iterations;
    float divergence_error_average;
    float divergence_error_max;
    float dt;
    double time_seconds;
    int32_t error_flags;
    /* DFSPH_P: the exact mean of the per-particle errors (FP64 sum), beside
     * the reference's metric above, sum(int64(err * 1000)) / (1000 n), which
     * drops every particle's error below 0.1%. */
    double error_average_exact;
    double divergence_error_average_exact;
} emerald_step_stats;

/* ---------------------------------------------------------------- setup */

/* Parameters() defaults (emerald/sph2d_box/parameters.h:12-41). */
int emerald_default_params(emerald_params* out);

/* Simulation_config (emerald/sph2d_box/config.cpp:16-132): out[0]
 * seconds_per_sub_step, out[1] mass_per_particle, out[2] draw_radius,
 * out[3] pressure_correction_denom. Overrides in *params are honoured. */
int emerald_config(emerald_params const* params, float* out);

/* The same template sums over an unjittered square lattice of spacing dx
 * (used by the block scenes): out[0] mass_per_particle, out[1] the PCISPH
 * pressure-correction denominator for sub-step dt. */
int emerald_lattice_config(emerald_params const* params, float dx, float dt, float* out);

/* z_index(x, y) (emerald/z_index/z_index.cpp:8-10). */
uint64_t emerald_z_index(uint32_t x, uint32_t y);

/* Seeded block scene: nx*ny fluid particles at (i+0.5)dx, (j+0.5)dx offset
 * by (x0, y0), each coordinate jittered by U(-jitter*dx, jitter*dx) from
 * std::mt19937_64{seed}. Writes nx*ny points; returns the count. */
size_t emerald_block_scene(uint32_t nx, uint32_t ny, float dx, float x0, float y0, float jitter,
                           uint64_t seed, float* xy);

/* Tank boundary: `layers` rows of particles at spacing dx below the floor
 * and outside both side walls of [0, length]^2. xy may be NULL to count. */
size_t emerald_wall_scene(float dx, float length, int32_t layers, float* xy);

/* The reference's default scene generators: world_walls_initial_solid_state
 * (emerald/sph2d_box/solids.cpp:139-213) and dam_break_initial_state
 * (emerald/sph2d_box/initial_state.cpp:14-97). Pass NULL to count. */
size_t emerald_world_walls(emerald_params const* params, float* xy);
size_t emerald_dam_break(emerald_params const* params, float const* solid_xy, size_t n_solid,
                         float* xy);

/* ------------------------------------------------------------ simulation */

typedef struct emerald_sim emerald_sim;

/* Creates a single-scene simulation on the current CUDA device: the
 * EZ_EXAMPLE_SIM state (emerald/sph2d_box/simulation.cpp:14-39) with the
 * given boundary and fluid particles. solid_volumes may be NULL, in which
 * case boundary volumes follow compute_volumes
 * (emerald/sph2d_box/solids.cpp:52-74). fluid_v may be NULL (zero). */
int emerald_sim_create(emerald_params const* params,
                       float const* solid_xy,
                       float const* solid_volumes,
                       size_t n_solid,
                       float const* fluid_xy,
                       float const* fluid_v,
                       size_t n_fluid,
                       emerald_sim** out);
int emerald_sim_destroy(emerald_sim* sim);

/* Per-frame temporaries of a fixed-dt run: the resize/reset of the method's
 * temporaries (e.g. emerald/sph2d_box/dfsph_p.cpp:214-229) and
 * compute_constant_volumes (emerald/sph_common/volume.cpp:7-14). */
int emerald_sim_begin_frame(emerald_sim* sim, int32_t method);

/* One solver sub-step with a caller-chosen dt: iisph_sub_step
 * (emerald/sph2d_box/iisph.cpp:23-151), iisph_ap_sub_step, iisph_pseudo_ap_sub_step,
 * dfsph_p_sub_step (dfsph_p.cpp:265-374) or pcisph_sub_step (pcisph.cpp:36-164). */
int emerald_sim_sub_step(emerald_sim* sim, int32_t method, float t, float dt,
                         emerald_step_stats* stats);

/* One frame, as X_simulation_step through EZ_EXAMPLE_SIM::step
 * (emerald/sph2d_box/simulation.cpp:41-93): CFL-adaptive sub-steps
 * (adaptive_time_step.h:35-122) or PCISPH's fixed sub-steps. With graphs on
 * (the default) the whole frame is one CUDA graph launch, its sub-step loop
 * a conditional while node on the device, and the call waits for the
 * device once; a frame that started earlier (after emerald_sim_advance) is
 * finished. stats->sub_steps counts the sub-steps this call ran. */
int emerald_sim_frame(emerald_sim* sim, int32_t method, emerald_step_stats* stats);

/* Advances n adaptive sub-steps, continuing and starting frames exactly as
 * successive emerald_sim_frame calls would. */
int emerald_sim_advance(emerald_sim* sim, int32_t method, int32_t n_substeps,
                        emerald_step_stats* stats);
/* emerald_sim_set_state(x_in, v_in), emerald_sim_advance and
 * emerald_sim_get_state(x_out, v_out) in one call, with one wait for the
 * device at the end: the copies and the sub-steps are queued back to back
 * on the simulation's stream. Any of the four buffers may be NULL; x_in may
 * be x_out (and v_in v_out). Pinned host memory copies at DMA speed. */
int emerald_sim_advance_host(emerald_sim* sim, int32_t method, int32_t n_substeps,
                             float const* x_in, float const* v_in, float* x_out, float* v_out,
                             emerald_step_stats* stats);

int emerald_sim_counts(emerald_sim const* sim, size_t* n_fluid, size_t* n_solid);
int emerald_sim_time(emerald_sim const* sim, int64_t* flicks);
int emerald_sim_get_state(emerald_sim* sim, float* x, float* v);
int emerald_sim_set_state(emerald_sim* sim, float const* x, float const* v);
int emerald_sim_get_solid(emerald_sim* sim, float* xy, float* volumes);
/* Replaces the boundary between sub-steps, for moving (kinematic) walls and
 * prescribed rigid motion. The reference's step functions take the
 * Solid_state by const reference on every call (e.g.
 * emerald/sph2d_box/dfsph_p.cpp:376-396), and its velocities enter the
 * divergence and density-star sums (emerald/sph_common/divergence.cpp:47-74,
 * emerald/sph2d_box/iisph_ops.cpp:87-221). solid_xy: the n_solid positions,
 * original order (NULL keeps them; new ones rebuild the boundary cell tables
 * as compute_neighbor_data_and_volumes does, emerald/sph2d_box/solids.cpp:76-137);
 * solid_v: velocities (NULL keeps them; they start at zero); solid_volumes:
 * NULL recomputes the volumes from new positions with compute_volumes
 * (solids.cpp:52-74) and keeps them otherwise. The count is fixed at
 * creation. */
int emerald_sim_set_solid(emerald_sim* sim, float const* solid_xy, float const* solid_v,
                          float const* solid_volumes);

/* External forces. The reference computes them once per sub-step through
 * compute_all_external_forces (emerald/sph2d_box/forces.cpp:11-33): the
 * forces start at zero and the user's User_forces_function
 * (emerald/sph2d_box/forces.h:13-21) adds to them, at the start of the
 * sub-step under IISPH, IISPH_AP, IISPH_PSEUDO_AP and PCISPH and after the
 * divergence solve under DFSPH_P. Two ways stand for that function here:
 *
 * force terms, evaluated on the device in the sub-step itself, in order,
 * each with the arithmetic of the reference function it names:
 *   EMERALD_FORCE_GRAVITY: accumulate_gravity_forces (forces.cpp:63-71),
 *     F.y -= mass * a;
 *   EMERALD_FORCE_POLE: accumulate_constant_pole_attraction_forces
 *     (forces.cpp:85-101), magnitude a, pole (b, c);
 *   EMERALD_FORCE_DRAG: accumulate_simple_drag_forces (forces.cpp:104-111),
 *     magnitude a, particle diameter b.
 * A new simulation has one gravity term with params->gravity, what
 * default_gravity_forces(gravity) (forces.cpp:73-83) computes. count 0
 * applies no external force; more than EMERALD_MAX_FORCE_TERMS terms, an
 * unknown kind or a non-finite argument is EMERALD_EINVAL. */
#define EMERALD_FORCE_GRAVITY 1
#define EMERALD_FORCE_POLE 2
#define EMERALD_FORCE_DRAG 3
#define EMERALD_MAX_FORCE_TERMS 4
typedef struct emerald_force_term {
    int32_t kind;
    float a, b, c;
} emerald_force_term;
int emerald_sim_set_forces(emerald_sim* sim, emerald_force_term const* terms, int32_t count);

/* or a host function with the User_forces_function argument list plus a
 * user pointer: once per sub-step, at the reference's force point, it gets
 * the particle count, the time in seconds (the sub-step's start; plus dt
 * under DFSPH_P, as dfsph_p.cpp:350 passes), dt, mass_per_particle,
 * draw_radius, the forces to add to (count x 2 floats, zeroed first) and
 * the positions and velocities at that point (original particle order).
 * While a callback is set the sub-steps run without CUDA graphs, with one
 * device-to-host and one host-to-device copy of the state per sub-step.
 * NULL removes the callback and the force terms apply again. */
typedef void (*emerald_forces_fn)(void* user, size_t count, float time, float dt, float mass,
                                  float radius, float* forces, float const* positions,
                                  float const* velocities);
int emerald_sim_set_force_callback(emerald_sim* sim, emerald_forces_fn fn, void* user);

/* Checkpoint and resume. The reference keeps a run's state in State and
 * Temp_data (emerald/sph2d_box/state.h:13-69) and has no checkpoint; the
 * DFSPH kappas there carry over between the sub-steps of a frame and are
 * zeroed per frame (dfsph_p.cpp:214-229), so a resumable state holds them.
 * emerald_sim_snapshot writes, between sub-steps, the frame clock in flicks
 * with the position inside the frame, the sub-step counters and the last
 * statistics, the positions, velocities and DFSPH kappas (original order),
 * the FP64 positions of a compensated scene and the boundary (positions,
 * velocities, volumes) into `buffer`; *size receives the bytes it needs
 * (buffer NULL: only the size; capacity too small: EMERALD_ENOSPC).
 * emerald_sim_restore loads one into a simulation of the same particle
 * counts and precision mode (EMERALD_EINVAL otherwise, or for a damaged
 * buffer); the sub-steps after it are bit-identical to those that followed
 * the snapshot. Parameters and force settings are not part of it. */
int emerald_sim_snapshot(emerald_sim* sim, void* buffer, size_t capacity, size_t* size);
int emerald_sim_restore(emerald_sim* sim, void const* buffer, size_t size);

/* Per-particle solver temporaries by their Temp_data name
 * (emerald/sph2d_box/state.h:34-69): "densities", "pressures",
 * "density_stars", "aiis", "alphas", "divergence_kappas", "density_kappas",
 * "diis", "sum_dij_pjs", "pressure_forces", "pressure_accelerations",
 * "velocity_external_forces", "position_stars", "velocity_stars".
 * *width receives 1 or 2 floats per particle; out may be NULL to query. */
int emerald_sim_get_array(emerald_sim* sim, char const* name, float* out, int32_t* width);

/* Neighbour lists of the last sub-step in the reference layout
 * (emerald/sph_common/neighborhood.h:126-160): counts[n], and n x 64 arrays
 * of indices, kernel values and kernel gradients (x, y). Any may be NULL. */
int emerald_sim_get_neighbors(emerald_sim* sim, int32_t solid, uint8_t* counts, uint32_t* idx,
                              float* w, float* gw);

/* Sort products of the last neighbour build (emerald/sph2d_box/state.h:34-40):
 * grid coords (n x 2), z keys, the sorted (z, index) pairs, block indices
 * and the [begin, end) blocks (nblocks x 2). Any output may be NULL. */
int emerald_sim_get_sort(emerald_sim* sim, int32_t solid, int32_t* grid_coords, uint64_t* z,
                         uint64_t* pair_z, uint64_t* pair_index, uint32_t* block_indices,
                         uint64_t* blocks, size_t* nblocks);

/* Device residency: the CUDA stream the simulation runs on (NULL keeps the
 * legacy default stream) and device pointers to its float2 positions and
 * velocities (original particle order). */
int emerald_sim_set_stream(emerald_sim* sim, void* cuda_stream);
int emerald_sim_device_state(emerald_sim* sim, void** x, void** v);

/* Accumulated device time per kernel name since the last reset, measured
 * with CUDA events around each launch when timing is enabled. */
int emerald_sim_enable_timing(emerald_sim* sim, int32_t enable);
int emerald_sim_kernel_times(emerald_sim* sim, char* names, size_t names_len, double* ms,
                             int32_t* launches, int32_t* count);

/* Execution mode: graphs != 0 (default) runs each sub-step as one CUDA graph
 * launch with the solver loops as conditional nodes; graphs == 0 launches
 * kernels one by one and tests the loop exit on the host after every
 * iteration, as the reference does. */
int emerald_sim_set_graphs(emerald_sim* sim, int32_t graphs);

/* Kernels this simulation has launched (graph nodes included, loop bodies
 * counted once per executed iteration). */
/* Times the simulation waited on the host for the device (stream or event
 * synchronisations). No counterpart in the reference; with graphs on, a
 * frame costs one. */
int emerald_sim_host_waits(emerald_sim* sim, int64_t* count);
int emerald_sim_kernel_launches(emerald_sim* sim, int64_t* count);

/* Number of kernel launches this library issued from the host since the
 * process started (a graph launch counts its kernels outside solver loops). */
int64_t emerald_kernel_launches(void);

/* ----------------------------------------------------------------- batches */

/* Many independent scenes advanced together: every kernel of a sub-step runs
 * once over all active scenes' particles (one CUDA graph launch per
 * sub-step), each scene with its own parameters, time step and convergence
 * state. The reference runs one scene per EZ_EXAMPLE_SIM; a scene here gives
 * the same bits as that scene run alone. */
typedef struct emerald_batch emerald_batch;

int emerald_batch_create(size_t fluid_capacity, size_t solid_capacity, int32_t max_scenes,
                         emerald_batch** out);
int emerald_batch_destroy(emerald_batch* batch);
/* Adds a scene (inactive until emerald_batch_set_active); *scene receives its
 * id. EMERALD_ENOSPC when the batch has no room for it. */
int emerald_batch_add_scene(emerald_batch* batch, emerald_params const* params,
                            float const* solid_xy, float const* solid_volumes, size_t n_solid,
                            float const* fluid_xy, float const* fluid_v, size_t n_fluid,
                            int32_t* scene);
int emerald_batch_remove_scene(emerald_batch* batch, int32_t scene);
int emerald_batch_set_active(emerald_batch* batch, int32_t scene, int32_t active);
/* n adaptive sub-steps (frames continue across calls) of `method` for every
 * active scene. Asynchronous on the batch's stream. */
int emerald_batch_step(emerald_batch* batch, int32_t method, int32_t n_substeps);
int emerald_batch_scene_stats(emerald_batch* batch, int32_t scene, emerald_step_stats* stats);
int emerald_batch_get_state(emerald_batch* batch, int32_t scene, float* x, float* v);
int emerald_batch_set_state(emerald_batch* batch, int32_t scene, float const* x, float const* v);
/* emerald_sim_set_solid for one scene of a batch. */
int emerald_batch_set_solid(emerald_batch* batch, int32_t scene, float const* solid_xy,
                            float const* solid_v, float const* solid_volumes);
/* emerald_sim_set_forces for one scene of a batch. */
int emerald_batch_set_forces(emerald_batch* batch, int32_t scene, emerald_force_term const* terms,
                             int32_t count);
/* Largest fluid range and scene slots still free. */
int emerald_batch_free(emerald_batch* batch, size_t* fluid, int32_t* scenes);
int emerald_batch_set_stream(emerald_batch* batch, void* cuda_stream);
int emerald_batch_synchronize(emerald_batch* batch);
int emerald_batch_kernel_launches(emerald_batch* batch, int64_t* count);

/* -------------------------------------------------------------- autotuning */

/* Neighbour entries each gather-sum kernel loads together (1, 4 or 8), and
 * how it brings its lists in (prefetch): 0 loads them as the sums need
 * them; 1 has each warp first ask L2 for its list rows;
 * EMERALD_TUNE_PERSISTENT (2) launches one grid of resident blocks of 128
 * threads whose warps walk their 32-particle tiles and request the next
 * tile's lists and inputs into L2 while they fold the current one;
 * EMERALD_TUNE_PERSISTENT_256 (3) the same in blocks of 256 threads;
 * EMERALD_TUNE_PERSISTENT_FUSED (4) and EMERALD_TUNE_PERSISTENT_256_FUSED (5)
 * the same, and on a solver loop's final kernel (apply for DFSPH_P, beta for
 * IISPH) the iteration's exit test runs in that kernel's last block instead
 * of a launch of its own.
 * Every choice gives the same bits. Autotuning (DFSPH_P and IISPH) times a
 * few whole sub-steps of `method` with each candidate setting, every
 * candidate from the same state (restored afterwards, so the simulation is
 * left as it was), after at least one sub-step of that method, and keeps
 * the fastest, also for later simulations (or, found on a batch, later
 * batches) of the same method and size class (log2 of the active particle
 * count). A batch times the persistent-warp candidates only (modes 2 to 5):
 * its solver loops run as long as its slowest scene's, and those kernels
 * walk just the scenes still iterating. candidate_ms[k]: mean
 * sub-step time of candidate k, whose chunks and prefetch modes are
 * candidate_chunks[k] and candidate_prefetch[k] (apply, divergence,
 * iisph_sum, iisph_beta; prefetch[] in the same order; the divergence
 * family's mode also applies to the DFSPH density and alpha pass). No
 * counterpart in the reference. */
#define EMERALD_TUNE_PERSISTENT 2
#define EMERALD_TUNE_PERSISTENT_256 3
#define EMERALD_TUNE_PERSISTENT_FUSED 4
#define EMERALD_TUNE_PERSISTENT_256_FUSED 5
#define EMERALD_TUNE_CANDIDATES 16
typedef struct emerald_tuning {
    int32_t apply_chunk, divergence_chunk, iisph_sum_chunk, iisph_beta_chunk;
    int32_t candidates;
    int32_t candidate_chunks[EMERALD_TUNE_CANDIDATES][4];
    float candidate_ms[EMERALD_TUNE_CANDIDATES];
    int32_t prefetch[4];
    int32_t candidate_prefetch[EMERALD_TUNE_CANDIDATES][4];
} emerald_tuning;

int emerald_sim_autotune(emerald_sim* sim, int32_t method, emerald_tuning* out);
int emerald_batch_autotune(emerald_batch* batch, int32_t method, emerald_tuning* out);
/* Pins the settings of *tuning (its chunks and prefetch modes; the candidate
 * fields are ignored) until the next call; NULL returns to the tuned or
 * default settings. */
int emerald_sim_set_tuning(emerald_sim* sim, emerald_tuning const* tuning);
int emerald_batch_set_tuning(emerald_batch* batch, emerald_tuning const* tuning);

/* ----------------------------------------------------------------- serving */

/* A request loop over batches: requests (a scene and a sub-step count) are
 * queued by any host thread, admitted as soon as an arena has room for them
 * (first fit: a large request waiting for room does not hold back smaller
 * ones behind it; each goes to the lane with the least resident work,
 * fluid particles times sub-steps left, among those with room), stepped
 * together with every other scene of its arena, and retired as soon as
 * their sub-steps are done, which frees their room for the queue. The queue
 * is in arrival order, or (order = 1) largest work first, which shortens
 * the tail of a burst. The device memory budget is split evenly over
 * `lanes` arenas, each with its own stream and host thread, sized once at
 * creation. No counterpart in the reference (one scene per process). */
typedef struct emerald_server emerald_server;

typedef struct emerald_server_config {
    size_t hbm_budget_bytes;         /* device bytes the arena may take */
    int32_t method;                  /* EMERALD_METHOD_* every request runs */
    int32_t max_scenes;              /* scenes resident at once */
    int32_t max_substeps_per_launch; /* sub-steps between admission points (0: 8) */
    int32_t lanes;                   /* arenas stepped concurrently (0: 4) */
    int32_t order;                   /* queue: 0 arrival order, 1 largest work first */
} emerald_server_config;

typedef struct emerald_server_stats {
    int64_t submitted, completed, rejected, queued, resident;
    int64_t batch_substeps;    /* batched sub-step launches */
    int64_t scene_substeps;    /* sum over scenes of their sub-steps */
    double particle_substeps;  /* sum over scenes of fluid count x sub-steps */
    double busy_seconds;       /* wall time with at least one scene resident */
    float step_ms_p50, step_ms_p99;       /* device time of one batched sub-step */
    float request_ms_p50, request_ms_p99; /* submit to result ready */
    float queue_ms_p50, queue_ms_p99;     /* submit to admission */
    size_t fluid_capacity, solid_capacity; /* of one lane */
    size_t device_bytes;                   /* all lanes */
    int32_t resident_peak;
    int32_t status; /* first error of the loop, EMERALD_OK while healthy */
    int64_t cancelled; /* requests retired by emerald_server_cancel */
} emerald_server_stats;

typedef struct emerald_request_timing {
    double queue_ms, run_ms, total_ms;
} emerald_request_timing;

int emerald_server_create(emerald_server_config const* config, emerald_server** out);
/* Stops the loop; requests not yet waited for are dropped. */
int emerald_server_destroy(emerald_server* server);
/* Copies the inputs and queues the request; *request receives its id.
 * EMERALD_ENOSPC when the scene is larger than the whole arena. */
int emerald_server_submit(emerald_server* server, emerald_params const* params,
                          float const* solid_xy, float const* solid_volumes, size_t n_solid,
                          float const* fluid_xy, float const* fluid_v, size_t n_fluid,
                          int32_t n_substeps, int64_t* request);
/* Waits for a request (timeout_ms < 0: without limit), copies out its final
 * positions and velocities (original order; NULL skips) and statistics, and
 * forgets it. EMERALD_ETIMEOUT when it is not done within the limit,
 * EMERALD_ENOTFOUND for an unknown or already collected id. */
int emerald_server_wait(emerald_server* server, int64_t request, int32_t timeout_ms, float* x,
                        float* v, emerald_step_stats* stats, emerald_request_timing* timing);
int emerald_server_get_stats(emerald_server* server, emerald_server_stats* out);
/* No counterpart in the reference (one scene per process, stopped by
 * killing it). Cancels a request: a queued one leaves the queue at once; a
 * resident one leaves its batch at the lane's next admission point, between
 * sub-steps, and its room is freed (the other scenes of the batch go on
 * unchanged, bit for bit); a finished one drops its result. emerald_server_wait
 * then returns EMERALD_ECANCELED for it. EMERALD_ENOTFOUND for an unknown or
 * already collected id. */
int emerald_server_cancel(emerald_server* server, int64_t request);

/* ------------------------------------------- sph_common functions on device */

/* The emerald/sph_common free functions on device memory, one call each, in
 * the reference's argument order (count first, outputs before inputs) and
 * arithmetic order: for the same inputs the outputs are bit-identical to the
 * reference's. Every pointer is device memory; V2f arrays are interleaved
 * (x, y) floats. Calls are asynchronous on `stream` (NULL: the legacy
 * default stream) and allocate nothing. Reductions write their result to
 * device memory. */

/* Neighborhood_pointers (emerald/sph_common/neighborhood.h:126-133): counts
 * per particle and, per particle, EMERALD_MAX_NEIGHBORS = 64 entries of
 * each array, row-major (particle i's entry k at i * 64 + k). Members a call
 * does not read may be NULL; a NULL `counts` in a solid neighbourhood skips
 * the boundary pass. */
typedef struct emerald_neighborhood {
    uint8_t const* counts;
    uint64_t const* indices;
    float const* distances;
    float const* vectors_to;       /* 2 floats per entry */
    float const* kernels;
    float const* kernel_gradients; /* 2 floats per entry */
} emerald_neighborhood;

/* compute_grid_coords (emerald/sph_common/common.cpp:57-67): int32 pairs. */
int emerald_compute_grid_coords(size_t n, float cell_size, float bounds_min_x, float bounds_min_y,
                                int32_t* grid_coords, float const* positions, void* stream);
/* compute_z_indices (emerald/sph_common/common.cpp:69-76). */
int emerald_compute_z_indices(size_t n, uint64_t* z_indices, int32_t const* grid_coords,
                              void* stream);

/* The z-order sort and the neighbour search (emerald/sph_common/neighborhood.h:41-97,
 * neighborhood.cpp:10-152). The reference's std::pair<uint64_t, size_t>
 * arrays (index pairs (z, index), blocks [begin, end)) are interleaved
 * uint64 pairs, their own memory layout on LP64. n is below 2^32 - 1. */
/* compute_index_pairs (neighborhood.cpp:10-16): index_pairs[i] = (z_indices[i], i). */
int emerald_compute_index_pairs(size_t n, uint64_t* index_pairs, uint64_t const* z_indices,
                                void* stream);
/* Bytes of device workspace emerald_sort_index_pairs and
 * emerald_compute_block_indices need for n pairs (256-byte aligned). */
int emerald_index_pairs_workspace(size_t n, size_t* bytes);
/* sort_index_pairs (neighborhood.cpp:18-26): ascending (z, index) order,
 * the order std::sort gives the pairs, in place. */
int emerald_sort_index_pairs(size_t n, uint64_t* index_pairs, void* workspace,
                             size_t workspace_bytes, void* stream);
/* compute_block_indices (neighborhood.cpp:28-64): per sorted pair, the
 * number of z changes before it (0 0 0 1 1 2 ...). The block count is
 * block_indices[n - 1] + 1, read by the caller as the reference's driver
 * does (emerald/sph2d_box/neighborhoods_from_state.cpp:32). */
int emerald_compute_block_indices(size_t n, uint32_t* block_indices,
                                  uint64_t const* sorted_index_pairs, void* workspace,
                                  size_t workspace_bytes, void* stream);
/* fill_blocks (neighborhood.cpp:66-93): blocks[b] = [first, last + 1) of
 * the pairs whose block index is b (non-decreasing block indices, as
 * emerald_compute_block_indices makes them). */
int emerald_fill_blocks(size_t n, uint64_t* blocks, uint32_t const* block_indices, void* stream);
/* Block_map (neighborhood.h:21-35): z key -> block, as a device hash table.
 * emerald_create_block_map (create_block_map, neighborhood.cpp:95-110)
 * clears the map and inserts every block under the z key of its first pair;
 * the table holds at least twice block_count slots and grows on demand, as
 * the reference's rehash does (growing waits for `stream`). A map is used
 * on the device that filled it. */
typedef struct emerald_block_map emerald_block_map;
int emerald_block_map_create(emerald_block_map** map);
int emerald_block_map_destroy(emerald_block_map* map);
int emerald_create_block_map(size_t block_count, emerald_block_map* into, uint64_t const* blocks,
                             uint64_t const* sorted_index_pairs, void* stream);
/* create_regular_neighborhoods (neighborhood.cpp:112-136, the search of
 * neighborhood.h:199-282): for each particle the other set's particles in
 * the 3x3 cells around its grid coordinate, closer than max_distance (the
 * particle itself excluded when other_positions == self_positions), at most
 * 64 taken in the reference's visiting order, sorted by (distance, index).
 * Rows are the Neighborhood_pointers layout (64 entries per particle);
 * entries past a particle's count are left as they were. */
int emerald_create_regular_neighborhoods(size_t n, float max_distance, uint8_t* counts,
                                         uint64_t* indices, float* distances, float* vectors_to,
                                         float const* self_positions,
                                         int32_t const* self_grid_coords,
                                         float const* other_positions,
                                         uint64_t const* other_sorted_index_pairs,
                                         emerald_block_map const* other_block_map, void* stream);
/* compute_neighbor_distances_and_vectors_to (emerald/sph_common/neighborhood.cpp:154-176). */
int emerald_compute_neighbor_distances_and_vectors_to(size_t n, float* distances,
                                                      float* vectors_to,
                                                      float const* self_positions,
                                                      float const* other_positions,
                                                      uint8_t const* counts,
                                                      uint64_t const* indices, void* stream);
/* compute_neighbor_kernels / compute_neighbor_kernel_gradients
 * (emerald/sph_common/neighborhood.cpp:178-210). */
int emerald_compute_neighbor_kernels(size_t n, float support, float* kernels,
                                     uint8_t const* counts, float const* distances, void* stream);
int emerald_compute_neighbor_kernel_gradients(size_t n, float support, float* kernel_gradients,
                                              uint8_t const* counts, float const* vectors_to,
                                              void* stream);
/* compute_densities (emerald/sph_common/density.cpp:47-72). */
int emerald_compute_densities(size_t n, float support, float target_density, float* densities,
                              float const* fluid_volumes, emerald_neighborhood fluid,
                              float const* solid_volumes, emerald_neighborhood solid,
                              void* stream);
/* compute_divergences (emerald/sph_common/divergence.cpp:47-74). */
int emerald_compute_divergences(size_t n, float target_density, float* divergences,
                                float const* fluid_volumes, float const* fluid_velocities,
                                emerald_neighborhood fluid, float const* solid_volumes,
                                float const* solid_velocities, emerald_neighborhood solid,
                                void* stream);
/* predict_density_stars (emerald/sph_common/density.cpp:85-109). */
int emerald_predict_density_stars(size_t n, float dt, float target_density, float* density_stars,
                                  float const* densities, float const* fluid_volumes,
                                  float const* fluid_velocities, emerald_neighborhood fluid,
                                  float const* solid_volumes, float const* solid_velocities,
                                  emerald_neighborhood solid, void* stream);
/* apply_pressures_in_place (emerald/sph_common/pressure.cpp:52-80). */
int emerald_apply_pressures_in_place(size_t n, float dt, float target_density, float* velocities,
                                     float const* densities, float const* pressures,
                                     float const* fluid_volumes, emerald_neighborhood fluid,
                                     float const* solid_volumes, emerald_neighborhood solid,
                                     void* stream);
/* compute_pressure_accelerations (emerald/sph_common/pressure.cpp:154-178). */
int emerald_compute_pressure_accelerations(size_t n, float target_density,
                                           float* pressure_accelerations, float const* pressures,
                                           float const* densities, float const* fluid_volumes,
                                           emerald_neighborhood fluid, float const* solid_volumes,
                                           emerald_neighborhood solid, void* stream);
/* integrate_velocities_in_place with forces / with accelerations, and
 * integrate_positions_in_place (emerald/sph_common/dynamics.cpp:24-51). */
int emerald_integrate_velocities_with_forces(size_t n, float dt, float target_density,
                                             float* velocities, float const* volumes,
                                             float const* forces, void* stream);
int emerald_integrate_velocities(size_t n, float dt, float* velocities,
                                 float const* accelerations, void* stream);
int emerald_integrate_positions(size_t n, float dt, float* positions, float const* velocities,
                                void* stream);
/* compute_constant_volumes (emerald/sph_common/volume.cpp:7-14). */
int emerald_compute_constant_volumes(size_t n, float target_density, float mass_per_particle,
                                     float* volumes, void* stream);
/* max_vector_squared_magnitude and max_density_error
 * (emerald/sph_common/common.cpp:78-92): *result (device) receives the value. */
int emerald_max_vector_squared_magnitude(size_t n, float* result, float const* vectors,
                                         void* stream);
int emerald_max_density_error(size_t n, float target_density, float* result,
                              float const* densities, void* stream);
/* cfl_maximum_time_step (emerald/sph_common/cfl.cpp:12-21): *flicks (device). */
int emerald_cfl_maximum_time_step(size_t n, float support, float factor, int64_t* flicks,
                                  float const* velocities, void* stream);
/* compute_scalar_average_and_max (emerald/sph_common/common.h:209-240):
 * average_and_max (device) receives {average, max}. */
int emerald_scalar_average_and_max(size_t n, float discretization, float* average_and_max,
                                   float const* values, void* stream);

/* ------------------------------------------ sph2d_box solver ops on device */

/* The solvers' operator functions (emerald/sph2d_box/{iisph,dfsph_p,pcisph,
 * iisph_ap,iisph_pseudo_ap}_ops.h) on device memory, with the conventions of
 * the sph_common section above: the reference's argument order and
 * arithmetic order, bit-identical outputs, asynchronous on `stream`, no
 * allocation, a NULL solid `counts` skipping the boundary terms. Where the
 * reference returns the iteration's (average, max) error pair, `result` is
 * device memory of EMERALD_ITERATION_RESULT_FLOATS floats, 8-byte aligned:
 * result[0] receives the average, result[1] the maximum, and the rest is
 * working storage. */
#define EMERALD_ITERATION_RESULT_FLOATS 4

/* iisph_compute_diis (emerald/sph2d_box/iisph_ops.h:13-24). */
int emerald_iisph_compute_diis(size_t n, float dt, float target_density, float* diis,
                               float const* self_densities, float const* fluid_volumes,
                               emerald_neighborhood fluid, float const* solid_volumes,
                               emerald_neighborhood solid, void* stream);
/* iisph_compute_aiis_and_density_stars (emerald/sph2d_box/iisph_ops.h:26-42). */
int emerald_iisph_compute_aiis_and_density_stars(
  size_t n, float dt, float target_density, float* aiis, float* density_stars, float const* diis,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream);
/* iisph_compute_sum_dij_pjs (emerald/sph2d_box/iisph_ops.h:44-51). */
int emerald_iisph_compute_sum_dij_pjs(size_t n, float dt, float target_density,
                                      float* sum_dij_pjs, float const* volumes,
                                      float const* densities, float const* pressures,
                                      emerald_neighborhood neighborhood, void* stream);
/* iisph_compute_betas (emerald/sph2d_box/iisph_ops.h:53-64). */
int emerald_iisph_compute_betas(size_t n, float dt, float target_density, float* betas,
                                float const* densities, float const* pressures,
                                float const* diis, float const* sum_dij_pjs,
                                float const* fluid_volumes, emerald_neighborhood fluid,
                                float const* solid_volumes, emerald_neighborhood solid,
                                void* stream);
/* iisph_compute_new_pressures (emerald/sph2d_box/iisph_ops.h:66-73). */
int emerald_iisph_compute_new_pressures(size_t n, float omega, float target_density,
                                        float* betas_in_new_pressures_out,
                                        float const* old_pressures, float const* alphas,
                                        float const* density_stars, float* result, void* stream);

/* dfsph_p_compute_shared_coeffs, _density_pseudo_pressures and
 * _divergence_pseudo_pressures (emerald/sph2d_box/dfsph_p_ops.h:13-37). */
int emerald_dfsph_p_compute_shared_coeffs(size_t n, float target_density, float* shared_coeffs,
                                          float const* densities, float const* fluid_volumes,
                                          emerald_neighborhood fluid, float const* solid_volumes,
                                          emerald_neighborhood solid, void* stream);
int emerald_dfsph_p_compute_density_pseudo_pressures(size_t n, float dt, float target_density,
                                                     float* density_pseudo_pressures,
                                                     float const* density_stars,
                                                     float const* shared_coeffs, void* stream);
int emerald_dfsph_p_compute_divergence_pseudo_pressures(size_t n, float dt, float target_density,
                                                        float* divergence_pseudo_pressures,
                                                        float const* divergences,
                                                        float const* shared_coeffs, void* stream);

/* The PCISPH operators (emerald/sph2d_box/pcisph_ops.h:12-61), with the
 * reference's separate neighbour arrays (64 entries per particle). */
int emerald_pcisph_compute_densities(size_t n, float mass_per_particle, float support,
                                     float* densities, uint8_t const* neighbor_counts,
                                     float const* neighbor_kernels, void* stream);
int emerald_pcisph_accumulate_density_from_solids(size_t n, float target_density,
                                                  float* densities, float const* solid_volumes,
                                                  uint8_t const* solid_neighbor_counts,
                                                  uint64_t const* solid_neighbor_indices,
                                                  float const* solid_neighbor_kernels,
                                                  void* stream);
int emerald_pcisph_update_pressures(size_t n, float target_density,
                                    float pressure_correction_denom, float* pressures,
                                    float const* densities, void* stream);
int emerald_pcisph_accumulate_pressure_forces(
  size_t n, float mass_per_particle, float support, float viscosity, float* pressure_forces,
  uint8_t const* neighbor_counts, uint64_t const* neighbor_indices,
  float const* neighbor_distances, float const* neighbor_vectors_to,
  float const* neighbor_kernel_gradients, float const* velocities, float const* pressures,
  float const* densities, void* stream);
int emerald_pcisph_accumulate_pressure_forces_from_solids(
  size_t n, float mass_per_particle, float target_density, float* pressure_forces,
  float const* solid_volumes, uint8_t const* solid_neighbor_counts,
  uint64_t const* solid_neighbor_indices, float const* solid_neighbor_kernel_gradients,
  float const* pressures, float const* densities, void* stream);

/* iisph_ap_density_stars_and_diagonals and iisph_ap_iterate_pressures_in_place
 * (emerald/sph2d_box/iisph_ap_ops.h:13-42). */
int emerald_iisph_ap_density_stars_and_diagonals(
  size_t n, float dt, float target_density, float* density_stars, float* diagonals,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream);
int emerald_iisph_ap_iterate_pressures_in_place(
  size_t n, float dt, float target_density, float omega, float* pressures,
  float const* density_stars, float const* pressure_accelerations, float const* diagonals,
  float const* fluid_volumes, emerald_neighborhood fluid, float const* solid_volumes,
  emerald_neighborhood solid, float* result, void* stream);

/* The IISPH_PSEUDO_AP operators (emerald/sph2d_box/iisph_pseudo_ap_ops.h:13-65). */
int emerald_iisph_pseudo_ap_density_stars_and_pseudo_diagonals(
  size_t n, float dt, float target_density, float* density_stars, float* pseudo_diagonals,
  float const* densities, float const* fluid_volumes, float const* fluid_velocities,
  emerald_neighborhood fluid, float const* solid_volumes, float const* solid_velocities,
  emerald_neighborhood solid, void* stream);
int emerald_iisph_pseudo_ap_compute_pseudo_pressure_displacements(
  size_t n, float target_density, float* pseudo_pressure_displacements,
  float const* pseudo_pressures, float const* densities, float const* fluid_volumes,
  emerald_neighborhood fluid, float const* solid_volumes, emerald_neighborhood solid,
  void* stream);
int emerald_iisph_pseudo_ap_iterate_pseudo_pressures_in_place(
  size_t n, float target_density, float omega, float* pseudo_pressures,
  float const* density_stars, float const* pseudo_pressure_displacements,
  float const* pseudo_diagonals, float const* fluid_volumes, emerald_neighborhood fluid,
  float const* solid_volumes, emerald_neighborhood solid, float* result, void* stream);
int emerald_iisph_pseudo_ap_integrate_velocities_and_positions_in_place(
  size_t n, float dt, float* velocities, float* positions,
  float const* pseudo_pressure_displacements, void* stream);

/* ---------------------------------------------------- allocation-free build */

/* No counterpart in the reference (which always allocates its std::vector
 * scratch). For callers that cannot allocate device memory: hosts that own
 * all device memory through their own allocator and forbid a library's own
 * cudaMalloc, and per-frame loops where cudaMalloc/cudaFree would synchronise
 * the device. Builds the neighbour lists of n points (device float2
 * positions) against themselves, cell size 2*support with the grid at the
 * origin, exactly as the simulation's fluid build: counts[n] and, slot-major,
 * idx/w/gw[k*stride + i] for the k-th neighbour of point i, k below
 * EMERALD_MAX_NEIGHBORS. Size the outputs for that many slots whatever
 * neighbour count you expect: d_idx and d_w hold EMERALD_MAX_NEIGHBORS *
 * stride 32-bit words, d_gw EMERALD_MAX_NEIGHBORS * stride float2, and a
 * dense point fills all 64 slots. d_xy and d_gw must be 8-byte aligned,
 * d_idx and d_w 4-byte aligned (EMERALD_EINVAL otherwise).
 * Allocates nothing: its scratch is a static device array sized for
 * EMERALD_STATIC_MAX_POINTS points, held by every device that loads the
 * library until exit. n above that limit returns EMERALD_EINVAL. Each call
 * looks up the array's device address with the caller's device current
 * (each device, and each new context after cudaDeviceReset, has its own
 * copy); make the first call on a device before any stream capture. All
 * calls share the array, so calls whose work overlaps on the GPU race; order
 * them on one stream. Work is enqueued on `stream` (NULL: the legacy default
 * stream). */
#define EMERALD_STATIC_MAX_POINTS 65536
int emerald_neighbors_static(void const* d_xy, uint32_t n, float support, uint8_t* d_counts,
                             uint32_t* d_idx, float* d_w, void* d_gw, uint32_t stride,
                             void* stream);

/* Message of the last failed call on this thread. */
char const* emerald_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
