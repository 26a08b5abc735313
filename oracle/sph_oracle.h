/*
 * Test infrastructure only: the CPU oracle for the emerald 2D SPH step.
 *
 * A plain-C restatement of the reference algorithm (emerald/z_index,
 * emerald/sph_common, emerald/sph2d_box). Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it; the product library never does.
 * Every function cites the reference file:line it restates. Single-precision
 * operations are written in the reference's source order and the file is
 * compiled with -ffp-contract=off, so results are bit-identical to the
 * reference compiled the same way (checked against oracle/_ref by the tests).
 */
#ifndef EMERALD_SPH_ORACLE_H
#define EMERALD_SPH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_NEIGHBORS 64

/* Mirrors emerald/sph2d_box/parameters.h:12-41 plus the derived
 * Simulation_config fields (emerald/sph2d_box/config.h:7-18). */
typedef struct oracle_params {
    int64_t time_per_step_flicks;
    int32_t sub_steps;
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
    float seconds_per_sub_step;
} oracle_params;

/* Per-sub-step solver statistics (not exposed by the reference, which keeps
 * its loop counters local). */
typedef struct oracle_stats {
    int32_t pressure_iterations;
    int32_t divergence_iterations;
    float error_average;
    float error_max;
    float divergence_error_average;
    float divergence_error_max;
} oracle_stats;

uint64_t oracle_z_index(uint32_t x, uint32_t y);
float oracle_kernel_w(float r, float h);
void oracle_kernel_grad_w(float dx, float dy, float h, float* out);
float oracle_vec2_length(float x, float y);

/* Neighbour build of one point set against another (or itself), grid
 * anchored at the origin. Outputs are n x 64 arrays (vec: n x 64 x 2). */
void oracle_neighborhoods(float const* self_xy,
                          size_t n,
                          float const* other_xy,
                          size_t m,
                          int same_set,
                          float cell_size,
                          uint8_t* counts,
                          uint32_t* idx,
                          float* dist,
                          float* vec);

/* Sort products for a point set: grid coords (n x 2), z keys, sorted
 * (z, index) pairs, block indices; returns the block count. */
size_t oracle_sort(float const* xy,
                   size_t n,
                   float cell_size,
                   int32_t* grid_coords,
                   uint64_t* z_indices,
                   uint64_t* pair_z,
                   uint64_t* pair_index,
                   uint32_t* block_indices,
                   uint64_t* blocks);

/* Boundary volumes V = numer / (W(0) + sum W) over the solid-solid
 * neighbourhood (emerald/sph2d_box/solids.cpp:52-74, numer 1.7 there). */
void oracle_solid_volumes(float const* xy, size_t n, float support, float numer, float* volumes);

typedef struct oracle_sim oracle_sim;

oracle_sim* oracle_sim_create(oracle_params const* params,
                              float const* solid_xy,
                              float const* solid_volumes,
                              size_t n_solid,
                              float const* fluid_xy,
                              float const* fluid_v,
                              size_t n_fluid);
void oracle_sim_destroy(oracle_sim* sim);
void oracle_set_threads(int n);
int oracle_sim_begin_frame(oracle_sim* sim, int method);
int oracle_sim_sub_step(oracle_sim* sim, int method, float t, float dt, oracle_stats* stats);
/* One CFL-adaptive frame (PCISPH: fixed sub-steps); returns sub-steps taken. */
int oracle_sim_frame(oracle_sim* sim, int method);
int64_t oracle_sim_time(oracle_sim const* sim);
void oracle_sim_get_state(oracle_sim const* sim, float* x, float* v);
void oracle_sim_set_state(oracle_sim* sim, float const* x, float const* v);
int oracle_sim_get_array(oracle_sim const* sim, char const* name, float* out);
void oracle_sim_get_neighbors(oracle_sim const* sim,
                              int solid,
                              uint8_t* counts,
                              uint32_t* idx,
                              float* w,
                              float* gw);

#ifdef __cplusplus
}
#endif

#endif
