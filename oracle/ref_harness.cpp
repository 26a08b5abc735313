// Test infrastructure only. A C-ABI harness around the UNMODIFIED emerald
// reference sources (emerald/z_index, emerald/sph_common, emerald/sph2d_box),
// compiled from where they lie by oracle/build_oracle.py against the
// project-written shims in oracle/ref_shim. Tests load the resulting
// oracle/_ref/libemerald_ref.so through ctypes to pin the C restatement and the
// CUDA path bit for bit; bench.py's reference arm times it on the host cores.
// Nothing in the product links or loads this file.
//
// The solver sub-step functions are file-static in the reference
// (emerald/sph2d_box/iisph.cpp:23, dfsph_p.cpp:265, pcisph.cpp:36,
// iisph_ap.cpp:44, iisph_pseudo_ap.cpp:64), so those translation units are
// included here to reach them with a fixed dt.
#include <emerald/sph2d_box/dfsph_p.cpp>
#include <emerald/sph2d_box/iisph.cpp>
#include <emerald/sph2d_box/iisph_ap.cpp>
#include <emerald/sph2d_box/iisph_pseudo_ap.cpp>
#include <emerald/sph2d_box/pcisph.cpp>

#include <emerald/sph2d_box/colors.h>
#include <emerald/sph2d_box/forces.h>
#include <emerald/sph2d_box/initial_state.h>
#include <emerald/sph2d_box/solids.h>
#include <emerald/sph_common/common.h>
#include <emerald/sph_common/neighborhood.h>
#include <emerald/sph_common/cfl.h>
#include <emerald/sph_common/density.h>
#include <emerald/sph_common/divergence.h>
#include <emerald/sph_common/dynamics.h>
#include <emerald/sph_common/pressure.h>
#include <emerald/sph_common/volume.h>
#include <emerald/z_index/z_index.h>

#include <tbb/tbb_shim.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <string>

using namespace emerald;
using namespace emerald::sph2d_box;
using namespace emerald::sph_common;

extern "C" {

// Mirrors emerald/sph2d_box/parameters.h:12-41 plus two optional overrides of
// Simulation_config fields (emerald/sph2d_box/config.h:7-18).
struct ref_params {
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
    float mass_per_particle_override;         // > 0 replaces config.mass_per_particle
    float pressure_correction_denom_override;  // > 0 replaces the PCISPH denominator
};

}  // extern "C"

namespace {

Parameters to_parameters(ref_params const& p) {
    Parameters params;
    params.seed = p.seed;
    params.time_per_step = flicks{p.time_per_step_flicks};
    params.sub_steps = p.sub_steps;
    params.length = p.length;
    params.support = p.support;
    params.gravity = p.gravity;
    params.viscosity = p.viscosity;
    params.target_density = p.target_density;
    params.iisph.max_pressure_iterations = p.iisph_max_pressure_iterations;
    params.iisph.error_average_threshold = p.iisph_error_average_threshold;
    params.iisph.error_max_threshold = p.iisph_error_max_threshold;
    params.iisph.omega = p.iisph_omega;
    params.dfsph.max_correction_iterations = p.dfsph_max_correction_iterations;
    params.dfsph.density_error_average_threshold = p.dfsph_density_error_average_threshold;
    params.dfsph.density_error_max_threshold = p.dfsph_density_error_max_threshold;
    params.dfsph.divergence_error_average_threshold =
      p.dfsph_divergence_error_average_threshold;
    params.dfsph.divergence_error_max_threshold = p.dfsph_divergence_error_max_threshold;
    return params;
}

Simulation_config to_config(ref_params const& p) {
    Simulation_config config{to_parameters(p)};
    if (p.mass_per_particle_override > 0.0f) {
        config.mass_per_particle = p.mass_per_particle_override;
    }
    if (p.pressure_correction_denom_override > 0.0f) {
        config.pressure_correction_denom = p.pressure_correction_denom_override;
    }
    return config;
}

struct Ref_sim {
    Simulation_config config;
    Solid_state solid_state;
    State state;
    Temp_data temp;
    User_forces_function forces;
    User_colors_function colors;
    flicks time{0};
    int64_t sub_steps_run = 0;  // sub-steps of ref_sim_run_window since creation
};

std::vector<V2f> to_v2f(float const* xy, size_t n) {
    std::vector<V2f> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = V2f{xy[2 * i], xy[2 * i + 1]};
    return out;
}

void copy_out(std::vector<V2f> const& v, float* out) {
    for (size_t i = 0; i < v.size(); ++i) {
        out[2 * i] = v[i][0];
        out[2 * i + 1] = v[i][1];
    }
}

void copy_out(std::vector<float> const& v, float* out) {
    std::memcpy(out, v.data(), v.size() * sizeof(float));
}

void copy_neighborhood(Neighborhood_vectors const& nb,
                       size_t n,
                       uint8_t* counts,
                       uint32_t* idx,
                       float* dist,
                       float* vec,
                       float* w,
                       float* gw) {
    for (size_t i = 0; i < n; ++i) {
        uint8_t const c = nb.counts[i];
        if (counts) counts[i] = c;
        for (size_t k = 0; k < NEIGHBORHOOD_MAX_COUNT; ++k) {
            size_t const o = i * NEIGHBORHOOD_MAX_COUNT + k;
            bool const live = k < c;
            if (idx) idx[o] = live ? static_cast<uint32_t>(nb.indices[i][k]) : 0u;
            if (dist) dist[o] = live && !nb.distances.empty() ? nb.distances[i][k] : 0.0f;
            if (vec) {
                vec[2 * o] = live && !nb.vectors_to.empty() ? nb.vectors_to[i][k][0] : 0.0f;
                vec[2 * o + 1] = live && !nb.vectors_to.empty() ? nb.vectors_to[i][k][1] : 0.0f;
            }
            if (w) w[o] = live && nb.kernels.size() == n ? nb.kernels[i][k] : 0.0f;
            if (gw) {
                bool const g = live && nb.kernel_gradients.size() == n;
                gw[2 * o] = g ? nb.kernel_gradients[i][k][0] : 0.0f;
                gw[2 * o + 1] = g ? nb.kernel_gradients[i][k][1] : 0.0f;
            }
        }
    }
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { tbb_shim::Pool::get().set_threads(n); }

int ref_get_threads() { return tbb_shim::Pool::get().threads(); }

uint64_t ref_z_index(uint32_t x, uint32_t y) { return z_index::z_index(x, y); }

void ref_default_params(ref_params* p) {
    Parameters const d;
    p->seed = d.seed;
    p->time_per_step_flicks = d.time_per_step.count();
    p->sub_steps = d.sub_steps;
    p->length = d.length;
    p->support = d.support;
    p->gravity = d.gravity;
    p->viscosity = d.viscosity;
    p->target_density = d.target_density;
    p->iisph_max_pressure_iterations = d.iisph.max_pressure_iterations;
    p->iisph_error_average_threshold = d.iisph.error_average_threshold;
    p->iisph_error_max_threshold = d.iisph.error_max_threshold;
    p->iisph_omega = d.iisph.omega;
    p->dfsph_max_correction_iterations = d.dfsph.max_correction_iterations;
    p->dfsph_density_error_average_threshold = d.dfsph.density_error_average_threshold;
    p->dfsph_density_error_max_threshold = d.dfsph.density_error_max_threshold;
    p->dfsph_divergence_error_average_threshold = d.dfsph.divergence_error_average_threshold;
    p->dfsph_divergence_error_max_threshold = d.dfsph.divergence_error_max_threshold;
    p->mass_per_particle_override = 0.0f;
    p->pressure_correction_denom_override = 0.0f;
}

// out: seconds_per_sub_step, mass_per_particle, draw_radius,
// pressure_correction_denom (emerald/sph2d_box/config.cpp:16-132).
void ref_config(ref_params const* p, float* out) {
    Simulation_config const c = to_config(*p);
    out[0] = c.seconds_per_sub_step;
    out[1] = c.mass_per_particle;
    out[2] = c.draw_radius;
    out[3] = c.pressure_correction_denom;
}

float ref_kernel_w(float r, float h) { return kernels::W(r, h); }

void ref_kernel_grad_w(float dx, float dy, float h, float* out) {
    V2f const g = kernels::GradW(V2f{dx, dy}, h);
    out[0] = g[0];
    out[1] = g[1];
}

float ref_vec2_length(float x, float y) { return V2f{x, y}.length(); }

// Seeded synthetic block scene: an nx-by-ny fluid lattice at spacing dx with
// origin offset (x0, y0), each coordinate jittered uniformly by +/- jitter*dx
// from std::mt19937_64{seed}; x then y per particle.
void ref_block_scene(uint32_t nx,
                     uint32_t ny,
                     float dx,
                     float x0,
                     float y0,
                     float jitter,
                     uint64_t seed,
                     float* xy) {
    std::mt19937_64 gen{seed};
    std::uniform_real_distribution<float> dist{-jitter * dx, jitter * dx};
    size_t k = 0;
    for (uint32_t j = 0; j < ny; ++j) {
        for (uint32_t i = 0; i < nx; ++i) {
            float const px = x0 + (static_cast<float>(i) + 0.5f) * dx;
            float const py = y0 + (static_cast<float>(j) + 0.5f) * dx;
            float const jx = dist(gen);
            float const jy = dist(gen);
            xy[2 * k] = px + jx;
            xy[2 * k + 1] = py + jy;
            ++k;
        }
    }
}

// The mass per particle and PCISPH denominator of a square lattice at
// spacing dx: the sums of the Simulation_config constructor
// (emerald/sph2d_box/config.cpp:16-132) taken over the lattice points
// (i dx, j dx), |i|, |j| <= ceil(2 support / dx) + 1, about the origin (rows
// j outer, columns i inner), with the reference's own kernels::W and GradW.
// out: mass_per_particle, pressure_correction_denom (dt in place of
// seconds_per_sub_step).
void ref_lattice_config(ref_params const* p, float dx, float dt, float* out) {
    float const h = p->support;
    int const reach = static_cast<int>(std::ceil(2.0 * double(h) / double(dx))) + 1;
    float muchness = 0.0f;
    V2f gradw_sum{0.0f, 0.0f};
    float gradw_dot_gradw_sum = 0.0f;
    for (int j = -reach; j <= reach; ++j) {
        for (int i = -reach; i <= reach; ++i) {
            V2f const point{static_cast<float>(i) * dx, static_cast<float>(j) * dx};
            V2f const delta_position = V2f{0.0f, 0.0f} - point;
            float const w = kernels::W(delta_position.length(), h);
            if (w > 0.0f) muchness += w;
            V2f const gradw = kernels::GradW(delta_position, h);
            gradw_sum += gradw;
            gradw_dot_gradw_sum += gradw.dot(gradw);
        }
    }
    out[0] = p->target_density / muchness;
    float const beta = 2.0f * sqr(dt / muchness);
    out[1] = beta * (gradw_sum.dot(gradw_sum) + gradw_dot_gradw_sum);
}

// Boundary rows of the synthetic dam-break tank [0, length]^2: `layers` rows
// at spacing dx below the floor (x from -layers to n + layers - 1 cells) and
// outside each side wall, row by row (floor, left, right), n = round(length /
// dx). Returns the point count; xy may be NULL to count only.
size_t ref_wall_scene(float dx, float length, int layers, float* xy) {
    int const n = static_cast<int>(std::lround(double(length) / double(dx)));
    size_t k = 0;
    auto put = [&](float x, float y) {
        if (xy) {
            xy[2 * k] = x;
            xy[2 * k + 1] = y;
        }
        ++k;
    };
    for (int l = 0; l < layers; ++l) {
        float const off = (static_cast<float>(l) + 0.5f) * dx;
        for (int i = -layers; i < n + layers; ++i) put((static_cast<float>(i) + 0.5f) * dx, -off);
        for (int j = 0; j < n; ++j) put(-off, (static_cast<float>(j) + 0.5f) * dx);
        for (int j = 0; j < n; ++j) put(length + off, (static_cast<float>(j) + 0.5f) * dx);
    }
    return k;
}

// n points with both coordinates drawn from
// std::uniform_real_distribution<float>{lo, hi} over std::mt19937_64{seed}, x
// then y per point: the fixture of emerald/sph_common/tests/test_common.cpp:18-31
// and test_neighborhood.cpp:18-31 (7927 points, seed 17272, [-100, 100]).
void ref_uniform_points(size_t n, uint64_t seed, float lo, float hi, float* xy) {
    std::mt19937_64 gen{seed};
    std::uniform_real_distribution<float> dist{lo, hi};
    for (size_t i = 0; i < n; ++i) {
        xy[2 * i] = dist(gen);
        xy[2 * i + 1] = dist(gen);
    }
}

void* ref_sim_create(ref_params const* p,
                     float const* solid_xy,
                     size_t n_solid,
                     float const* fluid_xy,
                     float const* fluid_v,
                     size_t n_fluid) {
    auto* sim = new Ref_sim;
    sim->config = to_config(*p);
    Parameters const& params = sim->config.params;
    if (solid_xy) {
        Solid_state solid;
        solid.positions = to_v2f(solid_xy, n_solid);
        solid.velocities.assign(n_solid, V2f{0.0f, 0.0f});
        solid.colors.assign(n_solid, C4f{0.784f, 0.608f, 0.078f, 1.0f});
        sim->solid_state = compute_neighbor_data_and_volumes(params, std::move(solid));
    } else {
        sim->solid_state = world_walls_initial_solid_state(params);
    }
    if (fluid_xy) {
        sim->state.positions = to_v2f(fluid_xy, n_fluid);
        if (fluid_v) {
            sim->state.velocities = to_v2f(fluid_v, n_fluid);
        } else {
            sim->state.velocities.assign(n_fluid, V2f{0.0f, 0.0f});
        }
        sim->state.colors.assign(n_fluid, C4f{0.5f, 0.5f, 1.0f, 1.0f});
    } else {
        sim->state = dam_break_initial_state(params, sim->solid_state);
    }
    sim->forces = default_gravity_forces(params.gravity);
    sim->colors = default_target_density_colors(params.target_density);
    return sim;
}

void ref_sim_destroy(void* h) { delete static_cast<Ref_sim*>(h); }

size_t ref_sim_fluid_count(void* h) { return static_cast<Ref_sim*>(h)->state.positions.size(); }

size_t ref_sim_solid_count(void* h) {
    return static_cast<Ref_sim*>(h)->solid_state.positions.size();
}

void ref_sim_get_solid(void* h, float* xy, float* volumes) {
    auto* sim = static_cast<Ref_sim*>(h);
    if (xy) copy_out(sim->solid_state.positions, xy);
    if (volumes) copy_out(sim->solid_state.volumes, volumes);
}

// Replaces the boundary volumes that compute_neighbor_data_and_volumes
// produced (Solid_state::volumes, emerald/sph2d_box/state.h:31).
void ref_sim_set_solid_volumes(void* h, float const* volumes) {
    auto* sim = static_cast<Ref_sim*>(h);
    std::memcpy(sim->solid_state.volumes.data(), volumes, sim->solid_state.volumes.size() * sizeof(float));
}

// Replaces the boundary between frames the way a caller of the step
// functions would: a new Solid_state from positions and velocities through
// compute_neighbor_data_and_volumes (emerald/sph2d_box/solids.cpp:76-137),
// whose volumes `volumes` overrides (NULL xy keeps the positions; NULL
// volumes with NULL xy keeps the volumes).
void ref_sim_set_solid(void* h, float const* xy, float const* v, float const* volumes) {
    auto* sim = static_cast<Ref_sim*>(h);
    size_t const n = sim->solid_state.positions.size();
    Solid_state solid;
    solid.positions = xy ? to_v2f(xy, n) : sim->solid_state.positions;
    solid.velocities = v ? to_v2f(v, n) : sim->solid_state.velocities;
    solid.colors = sim->solid_state.colors;
    std::vector<float> const old_volumes = sim->solid_state.volumes;
    sim->solid_state = compute_neighbor_data_and_volumes(sim->config.params, std::move(solid));
    if (volumes) {
        std::memcpy(sim->solid_state.volumes.data(), volumes, n * sizeof(float));
    } else if (!xy) {
        sim->solid_state.volumes = old_volumes;
    }
}

// Replaces the simulation's User_forces_function (default_gravity_forces,
// emerald/sph2d_box/forces.cpp:73-83, until then) with one that applies
// `count` terms in order through the reference's own force functions:
// kind 1 accumulate_gravity_forces (a = gravity), 2
// accumulate_constant_pole_attraction_forces (a = magnitude, pole (b, c)),
// 3 accumulate_simple_drag_forces (a = magnitude, b = diameter).
void ref_sim_set_forces(void* h, int32_t const* kinds, float const* args, int count) {
    auto* sim = static_cast<Ref_sim*>(h);
    std::vector<int32_t> const k(kinds, kinds + count);
    std::vector<float> const a(args, args + 3 * count);
    sim->forces = [k, a](size_t const n, float const, float const, float const mass,
                         float const, V2f* const forces, V2f const* const positions,
                         V2f const* const velocities) {
        for (size_t t = 0; t < k.size(); ++t) {
            float const x = a[3 * t], y = a[3 * t + 1], z = a[3 * t + 2];
            if (k[t] == 1) accumulate_gravity_forces(n, mass, x, forces);
            if (k[t] == 2) accumulate_constant_pole_attraction_forces(n, x, V2f{y, z}, forces, positions);
            if (k[t] == 3) accumulate_simple_drag_forces(n, x, y, forces, velocities);
        }
    };
}

// The reference's force functions on host arrays: n forces (x, y pairs,
// accumulated in place) from positions and velocities, with the terms of
// ref_sim_set_forces applied in order.
void ref_accumulate_forces(int32_t const* kinds, float const* args, int count, size_t n,
                           float mass, float* forces, float const* positions,
                           float const* velocities) {
    auto* f = reinterpret_cast<V2f*>(forces);
    auto const* x = reinterpret_cast<V2f const*>(positions);
    auto const* v = reinterpret_cast<V2f const*>(velocities);
    for (int t = 0; t < count; ++t) {
        float const a = args[3 * t], b = args[3 * t + 1], c = args[3 * t + 2];
        if (kinds[t] == 1) accumulate_gravity_forces(n, mass, a, f);
        if (kinds[t] == 2) accumulate_constant_pole_attraction_forces(n, a, V2f{b, c}, f, x);
        if (kinds[t] == 3) accumulate_simple_drag_forces(n, a, b, f, v);
    }
}

// A C function as the User_forces_function (argument list of
// emerald/sph2d_box/forces.h:13-21 plus a user pointer).
typedef void (*ref_forces_fn)(void* user, size_t count, float time, float dt, float mass,
                              float radius, float* forces, float const* positions,
                              float const* velocities);
void ref_sim_set_force_callback(void* h, ref_forces_fn fn, void* user) {
    auto* sim = static_cast<Ref_sim*>(h);
    sim->forces = [fn, user](size_t const n, float const t, float const dt, float const mass,
                             float const radius, V2f* const forces, V2f const* const positions,
                             V2f const* const velocities) {
        fn(user, n, t, dt, mass, radius, reinterpret_cast<float*>(forces),
           reinterpret_cast<float const*>(positions), reinterpret_cast<float const*>(velocities));
    };
}

int64_t ref_sim_time(void* h) { return static_cast<Ref_sim*>(h)->time.count(); }

// Method numbering follows EZ_EXAMPLE_SIM::Method
// (emerald/sph2d_box/simulation.h:25): 0 PCISPH, 1 IISPH, 2 IISPH_AP,
// 3 IISPH_PSEUDO_AP, 4 DFSPH_P.
int ref_sim_begin_frame(void* h, int method) {
    auto* sim = static_cast<Ref_sim*>(h);
    size_t const n = sim->state.positions.size();
    switch (method) {
    case 0: break;
    case 1: iisph_resize_temp_arrays(n, sim->temp); break;
    case 2: iisph_ap_resize_temp_arrays(n, sim->temp); break;
    case 3: iisph_pseudo_ap_resize_temp_arrays(n, sim->temp); break;
    case 4: dfsph_p_resize_and_init_temp_arrays(n, sim->temp); break;
    default: return -1;
    }
    if (method != 0) {
        compute_constant_volumes(n,
                                 sim->config.params.target_density,
                                 sim->config.mass_per_particle,
                                 sim->temp.fluid_volumes.data());
    }
    return 0;
}

int ref_sim_sub_step(void* h, int method, float t, float dt) {
    auto* sim = static_cast<Ref_sim*>(h);
    switch (method) {
    case 0:
        pcisph_sub_step(t, dt, sim->config, sim->state, sim->solid_state, sim->temp, sim->forces);
        break;
    case 1:
        iisph_sub_step(t, dt, sim->config, sim->state, sim->solid_state, sim->temp, sim->forces);
        break;
    case 2:
        iisph_ap_sub_step(
          t, dt, sim->config, sim->state, sim->solid_state, sim->temp, sim->forces);
        break;
    case 3:
        iisph_pseudo_ap_sub_step(
          t, dt, sim->config, sim->state, sim->solid_state, sim->temp, sim->forces);
        break;
    case 4:
        dfsph_p_sub_step(t, dt, sim->config, sim->state, sim->solid_state, sim->temp, sim->forces);
        break;
    default: return -1;
    }
    return 0;
}

// One frame through the reference's own frame functions, exactly as
// EZ_EXAMPLE_SIM::step (emerald/sph2d_box/simulation.cpp:41-93) calls them.
int ref_sim_frame(void* h, int method) {
    auto* sim = static_cast<Ref_sim*>(h);
    switch (method) {
    case 0:
        sim->state = pcisph_simulation_step(sim->time, sim->config, std::move(sim->state),
                                            sim->solid_state, sim->temp, sim->forces,
                                            sim->colors);
        break;
    case 1:
        sim->state = iisph_simulation_step(sim->time, sim->config, std::move(sim->state),
                                           sim->solid_state, sim->temp, sim->forces,
                                           sim->colors);
        break;
    case 2:
        sim->state = iisph_ap_simulation_step(sim->time, sim->config, std::move(sim->state),
                                              sim->solid_state, sim->temp, sim->forces,
                                              sim->colors);
        break;
    case 3:
        sim->state = iisph_pseudo_ap_simulation_step(sim->time, sim->config,
                                                     std::move(sim->state), sim->solid_state,
                                                     sim->temp, sim->forces, sim->colors);
        break;
    case 4:
        sim->state = dfsph_p_simulation_step(sim->time, sim->config, std::move(sim->state),
                                             sim->solid_state, sim->temp, sim->forces,
                                             sim->colors);
        break;
    default: return -1;
    }
    sim->time += sim->config.params.time_per_step;
    return 0;
}

// Runs CFL-adaptive frames through the reference's own frame loop
// (std_adaptive_time_step, emerald/sph2d_box/adaptive_time_step.h:35-122,
// with each method's sub-step function, resize function, denominators and
// CFL factor as its X_simulation_step passes them) and times a window of its
// sub-steps: sub-steps are numbered from 0 since the simulation's creation;
// those numbered [skip, skip + count) are timed one by one with a steady
// clock, those after the window are not run (the frame loop finishes with
// the state unchanged, so the state is that after skip + count sub-steps).
// Once the timed seconds pass max_seconds (> 0) the window ends early.
// Returns the number of sub-steps timed, -1 for PCISPH (no adaptive frames)
// or an unknown method; *seconds receives their total time.
int64_t ref_sim_run_window(void* h, int method, int64_t skip, int64_t count, double max_seconds,
                           double* seconds) {
    auto* sim = static_cast<Ref_sim*>(h);
    int64_t end = skip + count;
    int64_t timed = 0;
    double total = 0.0;
    using Sub = void (*)(float, float, Simulation_config const&, State&, Solid_state const&,
                         Temp_data&, User_forces_function const&);
    using Resize = void (*)(size_t, Temp_data&);
    Sub sub = nullptr;
    Resize resize = nullptr;
    int min_denom = 60, max_denom = 4;
    float cfl = 0.4f;
    switch (method) {
    case 1: sub = iisph_sub_step; resize = iisph_resize_temp_arrays; max_denom = 6; cfl = 0.2f; break;
    case 2: sub = iisph_ap_sub_step; resize = iisph_ap_resize_temp_arrays; break;
    case 3: sub = iisph_pseudo_ap_sub_step; resize = iisph_pseudo_ap_resize_temp_arrays; break;
    case 4: sub = dfsph_p_sub_step; resize = dfsph_p_resize_and_init_temp_arrays; break;
    default: return -1;
    }
    auto timed_sub = [&](float t, float dt, Simulation_config const& c, State& st,
                         Solid_state const& solid, Temp_data& temp,
                         User_forces_function const& forces) {
        int64_t const k = sim->sub_steps_run;
        if (k >= end) return;
        ++sim->sub_steps_run;
        if (k < skip) {
            sub(t, dt, c, st, solid, temp, forces);
            return;
        }
        auto const t0 = std::chrono::steady_clock::now();
        sub(t, dt, c, st, solid, temp, forces);
        total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        ++timed;
        if (max_seconds > 0.0 && total > max_seconds) end = sim->sub_steps_run;
    };
    while (sim->sub_steps_run < end) {
        sim->state = std_adaptive_time_step(std::nullopt, resize, timed_sub, min_denom, max_denom,
                                            cfl, sim->time, sim->config, std::move(sim->state),
                                            sim->solid_state, sim->temp, sim->forces,
                                            sim->colors);
        sim->time += sim->config.params.time_per_step;
    }
    if (seconds) *seconds = total;
    return timed;
}

void ref_sim_get_state(void* h, float* x, float* v) {
    auto* sim = static_cast<Ref_sim*>(h);
    if (x) copy_out(sim->state.positions, x);
    if (v) copy_out(sim->state.velocities, v);
}

void ref_sim_set_state(void* h, float const* x, float const* v) {
    auto* sim = static_cast<Ref_sim*>(h);
    size_t const n = sim->state.positions.size();
    if (x) sim->state.positions = to_v2f(x, n);
    if (v) sim->state.velocities = to_v2f(v, n);
}

// Copies a per-particle temporary of Temp_data (emerald/sph2d_box/state.h:34-69).
// Returns the number of floats per particle, 0 when the array is unset, or -1
// for an unknown name.
int ref_sim_get_array(void* h, char const* name, float* out) {
    auto* sim = static_cast<Ref_sim*>(h);
    auto& t = sim->temp;
    std::string const s{name};
    auto scalar = [&](std::vector<float> const& v) -> int {
        if (v.empty()) return 0;
        if (out) copy_out(v, out);
        return 1;
    };
    auto vector = [&](std::vector<V2f> const& v) -> int {
        if (v.empty()) return 0;
        if (out) copy_out(v, out);
        return 2;
    };
    if (s == "densities") return scalar(t.densities);
    if (s == "pressures") return scalar(t.pressures);
    if (s == "new_pressures") return scalar(t.new_pressures);
    if (s == "density_stars") return scalar(t.density_stars);
    if (s == "aiis") return scalar(t.aiis);
    if (s == "alphas") return scalar(t.alphas);
    if (s == "divergence_kappas") return scalar(t.divergence_kappas);
    if (s == "density_kappas") return scalar(t.density_kappas);
    if (s == "fluid_volumes") return scalar(t.fluid_volumes);
    if (s == "diis") return vector(t.diis);
    if (s == "sum_dij_pjs") return vector(t.sum_dij_pjs);
    if (s == "external_forces") return vector(t.external_forces);
    if (s == "pressure_forces") return vector(t.pressure_forces);
    if (s == "pressure_accelerations") return vector(t.pressure_accelerations);
    if (s == "velocity_external_forces") return vector(t.velocity_external_forces);
    if (s == "position_stars") return vector(t.position_stars);
    if (s == "velocity_stars") return vector(t.velocity_stars);
    return -1;
}

// Fluid (solid == 0) or boundary (solid == 1) neighbourhoods of the last
// sub-step, 64 slots per particle (emerald/sph_common/neighborhood.h:38).
void ref_sim_get_neighbors(void* h,
                           int solid,
                           uint8_t* counts,
                           uint32_t* idx,
                           float* dist,
                           float* vec,
                           float* w,
                           float* gw) {
    auto* sim = static_cast<Ref_sim*>(h);
    auto const& nb = solid ? sim->temp.solid_neighborhood : sim->temp.neighborhood;
    copy_neighborhood(nb, nb.counts.size(), counts, idx, dist, vec, w, gw);
}

// Sort products of the last neighbour build (emerald/sph2d_box/state.h:34-40).
size_t ref_sim_get_sort(void* h,
                        int solid,
                        int32_t* grid_coords,
                        uint64_t* z_indices,
                        uint64_t* pair_z,
                        uint64_t* pair_index,
                        uint32_t* block_indices,
                        uint64_t* blocks) {
    auto* sim = static_cast<Ref_sim*>(h);
    auto const& gc = solid ? sim->solid_state.grid_coords : sim->temp.grid_coords;
    auto const& z = solid ? sim->solid_state.z_indices : sim->temp.z_indices;
    auto const& pairs = solid ? sim->solid_state.index_pairs : sim->temp.index_pairs;
    auto const& bi = solid ? sim->solid_state.block_indices : sim->temp.block_indices;
    auto const& bl = solid ? sim->solid_state.blocks : sim->temp.blocks;
    for (size_t i = 0; i < gc.size(); ++i) {
        if (grid_coords) {
            grid_coords[2 * i] = gc[i][0];
            grid_coords[2 * i + 1] = gc[i][1];
        }
        if (z_indices) z_indices[i] = z[i];
        if (pair_z) pair_z[i] = pairs[i].first;
        if (pair_index) pair_index[i] = pairs[i].second;
        if (block_indices) block_indices[i] = bi[i];
    }
    if (blocks) {
        for (size_t b = 0; b < bl.size(); ++b) {
            blocks[2 * b] = bl[b].first;
            blocks[2 * b + 1] = bl[b].second;
        }
    }
    return bl.size();
}

// Stand-alone neighbour build over one point set against itself, with the
// grid anchored at the origin: the path of the reference's
// emerald/sph_common/tests/test_neighborhood.cpp:177-292.
void ref_self_neighborhoods(float const* xy,
                            size_t n,
                            float cell_size,
                            int32_t* grid_coords,
                            uint64_t* z_indices,
                            uint64_t* pair_index,
                            uint32_t* block_indices,
                            uint8_t* counts,
                            uint32_t* idx,
                            float* dist,
                            float* vec) {
    auto const positions = to_v2f(xy, n);
    std::vector<V2i> gc(n);
    compute_grid_coords(n, cell_size, V2f{0.0f, 0.0f}, gc.data(), positions.data());
    std::vector<uint64_t> z(n);
    compute_z_indices(n, z.data(), gc.data());
    std::vector<std::pair<uint64_t, size_t>> pairs(n);
    compute_index_pairs(n, pairs.data(), z.data());
    sort_index_pairs(n, pairs.data());
    std::vector<uint32_t> bi(n);
    compute_block_indices(n, bi.data(), pairs.data());
    size_t const block_count = n ? bi.back() + 1 : 0;
    std::vector<std::pair<size_t, size_t>> blocks(block_count);
    fill_blocks(n, blocks.data(), bi.data());
    Block_map map{block_count * 2};
    map = create_block_map(block_count, std::move(map), blocks.data(), pairs.data());
    Neighborhood_vectors nb;
    nb.resize(n);
    create_regular_neighborhoods(n,
                                 cell_size,
                                 nb.counts.data(),
                                 nb.indices.data(),
                                 nb.distances.data(),
                                 nb.vectors_to.data(),
                                 positions.data(),
                                 gc.data(),
                                 positions.data(),
                                 pairs.data(),
                                 map);
    nb.kernels.clear();
    nb.kernel_gradients.clear();
    for (size_t i = 0; i < n; ++i) {
        if (grid_coords) {
            grid_coords[2 * i] = gc[i][0];
            grid_coords[2 * i + 1] = gc[i][1];
        }
        if (z_indices) z_indices[i] = z[i];
        if (pair_index) pair_index[i] = pairs[i].second;
        if (block_indices) block_indices[i] = bi[i];
    }
    copy_neighborhood(nb, n, counts, idx, dist, vec, nullptr, nullptr);
}

float ref_max_density_error(size_t n, float target_density, float const* densities) {
    return max_density_error(n, target_density, densities);
}

float ref_max_vector_squared_magnitude(size_t n, float const* xy) {
    auto const v = to_v2f(xy, n);
    return max_vector_squared_magnitude(n, v.data());
}

int64_t ref_cfl_maximum_time_step(size_t n, float support, float factor, float const* v_xy) {
    auto const v = to_v2f(v_xy, n);
    return cfl_maximum_time_step(n, support, factor, v.data()).count();
}

}  // extern "C"

// ------------------------------------------------ sph_common free functions
//
// The reference's sph_common functions on flat host arrays, for comparing
// the library's device versions with them: neighbour lists arrive row-major
// (64 entries per particle, 64-bit indices) and are copied into the
// reference's Neighborhood_vectors.

namespace {

Neighborhood_vectors nbhd_from(size_t n, uint8_t const* counts, uint64_t const* idx,
                               float const* dist, float const* vec, float const* w,
                               float const* gw) {
    Neighborhood_vectors nb;
    nb.resize(n);
    for (size_t i = 0; i < n; ++i) {
        nb.counts[i] = counts ? counts[i] : 0;
        for (size_t k = 0; k < NEIGHBORHOOD_MAX_COUNT; ++k) {
            size_t const e = i * NEIGHBORHOOD_MAX_COUNT + k;
            nb.indices[i][k] = idx ? size_t(idx[e]) : 0;
            nb.distances[i][k] = dist ? dist[e] : 0.0f;
            nb.vectors_to[i][k] = vec ? V2f{vec[2 * e], vec[2 * e + 1]} : V2f{0.0f, 0.0f};
            nb.kernels[i][k] = w ? w[e] : 0.0f;
            nb.kernel_gradients[i][k] = gw ? V2f{gw[2 * e], gw[2 * e + 1]} : V2f{0.0f, 0.0f};
        }
    }
    return nb;
}

}  // namespace

extern "C" {

void ref_common_grid_coords(size_t n, float cell, float bx, float by, int32_t* gc,
                            float const* xy) {
    auto const p = to_v2f(xy, n);
    std::vector<V2i> out(n);
    compute_grid_coords(n, cell, V2f{bx, by}, out.data(), p.data());
    for (size_t i = 0; i < n; ++i) {
        gc[2 * i] = out[i][0];
        gc[2 * i + 1] = out[i][1];
    }
}

void ref_common_z_indices(size_t n, uint64_t* z, int32_t const* gc) {
    std::vector<V2i> g(n);
    for (size_t i = 0; i < n; ++i) g[i] = V2i{gc[2 * i], gc[2 * i + 1]};
    compute_z_indices(n, z, g.data());
}

// compute_index_pairs / sort_index_pairs / compute_block_indices /
// fill_blocks (emerald/sph_common/neighborhood.cpp:10-93) on interleaved
// (z, index) and (begin, end) uint64 pairs.
namespace {
std::vector<std::pair<uint64_t, size_t>> pairs_from(size_t n, uint64_t const* flat) {
    std::vector<std::pair<uint64_t, size_t>> p(n);
    for (size_t i = 0; i < n; ++i) p[i] = {flat[2 * i], size_t(flat[2 * i + 1])};
    return p;
}
void pairs_to(std::vector<std::pair<uint64_t, size_t>> const& p, uint64_t* flat) {
    for (size_t i = 0; i < p.size(); ++i) {
        flat[2 * i] = p[i].first;
        flat[2 * i + 1] = p[i].second;
    }
}
}  // namespace

void ref_common_index_pairs(size_t n, uint64_t* pairs, uint64_t const* z) {
    std::vector<std::pair<uint64_t, size_t>> p(n);
    compute_index_pairs(n, p.data(), z);
    pairs_to(p, pairs);
}

void ref_common_sort_index_pairs(size_t n, uint64_t* pairs) {
    auto p = pairs_from(n, pairs);
    sort_index_pairs(n, p.data());
    pairs_to(p, pairs);
}

void ref_common_block_indices(size_t n, uint32_t* block_indices, uint64_t const* pairs) {
    auto const p = pairs_from(n, pairs);
    compute_block_indices(n, block_indices, p.data());
}

void ref_common_fill_blocks(size_t n, size_t block_count, uint64_t* blocks,
                            uint32_t* block_indices) {
    std::vector<std::pair<size_t, size_t>> b(block_count);
    for (size_t k = 0; k < block_count; ++k) b[k] = {size_t(blocks[2 * k]), size_t(blocks[2 * k + 1])};
    fill_blocks(n, b.data(), block_indices);
    for (size_t k = 0; k < block_count; ++k) {
        blocks[2 * k] = b[k].first;
        blocks[2 * k + 1] = b[k].second;
    }
}

// create_block_map + create_regular_neighborhoods (neighborhood.cpp:95-136):
// the other set's block map from its blocks and sorted pairs, then the
// lists (row-major, 64 entries per particle). With `same` the other set is
// the self set (one positions array, so the reference skips each particle
// itself).
void ref_common_regular_neighborhoods(size_t n, size_t n_other, float max_distance,
                                      uint8_t* counts, uint64_t* idx, float* dist, float* vec,
                                      float const* self_xy, int32_t const* self_gc,
                                      float const* other_xy, int same, size_t n_pairs,
                                      uint64_t const* other_pairs, size_t block_count,
                                      uint64_t const* other_blocks) {
    auto const p = to_v2f(self_xy, n);
    auto const o = same ? std::vector<V2f>() : to_v2f(other_xy, n_other);
    std::vector<V2i> gc(n);
    for (size_t i = 0; i < n; ++i) gc[i] = V2i{self_gc[2 * i], self_gc[2 * i + 1]};
    auto const pairs = pairs_from(n_pairs, other_pairs);
    std::vector<std::pair<size_t, size_t>> blocks(block_count);
    for (size_t k = 0; k < block_count; ++k) {
        blocks[k] = {size_t(other_blocks[2 * k]), size_t(other_blocks[2 * k + 1])};
    }
    Block_map map{block_count * 2};
    map = create_block_map(block_count, std::move(map), blocks.data(), pairs.data());
    Neighborhood_vectors nb;
    nb.resize(n);
    create_regular_neighborhoods(n, max_distance, nb.counts.data(), nb.indices.data(),
                                 nb.distances.data(), nb.vectors_to.data(), p.data(), gc.data(),
                                 same ? p.data() : o.data(), pairs.data(), map);
    for (size_t i = 0; i < n; ++i) {
        counts[i] = nb.counts[i];
        for (size_t k = 0; k < nb.counts[i]; ++k) {
            size_t const e = i * NEIGHBORHOOD_MAX_COUNT + k;
            idx[e] = nb.indices[i][k];
            dist[e] = nb.distances[i][k];
            vec[2 * e] = nb.vectors_to[i][k][0];
            vec[2 * e + 1] = nb.vectors_to[i][k][1];
        }
    }
}

void ref_common_distances_vectors(size_t n, size_t n_other, float* dist, float* vec,
                                  float const* self_xy, float const* other_xy,
                                  uint8_t const* counts, uint64_t const* idx) {
    auto const p = to_v2f(self_xy, n);
    auto const o = to_v2f(other_xy, n_other);
    auto nb = nbhd_from(n, counts, idx, nullptr, nullptr, nullptr, nullptr);
    compute_neighbor_distances_and_vectors_to(n, nb.distances.data(), nb.vectors_to.data(),
                                              p.data(), o.data(), nb.counts.data(),
                                              nb.indices.data());
    for (size_t i = 0; i < n; ++i) {
        for (size_t k = 0; k < NEIGHBORHOOD_MAX_COUNT; ++k) {
            size_t const e = i * NEIGHBORHOOD_MAX_COUNT + k;
            dist[e] = nb.distances[i][k];
            vec[2 * e] = nb.vectors_to[i][k][0];
            vec[2 * e + 1] = nb.vectors_to[i][k][1];
        }
    }
}

void ref_common_kernels(size_t n, float support, float* w, float* gw, uint8_t const* counts,
                        float const* dist, float const* vec) {
    auto nb = nbhd_from(n, counts, nullptr, dist, vec, nullptr, nullptr);
    compute_neighbor_kernels(n, support, nb.kernels.data(), nb.counts.data(), nb.distances.data());
    compute_neighbor_kernel_gradients(n, support, nb.kernel_gradients.data(), nb.counts.data(),
                                      nb.vectors_to.data());
    for (size_t i = 0; i < n; ++i) {
        for (size_t k = 0; k < NEIGHBORHOOD_MAX_COUNT; ++k) {
            size_t const e = i * NEIGHBORHOOD_MAX_COUNT + k;
            w[e] = nb.kernels[i][k];
            gw[2 * e] = nb.kernel_gradients[i][k][0];
            gw[2 * e + 1] = nb.kernel_gradients[i][k][1];
        }
    }
}

void ref_common_densities(size_t n, float support, float rho0, float* out, float const* fvol,
                          uint8_t const* fc, uint64_t const* fi, float const* fw,
                          float const* svol, uint8_t const* sc, uint64_t const* si,
                          float const* sw) {
    auto const f = nbhd_from(n, fc, fi, nullptr, nullptr, fw, nullptr);
    auto const s = nbhd_from(n, sc, si, nullptr, nullptr, sw, nullptr);
    compute_densities(n, support, rho0, out, fvol, f.pointers(), svol, s.pointers());
}

void ref_common_divergences(size_t n, float rho0, float* out, float const* fvol,
                            float const* fvel, uint8_t const* fc, uint64_t const* fi,
                            float const* fgw, float const* svol, float const* svel, size_t n_solid,
                            uint8_t const* sc, uint64_t const* si, float const* sgw) {
    auto const f = nbhd_from(n, fc, fi, nullptr, nullptr, nullptr, fgw);
    auto const s = nbhd_from(n, sc, si, nullptr, nullptr, nullptr, sgw);
    auto const fv = to_v2f(fvel, n);
    auto const sv = to_v2f(svel, n_solid);
    compute_divergences(n, rho0, out, fvol, fv.data(), f.pointers(), svol, sv.data(),
                        s.pointers());
}

void ref_common_density_stars(size_t n, float dt, float rho0, float* out, float const* rho,
                              float const* fvol, float const* fvel, uint8_t const* fc,
                              uint64_t const* fi, float const* fgw, float const* svol,
                              float const* svel, size_t n_solid, uint8_t const* sc,
                              uint64_t const* si, float const* sgw) {
    auto const f = nbhd_from(n, fc, fi, nullptr, nullptr, nullptr, fgw);
    auto const s = nbhd_from(n, sc, si, nullptr, nullptr, nullptr, sgw);
    auto const fv = to_v2f(fvel, n);
    auto const sv = to_v2f(svel, n_solid);
    predict_density_stars(n, dt, rho0, out, rho, fvol, fv.data(), f.pointers(), svol, sv.data(),
                          s.pointers());
}

void ref_common_apply_pressures(size_t n, float dt, float rho0, float* vel, float const* rho,
                                float const* p, float const* fvol, uint8_t const* fc,
                                uint64_t const* fi, float const* fgw, float const* svol,
                                uint8_t const* sc, uint64_t const* si, float const* sgw) {
    auto const f = nbhd_from(n, fc, fi, nullptr, nullptr, nullptr, fgw);
    auto const s = nbhd_from(n, sc, si, nullptr, nullptr, nullptr, sgw);
    auto v = to_v2f(vel, n);
    apply_pressures_in_place(n, dt, rho0, v.data(), rho, p, fvol, f.pointers(), svol,
                             s.pointers());
    copy_out(v, vel);
}

void ref_common_pressure_accelerations(size_t n, float rho0, float* acc, float const* p,
                                       float const* rho, float const* fvol, uint8_t const* fc,
                                       uint64_t const* fi, float const* fgw, float const* svol,
                                       uint8_t const* sc, uint64_t const* si, float const* sgw) {
    auto const f = nbhd_from(n, fc, fi, nullptr, nullptr, nullptr, fgw);
    auto const s = nbhd_from(n, sc, si, nullptr, nullptr, nullptr, sgw);
    std::vector<V2f> a(n);
    compute_pressure_accelerations(n, rho0, a.data(), p, rho, fvol, f.pointers(), svol,
                                   s.pointers());
    copy_out(a, acc);
}

void ref_common_integrate(size_t n, float dt, float rho0, float* vel_forces, float* vel_acc,
                          float* pos, float const* vol, float const* forces, float const* acc,
                          float const* vel_for_pos) {
    auto vf = to_v2f(vel_forces, n);
    auto const f = to_v2f(forces, n);
    integrate_velocities_in_place(n, dt, rho0, vf.data(), vol, f.data());
    copy_out(vf, vel_forces);
    auto va = to_v2f(vel_acc, n);
    auto const a = to_v2f(acc, n);
    integrate_velocities_in_place(n, dt, va.data(), a.data());
    copy_out(va, vel_acc);
    auto x = to_v2f(pos, n);
    auto const v = to_v2f(vel_for_pos, n);
    integrate_positions_in_place(n, dt, x.data(), v.data());
    copy_out(x, pos);
}

void ref_common_constant_volumes(size_t n, float rho0, float mass, float* vol) {
    compute_constant_volumes(n, rho0, mass, vol);
}

void ref_common_average_and_max(size_t n, float discretization, float const* values,
                                float* out) {
    auto const r = compute_scalar_average_and_max(n, discretization, values);
    out[0] = r.first;
    out[1] = r.second;
}

}  // extern "C"

//------------------------------------------------------------------------------
// The reference's solver operator functions (emerald/sph2d_box/*_ops.cpp) on
// flat host arrays. A neighbour set arrives as six pointers in the layout of
// Neighborhood_pointers, row-major with 64-bit indices; V2f arrays are
// interleaved floats. The iteration functions' (average, max) pairs are
// written to out[0], out[1].

namespace {

struct ref_nb {
    uint8_t const* counts;
    uint64_t const* indices;
    float const* distances;
    float const* vectors_to;
    float const* kernels;
    float const* kernel_gradients;
};

Neighborhood_vectors nb_of(size_t n, ref_nb const* p) {
    return nbhd_from(n, p->counts, p->indices, p->distances, p->vectors_to, p->kernels,
                     p->kernel_gradients);
}

}  // namespace

extern "C" {

void ref_ops_iisph_diis(size_t n, float dt, float rho0, float* diis, float const* rho,
                        float const* fvol, ref_nb const* f, float const* svol, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    std::vector<V2f> d(n);
    iisph_compute_diis(n, dt, rho0, d.data(), rho, fvol, F.pointers(), svol, S.pointers());
    copy_out(d, diis);
}

void ref_ops_iisph_aiis_stars(size_t n, float dt, float rho0, float* aiis, float* stars,
                              float const* diis, float const* rho, float const* fvol,
                              float const* fvel, ref_nb const* f, float const* svol,
                              float const* svel, size_t n_solid, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto const d = to_v2f(diis, n);
    auto const fv = to_v2f(fvel, n);
    auto const sv = to_v2f(svel, n_solid);
    iisph_compute_aiis_and_density_stars(n, dt, rho0, aiis, stars, d.data(), rho, fvol, fv.data(),
                                         F.pointers(), svol, sv.data(), S.pointers());
}

void ref_ops_iisph_sum_dij_pjs(size_t n, float dt, float rho0, float* out, float const* vol,
                               float const* rho, float const* p, ref_nb const* nb) {
    auto const N = nb_of(n, nb);
    std::vector<V2f> o(n);
    iisph_compute_sum_dij_pjs(n, dt, rho0, o.data(), vol, rho, p, N.pointers());
    copy_out(o, out);
}

void ref_ops_iisph_betas(size_t n, float dt, float rho0, float* betas, float const* rho,
                         float const* p, float const* diis, float const* sdp, float const* fvol,
                         ref_nb const* f, float const* svol, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto const d = to_v2f(diis, n);
    auto const sd = to_v2f(sdp, n);
    iisph_compute_betas(n, dt, rho0, betas, rho, p, d.data(), sd.data(), fvol, F.pointers(), svol,
                        S.pointers());
}

void ref_ops_iisph_new_pressures(size_t n, float omega, float rho0, float* io,
                                 float const* old_p, float const* alphas, float const* stars,
                                 float* out) {
    auto const r = iisph_compute_new_pressures(n, omega, rho0, io, old_p, alphas, stars);
    out[0] = r.first;
    out[1] = r.second;
}

void ref_ops_dfsph_shared_coeffs(size_t n, float rho0, float* out, float const* rho,
                                 float const* fvol, ref_nb const* f, float const* svol,
                                 ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    dfsph_p_compute_shared_coeffs(n, rho0, out, rho, fvol, F.pointers(), svol, S.pointers());
}

void ref_ops_dfsph_pseudo_pressures(size_t n, float dt, float rho0, float* density_pp,
                                    float* divergence_pp, float const* stars, float const* div,
                                    float const* coeffs) {
    dfsph_p_compute_density_pseudo_pressures(n, dt, rho0, density_pp, stars, coeffs);
    dfsph_p_compute_divergence_pseudo_pressures(n, dt, rho0, divergence_pp, div, coeffs);
}

void ref_ops_pcisph_densities(size_t n, float mass, float support, float rho0, float* rho,
                              ref_nb const* f, float const* svol, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    pcisph_compute_densities(n, mass, support, rho, F.counts.data(), F.kernels.data());
    pcisph_accumulate_density_from_solids(n, rho0, rho, svol, S.counts.data(), S.indices.data(),
                                          S.kernels.data());
}

void ref_ops_pcisph_update_pressures(size_t n, float rho0, float denom, float* p,
                                     float const* rho) {
    pcisph_update_pressures(n, rho0, denom, p, rho);
}

void ref_ops_pcisph_forces(size_t n, float mass, float support, float viscosity, float rho0,
                           float* forces, ref_nb const* f, float const* vel, float const* p,
                           float const* rho, float const* svol, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto fo = to_v2f(forces, n);
    auto const v = to_v2f(vel, n);
    pcisph_accumulate_pressure_forces(n, mass, support, viscosity, fo.data(), F.counts.data(),
                                      F.indices.data(), F.distances.data(), F.vectors_to.data(),
                                      F.kernel_gradients.data(), v.data(), p, rho);
    pcisph_accumulate_pressure_forces_from_solids(n, mass, rho0, fo.data(), svol, S.counts.data(),
                                                  S.indices.data(), S.kernel_gradients.data(), p,
                                                  rho);
    copy_out(fo, forces);
}

void ref_ops_ap_stars_diagonals(int pseudo, size_t n, float dt, float rho0, float* stars,
                                float* diag, float const* rho, float const* fvol,
                                float const* fvel, ref_nb const* f, float const* svol,
                                float const* svel, size_t n_solid, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto const fv = to_v2f(fvel, n);
    auto const sv = to_v2f(svel, n_solid);
    if (pseudo) {
        iisph_pseudo_ap_density_stars_and_pseudo_diagonals(n, dt, rho0, stars, diag, rho, fvol,
                                                           fv.data(), F.pointers(), svol,
                                                           sv.data(), S.pointers());
    } else {
        iisph_ap_density_stars_and_diagonals(n, dt, rho0, stars, diag, rho, fvol, fv.data(),
                                             F.pointers(), svol, sv.data(), S.pointers());
    }
}

void ref_ops_ap_iterate(size_t n, float dt, float rho0, float omega, float* p,
                        float const* stars, float const* acc, float const* diag,
                        float const* fvol, ref_nb const* f, float const* svol, ref_nb const* s,
                        float* out) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto const a = to_v2f(acc, n);
    auto const r = iisph_ap_iterate_pressures_in_place(n, dt, rho0, omega, p, stars, a.data(),
                                                       diag, fvol, F.pointers(), svol,
                                                       S.pointers());
    out[0] = r.first;
    out[1] = r.second;
}

void ref_ops_pseudo_displacements(size_t n, float rho0, float* out, float const* pp,
                                  float const* rho, float const* fvol, ref_nb const* f,
                                  float const* svol, ref_nb const* s) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    std::vector<V2f> d(n);
    iisph_pseudo_ap_compute_pseudo_pressure_displacements(n, rho0, d.data(), pp, rho, fvol,
                                                          F.pointers(), svol, S.pointers());
    copy_out(d, out);
}

void ref_ops_pseudo_iterate(size_t n, float rho0, float omega, float* pp, float const* stars,
                            float const* disp, float const* diag, float const* fvol,
                            ref_nb const* f, float const* svol, ref_nb const* s, float* out) {
    auto const F = nb_of(n, f);
    auto const S = nb_of(n, s);
    auto const d = to_v2f(disp, n);
    auto const r = iisph_pseudo_ap_iterate_pseudo_pressures_in_place(
      n, rho0, omega, pp, stars, d.data(), diag, fvol, F.pointers(), svol, S.pointers());
    out[0] = r.first;
    out[1] = r.second;
}

void ref_ops_pseudo_integrate(size_t n, float dt, float* vel, float* pos, float const* disp) {
    auto v = to_v2f(vel, n);
    auto x = to_v2f(pos, n);
    auto const d = to_v2f(disp, n);
    iisph_pseudo_ap_integrate_velocities_and_positions_in_place(n, dt, v.data(), x.data(),
                                                                d.data());
    copy_out(v, vel);
    copy_out(x, pos);
}

}  // extern "C"
