// A caller written against the reference's sph2d_box step API, compiled
// against include/emerald_sph.hpp instead. The types below carry the
// reference's member names (emerald/sph2d_box/state.h:13-33,
// parameters.h:12-41, config.h:7-18, colors.h:13-21, forces.h:13-21); the
// step calls are spelled exactly as in EZ_EXAMPLE_SIM::step
// (emerald/sph2d_box/simulation.cpp:41-93).
//
//   step_dropin <method 0-4> <frames> <out.bin> [wall speed] [forces]
//
// Runs the reference's default dam break (world_walls + dam_break scenes)
// and writes positions, velocities and colours after the last frame. With a
// non-zero wall speed (m/s), the caller moves the boundary particles left of
// x = 0 along x before every frame (frame f, from 1, at f * speed * 2 ms)
// and gives them that velocity, as a caller of the reference moves a wall:
// by passing a changed Solid_state to the next step call. forces:
// "gravity" (default_gravity_forces, the default), "host" (a capturing
// lambda that adds gravity and a pole attraction with the reference's
// accumulate functions, called on the host) or "device" (the same two terms
// as Device_forces, run on the device).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <string>
#include <vector>

#include "emerald_sph.hpp"

namespace ref {
struct V2f {
    float x, y;
};
struct C4f {
    float r, g, b, a;
};
using flicks = std::chrono::duration<int64_t, std::ratio<1, 705600000>>;
struct Parameters {
    uint64_t seed = 1;
    flicks time_per_step{0};
    int sub_steps = 30;
    float length = 1.0f, support = 0.025f, gravity = 9.81f, viscosity = 0.01f;
    float target_density = 1000.0f;
    struct {
        int max_pressure_iterations;
        float error_average_threshold, error_max_threshold, omega;
    } iisph{};
    struct {
        int max_correction_iterations;
        float density_error_average_threshold, density_error_max_threshold;
        float divergence_error_average_threshold, divergence_error_max_threshold;
    } dfsph{};
};
struct Simulation_config {
    Parameters params;
    float seconds_per_sub_step = 1.0f, mass_per_particle = 1.0f, draw_radius = 1.0f;
    float pressure_correction_denom = 1.0f;
};
struct State {
    std::vector<V2f> positions, velocities;
    std::vector<C4f> colors;
};
struct Solid_state {
    std::vector<V2f> positions, velocities;
    std::vector<C4f> colors;
    std::vector<float> volumes;
};
struct Temp_data {};
using User_forces_function = std::function<void(size_t, float, float, float, float, V2f*,
                                                V2f const*, V2f const*)>;
using User_colors_function = std::function<void(size_t, float, float, float, C4f*, V2f const*,
                                                V2f const*, float const*)>;
}  // namespace ref

using namespace emerald_b200::sph2d_box;

int main(int argc, char** argv) {
    if (argc < 4 || argc > 6) return 2;
    int const method = std::atoi(argv[1]);
    int const frames = std::atoi(argv[2]);
    float const speed = argc >= 5 ? float(std::atof(argv[4])) : 0.0f;
    bool const moving = speed != 0.0f;
    std::string const force_mode = argc == 6 ? argv[5] : "gravity";
    emerald_params p{};
    emerald_b200::check(emerald_default_params(&p), "defaults");
    float cfg[4];
    emerald_b200::check(emerald_config(&p, cfg), "config");

    ref::Simulation_config config;
    config.params.seed = p.seed;
    config.params.time_per_step = ref::flicks(p.time_per_step_flicks);
    config.params.sub_steps = p.sub_steps;
    config.params.length = p.length;
    config.params.support = p.support;
    config.params.gravity = p.gravity;
    config.params.viscosity = p.viscosity;
    config.params.target_density = p.target_density;
    config.params.iisph = {p.iisph_max_pressure_iterations, p.iisph_error_average_threshold,
                           p.iisph_error_max_threshold, p.iisph_omega};
    config.params.dfsph = {p.dfsph_max_correction_iterations,
                           p.dfsph_density_error_average_threshold,
                           p.dfsph_density_error_max_threshold,
                           p.dfsph_divergence_error_average_threshold,
                           p.dfsph_divergence_error_max_threshold};
    config.seconds_per_sub_step = cfg[0];
    config.mass_per_particle = cfg[1];
    config.draw_radius = cfg[2];
    config.pressure_correction_denom = cfg[3];

    ref::Solid_state solid_state;
    solid_state.positions.resize(emerald_world_walls(&p, nullptr));
    emerald_world_walls(&p, reinterpret_cast<float*>(solid_state.positions.data()));
    solid_state.velocities.assign(solid_state.positions.size(), {0.0f, 0.0f});
    ref::State state;
    size_t const n = emerald_dam_break(&p, reinterpret_cast<float const*>(solid_state.positions.data()),
                                       solid_state.positions.size(), nullptr);
    state.positions.resize(n);
    emerald_dam_break(&p, reinterpret_cast<float const*>(solid_state.positions.data()),
                      solid_state.positions.size(), reinterpret_cast<float*>(state.positions.data()));
    state.velocities.assign(n, {0.0f, 0.0f});

    ref::Temp_data temp_data;
    // The pole pull of the reference's commented-out example
    // (emerald/sph2d_box/forces.cpp:24-28): a quarter of gravity towards the
    // tank's centre.
    float const g = config.params.gravity;
    float const pole_magnitude = 0.25f * g * config.mass_per_particle;
    ref::User_forces_function user_forces = default_gravity_forces(g);
    if (force_mode == "host") {
        user_forces = [g, pole_magnitude](size_t count, float, float, float mass, float,
                                          ref::V2f* forces, ref::V2f const* positions,
                                          ref::V2f const*) {
            accumulate_gravity_forces(count, mass, g, forces);
            accumulate_constant_pole_attraction_forces(count, pole_magnitude, ref::V2f{0.5f, 0.5f},
                                                       forces, positions);
        };
    } else if (force_mode == "device") {
        user_forces = Device_forces{{EMERALD_FORCE_GRAVITY, g, 0.0f, 0.0f},
                                    {EMERALD_FORCE_POLE, pole_magnitude, 0.5f, 0.5f}};
    } else if (force_mode != "gravity") {
        return 2;
    }
    float const rho0 = config.params.target_density;
    ref::User_colors_function user_colors = [rho0](size_t count, float, float, float,
                                                   ref::C4f* colors, ref::V2f const*,
                                                   ref::V2f const*, float const* densities) {
        for (size_t i = 0; i < count; ++i) {
            float const norm_d = densities[i] / (1.1f * rho0);
            float c = 1.0f - norm_d;
            c = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
            colors[i] = {c, c, 1.0f, 1.0f};
        }
    };
    std::vector<ref::V2f> const walls0 = solid_state.positions;
    float const step = float(double(speed) * 0.002);
    ref::flicks time{0};
    try {
        for (int f = 0; f < frames; ++f) {
            if (moving) {
                for (size_t k = 0; k < walls0.size(); ++k) {
                    if (walls0[k].x < 0.0f) {
                        solid_state.positions[k].x = walls0[k].x + float(f + 1) * step;
                        solid_state.velocities[k] = {speed, 0.0f};
                    }
                }
            }
            switch (method) {
            case 0:
                state = pcisph_simulation_step(time, config, std::move(state), solid_state,
                                               temp_data, user_forces, user_colors);
                break;
            case 1:
                state = iisph_simulation_step(time, config, std::move(state), solid_state,
                                              temp_data, user_forces, user_colors);
                break;
            case 2:
                state = iisph_ap_simulation_step(time, config, std::move(state), solid_state,
                                                 temp_data, user_forces, user_colors);
                break;
            case 3:
                state = iisph_pseudo_ap_simulation_step(time, config, std::move(state),
                                                        solid_state, temp_data, user_forces,
                                                        user_colors);
                break;
            default:
                state = dfsph_p_simulation_step(time, config, std::move(state), solid_state,
                                                temp_data, user_forces, user_colors);
                break;
            }
            time += config.params.time_per_step;
        }
    } catch (emerald_b200::Error const& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    emerald_b200::release(temp_data);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 3;
    uint64_t const count = n;
    std::fwrite(&count, 8, 1, f);
    std::fwrite(state.positions.data(), 8, n, f);
    std::fwrite(state.velocities.data(), 8, n, f);
    std::fwrite(state.colors.data(), 16, n, f);
    std::fclose(f);
    return 0;
}
