// C++ drop-in for the reference's step functions over the C ABI.
//
// emerald/sph2d_box declares, per solver (e.g. emerald/sph2d_box/iisph.h),
//
//     State iisph_simulation_step(flicks global_time, Simulation_config const& config,
//                                 State&& state, Solid_state const& solid_state,
//                                 Temp_data& temp, User_forces_function const& user_forces,
//                                 User_colors_function const& user_colors);
//
// and EZ_EXAMPLE_SIM::step (emerald/sph2d_box/simulation.cpp:41-93) calls one of
// them per frame. The templates below take the caller's own types with the
// same argument list, so that code written against the reference compiles
// unchanged after `using namespace emerald_b200::sph2d_box;`:
//
//   * State / Solid_state: anything with `positions` and `velocities`
//     (std::vector of a two-float vector type such as Imath::V2f) and, for
//     State, `colors` (a vector of a four-float colour type);
//   * Simulation_config: anything with `params` (the reference's Parameters
//     member names) and `mass_per_particle`, `pressure_correction_denom`,
//     `draw_radius`;
//   * Temp_data: any object; its address keys the device simulation that
//     stands for it (release it with emerald_b200::release(temp) before the
//     object goes away);
//   * flicks: anything with `.count()` (std::chrono::duration) or an integer.
//
// Each call uploads the state, passes on a boundary whose positions or
// velocities differ from the previous call's (a moving wall: the reference
// takes the Solid_state anew on every call), runs one frame on the GPU,
// downloads the new state and, unless user_colors is empty, calls it on the
// host with the
// frame's densities, as compute_colors does (emerald/sph2d_box/colors.cpp:22-38).
//
// user_forces (emerald/sph2d_box/forces.h:13-21) is honoured as the
// reference honours it, once per sub-step at the solver's force point:
//   * default_gravity_forces(g) and Device_forces{...} from this header
//     (the std::function holds them, found with target<>()) become force
//     terms evaluated on the device inside the sub-step;
//   * any other callable is called on the host with the state of that
//     point of the sub-step (emerald_sim_set_force_callback; the sub-steps
//     then run without graphs);
//   * an empty function throws std::bad_function_call, as calling it in the
//     reference does.
// accumulate_gravity_forces, accumulate_constant_pole_attraction_forces and
// accumulate_simple_drag_forces (emerald/sph2d_box/forces.cpp:63-111) are
// provided for host force functions written against the reference.
#pragma once

#include <algorithm>
#include <cstdint>
#include <functional>
#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <cmath>
#include <limits>
#include <type_traits>
#include <utility>
#include <vector>

#include "emerald_sph.h"

namespace emerald_b200 {

class Error : public std::runtime_error {
public:
    Error(int code, std::string const& what)
      : std::runtime_error(what + " (" + std::to_string(code) + "): " + emerald_last_error()),
        code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, char const* what) {
    if (rc != EMERALD_OK) throw Error(rc, what);
}

namespace sph2d_box {

// The reference's force functions (emerald/sph2d_box/forces.cpp:63-111) for
// host force functions, on any two-float vector type with x and y members,
// with the reference's arithmetic (Imath 2.x Vec2 operations).
template <class V>
void accumulate_gravity_forces(size_t const count, float const mass_per_particle,
                               float const gravity, V* const forces) {
    for (size_t i = 0; i < count; ++i) forces[i].y -= mass_per_particle * gravity;
}

template <class V>
void accumulate_constant_pole_attraction_forces(size_t const count, float const magnitude,
                                                V const pole, V* const forces,
                                                V const* const positions) {
    for (size_t i = 0; i < count; ++i) {
        float const rx = positions[i].x - pole.x;
        float const ry = positions[i].y - pole.y;
        // Imath Vec2::length with its tiny-length rescale, then normalized()
        float len;
        float const l2 = rx * rx + ry * ry;
        if (l2 < 2.0f * std::numeric_limits<float>::min()) {
            float ax = rx >= 0.0f ? rx : -rx;
            float ay = ry >= 0.0f ? ry : -ry;
            float m = ax;
            if (m < ay) m = ay;
            if (m == 0.0f) {
                len = 0.0f;
            } else {
                ax /= m;
                ay /= m;
                len = m * std::sqrt(ax * ax + ay * ay);
            }
        } else {
            len = std::sqrt(l2);
        }
        float const nx = len == 0.0f ? 0.0f : rx / len;
        float const ny = len == 0.0f ? 0.0f : ry / len;
        forces[i].x -= magnitude * nx;
        forces[i].y -= magnitude * ny;
        // (0, 0, magnitude / 8) x (nx, ny, 0)
        float const tz = 0.125f * magnitude;
        float const zero = 0.0f;
        forces[i].x += zero * zero - tz * ny;
        forces[i].y += tz * nx - zero * zero;
    }
}

template <class V>
void accumulate_simple_drag_forces(size_t const count, float const magnitude,
                                   float const particle_diameter, V* const forces,
                                   V const* const velocities) {
    float const m = -magnitude * particle_diameter;
    for (size_t i = 0; i < count; ++i) {
        forces[i].x += m * velocities[i].x;
        forces[i].y += m * velocities[i].y;
    }
}

// default_gravity_forces (emerald/sph2d_box/forces.cpp:73-83) as a functor
// the step functions recognise and run on the device.
struct Gravity_forces {
    float gravity;
    template <class V>
    void operator()(size_t const count, float, float, float const mass_per_particle, float,
                    V* const forces, V const* const, V const* const) const {
        accumulate_gravity_forces(count, mass_per_particle, gravity, forces);
    }
};

inline Gravity_forces default_gravity_forces(float const gravity) { return Gravity_forces{gravity}; }

// Up to EMERALD_MAX_FORCE_TERMS device force terms (emerald_force_term) as a
// User_forces_function: the step functions run them on the device; called
// on the host it computes the same forces.
struct Device_forces {
    std::vector<emerald_force_term> terms;
    Device_forces(std::initializer_list<emerald_force_term> t) : terms(t) {}
    template <class V>
    void operator()(size_t const count, float, float, float const mass_per_particle, float,
                    V* const forces, V const* const positions, V const* const velocities) const {
        for (auto const& t : terms) {
            if (t.kind == EMERALD_FORCE_GRAVITY) {
                accumulate_gravity_forces(count, mass_per_particle, t.a, forces);
            } else if (t.kind == EMERALD_FORCE_POLE) {
                V pole;
                pole.x = t.b;
                pole.y = t.c;
                accumulate_constant_pole_attraction_forces(count, t.a, pole, forces, positions);
            } else if (t.kind == EMERALD_FORCE_DRAG) {
                accumulate_simple_drag_forces(count, t.a, t.b, forces, velocities);
            }
        }
    }
};

}  // namespace sph2d_box

namespace detail {

template <class T, class = void>
struct has_volumes : std::false_type {};
template <class T>
struct has_volumes<T, std::void_t<decltype(std::declval<T const&>().volumes)>>
  : std::is_same<typename std::decay<decltype(std::declval<T const&>().volumes)>::type,
                 std::vector<float>> {};

template <class T, class = void>
struct has_velocities : std::false_type {};
template <class T>
struct has_velocities<T, std::void_t<decltype(std::declval<T const&>().velocities)>>
  : std::true_type {};

template <class V>
float const* floats(std::vector<V> const& v) {
    static_assert(sizeof(V) == 2 * sizeof(float) && std::is_standard_layout<V>::value,
                  "positions and velocities must be vectors of two packed floats");
    return reinterpret_cast<float const*>(v.data());
}

template <class V>
float* floats(std::vector<V>& v) {
    static_assert(sizeof(V) == 2 * sizeof(float) && std::is_standard_layout<V>::value,
                  "positions and velocities must be vectors of two packed floats");
    return reinterpret_cast<float*>(v.data());
}

template <class T>
auto ticks(T const& t, int) -> decltype(int64_t(t.count())) {
    return int64_t(t.count());
}
template <class T>
int64_t ticks(T const& t, long) {
    return int64_t(t);
}

// An empty std::function (or a null function pointer, or nullptr): the
// only callables that can be empty. Lambdas and functors never are.
template <class F>
auto is_empty(F const& f, int) -> decltype(!bool(f)) {
    return !bool(f);
}
template <class F>
bool is_empty(F const&, long) {
    return false;
}

// Parameters + Simulation_config (emerald/sph2d_box/parameters.h:12-41,
// emerald/sph2d_box/config.h:7-18) to emerald_params.
template <class Config>
emerald_params to_params(Config const& config) {
    emerald_params p{};
    check(emerald_default_params(&p), "emerald_default_params");
    auto const& in = config.params;
    p.seed = uint64_t(in.seed);
    p.time_per_step_flicks = ticks(in.time_per_step, 0);
    p.sub_steps = int32_t(in.sub_steps);
    p.length = float(in.length);
    p.support = float(in.support);
    p.gravity = float(in.gravity);
    p.viscosity = float(in.viscosity);
    p.target_density = float(in.target_density);
    p.iisph_max_pressure_iterations = int32_t(in.iisph.max_pressure_iterations);
    p.iisph_error_average_threshold = float(in.iisph.error_average_threshold);
    p.iisph_error_max_threshold = float(in.iisph.error_max_threshold);
    p.iisph_omega = float(in.iisph.omega);
    p.dfsph_max_correction_iterations = int32_t(in.dfsph.max_correction_iterations);
    p.dfsph_density_error_average_threshold = float(in.dfsph.density_error_average_threshold);
    p.dfsph_density_error_max_threshold = float(in.dfsph.density_error_max_threshold);
    p.dfsph_divergence_error_average_threshold = float(in.dfsph.divergence_error_average_threshold);
    p.dfsph_divergence_error_max_threshold = float(in.dfsph.divergence_error_max_threshold);
    p.mass_per_particle = float(config.mass_per_particle);
    p.pressure_correction_denom = float(config.pressure_correction_denom);
    return p;
}

// The device simulation standing for one Temp_data object.
struct Context {
    emerald_sim* sim = nullptr;
    size_t n_fluid = 0;
    int64_t time = 0;
    std::vector<float> densities;
    std::vector<float> solid_xy, solid_v;  // the boundary the device holds
    ~Context() {
        if (sim) emerald_sim_destroy(sim);
    }
};

inline std::map<void const*, std::unique_ptr<Context>>& registry() {
    static std::map<void const*, std::unique_ptr<Context>> r;
    return r;
}
inline std::mutex& registry_mutex() {
    static std::mutex m;
    return m;
}

template <class Config, class Solid_state>
Context& context(void const* key, Config const& config, Solid_state const& solid, size_t n_fluid,
                 float const* x, float const* v, int64_t time) {
    std::lock_guard<std::mutex> lock(registry_mutex());
    auto& slot = registry()[key];
    if (slot && slot->n_fluid == n_fluid) return *slot;
    slot.reset(new Context);
    emerald_params const p = to_params(config);
    float const* vols = nullptr;
    if constexpr (has_volumes<typename std::decay<Solid_state>::type>::value) {
        // the reference's compute_neighbor_data_and_volumes results, if filled
        if (solid.volumes.size() == solid.positions.size()) vols = solid.volumes.data();
    }
    check(emerald_sim_create(&p, floats(solid.positions), vols, solid.positions.size(), x, v,
                             n_fluid, &slot->sim),
          "emerald_sim_create");
    slot->n_fluid = n_fluid;
    slot->time = time;
    size_t const ns = solid.positions.size();
    slot->solid_xy.assign(floats(solid.positions), floats(solid.positions) + 2 * ns);
    slot->solid_v.assign(2 * ns, 0.0f);
    return *slot;
}

// Sends the caller's boundary to the device when its positions or
// velocities changed since the last call (same count; a different count
// needs a new simulation).
template <class Solid_state>
void sync_solid(Context& ctx, Solid_state const& solid) {
    size_t const ns = solid.positions.size();
    if (2 * ns != ctx.solid_xy.size()) {
        throw std::invalid_argument("the boundary particle count changed");
    }
    float const* xy = floats(solid.positions);
    bool const moved = ns && !std::equal(xy, xy + 2 * ns, ctx.solid_xy.begin());
    float const* v = nullptr;
    bool vchanged = false;
    if constexpr (has_velocities<typename std::decay<Solid_state>::type>::value) {
        if (solid.velocities.size() == ns && ns) {
            v = floats(solid.velocities);
            vchanged = !std::equal(v, v + 2 * ns, ctx.solid_v.begin());
        }
    }
    if (!moved && !vchanged) return;
    float const* vols = nullptr;
    if constexpr (has_volumes<typename std::decay<Solid_state>::type>::value) {
        if (moved && solid.volumes.size() == ns) vols = solid.volumes.data();
    }
    check(emerald_sim_set_solid(ctx.sim, moved ? xy : nullptr, vchanged ? v : nullptr, vols),
          "emerald_sim_set_solid");
    if (moved) std::copy(xy, xy + 2 * ns, ctx.solid_xy.begin());
    if (vchanged) std::copy(v, v + 2 * ns, ctx.solid_v.begin());
}

template <class T, class F>
auto held(F const& f, int) -> decltype(f.template target<T>()) {
    return f.template target<T>();
}
template <class T, class F>
T const* held(F const& f, long) {
    if constexpr (std::is_same<typename std::decay<F>::type, T>::value) {
        return &f;
    } else {
        return nullptr;
    }
}

// Calls the caller's force function with its own vector type.
template <class Forces, class V>
void call_forces(void* user, size_t count, float time, float dt, float mass, float radius,
                 float* forces, float const* positions, float const* velocities) {
    (*static_cast<Forces const*>(user))(count, time, dt, mass, radius,
                                        reinterpret_cast<V*>(forces),
                                        reinterpret_cast<V const*>(positions),
                                        reinterpret_cast<V const*>(velocities));
}

// Points the device simulation at the caller's forces for this call.
template <class V, class Forces>
void set_forces(Context& ctx, Forces const& user_forces) {
    using sph2d_box::Device_forces;
    using sph2d_box::Gravity_forces;
    if (Gravity_forces const* g = held<Gravity_forces>(user_forces, 0)) {
        emerald_force_term const t{EMERALD_FORCE_GRAVITY, g->gravity, 0.0f, 0.0f};
        check(emerald_sim_set_force_callback(ctx.sim, nullptr, nullptr), "force callback");
        check(emerald_sim_set_forces(ctx.sim, &t, 1), "emerald_sim_set_forces");
        return;
    }
    if (Device_forces const* d = held<Device_forces>(user_forces, 0)) {
        check(emerald_sim_set_force_callback(ctx.sim, nullptr, nullptr), "force callback");
        check(emerald_sim_set_forces(ctx.sim, d->terms.data(), int32_t(d->terms.size())),
              "emerald_sim_set_forces");
        return;
    }
    if (is_empty(user_forces, 0)) throw std::bad_function_call();
    check(emerald_sim_set_force_callback(
            ctx.sim, &call_forces<typename std::decay<Forces>::type, V>,
            const_cast<void*>(static_cast<void const*>(&user_forces))),
          "emerald_sim_set_force_callback");
}

template <class State, class Config, class Solid_state, class Forces, class Colors>
State step(int32_t method, int64_t global_time, Config const& config, State&& state,
           Solid_state const& solid, void const* temp_key, Forces const& user_forces,
           Colors const& user_colors) {
    size_t const n = state.positions.size();
    if (state.velocities.size() != n) {
        throw std::invalid_argument("positions and velocities differ in size");
    }
    Context& ctx = context(temp_key, config, solid, n, floats(state.positions),
                           floats(state.velocities), global_time);
    if (ctx.time != global_time) {
        throw std::invalid_argument("global_time does not continue the device simulation's clock");
    }
    sync_solid(ctx, solid);
    check(emerald_sim_set_state(ctx.sim, floats(state.positions), floats(state.velocities)),
          "emerald_sim_set_state");
    using V2 = typename std::decay<decltype(state.positions[0])>::type;
    set_forces<V2>(ctx, user_forces);
    emerald_step_stats stats{};
    int const rc = emerald_sim_frame(ctx.sim, method, &stats);
    // the callback points at user_forces, which lives only for this call
    emerald_sim_set_force_callback(ctx.sim, nullptr, nullptr);
    check(rc, "emerald_sim_frame");
    check(emerald_sim_get_state(ctx.sim, floats(state.positions), floats(state.velocities)),
          "emerald_sim_get_state");
    ctx.time += to_params(config).time_per_step_flicks;
    if (!is_empty(user_colors, 0)) {
        ctx.densities.resize(n);
        int32_t width = 0;
        check(emerald_sim_get_array(ctx.sim, "densities", ctx.densities.data(), &width),
              "emerald_sim_get_array");
        state.colors.resize(n);
        user_colors(n, float(double(global_time) / 705600000.0), config.mass_per_particle,
                    config.draw_radius, state.colors.data(), state.positions.data(),
                    state.velocities.data(), ctx.densities.data());
    }
    return std::move(state);
}

}  // namespace detail

// Destroys the device simulation that stands for `temp`.
template <class Temp>
void release(Temp const& temp) {
    std::lock_guard<std::mutex> lock(detail::registry_mutex());
    detail::registry().erase(static_cast<void const*>(&temp));
}

namespace sph2d_box {

#define EMERALD_B200_STEP(name, method)                                                        \
    template <class Flicks, class Config, class State, class Solid_state, class Temp,          \
              class Forces, class Colors>                                                      \
    typename std::decay<State>::type name(Flicks const global_time, Config const& config,      \
                                          State&& state, Solid_state const& solid_state,       \
                                          Temp& temp, Forces const& user_forces,               \
                                          Colors const& user_colors) {                         \
        return detail::step(method, detail::ticks(global_time, 0), config,                     \
                            std::forward<State>(state), solid_state,                           \
                            static_cast<void const*>(&temp), user_forces, user_colors);        \
    }

// emerald/sph2d_box/pcisph.cpp:166-204
EMERALD_B200_STEP(pcisph_simulation_step, EMERALD_PCISPH)
// emerald/sph2d_box/iisph.cpp:168-188
EMERALD_B200_STEP(iisph_simulation_step, EMERALD_IISPH)
// emerald/sph2d_box/iisph_ap.cpp
EMERALD_B200_STEP(iisph_ap_simulation_step, EMERALD_IISPH_AP)
// emerald/sph2d_box/iisph_pseudo_ap.cpp
EMERALD_B200_STEP(iisph_pseudo_ap_simulation_step, EMERALD_IISPH_PSEUDO_AP)
// emerald/sph2d_box/dfsph_p.cpp:376-396
EMERALD_B200_STEP(dfsph_p_simulation_step, EMERALD_DFSPH_P)

#undef EMERALD_B200_STEP

}  // namespace sph2d_box

}  // namespace emerald_b200
