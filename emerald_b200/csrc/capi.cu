// extern "C" entry points of include/emerald_sph.h over the Engine.
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/emerald_sph.h"
#include "engine.hpp"
#include "kernels.cuh"
#include "server.hpp"

namespace emerald {
void lattice_config(emerald_params const& p, float dx, float dt, float& mass, float& denom);
size_t block_scene(uint32_t nx, uint32_t ny, float dx, float x0, float y0, float jitter,
                   uint64_t seed, float* xy);
size_t wall_scene(float dx, float length, int layers, float* xy);
std::vector<float2> world_walls(emerald_params const& p);
std::vector<float2> dam_break(emerald_params const& p, float2 const* solid, size_t n_solid);
}  // namespace emerald

using namespace emerald;

struct emerald_batch {
    Engine engine;
    emerald_batch(uint32_t n, uint32_t ns, int scenes) : engine(n, ns, scenes) {}
};

struct emerald_server {
    Server server;
    explicit emerald_server(emerald_server_config const& c) : server(c) {}
};

struct emerald_sim {
    Engine engine;
    int scene;
    emerald_params params;
    emerald_sim(uint32_t n, uint32_t ns) : engine(n, ns, 1), scene(-1), params{} {}
};

namespace {

thread_local std::string t_error;

int fail(int code, std::string const& msg) {
    t_error = msg;
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (std::bad_alloc const&) {
        return fail(EMERALD_ENOMEM, "device or host allocation failed");
    } catch (std::exception const& e) {
        return fail(EMERALD_ECUDA, e.what());
    }
}

bool valid_method(int32_t m) { return m >= 0 && m <= 4; }

// An infinity or a NaN among n host floats (the reference would carry it
// into every neighbour sum; emerald/util/assert.h has no check for it).
int check_finite(float const* p, size_t n, char const* what) {
    if (!p) return EMERALD_OK;
    for (size_t k = 0; k < n; ++k) {
        if (!std::isfinite(p[k])) {
            return fail(EMERALD_EINVAL, std::string(what) + " holds a non-finite value at float " +
                                          std::to_string(k));
        }
    }
    return EMERALD_OK;
}

int check_particles(float const* fluid_xy, float const* fluid_v, size_t n_fluid,
                    float const* solid_xy, float const* solid_volumes, size_t n_solid) {
    if (int rc = check_finite(fluid_xy, 2 * n_fluid, "fluid positions")) return rc;
    if (int rc = check_finite(fluid_v, 2 * n_fluid, "fluid velocities")) return rc;
    if (int rc = check_finite(solid_xy, 2 * n_solid, "boundary positions")) return rc;
    return check_finite(solid_volumes, n_solid, "boundary volumes");
}

int check_forces(emerald_force_term const* terms, int32_t count) {
    if (count < 0 || count > EMERALD_MAX_FORCE_TERMS) {
        return fail(EMERALD_EINVAL, "between 0 and EMERALD_MAX_FORCE_TERMS force terms");
    }
    if (count && !terms) return fail(EMERALD_EINVAL, "terms is NULL");
    for (int32_t k = 0; k < count; ++k) {
        emerald_force_term const& t = terms[k];
        if (t.kind != EMERALD_FORCE_GRAVITY && t.kind != EMERALD_FORCE_POLE &&
            t.kind != EMERALD_FORCE_DRAG) {
            return fail(EMERALD_EINVAL, "unknown force term kind");
        }
        if (!std::isfinite(t.a) || !std::isfinite(t.b) || !std::isfinite(t.c)) {
            return fail(EMERALD_EINVAL, "force term arguments must be finite");
        }
    }
    return EMERALD_OK;
}

std::vector<ForceTerm> to_terms(emerald_force_term const* terms, int32_t count) {
    std::vector<ForceTerm> out(size_t(count) + 1);
    for (int32_t k = 0; k < count; ++k) {
        out[k] = ForceTerm{terms[k].kind, terms[k].a, terms[k].b, terms[k].c};
    }
    return out;
}

int check_params(emerald_params const* p) {
    if (!p) return fail(EMERALD_EINVAL, "params is NULL");
    if (!(p->support > 0.0f)) return fail(EMERALD_EINVAL, "support must be positive");
    if (!(p->target_density > 0.0f)) return fail(EMERALD_EINVAL, "target_density must be positive");
    if (p->time_per_step_flicks <= 0) return fail(EMERALD_EINVAL, "time_per_step must be positive");
    if (p->sub_steps <= 0) return fail(EMERALD_EINVAL, "sub_steps must be positive");
    if (p->precision != EMERALD_PRECISION_REFERENCE && p->precision != EMERALD_PRECISION_COMPENSATED) {
        return fail(EMERALD_EINVAL, "unknown precision mode");
    }
    float const values[] = {p->length, p->gravity, p->viscosity, p->iisph_error_average_threshold,
                            p->iisph_error_max_threshold, p->iisph_omega,
                            p->dfsph_density_error_average_threshold,
                            p->dfsph_density_error_max_threshold,
                            p->dfsph_divergence_error_average_threshold,
                            p->dfsph_divergence_error_max_threshold, p->mass_per_particle,
                            p->pressure_correction_denom, p->support, p->target_density};
    for (float const v : values) {
        if (!std::isfinite(v)) return fail(EMERALD_EINVAL, "a parameter is not finite");
    }
    return EMERALD_OK;
}

void fill_stats(SceneState const& s, emerald_step_stats* out, int substeps) {
    if (!out) return;
    out->sub_steps = substeps;
    out->pressure_iterations = s.stat_iters;
    out->error_average = s.stat_avg;
    out->error_max = s.stat_max;
    out->divergence_iterations = s.stat_div_iters;
    out->divergence_error_average = s.stat_div_avg;
    out->divergence_error_max = s.stat_div_max;
    out->dt = s.dt;
    out->time_seconds = double(s.frame_time + s.elapsed) / 705600000.0;
    out->error_flags = s.error;
    out->error_average_exact = s.stat_avg_exact;
    out->divergence_error_average_exact = s.stat_div_avg_exact;
}

}  // namespace

namespace emerald {
int set_last_error(int code, char const* msg) { return fail(code, msg); }
}  // namespace emerald

extern "C" {

char const* emerald_last_error(void) { return t_error.c_str(); }

int64_t emerald_kernel_launches(void) { return kernel_launch_count(); }

int emerald_default_params(emerald_params* out) {
    if (!out) return fail(EMERALD_EINVAL, "out is NULL");
    default_params(*out);
    return EMERALD_OK;
}

int emerald_config(emerald_params const* params, float* out) {
    if (int rc = check_params(params)) return rc;
    if (!out) return fail(EMERALD_EINVAL, "out is NULL");
    DerivedConfig const c = derive_config(*params);
    out[0] = c.seconds_per_sub_step;
    out[1] = c.mass_per_particle;
    out[2] = c.draw_radius;
    out[3] = c.pressure_correction_denom;
    return EMERALD_OK;
}

int emerald_lattice_config(emerald_params const* params, float dx, float dt, float* out) {
    if (int rc = check_params(params)) return rc;
    if (!out || !(dx > 0.0f)) return fail(EMERALD_EINVAL, "bad lattice arguments");
    lattice_config(*params, dx, dt, out[0], out[1]);
    return EMERALD_OK;
}

uint64_t emerald_z_index(uint32_t x, uint32_t y) { return morton2(x, y); }

size_t emerald_block_scene(uint32_t nx, uint32_t ny, float dx, float x0, float y0, float jitter,
                           uint64_t seed, float* xy) {
    return block_scene(nx, ny, dx, x0, y0, jitter, seed, xy);
}

size_t emerald_wall_scene(float dx, float length, int32_t layers, float* xy) {
    if (!(dx > 0.0f) || layers < 0) return 0;
    return wall_scene(dx, length, layers, xy);
}

size_t emerald_world_walls(emerald_params const* params, float* xy) {
    if (check_params(params)) return 0;
    auto const pts = world_walls(*params);
    if (xy) std::memcpy(xy, pts.data(), pts.size() * sizeof(float2));
    return pts.size();
}

size_t emerald_dam_break(emerald_params const* params, float const* solid_xy, size_t n_solid,
                         float* xy) {
    if (check_params(params)) return 0;
    auto const pts = dam_break(*params, reinterpret_cast<float2 const*>(solid_xy), n_solid);
    if (xy) std::memcpy(xy, pts.data(), pts.size() * sizeof(float2));
    return pts.size();
}

int emerald_sim_create(emerald_params const* params,
                       float const* solid_xy,
                       float const* solid_volumes,
                       size_t n_solid,
                       float const* fluid_xy,
                       float const* fluid_v,
                       size_t n_fluid,
                       emerald_sim** out) {
    if (int rc = check_params(params)) return rc;
    if (!out) return fail(EMERALD_EINVAL, "out is NULL");
    if ((n_fluid && !fluid_xy) || (n_solid && !solid_xy)) {
        return fail(EMERALD_EINVAL, "particle arrays are NULL");
    }
    if (n_fluid > (1u << 30) || n_solid > (1u << 30)) return fail(EMERALD_EINVAL, "too many particles");
    if (int rc = check_particles(fluid_xy, fluid_v, n_fluid, solid_xy, solid_volumes, n_solid)) {
        return rc;
    }
    return guarded([&] {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            return fail(EMERALD_ECUDA, "no CUDA device");
        }
        auto* sim = new emerald_sim(uint32_t(n_fluid), uint32_t(n_solid));
        sim->params = *params;
        SceneSpec spec;
        spec.params = *params;
        spec.method = kDfsph;
        spec.mode = kFrame;
        spec.solid_xy = solid_xy;
        spec.solid_volumes = solid_volumes;
        spec.n_solid = uint32_t(n_solid);
        spec.fluid_xy = fluid_xy;
        spec.fluid_v = fluid_v;
        spec.n_fluid = uint32_t(n_fluid);
        sim->scene = sim->engine.add_scene(spec);
        if (sim->scene < 0) {
            delete sim;
            return fail(EMERALD_ENOMEM, "scene does not fit");
        }
        sim->engine.set_active(sim->scene, true);
        *out = sim;
        return EMERALD_OK;
    });
}

int emerald_sim_destroy(emerald_sim* sim) {
    delete sim;
    return EMERALD_OK;
}

int emerald_sim_begin_frame(emerald_sim* sim, int32_t method) {
    if (!sim || !valid_method(method)) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        sim->engine.begin_frame(method);
        sim->engine.check("begin_frame");
        return EMERALD_OK;
    });
}

int emerald_sim_sub_step(emerald_sim* sim, int32_t method, float t, float dt,
                         emerald_step_stats* stats) {
    if (!sim || !valid_method(method)) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        sim->engine.set_mode(sim->scene, kFixedDt, dt, t);
        sim->engine.substep(method);
        if (stats) fill_stats(sim->engine.scene_state(sim->scene), stats, 1);
        return EMERALD_OK;
    });
}

int emerald_sim_frame(emerald_sim* sim, int32_t method, emerald_step_stats* stats) {
    if (!sim || !valid_method(method)) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        sim->engine.set_mode(sim->scene, kFrame, 0.0f);
        SceneState s{};
        int const n = sim->engine.frame(sim->scene, method, s);
        fill_stats(s, stats, n);
        return EMERALD_OK;
    });
}

int emerald_sim_advance(emerald_sim* sim, int32_t method, int32_t n_substeps,
                        emerald_step_stats* stats) {
    if (!sim || !valid_method(method) || n_substeps < 0) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        sim->engine.set_mode(sim->scene, kFrame, 0.0f);
        for (int k = 0; k < n_substeps; ++k) sim->engine.substep(method);
        if (stats) fill_stats(sim->engine.scene_state(sim->scene), stats, n_substeps);
        return EMERALD_OK;
    });
}

int emerald_sim_advance_host(emerald_sim* sim, int32_t method, int32_t n_substeps,
                             float const* x_in, float const* v_in, float* x_out, float* v_out,
                             emerald_step_stats* stats) {
    if (!sim || !valid_method(method) || n_substeps < 0) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        if (!sim->engine.set_state(sim->scene, x_in, v_in, false)) {
            return fail(EMERALD_EINVAL, "non-finite positions or velocities (state unchanged)");
        }
        sim->engine.set_mode(sim->scene, kFrame, 0.0f);
        for (int k = 0; k < n_substeps; ++k) sim->engine.substep(method);
        sim->engine.get_state(sim->scene, x_out, v_out, true);
        if (stats) fill_stats(sim->engine.scene_state(sim->scene), stats, n_substeps);
        return EMERALD_OK;
    });
}

int emerald_sim_counts(emerald_sim const* sim, size_t* n_fluid, size_t* n_solid) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    if (n_fluid) *n_fluid = sim->engine.fluid_count(sim->scene);
    if (n_solid) *n_solid = sim->engine.solid_count(sim->scene);
    return EMERALD_OK;
}

int emerald_sim_time(emerald_sim const* sim, int64_t* flicks) {
    if (!sim || !flicks) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        SceneState const s = const_cast<emerald_sim*>(sim)->engine.scene_state(sim->scene);
        *flicks = s.frame_time + s.elapsed;
        return EMERALD_OK;
    });
}

int emerald_sim_get_state(emerald_sim* sim, float* x, float* v) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        sim->engine.get_state(sim->scene, x, v);
        return EMERALD_OK;
    });
}

int emerald_sim_set_state(emerald_sim* sim, float const* x, float const* v) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        if (!sim->engine.set_state(sim->scene, x, v)) {
            return fail(EMERALD_EINVAL, "non-finite positions or velocities (state unchanged)");
        }
        return EMERALD_OK;
    });
}

int emerald_sim_get_solid(emerald_sim* sim, float* xy, float* volumes) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        sim->engine.get_solid(sim->scene, xy, volumes);
        return EMERALD_OK;
    });
}

int emerald_sim_set_solid(emerald_sim* sim, float const* solid_xy, float const* solid_v,
                          float const* solid_volumes) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    size_t const ns = sim->engine.solid_count(sim->scene);
    if (int rc = check_particles(nullptr, nullptr, 0, solid_xy, solid_volumes, ns)) return rc;
    if (int rc = check_finite(solid_v, 2 * ns, "boundary velocities")) return rc;
    return guarded([&] {
        sim->engine.set_solid(sim->scene, solid_xy, solid_v, solid_volumes);
        return EMERALD_OK;
    });
}

int emerald_sim_snapshot(emerald_sim* sim, void* buffer, size_t capacity, size_t* size) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        size_t const need = sim->engine.snapshot_size(sim->scene);
        if (size) *size = need;
        if (!buffer) return EMERALD_OK;
        if (capacity < need) return fail(EMERALD_ENOSPC, "snapshot buffer too small");
        sim->engine.snapshot(sim->scene, buffer);
        return EMERALD_OK;
    });
}

int emerald_sim_restore(emerald_sim* sim, void const* buffer, size_t size) {
    if (!sim || !buffer) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        try {
            sim->engine.restore(sim->scene, buffer, size);
        } catch (std::invalid_argument const& e) {
            return fail(EMERALD_EINVAL, e.what());
        }
        return EMERALD_OK;
    });
}

int emerald_sim_set_forces(emerald_sim* sim, emerald_force_term const* terms, int32_t count) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    if (int rc = check_forces(terms, count)) return rc;
    return guarded([&] {
        std::vector<ForceTerm> const t = to_terms(terms, count);
        sim->engine.set_forces(sim->scene, t.data(), count);
        return EMERALD_OK;
    });
}

int emerald_sim_set_force_callback(emerald_sim* sim, emerald_forces_fn fn, void* user) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        sim->engine.set_force_callback(sim->scene, fn, user);
        return EMERALD_OK;
    });
}

int emerald_sim_get_array(emerald_sim* sim, char const* name, float* out, int32_t* width) {
    if (!sim || !name) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        int w = 0;
        if (!sim->engine.get_array(sim->scene, name, out, w)) {
            return fail(EMERALD_ENOTFOUND, std::string("no array ") + name);
        }
        if (width) *width = w;
        return EMERALD_OK;
    });
}

int emerald_sim_get_neighbors(emerald_sim* sim, int32_t solid, uint8_t* counts, uint32_t* idx,
                              float* w, float* gw) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        sim->engine.get_neighbors(sim->scene, solid != 0, counts, idx, w, gw);
        return EMERALD_OK;
    });
}

int emerald_sim_get_sort(emerald_sim* sim, int32_t solid, int32_t* grid_coords, uint64_t* z,
                         uint64_t* pair_z, uint64_t* pair_index, uint32_t* block_indices,
                         uint64_t* blocks, size_t* nblocks) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        size_t const nb = sim->engine.get_sort(sim->scene, solid != 0, grid_coords, z, pair_z,
                                               pair_index, block_indices, blocks);
        if (nblocks) *nblocks = nb;
        return EMERALD_OK;
    });
}

int emerald_sim_set_stream(emerald_sim* sim, void* cuda_stream) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    sim->engine.set_stream(static_cast<cudaStream_t>(cuda_stream));
    return EMERALD_OK;
}

int emerald_sim_device_state(emerald_sim* sim, void** x, void** v) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    if (x) *x = sim->engine.device_x(sim->scene);
    if (v) *v = sim->engine.device_v(sim->scene);
    return EMERALD_OK;
}

int emerald_batch_create(size_t fluid_capacity, size_t solid_capacity, int32_t max_scenes,
                         emerald_batch** out) {
    if (!out || max_scenes < 1 || fluid_capacity > (size_t(1) << 30) ||
        solid_capacity > (size_t(1) << 30)) {
        return fail(EMERALD_EINVAL, "bad batch capacity");
    }
    return guarded([&] {
        *out = new emerald_batch(uint32_t(fluid_capacity), uint32_t(solid_capacity), max_scenes);
        return EMERALD_OK;
    });
}

int emerald_batch_destroy(emerald_batch* batch) {
    delete batch;
    return EMERALD_OK;
}

int emerald_batch_add_scene(emerald_batch* batch, emerald_params const* params,
                            float const* solid_xy, float const* solid_volumes, size_t n_solid,
                            float const* fluid_xy, float const* fluid_v, size_t n_fluid,
                            int32_t* scene) {
    if (!batch || !scene) return fail(EMERALD_EINVAL, "bad arguments");
    if (int rc = check_params(params)) return rc;
    if ((n_fluid && !fluid_xy) || (n_solid && !solid_xy)) {
        return fail(EMERALD_EINVAL, "particle arrays are NULL");
    }
    if (int rc = check_particles(fluid_xy, fluid_v, n_fluid, solid_xy, solid_volumes, n_solid)) {
        return rc;
    }
    return guarded([&] {
        SceneSpec spec;
        spec.params = *params;
        spec.method = kDfsph;
        spec.mode = kFrame;
        spec.solid_xy = solid_xy;
        spec.solid_volumes = solid_volumes;
        spec.n_solid = uint32_t(n_solid);
        spec.fluid_xy = fluid_xy;
        spec.fluid_v = fluid_v;
        spec.n_fluid = uint32_t(n_fluid);
        int const id = batch->engine.add_scene(spec);
        if (id < 0) return fail(EMERALD_ENOSPC, "no room in the batch for this scene");
        *scene = id;
        return EMERALD_OK;
    });
}

int emerald_batch_remove_scene(emerald_batch* batch, int32_t scene) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    return guarded([&] {
        batch->engine.remove_scene(scene);
        return EMERALD_OK;
    });
}

int emerald_batch_set_active(emerald_batch* batch, int32_t scene, int32_t active) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    return guarded([&] {
        batch->engine.set_active(scene, active != 0);
        return EMERALD_OK;
    });
}

int emerald_batch_step(emerald_batch* batch, int32_t method, int32_t n_substeps) {
    if (!batch || !valid_method(method) || n_substeps < 0) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        for (int k = 0; k < n_substeps; ++k) batch->engine.substep(method);
        return EMERALD_OK;
    });
}

int emerald_batch_scene_stats(emerald_batch* batch, int32_t scene, emerald_step_stats* stats) {
    if (!batch || !stats || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    return guarded([&] {
        SceneState const s = batch->engine.scene_state(scene);
        fill_stats(s, stats, s.substeps_total);
        return EMERALD_OK;
    });
}

int emerald_batch_get_state(emerald_batch* batch, int32_t scene, float* x, float* v) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    return guarded([&] {
        batch->engine.get_state(scene, x, v);
        return EMERALD_OK;
    });
}

int emerald_batch_set_state(emerald_batch* batch, int32_t scene, float const* x, float const* v) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    return guarded([&] {
        if (!batch->engine.set_state(scene, x, v)) {
            return fail(EMERALD_EINVAL, "non-finite positions or velocities (state unchanged)");
        }
        return EMERALD_OK;
    });
}

int emerald_batch_set_solid(emerald_batch* batch, int32_t scene, float const* solid_xy,
                            float const* solid_v, float const* solid_volumes) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    size_t const ns = batch->engine.solid_count(scene);
    if (int rc = check_particles(nullptr, nullptr, 0, solid_xy, solid_volumes, ns)) return rc;
    if (int rc = check_finite(solid_v, 2 * ns, "boundary velocities")) return rc;
    return guarded([&] {
        batch->engine.set_solid(scene, solid_xy, solid_v, solid_volumes);
        return EMERALD_OK;
    });
}

int emerald_batch_set_forces(emerald_batch* batch, int32_t scene, emerald_force_term const* terms,
                             int32_t count) {
    if (!batch || !batch->engine.scene_used(scene)) return fail(EMERALD_EINVAL, "bad scene");
    if (int rc = check_forces(terms, count)) return rc;
    return guarded([&] {
        std::vector<ForceTerm> const t = to_terms(terms, count);
        batch->engine.set_forces(scene, t.data(), count);
        return EMERALD_OK;
    });
}

int emerald_batch_free(emerald_batch* batch, size_t* fluid, int32_t* scenes) {
    if (!batch) return fail(EMERALD_EINVAL, "batch is NULL");
    if (fluid) *fluid = batch->engine.free_fluid();
    if (scenes) *scenes = batch->engine.free_scene_slots();
    return EMERALD_OK;
}

int emerald_batch_set_stream(emerald_batch* batch, void* cuda_stream) {
    if (!batch) return fail(EMERALD_EINVAL, "batch is NULL");
    batch->engine.set_stream(static_cast<cudaStream_t>(cuda_stream));
    return EMERALD_OK;
}

int emerald_batch_synchronize(emerald_batch* batch) {
    if (!batch) return fail(EMERALD_EINVAL, "batch is NULL");
    return guarded([&] {
        cudaStreamSynchronize(batch->engine.stream());
        batch->engine.check("synchronize");
        return EMERALD_OK;
    });
}

int emerald_batch_kernel_launches(emerald_batch* batch, int64_t* count) {
    if (!batch || !count) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        *count = batch->engine.kernel_launches();
        return EMERALD_OK;
    });
}

namespace {
int autotune_into(Engine& engine, int32_t method, emerald_tuning* out) {
    if (!valid_method(method)) return fail(EMERALD_EINVAL, "bad method");
    return guarded([&] {
        try {
            Engine::TuneReport const r = engine.autotune(method);
            if (out) {
                *out = emerald_tuning{};
                auto split = [](int v, int32_t& chunk, int32_t& prefetch) {
                    chunk = v & kChunkMask;
                    prefetch = (v & kPersistentWarps)
                                 ? ((v & kPersistentBlocks256) ? EMERALD_TUNE_PERSISTENT_256
                                                               : EMERALD_TUNE_PERSISTENT) +
                                     ((v & kFusedExitTest) ? 2 : 0)
                                 : ((v & kPrefetchLists) ? 1 : 0);
                };
                split(r.chosen.apply, out->apply_chunk, out->prefetch[0]);
                split(r.chosen.divergence, out->divergence_chunk, out->prefetch[1]);
                split(r.chosen.iisph_sum, out->iisph_sum_chunk, out->prefetch[2]);
                split(r.chosen.iisph_beta, out->iisph_beta_chunk, out->prefetch[3]);
                out->candidates = r.count;
                for (int k = 0; k < r.count && k < EMERALD_TUNE_CANDIDATES; ++k) {
                    Engine::Tuning const& t = r.candidates[k];
                    split(t.apply, out->candidate_chunks[k][0], out->candidate_prefetch[k][0]);
                    split(t.divergence, out->candidate_chunks[k][1], out->candidate_prefetch[k][1]);
                    split(t.iisph_sum, out->candidate_chunks[k][2], out->candidate_prefetch[k][2]);
                    split(t.iisph_beta, out->candidate_chunks[k][3], out->candidate_prefetch[k][3]);
                    out->candidate_ms[k] = r.ms[k];
                }
            }
        } catch (std::invalid_argument const& e) {
            return fail(EMERALD_EINVAL, e.what());
        }
        return EMERALD_OK;
    });
}
}  // namespace

namespace {
int set_tuning_of(Engine& engine, emerald_tuning const* t) {
    if (!t) {
        engine.set_tuning(nullptr);
        return EMERALD_OK;
    }
    int32_t const chunks[4] = {t->apply_chunk, t->divergence_chunk, t->iisph_sum_chunk,
                               t->iisph_beta_chunk};
    int v[4];
    for (int k = 0; k < 4; ++k) {
        if (chunks[k] != 1 && chunks[k] != 4 && chunks[k] != 8) {
            return fail(EMERALD_EINVAL, "chunks must be 1, 4 or 8");
        }
        int32_t const mode = t->prefetch[k];
        if (mode < 0 || mode > EMERALD_TUNE_PERSISTENT_256_FUSED) {
            return fail(EMERALD_EINVAL, "prefetch must be between 0 and 5");
        }
        v[k] = chunks[k] | (mode == 1 ? kPrefetchLists : 0) |
               (mode >= EMERALD_TUNE_PERSISTENT ? kPersistentWarps : 0) |
               ((mode == EMERALD_TUNE_PERSISTENT_256 || mode == EMERALD_TUNE_PERSISTENT_256_FUSED)
                  ? kPersistentBlocks256
                  : 0) |
               (mode >= EMERALD_TUNE_PERSISTENT_FUSED ? kFusedExitTest : 0);
    }
    Engine::Tuning tu;
    tu.apply = v[0];
    tu.divergence = v[1];
    tu.iisph_sum = v[2];
    tu.iisph_beta = v[3];
    return guarded([&] {
        engine.set_tuning(&tu);
        return EMERALD_OK;
    });
}
}  // namespace

int emerald_sim_set_tuning(emerald_sim* sim, emerald_tuning const* tuning) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return set_tuning_of(sim->engine, tuning);
}

int emerald_batch_set_tuning(emerald_batch* batch, emerald_tuning const* tuning) {
    if (!batch) return fail(EMERALD_EINVAL, "batch is NULL");
    return set_tuning_of(batch->engine, tuning);
}

int emerald_sim_autotune(emerald_sim* sim, int32_t method, emerald_tuning* out) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return autotune_into(sim->engine, method, out);
}

int emerald_batch_autotune(emerald_batch* batch, int32_t method, emerald_tuning* out) {
    if (!batch) return fail(EMERALD_EINVAL, "batch is NULL");
    return autotune_into(batch->engine, method, out);
}

int emerald_server_create(emerald_server_config const* config, emerald_server** out) {
    if (!config || !out || !valid_method(config->method) || config->hbm_budget_bytes == 0) {
        return fail(EMERALD_EINVAL, "bad server configuration");
    }
    return guarded([&] {
        *out = new emerald_server(*config);
        return EMERALD_OK;
    });
}

int emerald_server_destroy(emerald_server* server) {
    delete server;
    return EMERALD_OK;
}

int emerald_server_submit(emerald_server* server, emerald_params const* params,
                          float const* solid_xy, float const* solid_volumes, size_t n_solid,
                          float const* fluid_xy, float const* fluid_v, size_t n_fluid,
                          int32_t n_substeps, int64_t* request) {
    if (!server || !request || n_substeps < 0) return fail(EMERALD_EINVAL, "bad arguments");
    if (int rc = check_params(params)) return rc;
    if ((n_fluid && !fluid_xy) || (n_solid && !solid_xy) || n_fluid > (size_t(1) << 30) ||
        n_solid > (size_t(1) << 30)) {
        return fail(EMERALD_EINVAL, "bad particle arrays");
    }
    if (int rc = check_particles(fluid_xy, fluid_v, n_fluid, solid_xy, solid_volumes, n_solid)) {
        return rc;
    }
    return guarded([&] {
        std::unique_ptr<ServerRequest> r(new ServerRequest);
        r->params = *params;
        r->n_fluid = uint32_t(n_fluid);
        r->n_solid = uint32_t(n_solid);
        r->substeps = n_substeps;
        r->fluid_xy.assign(fluid_xy, fluid_xy + 2 * n_fluid);
        if (fluid_v) r->fluid_v.assign(fluid_v, fluid_v + 2 * n_fluid);
        if (n_solid) r->solid_xy.assign(solid_xy, solid_xy + 2 * n_solid);
        if (solid_volumes) r->solid_volumes.assign(solid_volumes, solid_volumes + n_solid);
        int const rc = server->server.submit(std::move(r), *request);
        if (rc == EMERALD_ENOSPC) return fail(rc, "scene larger than the server's arena");
        if (rc != EMERALD_OK) return fail(rc, "server loop failed");
        return EMERALD_OK;
    });
}

int emerald_server_wait(emerald_server* server, int64_t request, int32_t timeout_ms, float* x,
                        float* v, emerald_step_stats* stats, emerald_request_timing* timing) {
    if (!server) return fail(EMERALD_EINVAL, "server is NULL");
    return guarded([&] {
        int const rc = server->server.wait(request, timeout_ms, x, v, stats, timing);
        if (rc == EMERALD_ETIMEOUT) return fail(rc, "request not done yet");
        if (rc == EMERALD_ENOTFOUND) return fail(rc, "unknown request");
        if (rc == EMERALD_ECANCELED) return fail(rc, "request was cancelled");
        if (rc != EMERALD_OK) return fail(rc, "request failed");
        return EMERALD_OK;
    });
}

int emerald_server_cancel(emerald_server* server, int64_t request) {
    if (!server) return fail(EMERALD_EINVAL, "server is NULL");
    return guarded([&] {
        int const rc = server->server.cancel(request);
        if (rc == EMERALD_ENOTFOUND) return fail(rc, "unknown request");
        return rc;
    });
}

int emerald_server_get_stats(emerald_server* server, emerald_server_stats* out) {
    if (!server || !out) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        server->server.stats(*out);
        return EMERALD_OK;
    });
}

int emerald_sim_set_graphs(emerald_sim* sim, int32_t graphs) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    sim->engine.set_graphs(graphs != 0);
    return EMERALD_OK;
}

int emerald_sim_host_waits(emerald_sim* sim, int64_t* count) {
    if (!sim || !count) return fail(EMERALD_EINVAL, "bad arguments");
    *count = sim->engine.host_waits();
    return EMERALD_OK;
}

int emerald_sim_kernel_launches(emerald_sim* sim, int64_t* count) {
    if (!sim || !count) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        *count = sim->engine.kernel_launches();
        return EMERALD_OK;
    });
}

int emerald_sim_enable_timing(emerald_sim* sim, int32_t enable) {
    if (!sim) return fail(EMERALD_EINVAL, "sim is NULL");
    return guarded([&] {
        sim->engine.reset_timing();
        sim->engine.enable_timing(enable != 0);
        return EMERALD_OK;
    });
}

int emerald_sim_kernel_times(emerald_sim* sim, char* names, size_t names_len, double* ms,
                             int32_t* launches, int32_t* count) {
    if (!sim || !count) return fail(EMERALD_EINVAL, "bad arguments");
    return guarded([&] {
        KernelTimes const& t = sim->engine.kernel_times();
        int const cap = *count;
        int k = 0;
        std::string joined;
        for (auto const& kv : t.ms) {
            if (k < cap) {
                if (ms) ms[k] = kv.second;
                if (launches) launches[k] = t.launches.at(kv.first);
            }
            if (!joined.empty()) joined += '\n';
            joined += kv.first;
            ++k;
        }
        if (names && names_len) {
            std::strncpy(names, joined.c_str(), names_len - 1);
            names[names_len - 1] = '\0';
        }
        *count = k;
        return EMERALD_OK;
    });
}

}  // extern "C"
