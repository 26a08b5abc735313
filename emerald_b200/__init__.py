"""emerald_b200: B200 implementation of the emerald 2D SPH step.

A Python mirror of the reference's solver API (emerald/sph2d_box/simulation.h,
EZ_EXAMPLE_SIM and the X_simulation_step functions) over the C ABI in
include/emerald_sph.h. All compute runs in libemerald_b200.so on the GPU;
this module only marshals arrays. Importing it fails loudly when the library
is missing.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemerald_b200.so")

METHODS = {"pcisph": 0, "iisph": 1, "iisph_ap": 2, "iisph_pseudo_ap": 3, "dfsph_p": 4}
PRECISION_REFERENCE = 0
PRECISION_COMPENSATED = 1
FLICKS_PER_SECOND = 705600000

c_f = ctypes.c_float
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_sz = ctypes.c_size_t
c_vp = ctypes.c_void_p


class EmeraldError(RuntimeError):
    """A failed C-ABI call; `code` is its EMERALD_* status."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


class Params(ctypes.Structure):
    """emerald_params (mirrors emerald/sph2d_box/parameters.h:12-41)."""

    _fields_ = [
        ("seed", c_u64), ("time_per_step_flicks", c_i64), ("sub_steps", c_i32),
        ("length", c_f), ("support", c_f), ("gravity", c_f), ("viscosity", c_f),
        ("target_density", c_f), ("iisph_max_pressure_iterations", c_i32),
        ("iisph_error_average_threshold", c_f), ("iisph_error_max_threshold", c_f),
        ("iisph_omega", c_f), ("dfsph_max_correction_iterations", c_i32),
        ("dfsph_density_error_average_threshold", c_f),
        ("dfsph_density_error_max_threshold", c_f),
        ("dfsph_divergence_error_average_threshold", c_f),
        ("dfsph_divergence_error_max_threshold", c_f),
        ("mass_per_particle", c_f), ("pressure_correction_denom", c_f),
        ("precision", c_i32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StepStats(ctypes.Structure):
    _fields_ = [
        ("sub_steps", c_i32), ("pressure_iterations", c_i32), ("error_average", c_f),
        ("error_max", c_f), ("divergence_iterations", c_i32), ("divergence_error_average", c_f),
        ("divergence_error_max", c_f), ("dt", c_f), ("time_seconds", ctypes.c_double),
        ("error_flags", c_i32), ("error_average_exact", ctypes.c_double),
        ("divergence_error_average_exact", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", c_sz), ("method", c_i32), ("max_scenes", c_i32),
                ("max_substeps_per_launch", c_i32), ("lanes", c_i32), ("order", c_i32)]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", c_i64), ("completed", c_i64), ("rejected", c_i64), ("queued", c_i64),
        ("resident", c_i64), ("batch_substeps", c_i64), ("scene_substeps", c_i64),
        ("particle_substeps", ctypes.c_double), ("busy_seconds", ctypes.c_double),
        ("step_ms_p50", c_f), ("step_ms_p99", c_f), ("request_ms_p50", c_f),
        ("request_ms_p99", c_f), ("queue_ms_p50", c_f), ("queue_ms_p99", c_f),
        ("fluid_capacity", c_sz), ("solid_capacity", c_sz), ("device_bytes", c_sz),
        ("resident_peak", c_i32), ("status", c_i32), ("cancelled", c_i64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestTiming(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("apply_chunk", c_i32), ("divergence_chunk", c_i32), ("iisph_sum_chunk", c_i32),
                ("iisph_beta_chunk", c_i32), ("candidates", c_i32),
                ("candidate_chunks", (c_i32 * 4) * 16), ("candidate_ms", c_f * 16),
                ("prefetch", c_i32 * 4), ("candidate_prefetch", (c_i32 * 4) * 16)]

    def as_dict(self):
        fams = ("apply", "divergence", "iisph_sum", "iisph_beta")
        return {"chunks": {f: getattr(self, f + "_chunk") for f in fams},
                "prefetch": dict(zip(fams, list(self.prefetch))),
                "candidates": [{"chunks": dict(zip(fams, list(self.candidate_chunks[k]))),
                                "prefetch": dict(zip(fams, list(self.candidate_prefetch[k]))),
                                "ms_per_substep": round(self.candidate_ms[k], 4)}
                               for k in range(self.candidates)]}


def _tuning_struct(chunks, prefetch=None):
    """A Tuning from {family: chunk} and {family: 0/1} (None unpins)."""
    if chunks is None:
        return None
    fams = ("apply", "divergence", "iisph_sum", "iisph_beta")
    t = Tuning()
    for k, f in enumerate(fams):
        setattr(t, f + "_chunk", int(chunks[f]))
        t.prefetch[k] = int((prefetch or {}).get(f, 0))
    return t


class Neighborhood(ctypes.Structure):
    """emerald_neighborhood: device pointers of the reference's
    Neighborhood_pointers layout (64 entries per particle, row-major)."""
    _fields_ = [("counts", c_vp), ("indices", c_vp), ("distances", c_vp), ("vectors_to", c_vp),
                ("kernels", c_vp), ("kernel_gradients", c_vp)]


class ForceTerm(ctypes.Structure):
    """emerald_force_term: kind (FORCE_GRAVITY, FORCE_POLE, FORCE_DRAG) and
    its arguments a, b, c."""
    _fields_ = [("kind", c_i32), ("a", c_f), ("b", c_f), ("c", c_f)]


FORCE_GRAVITY, FORCE_POLE, FORCE_DRAG = 1, 2, 3
MAX_FORCE_TERMS = 4
# emerald_forces_fn(user, count, time, dt, mass, radius, forces, positions, velocities)
FORCES_FN = ctypes.CFUNCTYPE(None, c_vp, ctypes.c_size_t, c_f, c_f, c_f, c_f,
                             ctypes.POINTER(c_f), ctypes.POINTER(c_f), ctypes.POINTER(c_f))


def force_terms(terms):
    """A ctypes array of emerald_force_term from (kind, a, b, c) tuples
    (missing arguments are zero)."""
    arr = (ForceTerm * max(len(terms), 1))()
    for k, t in enumerate(terms):
        t = tuple(t) + (0.0,) * (4 - len(t))
        arr[k] = ForceTerm(int(t[0]), float(t[1]), float(t[2]), float(t[3]))
    return arr


EXPORTS = {
    "emerald_default_params": (c_i32, [ctypes.POINTER(Params)]),
    "emerald_config": (c_i32, [ctypes.POINTER(Params), c_vp]),
    "emerald_lattice_config": (c_i32, [ctypes.POINTER(Params), c_f, c_f, c_vp]),
    "emerald_z_index": (c_u64, [c_u32, c_u32]),
    "emerald_block_scene": (c_sz, [c_u32, c_u32, c_f, c_f, c_f, c_f, c_u64, c_vp]),
    "emerald_wall_scene": (c_sz, [c_f, c_f, c_i32, c_vp]),
    "emerald_world_walls": (c_sz, [ctypes.POINTER(Params), c_vp]),
    "emerald_dam_break": (c_sz, [ctypes.POINTER(Params), c_vp, c_sz, c_vp]),
    "emerald_sim_create": (c_i32, [ctypes.POINTER(Params), c_vp, c_vp, c_sz, c_vp, c_vp, c_sz,
                                   ctypes.POINTER(c_vp)]),
    "emerald_sim_destroy": (c_i32, [c_vp]),
    "emerald_sim_begin_frame": (c_i32, [c_vp, c_i32]),
    "emerald_sim_sub_step": (c_i32, [c_vp, c_i32, c_f, c_f, ctypes.POINTER(StepStats)]),
    "emerald_sim_frame": (c_i32, [c_vp, c_i32, ctypes.POINTER(StepStats)]),
    "emerald_sim_advance": (c_i32, [c_vp, c_i32, c_i32, ctypes.POINTER(StepStats)]),
    "emerald_sim_advance_host": (c_i32, [c_vp, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp,
                                         ctypes.POINTER(StepStats)]),
    "emerald_sim_counts": (c_i32, [c_vp, ctypes.POINTER(c_sz), ctypes.POINTER(c_sz)]),
    "emerald_sim_time": (c_i32, [c_vp, ctypes.POINTER(c_i64)]),
    "emerald_sim_get_state": (c_i32, [c_vp, c_vp, c_vp]),
    "emerald_sim_set_state": (c_i32, [c_vp, c_vp, c_vp]),
    "emerald_sim_get_solid": (c_i32, [c_vp, c_vp, c_vp]),
    "emerald_sim_set_solid": (c_i32, [c_vp, c_vp, c_vp, c_vp]),
    "emerald_sim_set_forces": (c_i32, [c_vp, c_vp, c_i32]),
    "emerald_sim_set_force_callback": (c_i32, [c_vp, FORCES_FN, c_vp]),
    "emerald_sim_snapshot": (c_i32, [c_vp, c_vp, c_sz, ctypes.POINTER(c_sz)]),
    "emerald_sim_host_waits": (c_i32, [c_vp, ctypes.POINTER(c_i64)]),
    "emerald_sim_restore": (c_i32, [c_vp, c_vp, c_sz]),
    "emerald_sim_get_array": (c_i32, [c_vp, ctypes.c_char_p, c_vp, ctypes.POINTER(c_i32)]),
    "emerald_sim_get_neighbors": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp]),
    "emerald_sim_get_sort": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                     ctypes.POINTER(c_sz)]),
    "emerald_sim_set_stream": (c_i32, [c_vp, c_vp]),
    "emerald_sim_device_state": (c_i32, [c_vp, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp)]),
    "emerald_sim_enable_timing": (c_i32, [c_vp, c_i32]),
    "emerald_sim_kernel_times": (c_i32, [c_vp, ctypes.c_char_p, c_sz, c_vp, c_vp,
                                         ctypes.POINTER(c_i32)]),
    "emerald_sim_set_graphs": (c_i32, [c_vp, c_i32]),
    "emerald_sim_kernel_launches": (c_i32, [c_vp, ctypes.POINTER(c_i64)]),
    "emerald_batch_create": (c_i32, [c_sz, c_sz, c_i32, ctypes.POINTER(c_vp)]),
    "emerald_batch_destroy": (c_i32, [c_vp]),
    "emerald_batch_add_scene": (c_i32, [c_vp, ctypes.POINTER(Params), c_vp, c_vp, c_sz, c_vp, c_vp,
                                        c_sz, ctypes.POINTER(c_i32)]),
    "emerald_batch_remove_scene": (c_i32, [c_vp, c_i32]),
    "emerald_batch_set_active": (c_i32, [c_vp, c_i32, c_i32]),
    "emerald_batch_step": (c_i32, [c_vp, c_i32, c_i32]),
    "emerald_batch_scene_stats": (c_i32, [c_vp, c_i32, ctypes.POINTER(StepStats)]),
    "emerald_batch_get_state": (c_i32, [c_vp, c_i32, c_vp, c_vp]),
    "emerald_batch_set_state": (c_i32, [c_vp, c_i32, c_vp, c_vp]),
    "emerald_batch_set_solid": (c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp]),
    "emerald_batch_set_forces": (c_i32, [c_vp, c_i32, c_vp, c_i32]),
    "emerald_batch_free": (c_i32, [c_vp, ctypes.POINTER(c_sz), ctypes.POINTER(c_i32)]),
    "emerald_batch_set_stream": (c_i32, [c_vp, c_vp]),
    "emerald_batch_synchronize": (c_i32, [c_vp]),
    "emerald_batch_kernel_launches": (c_i32, [c_vp, ctypes.POINTER(c_i64)]),
    "emerald_server_create": (c_i32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(c_vp)]),
    "emerald_server_destroy": (c_i32, [c_vp]),
    "emerald_server_submit": (c_i32, [c_vp, ctypes.POINTER(Params), c_vp, c_vp, c_sz, c_vp, c_vp,
                                      c_sz, c_i32, ctypes.POINTER(c_i64)]),
    "emerald_server_wait": (c_i32, [c_vp, c_i64, c_i32, c_vp, c_vp, ctypes.POINTER(StepStats),
                                    ctypes.POINTER(RequestTiming)]),
    "emerald_server_get_stats": (c_i32, [c_vp, ctypes.POINTER(ServerStats)]),
    "emerald_server_cancel": (c_i32, [c_vp, c_i64]),
    "emerald_sim_autotune": (c_i32, [c_vp, c_i32, ctypes.POINTER(Tuning)]),
    "emerald_sim_set_tuning": (c_i32, [c_vp, ctypes.POINTER(Tuning)]),
    "emerald_batch_set_tuning": (c_i32, [c_vp, ctypes.POINTER(Tuning)]),
    "emerald_batch_autotune": (c_i32, [c_vp, c_i32, ctypes.POINTER(Tuning)]),
    "emerald_compute_grid_coords": (c_i32, [c_sz, c_f, c_f, c_f, c_vp, c_vp, c_vp]),
    "emerald_compute_z_indices": (c_i32, [c_sz, c_vp, c_vp, c_vp]),
    "emerald_compute_index_pairs": (c_i32, [c_sz, c_vp, c_vp, c_vp]),
    "emerald_index_pairs_workspace": (c_i32, [c_sz, ctypes.POINTER(c_sz)]),
    "emerald_sort_index_pairs": (c_i32, [c_sz, c_vp, c_vp, c_sz, c_vp]),
    "emerald_compute_block_indices": (c_i32, [c_sz, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "emerald_fill_blocks": (c_i32, [c_sz, c_vp, c_vp, c_vp]),
    "emerald_block_map_create": (c_i32, [ctypes.POINTER(c_vp)]),
    "emerald_block_map_destroy": (c_i32, [c_vp]),
    "emerald_create_block_map": (c_i32, [c_sz, c_vp, c_vp, c_vp, c_vp]),
    "emerald_create_regular_neighborhoods": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp, c_vp,
                                                     c_vp, c_vp, c_vp, c_vp, c_vp]),
    "emerald_compute_neighbor_distances_and_vectors_to": (c_i32, [c_sz, c_vp, c_vp, c_vp, c_vp,
                                                                  c_vp, c_vp, c_vp]),
    "emerald_compute_neighbor_kernels": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp]),
    "emerald_compute_neighbor_kernel_gradients": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp]),
    "emerald_compute_densities": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, Neighborhood, c_vp,
                                          Neighborhood, c_vp]),
    "emerald_compute_divergences": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, Neighborhood, c_vp, c_vp,
                                            Neighborhood, c_vp]),
    "emerald_predict_density_stars": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp,
                                              Neighborhood, c_vp, c_vp, Neighborhood, c_vp]),
    "emerald_apply_pressures_in_place": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp,
                                                 Neighborhood, c_vp, Neighborhood, c_vp]),
    "emerald_compute_pressure_accelerations": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp,
                                                       Neighborhood, c_vp, Neighborhood, c_vp]),
    "emerald_integrate_velocities_with_forces": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp]),
    "emerald_integrate_velocities": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp]),
    "emerald_integrate_positions": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp]),
    "emerald_compute_constant_volumes": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp]),
    "emerald_max_vector_squared_magnitude": (c_i32, [c_sz, c_vp, c_vp, c_vp]),
    "emerald_max_density_error": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp]),
    "emerald_cfl_maximum_time_step": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp]),
    "emerald_scalar_average_and_max": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp]),
    "emerald_iisph_compute_diis": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, Neighborhood, c_vp,
                                           Neighborhood, c_vp]),
    "emerald_iisph_compute_aiis_and_density_stars": (
        c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp, c_vp,
                Neighborhood, c_vp]),
    "emerald_iisph_compute_sum_dij_pjs": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp,
                                                  Neighborhood, c_vp]),
    "emerald_iisph_compute_betas": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                            Neighborhood, c_vp, Neighborhood, c_vp]),
    "emerald_iisph_compute_new_pressures": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp,
                                                    c_vp]),
    "emerald_dfsph_p_compute_shared_coeffs": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, Neighborhood,
                                                      c_vp, Neighborhood, c_vp]),
    "emerald_dfsph_p_compute_density_pseudo_pressures": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp,
                                                                 c_vp, c_vp]),
    "emerald_dfsph_p_compute_divergence_pseudo_pressures": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp,
                                                                    c_vp, c_vp]),
    "emerald_pcisph_compute_densities": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp]),
    "emerald_pcisph_accumulate_density_from_solids": (c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp,
                                                              c_vp, c_vp]),
    "emerald_pcisph_update_pressures": (c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp]),
    "emerald_pcisph_accumulate_pressure_forces": (c_i32, [c_sz, c_f, c_f, c_f] + [c_vp] * 10),
    "emerald_pcisph_accumulate_pressure_forces_from_solids": (c_i32, [c_sz, c_f, c_f] +
                                                              [c_vp] * 8),
    "emerald_iisph_ap_density_stars_and_diagonals": (
        c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp, c_vp,
                Neighborhood, c_vp]),
    "emerald_iisph_ap_iterate_pressures_in_place": (
        c_i32, [c_sz, c_f, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp,
                Neighborhood, c_vp, c_vp]),
    "emerald_iisph_pseudo_ap_density_stars_and_pseudo_diagonals": (
        c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp, c_vp,
                Neighborhood, c_vp]),
    "emerald_iisph_pseudo_ap_compute_pseudo_pressure_displacements": (
        c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp, Neighborhood, c_vp]),
    "emerald_iisph_pseudo_ap_iterate_pseudo_pressures_in_place": (
        c_i32, [c_sz, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, Neighborhood, c_vp, Neighborhood,
                c_vp, c_vp]),
    "emerald_iisph_pseudo_ap_integrate_velocities_and_positions_in_place": (
        c_i32, [c_sz, c_f, c_vp, c_vp, c_vp, c_vp]),
    "emerald_neighbors_static": (c_i32, [c_vp, c_u32, c_f, c_vp, c_vp, c_vp, c_vp, c_u32, c_vp]),
    "emerald_kernel_launches": (c_i64, []),
    "emerald_last_error": (ctypes.c_char_p, []),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "emerald_b200: %s is missing; build it with `python emerald_b200/build.py` "
            "(there is no CPU fallback)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(c_vp)


def _check(rc, what):
    if rc != 0:
        msg = lib.emerald_last_error()
        raise EmeraldError("%s failed (%d): %s" % (what, rc, msg.decode() if msg else ""), rc)


def _f32(a, shape_tail=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def _out_array(a, n):
    if a is None:
        return np.zeros((n, 2), np.float32)
    if a.dtype != np.float32 or a.shape != (n, 2) or not a.flags.c_contiguous:
        raise ValueError("output array must be C-contiguous float32 of shape (%d, 2)" % n)
    return a


def method_id(method):
    return METHODS[method] if isinstance(method, str) else int(method)


def default_params(**overrides):
    p = Params()
    _check(lib.emerald_default_params(ctypes.byref(p)), "emerald_default_params")
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def config(params):
    """Simulation_config values: seconds_per_sub_step, mass_per_particle,
    draw_radius, pressure_correction_denom (emerald/sph2d_box/config.cpp)."""
    out = np.zeros(4, np.float32)
    _check(lib.emerald_config(ctypes.byref(params), _ptr(out)), "emerald_config")
    return dict(seconds_per_sub_step=out[0], mass_per_particle=out[1], draw_radius=out[2],
                pressure_correction_denom=out[3])


def lattice_config(params, dx, dt):
    out = np.zeros(2, np.float32)
    _check(lib.emerald_lattice_config(ctypes.byref(params), dx, dt, _ptr(out)),
           "emerald_lattice_config")
    return out[0], out[1]


def z_index(x, y):
    return lib.emerald_z_index(x & 0xFFFFFFFF, y & 0xFFFFFFFF)


def block_scene(nx, ny, dx, x0=0.0, y0=0.0, jitter=0.01, seed=1):
    xy = np.zeros((nx * ny, 2), np.float32)
    lib.emerald_block_scene(nx, ny, dx, x0, y0, jitter, seed, _ptr(xy))
    return xy


def wall_scene(dx, length=1.0, layers=3):
    n = lib.emerald_wall_scene(dx, length, layers, None)
    xy = np.zeros((n, 2), np.float32)
    lib.emerald_wall_scene(dx, length, layers, _ptr(xy))
    return xy


def world_walls(params):
    n = lib.emerald_world_walls(ctypes.byref(params), None)
    xy = np.zeros((n, 2), np.float32)
    lib.emerald_world_walls(ctypes.byref(params), _ptr(xy))
    return xy


def dam_break(params, solid_xy):
    solid_xy = _f32(solid_xy)
    n = lib.emerald_dam_break(ctypes.byref(params), _ptr(solid_xy), len(solid_xy), None)
    xy = np.zeros((n, 2), np.float32)
    lib.emerald_dam_break(ctypes.byref(params), _ptr(solid_xy), len(solid_xy), _ptr(xy))
    return xy


def kernel_launches():
    return lib.emerald_kernel_launches()


STATIC_MAX_POINTS = 65536
MAX_NEIGHBORS = 64  # EMERALD_MAX_NEIGHBORS


def neighbors_static(d_xy, n, support, d_counts, d_idx, d_w, d_gw, stride, stream=None):
    """emerald_neighbors_static on raw device pointers (integers): the
    allocation-free neighbour build for callers that cannot allocate."""
    _check(lib.emerald_neighbors_static(d_xy, n, support, d_counts, d_idx, d_w, d_gw, stride,
                                        stream), "emerald_neighbors_static")


class BlockScene:
    """A seeded dam-break block scene: an nx-by-ny fluid lattice at spacing dx
    (jitter +/- jitter*dx from std::mt19937_64{seed}) inside a [0, length]^2
    tank with `layers` boundary rows at the same spacing on the floor and side
    walls. support = support_ratio * dx. Boundary volumes are the fluid
    particle volume (the rows act as frozen fluid at the lattice spacing) and
    the mass per particle gives the unjittered lattice the target density."""

    def __init__(self, n_side, dx=None, ny=None, length=1.0, support_ratio=1.0, jitter=0.01,
                 seed=1, layers=3, dt=5e-4, **param_overrides):
        self.nx = n_side
        self.ny = ny or n_side
        self.dx = np.float32(dx if dx is not None else 1.0 / (2 * n_side))
        self.support = np.float32(support_ratio * self.dx)
        self.params = default_params(support=self.support, length=length, seed=seed)
        for k, v in param_overrides.items():
            setattr(self.params, k, v)
        mass, denom = lattice_config(self.params, self.dx, dt)
        self.params.mass_per_particle = mass
        self.params.pressure_correction_denom = denom
        self.fluid = block_scene(self.nx, self.ny, self.dx, 0.0, 0.0, jitter, seed)
        self.solid = wall_scene(self.dx, length, layers)
        self.solid_volumes = np.full(len(self.solid), np.float32(mass) / np.float32(
            self.params.target_density), np.float32)


class Simulation:
    """One scene on the GPU: the EZ_EXAMPLE_SIM state
    (emerald/sph2d_box/simulation.h:24-44) with step functions."""

    def __init__(self, params, solid_xy, fluid_xy, fluid_v=None, solid_volumes=None):
        self.params = params
        s = _f32(solid_xy).reshape(-1, 2)
        f = _f32(fluid_xy).reshape(-1, 2)
        v = None if fluid_v is None else _f32(fluid_v).reshape(-1, 2)
        vol = None if solid_volumes is None else _f32(solid_volumes)
        h = c_vp()
        _check(lib.emerald_sim_create(ctypes.byref(params), _ptr(s), _ptr(vol), len(s), _ptr(f),
                                      _ptr(v), len(f), ctypes.byref(h)), "emerald_sim_create")
        self._h = h
        self.n = len(f)
        self.ns = len(s)

    @classmethod
    def from_block_scene(cls, scene):
        return cls(scene.params, scene.solid, scene.fluid, None, scene.solid_volumes)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.emerald_sim_destroy(self._h)
            self._h = c_vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def begin_frame(self, method):
        _check(lib.emerald_sim_begin_frame(self._h, method_id(method)), "begin_frame")

    def sub_step(self, method, t, dt):
        st = StepStats()
        _check(lib.emerald_sim_sub_step(self._h, method_id(method), t, dt, ctypes.byref(st)),
               "sub_step")
        return st.as_dict()

    def frame(self, method):
        st = StepStats()
        _check(lib.emerald_sim_frame(self._h, method_id(method), ctypes.byref(st)), "frame")
        return st.as_dict()

    def advance(self, method, n_substeps, stats=True):
        st = StepStats()
        _check(lib.emerald_sim_advance(self._h, method_id(method), n_substeps,
                                       ctypes.byref(st) if stats else None), "advance")
        return st.as_dict()

    def advance_host(self, method, n_substeps, x, v, stats=False):
        """Copies x, v (C-contiguous float32 (n, 2) host arrays, e.g. pinned)
        in, advances n sub-steps and copies the new state back into them,
        with one wait for the device."""
        st = StepStats()
        _check(lib.emerald_sim_advance_host(self._h, method_id(method), n_substeps, _ptr(x),
                                            _ptr(v), _ptr(x), _ptr(v),
                                            ctypes.byref(st) if stats else None), "advance_host")
        return st.as_dict() if stats else None

    def time(self):
        t = c_i64()
        _check(lib.emerald_sim_time(self._h, ctypes.byref(t)), "time")
        return t.value

    def state(self, x=None, v=None):
        """Positions and velocities (original order). Given x / v (C-contiguous
        float32 arrays of shape (n, 2), e.g. pinned host memory) are filled in
        place instead of new arrays."""
        x = _out_array(x, self.n)
        v = _out_array(v, self.n)
        _check(lib.emerald_sim_get_state(self._h, _ptr(x), _ptr(v)), "get_state")
        return x, v

    def set_state(self, x=None, v=None):
        x = None if x is None else _f32(x)
        v = None if v is None else _f32(v)
        _check(lib.emerald_sim_set_state(self._h, _ptr(x), _ptr(v)), "set_state")

    def set_solid(self, xy=None, v=None, volumes=None):
        """Moves the boundary between sub-steps: new positions (rebuilding its
        cell tables and, unless `volumes` is given, its volumes), velocities
        or volumes; None keeps each."""
        xy = None if xy is None else _f32(xy)
        v = None if v is None else _f32(v)
        volumes = None if volumes is None else np.ascontiguousarray(volumes, np.float32)
        _check(lib.emerald_sim_set_solid(self._h, _ptr(xy), _ptr(v), _ptr(volumes)), "set_solid")

    def host_waits(self):
        """Times the simulation waited on the host for the device."""
        n = c_i64()
        _check(lib.emerald_sim_host_waits(self._h, ctypes.byref(n)), "host_waits")
        return n.value

    def snapshot(self):
        """The simulation's checkpoint (emerald_sim_snapshot) as bytes."""
        size = c_sz()
        _check(lib.emerald_sim_snapshot(self._h, None, 0, ctypes.byref(size)), "snapshot")
        buf = ctypes.create_string_buffer(size.value)
        _check(lib.emerald_sim_snapshot(self._h, buf, size.value, ctypes.byref(size)), "snapshot")
        return buf.raw

    def restore(self, data):
        """Loads a checkpoint taken by snapshot() (emerald_sim_restore)."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        _check(lib.emerald_sim_restore(self._h, buf, len(data)), "restore")

    def set_forces(self, terms):
        """Device force terms, (kind, a, b, c) tuples evaluated in order
        (emerald_sim_set_forces); [] applies no external force."""
        arr = force_terms(terms)
        _check(lib.emerald_sim_set_forces(self._h, ctypes.cast(arr, c_vp), len(terms)),
               "set_forces")

    def set_force_callback(self, fn):
        """A host force function called once per sub-step at the solver's
        force point: fn(time, dt, mass, radius, forces, positions, velocities)
        with (n, 2) float32 views, forces zeroed, to be filled in place. None
        removes it."""
        if fn is None:
            self._force_cb = None
            _check(lib.emerald_sim_set_force_callback(self._h, FORCES_FN(), None),
                   "set_force_callback")
            return
        n = self.n

        def trampoline(user, count, time, dt, mass, radius, f, x, v):
            view = lambda p: np.ctypeslib.as_array(p, shape=(count, 2))
            fn(time, dt, mass, radius, view(f), view(x), view(v))

        self._force_cb = FORCES_FN(trampoline)
        _check(lib.emerald_sim_set_force_callback(self._h, self._force_cb, None),
               "set_force_callback")

    def solid(self):
        xy = np.zeros((self.ns, 2), np.float32)
        vol = np.zeros(self.ns, np.float32)
        _check(lib.emerald_sim_get_solid(self._h, _ptr(xy), _ptr(vol)), "get_solid")
        return xy, vol

    def array(self, name):
        w = c_i32()
        _check(lib.emerald_sim_get_array(self._h, name.encode(), None, ctypes.byref(w)),
               "get_array")
        out = np.zeros((self.n, w.value) if w.value > 1 else self.n, np.float32)
        _check(lib.emerald_sim_get_array(self._h, name.encode(), _ptr(out), ctypes.byref(w)),
               "get_array")
        return out

    def neighbors(self, solid=False):
        counts = np.zeros(self.n, np.uint8)
        idx = np.zeros((self.n, 64), np.uint32)
        w = np.zeros((self.n, 64), np.float32)
        gw = np.zeros((self.n, 64, 2), np.float32)
        _check(lib.emerald_sim_get_neighbors(self._h, int(solid), _ptr(counts), _ptr(idx),
                                             _ptr(w), _ptr(gw)), "get_neighbors")
        return counts, idx, w, gw

    def sort(self, solid=False):
        n = self.ns if solid else self.n
        gc = np.zeros((n, 2), np.int32)
        z = np.zeros(n, np.uint64)
        pz = np.zeros(n, np.uint64)
        pi = np.zeros(n, np.uint64)
        bi = np.zeros(n, np.uint32)
        blocks = np.zeros((max(n, 1), 2), np.uint64)
        nb = c_sz()
        _check(lib.emerald_sim_get_sort(self._h, int(solid), _ptr(gc), _ptr(z), _ptr(pz), _ptr(pi),
                                        _ptr(bi), _ptr(blocks), ctypes.byref(nb)), "get_sort")
        return dict(grid_coords=gc, z_indices=z, pair_z=pz, pair_index=pi, block_indices=bi,
                    blocks=blocks[:nb.value])

    def set_stream(self, stream_ptr):
        _check(lib.emerald_sim_set_stream(self._h, stream_ptr), "set_stream")

    def device_state(self):
        x = c_vp()
        v = c_vp()
        _check(lib.emerald_sim_device_state(self._h, ctypes.byref(x), ctypes.byref(v)),
               "device_state")
        return x.value, v.value

    def set_graphs(self, on=True):
        _check(lib.emerald_sim_set_graphs(self._h, int(on)), "set_graphs")

    def kernel_launches(self):
        n = c_i64()
        _check(lib.emerald_sim_kernel_launches(self._h, ctypes.byref(n)), "kernel_launches")
        return n.value

    def autotune(self, method):
        t = Tuning()
        _check(lib.emerald_sim_autotune(self._h, method_id(method), ctypes.byref(t)), "autotune")
        return t.as_dict()

    def set_tuning(self, chunks=None, prefetch=None):
        """Pins the gather kernels' chunks and prefetch flags (as autotune
        reports them); no arguments unpins."""
        t = _tuning_struct(chunks, prefetch)
        _check(lib.emerald_sim_set_tuning(self._h, None if t is None else ctypes.byref(t)),
               "set_tuning")

    def enable_timing(self, on=True):
        _check(lib.emerald_sim_enable_timing(self._h, int(on)), "enable_timing")

    def kernel_times(self):
        count = c_i32(256)
        ms = np.zeros(256, np.float64)
        launches = np.zeros(256, np.int32)
        names = ctypes.create_string_buffer(1 << 16)
        _check(lib.emerald_sim_kernel_times(self._h, names, len(names), _ptr(ms), _ptr(launches),
                                            ctypes.byref(count)), "kernel_times")
        keys = names.value.decode().split("\n") if names.value else []
        return {k: (float(ms[i]), int(launches[i])) for i, k in enumerate(keys[:count.value])}


class Batch:
    """Many independent scenes advanced together on one GPU: each kernel of a
    sub-step runs once over every active scene. A scene's results are the
    bits it gives when run alone."""

    def __init__(self, fluid_capacity, solid_capacity, max_scenes):
        h = c_vp()
        _check(lib.emerald_batch_create(fluid_capacity, solid_capacity, max_scenes,
                                        ctypes.byref(h)), "emerald_batch_create")
        self._h = h
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.emerald_batch_destroy(self._h)
            self._h = c_vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, params, solid_xy, fluid_xy, fluid_v=None, solid_volumes=None,
                  active=True):
        """Returns the scene id, or None when the batch has no room."""
        s = _f32(solid_xy).reshape(-1, 2)
        f = _f32(fluid_xy).reshape(-1, 2)
        v = None if fluid_v is None else _f32(fluid_v).reshape(-1, 2)
        vol = None if solid_volumes is None else _f32(solid_volumes)
        sid = c_i32()
        rc = lib.emerald_batch_add_scene(self._h, ctypes.byref(params), _ptr(s), _ptr(vol), len(s),
                                         _ptr(f), _ptr(v), len(f), ctypes.byref(sid))
        if rc == 28:
            return None
        _check(rc, "emerald_batch_add_scene")
        self._sizes[sid.value] = len(f)
        if active:
            self.set_active(sid.value, True)
        return sid.value

    def add_block_scene(self, scene, active=True):
        return self.add_scene(scene.params, scene.solid, scene.fluid, None, scene.solid_volumes,
                              active)

    def remove_scene(self, sid):
        _check(lib.emerald_batch_remove_scene(self._h, sid), "remove_scene")
        self._sizes.pop(sid, None)

    def set_active(self, sid, on=True):
        _check(lib.emerald_batch_set_active(self._h, sid, int(on)), "set_active")

    def step(self, method, n_substeps=1):
        _check(lib.emerald_batch_step(self._h, method_id(method), n_substeps), "batch_step")

    def stats(self, sid):
        st = StepStats()
        _check(lib.emerald_batch_scene_stats(self._h, sid, ctypes.byref(st)), "scene_stats")
        return st.as_dict()

    def state(self, sid):
        n = self._sizes[sid]
        x = np.zeros((n, 2), np.float32)
        v = np.zeros((n, 2), np.float32)
        _check(lib.emerald_batch_get_state(self._h, sid, _ptr(x), _ptr(v)), "get_state")
        return x, v

    def set_state(self, sid, x=None, v=None):
        x = None if x is None else _f32(x)
        v = None if v is None else _f32(v)
        _check(lib.emerald_batch_set_state(self._h, sid, _ptr(x), _ptr(v)), "set_state")

    def set_solid(self, sid, xy=None, v=None, volumes=None):
        xy = None if xy is None else _f32(xy)
        v = None if v is None else _f32(v)
        volumes = None if volumes is None else np.ascontiguousarray(volumes, np.float32)
        _check(lib.emerald_batch_set_solid(self._h, sid, _ptr(xy), _ptr(v), _ptr(volumes)),
               "set_solid")

    def set_forces(self, sid, terms):
        """Device force terms of one scene (emerald_batch_set_forces)."""
        arr = force_terms(terms)
        _check(lib.emerald_batch_set_forces(self._h, sid, ctypes.cast(arr, c_vp), len(terms)),
               "set_forces")

    def free(self):
        n = c_sz()
        k = c_i32()
        _check(lib.emerald_batch_free(self._h, ctypes.byref(n), ctypes.byref(k)), "batch_free")
        return n.value, k.value

    def set_stream(self, stream_ptr):
        _check(lib.emerald_batch_set_stream(self._h, stream_ptr), "set_stream")

    def synchronize(self):
        _check(lib.emerald_batch_synchronize(self._h), "synchronize")

    def kernel_launches(self):
        n = c_i64()
        _check(lib.emerald_batch_kernel_launches(self._h, ctypes.byref(n)), "kernel_launches")
        return n.value

    def autotune(self, method):
        t = Tuning()
        _check(lib.emerald_batch_autotune(self._h, method_id(method), ctypes.byref(t)), "autotune")
        return t.as_dict()

    def set_tuning(self, chunks=None, prefetch=None):
        t = _tuning_struct(chunks, prefetch)
        _check(lib.emerald_batch_set_tuning(self._h, None if t is None else ctypes.byref(t)),
               "set_tuning")


class Server:
    """Request loop over one batch arena sized from a device-memory budget:
    submitted scenes are admitted as room frees up, stepped together with
    every resident scene, and retired when their sub-steps are done."""

    ENOSPC = 28
    ETIMEOUT = 110
    ECANCELED = 125

    def __init__(self, hbm_budget_bytes, method="dfsph_p", max_scenes=256,
                 max_substeps_per_launch=8, lanes=4, order="arrival"):
        cfg = ServerConfig(int(hbm_budget_bytes), method_id(method), int(max_scenes),
                           int(max_substeps_per_launch), int(lanes),
                           {"arrival": 0, "largest_first": 1}[order])
        h = c_vp()
        _check(lib.emerald_server_create(ctypes.byref(cfg), ctypes.byref(h)),
               "emerald_server_create")
        self._h = h
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.emerald_server_destroy(self._h)
            self._h = c_vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, params, solid_xy, fluid_xy, n_substeps, fluid_v=None, solid_volumes=None):
        """Queues a request and returns its id (None if it can never fit)."""
        s = _f32(solid_xy).reshape(-1, 2)
        f = _f32(fluid_xy).reshape(-1, 2)
        v = None if fluid_v is None else _f32(fluid_v).reshape(-1, 2)
        vol = None if solid_volumes is None else _f32(solid_volumes)
        rid = c_i64()
        rc = lib.emerald_server_submit(self._h, ctypes.byref(params), _ptr(s), _ptr(vol), len(s),
                                       _ptr(f), _ptr(v), len(f), int(n_substeps),
                                       ctypes.byref(rid))
        if rc == self.ENOSPC:
            return None
        _check(rc, "emerald_server_submit")
        self._sizes[rid.value] = len(f)
        return rid.value

    def submit_block_scene(self, scene, n_substeps):
        return self.submit(scene.params, scene.solid, scene.fluid, n_substeps,
                           solid_volumes=scene.solid_volumes)

    def wait(self, rid, timeout_ms=-1):
        """(x, v, stats, timing) of a finished request, or None on timeout."""
        n = self._sizes.get(rid, 0)
        x = np.zeros((n, 2), np.float32)
        v = np.zeros((n, 2), np.float32)
        st = StepStats()
        tm = RequestTiming()
        rc = lib.emerald_server_wait(self._h, rid, int(timeout_ms), _ptr(x), _ptr(v),
                                     ctypes.byref(st), ctypes.byref(tm))
        if rc == self.ETIMEOUT:
            return None
        _check(rc, "emerald_server_wait")
        self._sizes.pop(rid, None)
        return x, v, st.as_dict(), {k: getattr(tm, k) for k, _ in tm._fields_}

    def stats(self):
        out = ServerStats()
        _check(lib.emerald_server_get_stats(self._h, ctypes.byref(out)), "server_stats")
        return out.as_dict()

    def cancel(self, rid):
        """Cancels a queued, resident or finished request; wait() then
        raises EmeraldError with code ECANCELED for it."""
        _check(lib.emerald_server_cancel(self._h, int(rid)), "emerald_server_cancel")
