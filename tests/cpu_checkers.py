"""ctypes bindings for the CPU checkers (test infrastructure only).

``Oracle`` wraps oracle/liboracle_sph.so, the project's C restatement of the
reference SPH path. ``Reference`` wraps oracle/_ref/libemerald_ref.so, the
unmodified emerald sources compiled against project-written shims (present
only where it was built). Only tests, the smoke check and bench.py's CPU
baseline use these; the product never does.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle_sph.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libemerald_ref.so")

METHODS = {"pcisph": 0, "iisph": 1, "iisph_ap": 2, "iisph_pseudo_ap": 3, "dfsph_p": 4}

c_f = ctypes.c_float
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_u64 = ctypes.c_uint64
c_sz = ctypes.c_size_t
c_vp = ctypes.c_void_p


def ptr(a):
    return None if a is None else a.ctypes.data_as(c_vp)


def ensure_built():
    import sys
    sys.path.insert(0, ORACLE_DIR)
    try:
        import build_oracle
        build_oracle.build_oracle()
        build_oracle.build_reference()
    finally:
        sys.path.pop(0)


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("time_per_step_flicks", c_i64), ("sub_steps", c_i32), ("support", c_f),
        ("gravity", c_f), ("viscosity", c_f), ("target_density", c_f),
        ("iisph_max_pressure_iterations", c_i32), ("iisph_error_average_threshold", c_f),
        ("iisph_error_max_threshold", c_f), ("iisph_omega", c_f),
        ("dfsph_max_correction_iterations", c_i32),
        ("dfsph_density_error_average_threshold", c_f),
        ("dfsph_density_error_max_threshold", c_f),
        ("dfsph_divergence_error_average_threshold", c_f),
        ("dfsph_divergence_error_max_threshold", c_f),
        ("mass_per_particle", c_f), ("pressure_correction_denom", c_f),
        ("seconds_per_sub_step", c_f),
    ]


class OracleStats(ctypes.Structure):
    _fields_ = [("pressure_iterations", c_i32), ("divergence_iterations", c_i32),
                ("error_average", c_f), ("error_max", c_f),
                ("divergence_error_average", c_f), ("divergence_error_max", c_f)]


class RefParams(ctypes.Structure):
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
        ("mass_per_particle_override", c_f), ("pressure_correction_denom_override", c_f),
    ]


_ARRAYS = ["densities", "pressures", "new_pressures", "density_stars", "aiis", "alphas",
           "divergence_kappas", "density_kappas", "fluid_volumes", "diis", "sum_dij_pjs",
           "external_forces", "pressure_forces", "pressure_accelerations",
           "velocity_external_forces", "position_stars", "velocity_stars"]


class Oracle:
    """The C restatement (oracle/sph_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            ensure_built()
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_z_index.restype = c_u64
        L.oracle_z_index.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_kernel_w.restype = c_f
        L.oracle_kernel_w.argtypes = [c_f, c_f]
        L.oracle_kernel_grad_w.argtypes = [c_f, c_f, c_f, c_vp]
        L.oracle_vec2_length.restype = c_f
        L.oracle_vec2_length.argtypes = [c_f, c_f]
        L.oracle_neighborhoods.argtypes = [c_vp, c_sz, c_vp, c_sz, ctypes.c_int, c_f,
                                           c_vp, c_vp, c_vp, c_vp]
        L.oracle_sort.restype = c_sz
        L.oracle_sort.argtypes = [c_vp, c_sz, c_f, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]
        L.oracle_solid_volumes.argtypes = [c_vp, c_sz, c_f, c_f, c_vp]
        L.oracle_sim_create.restype = c_vp
        L.oracle_sim_create.argtypes = [ctypes.POINTER(OracleParams), c_vp, c_vp, c_sz,
                                        c_vp, c_vp, c_sz]
        L.oracle_sim_destroy.argtypes = [c_vp]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_sim_begin_frame.argtypes = [c_vp, ctypes.c_int]
        L.oracle_sim_sub_step.argtypes = [c_vp, ctypes.c_int, c_f, c_f,
                                          ctypes.POINTER(OracleStats)]
        L.oracle_sim_frame.argtypes = [c_vp, ctypes.c_int]
        L.oracle_sim_time.restype = c_i64
        L.oracle_sim_time.argtypes = [c_vp]
        L.oracle_sim_get_state.argtypes = [c_vp, c_vp, c_vp]
        L.oracle_sim_set_state.argtypes = [c_vp, c_vp, c_vp]
        L.oracle_sim_get_array.argtypes = [c_vp, ctypes.c_char_p, c_vp]
        L.oracle_sim_get_neighbors.argtypes = [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp]
        self.L = L

    def z_index(self, x, y):
        return self.L.oracle_z_index(x & 0xFFFFFFFF, y & 0xFFFFFFFF)

    def kernel_w(self, r, h):
        return self.L.oracle_kernel_w(r, h)

    def kernel_grad_w(self, dx, dy, h):
        out = np.zeros(2, np.float32)
        self.L.oracle_kernel_grad_w(dx, dy, h, ptr(out))
        return out

    def neighborhoods(self, self_xy, other_xy, same_set, cell_size):
        self_xy = np.ascontiguousarray(self_xy, np.float32)
        other_xy = np.ascontiguousarray(other_xy, np.float32)
        n = len(self_xy)
        counts = np.zeros(n, np.uint8)
        idx = np.zeros((n, 64), np.uint32)
        dist = np.zeros((n, 64), np.float32)
        vec = np.zeros((n, 64, 2), np.float32)
        self.L.oracle_neighborhoods(ptr(self_xy), n, ptr(other_xy), len(other_xy),
                                    int(same_set), cell_size, ptr(counts), ptr(idx),
                                    ptr(dist), ptr(vec))
        return counts, idx, dist, vec

    def sort(self, xy, cell_size):
        xy = np.ascontiguousarray(xy, np.float32)
        n = len(xy)
        gc = np.zeros((n, 2), np.int32)
        z = np.zeros(n, np.uint64)
        pz = np.zeros(n, np.uint64)
        pi = np.zeros(n, np.uint64)
        bi = np.zeros(n, np.uint32)
        blocks = np.zeros((max(n, 1), 2), np.uint64)
        nb = self.L.oracle_sort(ptr(xy), n, cell_size, ptr(gc), ptr(z), ptr(pz), ptr(pi),
                                ptr(bi), ptr(blocks))
        return dict(grid_coords=gc, z_indices=z, pair_z=pz, pair_index=pi,
                    block_indices=bi, blocks=blocks[:nb])

    def solid_volumes(self, xy, support, numer=1.7):
        xy = np.ascontiguousarray(xy, np.float32)
        out = np.zeros(len(xy), np.float32)
        self.L.oracle_solid_volumes(ptr(xy), len(xy), support, numer, ptr(out))
        return out

    def set_threads(self, n):
        self.L.oracle_set_threads(n)

    def sim(self, params, solid_xy, solid_volumes, fluid_xy, fluid_v=None):
        return OracleSim(self, params, solid_xy, solid_volumes, fluid_xy, fluid_v)


class OracleSim:
    def __init__(self, lib, params, solid_xy, solid_volumes, fluid_xy, fluid_v):
        self.lib = lib
        L = lib.L
        p = OracleParams()
        for name, _ in OracleParams._fields_:
            setattr(p, name, params[name])
        self._solid = np.ascontiguousarray(solid_xy, np.float32)
        self._vol = None if solid_volumes is None else np.ascontiguousarray(solid_volumes, np.float32)
        fx = np.ascontiguousarray(fluid_xy, np.float32)
        fv = None if fluid_v is None else np.ascontiguousarray(fluid_v, np.float32)
        self.n = len(fx)
        self.h = L.oracle_sim_create(ctypes.byref(p), ptr(self._solid), ptr(self._vol),
                                     len(self._solid), ptr(fx), ptr(fv), self.n)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.oracle_sim_destroy(self.h)
            self.h = None

    def begin_frame(self, method):
        assert self.lib.L.oracle_sim_begin_frame(self.h, METHODS.get(method, method)) == 0

    def sub_step(self, method, t, dt):
        st = OracleStats()
        assert self.lib.L.oracle_sim_sub_step(self.h, METHODS.get(method, method), t, dt,
                                              ctypes.byref(st)) == 0
        return {k: getattr(st, k) for k, _ in OracleStats._fields_}

    def frame(self, method):
        return self.lib.L.oracle_sim_frame(self.h, METHODS.get(method, method))

    def time(self):
        return self.lib.L.oracle_sim_time(self.h)

    def state(self):
        x = np.zeros((self.n, 2), np.float32)
        v = np.zeros((self.n, 2), np.float32)
        self.lib.L.oracle_sim_get_state(self.h, ptr(x), ptr(v))
        return x, v

    def set_state(self, x=None, v=None):
        x = None if x is None else np.ascontiguousarray(x, np.float32)
        v = None if v is None else np.ascontiguousarray(v, np.float32)
        self.lib.L.oracle_sim_set_state(self.h, ptr(x), ptr(v))

    def array(self, name):
        w = self.lib.L.oracle_sim_get_array(self.h, name.encode(), None)
        if w < 0:
            raise KeyError(name)
        n = len(self._solid) if name == "solid_volumes" else self.n
        out = np.zeros((n, w) if w > 1 else n, np.float32)
        self.lib.L.oracle_sim_get_array(self.h, name.encode(), ptr(out))
        return out

    def neighbors(self, solid=False):
        counts = np.zeros(self.n, np.uint8)
        idx = np.zeros((self.n, 64), np.uint32)
        w = np.zeros((self.n, 64), np.float32)
        gw = np.zeros((self.n, 64, 2), np.float32)
        self.lib.L.oracle_sim_get_neighbors(self.h, int(solid), ptr(counts), ptr(idx),
                                            ptr(w), ptr(gw))
        return counts, idx, w, gw


class Reference:
    """The unmodified emerald reference built against shims (oracle/_ref)."""

    available = os.path.exists(REF_SO)

    def __init__(self):
        L = ctypes.CDLL(REF_SO)
        L.ref_z_index.restype = c_u64
        L.ref_z_index.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.ref_default_params.argtypes = [ctypes.POINTER(RefParams)]
        L.ref_config.argtypes = [ctypes.POINTER(RefParams), c_vp]
        L.ref_kernel_w.restype = c_f
        L.ref_kernel_w.argtypes = [c_f, c_f]
        L.ref_kernel_grad_w.argtypes = [c_f, c_f, c_f, c_vp]
        L.ref_vec2_length.restype = c_f
        L.ref_vec2_length.argtypes = [c_f, c_f]
        L.ref_block_scene.argtypes = [ctypes.c_uint32, ctypes.c_uint32, c_f, c_f, c_f, c_f,
                                      c_u64, c_vp]
        L.ref_uniform_points.argtypes = [c_sz, c_u64, c_f, c_f, c_vp]
        L.ref_lattice_config.argtypes = [ctypes.POINTER(RefParams), c_f, c_f, c_vp]
        L.ref_wall_scene.restype = c_sz
        L.ref_wall_scene.argtypes = [c_f, c_f, ctypes.c_int, c_vp]
        L.ref_sim_set_forces.argtypes = [c_vp, c_vp, c_vp, ctypes.c_int]
        L.ref_sim_set_force_callback.argtypes = [c_vp, c_vp, c_vp]
        L.ref_sim_run_window.restype = c_i64
        L.ref_sim_run_window.argtypes = [c_vp, ctypes.c_int, c_i64, c_i64, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_double)]
        L.ref_sim_create.restype = c_vp
        L.ref_sim_create.argtypes = [ctypes.POINTER(RefParams), c_vp, c_sz, c_vp, c_vp, c_sz]
        L.ref_sim_destroy.argtypes = [c_vp]
        L.ref_sim_fluid_count.restype = c_sz
        L.ref_sim_fluid_count.argtypes = [c_vp]
        L.ref_sim_solid_count.restype = c_sz
        L.ref_sim_solid_count.argtypes = [c_vp]
        L.ref_sim_get_solid.argtypes = [c_vp, c_vp, c_vp]
        L.ref_sim_set_solid_volumes.argtypes = [c_vp, c_vp]
        L.ref_sim_time.restype = c_i64
        L.ref_sim_time.argtypes = [c_vp]
        L.ref_sim_begin_frame.argtypes = [c_vp, ctypes.c_int]
        L.ref_sim_sub_step.argtypes = [c_vp, ctypes.c_int, c_f, c_f]
        L.ref_sim_frame.argtypes = [c_vp, ctypes.c_int]
        L.ref_sim_get_state.argtypes = [c_vp, c_vp, c_vp]
        L.ref_sim_set_solid.argtypes = [c_vp, c_vp, c_vp, c_vp]
        L.ref_sim_set_state.argtypes = [c_vp, c_vp, c_vp]
        L.ref_sim_get_array.argtypes = [c_vp, ctypes.c_char_p, c_vp]
        L.ref_sim_get_neighbors.argtypes = [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp,
                                            c_vp]
        L.ref_sim_get_sort.restype = c_sz
        L.ref_sim_get_sort.argtypes = [c_vp, ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]
        L.ref_self_neighborhoods.argtypes = [c_vp, c_sz, c_f, c_vp, c_vp, c_vp, c_vp, c_vp,
                                             c_vp, c_vp, c_vp]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_density_error.restype = c_f
        L.ref_max_density_error.argtypes = [c_sz, c_f, c_vp]
        L.ref_max_vector_squared_magnitude.restype = c_f
        L.ref_max_vector_squared_magnitude.argtypes = [c_sz, c_vp]
        L.ref_cfl_maximum_time_step.restype = c_i64
        L.ref_cfl_maximum_time_step.argtypes = [c_sz, c_f, c_f, c_vp]
        # the sph_common functions on flat arrays (row-major 64-entry lists)
        L.ref_common_grid_coords.argtypes = [c_sz, c_f, c_f, c_f, c_vp, c_vp]
        L.ref_common_z_indices.argtypes = [c_sz, c_vp, c_vp]
        L.ref_common_index_pairs.argtypes = [c_sz, c_vp, c_vp]
        L.ref_common_sort_index_pairs.argtypes = [c_sz, c_vp]
        L.ref_common_block_indices.argtypes = [c_sz, c_vp, c_vp]
        L.ref_common_fill_blocks.argtypes = [c_sz, c_sz, c_vp, c_vp]
        L.ref_common_regular_neighborhoods.argtypes = [c_sz, c_sz, c_f] + [c_vp] * 7 + \
            [ctypes.c_int, c_sz, c_vp, c_sz, c_vp]
        L.ref_common_distances_vectors.argtypes = [c_sz, c_sz, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]
        L.ref_common_kernels.argtypes = [c_sz, c_f, c_vp, c_vp, c_vp, c_vp, c_vp]
        L.ref_common_densities.argtypes = [c_sz, c_f, c_f] + [c_vp] * 9
        L.ref_common_divergences.argtypes = [c_sz, c_f] + [c_vp] * 8 + [c_sz] + [c_vp] * 3
        L.ref_common_density_stars.argtypes = [c_sz, c_f, c_f] + [c_vp] * 9 + [c_sz] + [c_vp] * 3
        L.ref_common_apply_pressures.argtypes = [c_sz, c_f, c_f] + [c_vp] * 11
        L.ref_common_pressure_accelerations.argtypes = [c_sz, c_f] + [c_vp] * 11
        L.ref_common_integrate.argtypes = [c_sz, c_f, c_f] + [c_vp] * 7
        L.ref_common_constant_volumes.argtypes = [c_sz, c_f, c_f, c_vp]
        L.ref_common_average_and_max.argtypes = [c_sz, c_f, c_vp, c_vp]
        # the solver operator functions; neighbour sets by pointer to six
        # pointers (RefNb)
        L.ref_ops_iisph_diis.argtypes = [c_sz, c_f, c_f] + [c_vp] * 6
        L.ref_ops_iisph_aiis_stars.argtypes = [c_sz, c_f, c_f] + [c_vp] * 9 + [c_sz, c_vp]
        L.ref_ops_iisph_sum_dij_pjs.argtypes = [c_sz, c_f, c_f] + [c_vp] * 5
        L.ref_ops_iisph_betas.argtypes = [c_sz, c_f, c_f] + [c_vp] * 9
        L.ref_ops_iisph_new_pressures.argtypes = [c_sz, c_f, c_f] + [c_vp] * 5
        L.ref_ops_dfsph_shared_coeffs.argtypes = [c_sz, c_f] + [c_vp] * 6
        L.ref_ops_dfsph_pseudo_pressures.argtypes = [c_sz, c_f, c_f] + [c_vp] * 5
        L.ref_ops_pcisph_densities.argtypes = [c_sz, c_f, c_f, c_f] + [c_vp] * 4
        L.ref_ops_pcisph_update_pressures.argtypes = [c_sz, c_f, c_f, c_vp, c_vp]
        L.ref_ops_pcisph_forces.argtypes = [c_sz, c_f, c_f, c_f, c_f] + [c_vp] * 7
        L.ref_ops_ap_stars_diagonals.argtypes = [ctypes.c_int, c_sz, c_f, c_f] + [c_vp] * 8 + \
            [c_sz, c_vp]
        L.ref_ops_ap_iterate.argtypes = [c_sz, c_f, c_f, c_f] + [c_vp] * 9
        L.ref_ops_pseudo_displacements.argtypes = [c_sz, c_f] + [c_vp] * 7
        L.ref_ops_pseudo_iterate.argtypes = [c_sz, c_f, c_f] + [c_vp] * 9
        L.ref_ops_pseudo_integrate.argtypes = [c_sz, c_f, c_vp, c_vp, c_vp]
        self.L = L

    def default_params(self):
        p = RefParams()
        self.L.ref_default_params(ctypes.byref(p))
        return {k: getattr(p, k) for k, _ in RefParams._fields_}

    def config(self, params):
        p = self._params(params)
        out = np.zeros(4, np.float32)
        self.L.ref_config(ctypes.byref(p), ptr(out))
        return dict(seconds_per_sub_step=out[0], mass_per_particle=out[1], draw_radius=out[2],
                    pressure_correction_denom=out[3])

    @staticmethod
    def _params(params):
        p = RefParams()
        for name, _ in RefParams._fields_:
            setattr(p, name, params[name])
        return p

    def z_index(self, x, y):
        return self.L.ref_z_index(x & 0xFFFFFFFF, y & 0xFFFFFFFF)

    def block_scene(self, nx, ny, dx, x0=0.0, y0=0.0, jitter=0.01, seed=1):
        xy = np.zeros((nx * ny, 2), np.float32)
        self.L.ref_block_scene(nx, ny, dx, x0, y0, jitter, seed, ptr(xy))
        return xy

    def lattice_config(self, params, dx, dt):
        """(mass_per_particle, pressure_correction_denom) of a square lattice
        at spacing dx, from the reference's kernels."""
        out = np.zeros(2, np.float32)
        self.L.ref_lattice_config(ctypes.byref(self._params(params)), dx, dt, ptr(out))
        return out[0], out[1]

    def wall_scene(self, dx, length=1.0, layers=3):
        n = self.L.ref_wall_scene(dx, length, layers, None)
        xy = np.zeros((n, 2), np.float32)
        self.L.ref_wall_scene(dx, length, layers, ptr(xy))
        return xy

    def uniform_points(self, n, seed, lo, hi):
        xy = np.zeros((n, 2), np.float32)
        self.L.ref_uniform_points(n, seed, lo, hi, ptr(xy))
        return xy

    def self_neighborhoods(self, xy, cell_size):
        xy = np.ascontiguousarray(xy, np.float32)
        n = len(xy)
        out = dict(grid_coords=np.zeros((n, 2), np.int32), z_indices=np.zeros(n, np.uint64),
                   pair_index=np.zeros(n, np.uint64), block_indices=np.zeros(n, np.uint32),
                   counts=np.zeros(n, np.uint8), idx=np.zeros((n, 64), np.uint32),
                   dist=np.zeros((n, 64), np.float32), vec=np.zeros((n, 64, 2), np.float32))
        self.L.ref_self_neighborhoods(ptr(xy), n, cell_size, ptr(out["grid_coords"]),
                                      ptr(out["z_indices"]), ptr(out["pair_index"]),
                                      ptr(out["block_indices"]), ptr(out["counts"]),
                                      ptr(out["idx"]), ptr(out["dist"]), ptr(out["vec"]))
        return out

    def set_threads(self, n):
        self.L.ref_set_threads(n)

    def sim(self, params, solid_xy=None, fluid_xy=None, fluid_v=None, solid_volumes=None):
        return RefSim(self, params, solid_xy, fluid_xy, fluid_v, solid_volumes)


class RefSim:
    def __init__(self, lib, params, solid_xy, fluid_xy, fluid_v, solid_volumes):
        self.lib = lib
        L = lib.L
        p = Reference._params(params)
        s = None if solid_xy is None else np.ascontiguousarray(solid_xy, np.float32)
        f = None if fluid_xy is None else np.ascontiguousarray(fluid_xy, np.float32)
        v = None if fluid_v is None else np.ascontiguousarray(fluid_v, np.float32)
        self.h = L.ref_sim_create(ctypes.byref(p), ptr(s), 0 if s is None else len(s), ptr(f),
                                  ptr(v), 0 if f is None else len(f))
        self.n = L.ref_sim_fluid_count(self.h)
        self.ns = L.ref_sim_solid_count(self.h)
        if solid_volumes is not None:
            vol = np.ascontiguousarray(solid_volumes, np.float32)
            assert len(vol) == self.ns
            L.ref_sim_set_solid_volumes(self.h, ptr(vol))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.ref_sim_destroy(self.h)
            self.h = None

    def solid(self):
        xy = np.zeros((self.ns, 2), np.float32)
        vol = np.zeros(self.ns, np.float32)
        self.lib.L.ref_sim_get_solid(self.h, ptr(xy), ptr(vol))
        return xy, vol

    def begin_frame(self, method):
        assert self.lib.L.ref_sim_begin_frame(self.h, METHODS.get(method, method)) == 0

    def sub_step(self, method, t, dt):
        assert self.lib.L.ref_sim_sub_step(self.h, METHODS.get(method, method), t, dt) == 0

    def frame(self, method):
        assert self.lib.L.ref_sim_frame(self.h, METHODS.get(method, method)) == 0

    def set_forces(self, terms):
        """The reference's force functions in order, (kind, a, b, c) tuples:
        1 gravity, 2 constant pole attraction, 3 simple drag."""
        kinds = np.array([t[0] for t in terms] or [0], np.int32)
        args = np.array([(tuple(t[1:]) + (0.0,) * 3)[:3] for t in terms] or [(0, 0, 0)],
                        np.float32)
        self.lib.L.ref_sim_set_forces(self.h, ptr(kinds), ptr(args), len(terms))

    def set_force_callback(self, cfunc):
        """A ctypes emerald_forces_fn-compatible callback as the
        User_forces_function; the caller keeps `cfunc` alive."""
        self._cb = cfunc
        self.lib.L.ref_sim_set_force_callback(self.h, ctypes.cast(cfunc, c_vp), None)

    def run_window(self, method, skip, count, max_seconds=0.0):
        """Adaptive frames through the reference's frame loop; sub-steps
        [skip, skip + count) since creation timed one by one (ended early once
        max_seconds > 0 is passed). Returns (sub-steps timed, seconds)."""
        sec = ctypes.c_double(0.0)
        k = self.lib.L.ref_sim_run_window(self.h, METHODS.get(method, method), skip, count,
                                          max_seconds, ctypes.byref(sec))
        assert k >= 0
        return int(k), sec.value

    def time(self):
        return self.lib.L.ref_sim_time(self.h)

    def state(self):
        x = np.zeros((self.n, 2), np.float32)
        v = np.zeros((self.n, 2), np.float32)
        self.lib.L.ref_sim_get_state(self.h, ptr(x), ptr(v))
        return x, v

    def set_state(self, x=None, v=None):
        x = None if x is None else np.ascontiguousarray(x, np.float32)
        v = None if v is None else np.ascontiguousarray(v, np.float32)
        self.lib.L.ref_sim_set_state(self.h, ptr(x), ptr(v))

    def set_solid(self, xy=None, v=None, volumes=None):
        xy = None if xy is None else np.ascontiguousarray(xy, np.float32)
        v = None if v is None else np.ascontiguousarray(v, np.float32)
        volumes = None if volumes is None else np.ascontiguousarray(volumes, np.float32)
        self.lib.L.ref_sim_set_solid(self.h, ptr(xy), ptr(v), ptr(volumes))

    def array(self, name):
        w = self.lib.L.ref_sim_get_array(self.h, name.encode(), None)
        if w < 0:
            raise KeyError(name)
        if w == 0:
            return None
        out = np.zeros((self.n, w) if w > 1 else self.n, np.float32)
        self.lib.L.ref_sim_get_array(self.h, name.encode(), ptr(out))
        return out

    def neighbors(self, solid=False):
        n = self.n
        counts = np.zeros(n, np.uint8)
        idx = np.zeros((n, 64), np.uint32)
        dist = np.zeros((n, 64), np.float32)
        vec = np.zeros((n, 64, 2), np.float32)
        w = np.zeros((n, 64), np.float32)
        gw = np.zeros((n, 64, 2), np.float32)
        self.lib.L.ref_sim_get_neighbors(self.h, int(solid), ptr(counts), ptr(idx), ptr(dist),
                                         ptr(vec), ptr(w), ptr(gw))
        return counts, idx, w, gw

    def sort(self, solid=False):
        n = self.ns if solid else self.n
        gc = np.zeros((n, 2), np.int32)
        z = np.zeros(n, np.uint64)
        pz = np.zeros(n, np.uint64)
        pi = np.zeros(n, np.uint64)
        bi = np.zeros(n, np.uint32)
        blocks = np.zeros((max(n, 1), 2), np.uint64)
        nb = self.lib.L.ref_sim_get_sort(self.h, int(solid), ptr(gc), ptr(z), ptr(pz), ptr(pi),
                                         ptr(bi), ptr(blocks))
        return dict(grid_coords=gc, z_indices=z, pair_z=pz, pair_index=pi, block_indices=bi,
                    blocks=blocks[:nb])


class FP64Oracle:
    """The FP64 GPU oracle of the DFSPH_P and IISPH sub-steps
    (oracle/fp64/dfsph_fp64.cu): the same formulas and list order in double,
    driven with each FP32 sub-step's dt and iteration counts."""

    path = os.path.join(ORACLE_DIR, "libfp64_oracle.so")

    class Params(ctypes.Structure):
        _fields_ = [("support", ctypes.c_double), ("rho0", ctypes.c_double),
                    ("mass", ctypes.c_double), ("fluid_volume", ctypes.c_double),
                    ("gravity", ctypes.c_double)]

    def __init__(self):
        lib = ctypes.CDLL(self.path)
        vp = ctypes.c_void_p
        lib.fp64_create.argtypes = [ctypes.POINTER(FP64Oracle.Params), vp, vp, ctypes.c_size_t,
                                    vp, vp, ctypes.c_size_t, ctypes.POINTER(vp)]
        lib.fp64_destroy.argtypes = [vp]
        lib.fp64_sub_step.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int]
        lib.fp64_sub_step_iisph.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        lib.fp64_sub_step_ap.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int]
        lib.fp64_sub_step_pcisph.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double]
        lib.fp64_get.argtypes = [vp, ctypes.c_char_p, vp]
        self.lib = lib

    def sim(self, support, rho0, mass, gravity, solid_xy, solid_vols, fluid_xy, fluid_v=None):
        return FP64Sim(self, support, rho0, mass, gravity, solid_xy, solid_vols, fluid_xy, fluid_v)


class FP64Sim:
    def __init__(self, o, support, rho0, mass, gravity, solid_xy, solid_vols, fluid_xy, fluid_v):
        self.o = o
        p = FP64Oracle.Params(float(support), float(rho0), float(mass),
                              float(mass) / float(rho0), float(gravity))
        s = np.ascontiguousarray(solid_xy, np.float64).reshape(-1, 2)
        sv = np.ascontiguousarray(solid_vols, np.float64)
        f = np.ascontiguousarray(fluid_xy, np.float64).reshape(-1, 2)
        v = None if fluid_v is None else np.ascontiguousarray(fluid_v, np.float64).reshape(-1, 2)
        h = ctypes.c_void_p()
        rc = o.lib.fp64_create(ctypes.byref(p), s.ctypes.data, sv.ctypes.data, len(s),
                               f.ctypes.data, None if v is None else v.ctypes.data, len(f),
                               ctypes.byref(h))
        assert rc == 0, rc
        self.h = h
        self.n = len(f)

    def sub_step(self, dt, new_frame, div_iters, dens_iters):
        rc = self.o.lib.fp64_sub_step(self.h, float(dt), int(new_frame), int(div_iters),
                                      int(dens_iters))
        assert rc == 0, rc

    def sub_step_iisph(self, dt, iters, omega):
        rc = self.o.lib.fp64_sub_step_iisph(self.h, float(dt), int(iters), float(omega))
        assert rc == 0, rc

    def sub_step_ap(self, dt, iters, omega, pseudo):
        rc = self.o.lib.fp64_sub_step_ap(self.h, float(dt), int(iters), float(omega), int(pseudo))
        assert rc == 0, rc

    def sub_step_pcisph(self, dt, passes, viscosity, denom):
        rc = self.o.lib.fp64_sub_step_pcisph(self.h, float(dt), int(passes), float(viscosity),
                                             float(denom))
        assert rc == 0, rc

    def get(self, name):
        w = 2 if name in ("x", "v") else 1
        out = np.zeros((self.n, w) if w > 1 else self.n, np.float64)
        rc = self.o.lib.fp64_get(self.h, name.encode(), out.ctypes.data)
        assert rc == 0, rc
        return out

    def close(self):
        if self.h:
            self.o.lib.fp64_destroy(self.h)
            self.h = None
