"""Host-side parts of the product library that need no GPU: the C ABI
exports, parameter validation, configuration and scene generators."""
import ctypes
import os
import re

import numpy as np
import pytest

import emerald_b200 as E
from conftest import assert_bitwise
from scenes import F, lattice_template, walls

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def header_symbols():
    text = open(os.path.join(ROOT, "include", "emerald_sph.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(emerald_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(E.LIB_PATH)
    names = header_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_header():
    assert set(header_symbols()) == set(E.EXPORTS)


def header_arities():
    text = open(os.path.join(ROOT, "include", "emerald_sph.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(emerald_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_bindings_match_header_arity():
    """Each binding's argument list has as many entries as the prototype."""
    arity = header_arities()
    wrong = {n: (arity[n], len(E.EXPORTS[n][1])) for n in arity
             if len(E.EXPORTS[n][1]) != arity[n]}
    assert not wrong, wrong


@pytest.mark.parametrize("x,y,z", [(0b111, 0b111, 0b111111), (0xFFFF, 0xFFFF, 0xFFFFFFFF),
                                   (0, 0xFFFF, 0xAAAAAAAA),
                                   (0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFFFFFFFFFF)])
def test_z_index(x, y, z):
    assert E.z_index(x, y) == z


def test_invalid_arguments_return_einval():
    p = E.default_params(support=0.0)
    h = ctypes.c_void_p()
    rc = E.lib.emerald_sim_create(ctypes.byref(p), None, None, 0, None, None, 0, ctypes.byref(h))
    assert rc == 22
    assert b"support" in E.lib.emerald_last_error()
    p = E.default_params()
    rc = E.lib.emerald_sim_create(ctypes.byref(p), None, None, 5, None, None, 0, ctypes.byref(h))
    assert rc == 22
    assert E.lib.emerald_sim_sub_step(None, 1, 0.0, 1e-4, None) == 22
    assert E.lib.emerald_sim_frame(None, 9, None) == 22


def test_default_config_matches_reference_values():
    c = E.config(E.default_params())
    # emerald/sph2d_box/config.cpp for the default Parameters
    assert c["seconds_per_sub_step"] == F(1.0 / 900.0)
    assert c["draw_radius"] == F(0.99) * (F(0.025) * F(0.5))


def test_config_matches_reference(reference):
    for sup in (0.025, 0.01, 1 / 512, 1 / 2048):
        p = E.default_params(support=F(sup))
        rp = reference.default_params()
        rp["support"] = F(sup)
        a = E.config(p)
        b = reference.config(rp)
        for k in a:
            assert F(a[k]) == F(b[k]), (sup, k)


def test_lattice_config_matches_restatement(oracle):
    for dx in (F(1 / 64), F(1 / 1024)):
        p = E.default_params(support=dx)
        got = E.lattice_config(p, dx, F(5e-4))
        want = lattice_template(oracle.kernel_w, oracle.kernel_grad_w, oracle.L.oracle_vec2_length,
                                dx, dx, 1000.0, F(5e-4))
        assert F(got[0]) == F(want[0]) and F(got[1]) == F(want[1])


def test_block_scene_and_walls_match_golden():
    g = dict(np.load(os.path.join(GOLDEN, "run_iisph.npz")))
    dx = F(1 / 48)
    assert_bitwise(E.block_scene(24, 24, dx), g["fluid"], "block scene")
    assert_bitwise(E.wall_scene(dx), g["solid"], "walls")
    assert_bitwise(E.wall_scene(dx), walls(dx), "walls restated")
    m, d = E.lattice_config(E.default_params(support=dx), dx, F(352800 / 705600000.0))
    assert F(m) == F(g["mass"]) and F(d) == F(g["denom"])


def test_reference_scene_generators_match_golden():
    g = dict(np.load(os.path.join(GOLDEN, "frames_default.npz")))
    p = E.default_params()
    ww = E.world_walls(p)
    assert_bitwise(ww, g["solid"], "world walls")
    assert_bitwise(E.dam_break(p, ww), g["fluid"], "dam break")


def test_block_scene_matches_reference_generator(reference):
    a = E.block_scene(33, 17, F(1 / 100), 0.25, 0.5, 0.02, 11)
    b = reference.block_scene(33, 17, F(1 / 100), 0.25, 0.5, 0.02, 11)
    assert_bitwise(a, b, "block scene")


def test_dropin_header_compiles():
    """include/emerald_sph.hpp compiles against a caller spelled like the
    reference's EZ_EXAMPLE_SIM::step and links against the library."""
    import shutil
    import subprocess
    import tempfile
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "emerald_b200")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "step_dropin")
        r = subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                            os.path.join(root, "include"),
                            os.path.join(root, "tests", "cpp", "step_dropin.cpp"), "-L", lib,
                            "-lemerald_b200", "-o", out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_non_finite_inputs_are_rejected_before_any_device_work():
    """emerald_sim_create screens its host arrays (positions, velocities,
    boundary positions and volumes) and the parameters for infinities and
    NaNs and returns EMERALD_EINVAL naming the array, before it touches a
    device (so this runs without a GPU)."""
    p = E.default_params()
    fluid = np.array([[0.1, 0.1], [0.2, 0.1], [0.3, 0.1]], np.float32)
    solid = np.array([[0.0, -0.01], [0.1, -0.01]], np.float32)
    h = ctypes.c_void_p()

    def create(f, v, s, vol, params=p):
        return E.lib.emerald_sim_create(ctypes.byref(params), E._ptr(s), E._ptr(vol), len(s),
                                        E._ptr(f), E._ptr(v), len(f), ctypes.byref(h))

    bad = fluid.copy()
    bad[1, 0] = np.nan
    assert create(bad, None, solid, None) == 22
    assert b"fluid positions" in E.lib.emerald_last_error()
    v = np.zeros_like(fluid)
    v[2, 1] = np.inf
    assert create(fluid, v, solid, None) == 22
    assert b"fluid velocities" in E.lib.emerald_last_error()
    s = solid.copy()
    s[0, 1] = -np.inf
    assert create(fluid, None, s, None) == 22
    assert b"boundary positions" in E.lib.emerald_last_error()
    vol = np.array([1.0, np.nan], np.float32)
    assert create(fluid, None, solid, vol) == 22
    assert b"boundary volumes" in E.lib.emerald_last_error()
    q = E.default_params(gravity=float("nan"))
    assert create(fluid, None, solid, None, q) == 22
    assert b"not finite" in E.lib.emerald_last_error()
    out = np.zeros(4, np.float32)
    assert E.lib.emerald_config(ctypes.byref(q), E._ptr(out)) == 22


def test_sort_entry_points_host_side():
    """The z-order sort and search entry points: the workspace size grows with
    n, a block map is created and destroyed on the host, and NULL arguments
    are refused before any device work (no GPU needed)."""
    import emerald_b200 as E
    sizes = []
    for n in (0, 1, 1000, 1 << 20):
        b = ctypes.c_size_t()
        assert E.lib.emerald_index_pairs_workspace(n, ctypes.byref(b)) == 0
        assert b.value > 0
        sizes.append(b.value)
    assert sizes == sorted(sizes) and sizes[-1] >= 16 << 20
    assert E.lib.emerald_index_pairs_workspace(1 << 33, ctypes.byref(ctypes.c_size_t())) == 22
    assert E.lib.emerald_index_pairs_workspace(10, None) == 22
    m = ctypes.c_void_p()
    assert E.lib.emerald_block_map_create(ctypes.byref(m)) == 0 and m.value
    assert E.lib.emerald_create_regular_neighborhoods(5, 0.1, None, None, None, None, None, None,
                                                      None, None, m.value, None) == 22
    # a map that was never filled is refused
    fake = ctypes.c_void_p(8)
    assert E.lib.emerald_create_regular_neighborhoods(5, 0.1, fake, fake, fake, fake, fake, fake,
                                                      fake, fake, m.value, None) == 22
    assert b"filled" in E.lib.emerald_last_error()
    assert E.lib.emerald_block_map_destroy(m.value) == 0
    assert E.lib.emerald_block_map_destroy(None) == 0
    assert E.lib.emerald_create_block_map(3, None, None, None, None) == 22
    assert E.lib.emerald_sort_index_pairs(10, None, None, 0, None) == 22
    assert E.lib.emerald_compute_block_indices(10, None, None, None, 0, None) == 22
