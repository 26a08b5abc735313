"""The drop-in header's host force functions against the reference's own
(emerald/sph2d_box/forces.cpp:63-111), bit for bit, on the CPU: random
points plus the edge cases of the pole pull (a point exactly on the pole,
offsets small enough to take Imath's tiny-length rescale, signed zeros)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import assert_bitwise

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def host_forces(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("forces_host") / "forces_host")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "forces_host.cpp"),
                    "-o", out], check=True)
    return out


def points():
    rng = np.random.default_rng(31)
    x = rng.uniform(-0.5, 1.5, (4000, 2)).astype(np.float32)
    pole = np.float32([0.5, 0.5])
    tiny = np.float32(1e-20)
    edge = np.array([pole, pole + [tiny, 0], pole + [0, -tiny], pole + [tiny, tiny],
                     pole + [np.float32(1e-38), np.float32(3e-39)], [0.5, -0.0], [-0.0, 0.5],
                     pole + [np.float32(1e-19), np.float32(-2e-19)]], np.float32)
    x = np.concatenate([edge, x]).astype(np.float32)
    v = rng.normal(0, 2, x.shape).astype(np.float32)
    v[:3] = [[0.0, -0.0], [-0.0, 0.0], [1e-40, -1e-40]]
    f = rng.normal(0, 1, x.shape).astype(np.float32)
    return x, v, f


@pytest.mark.parametrize("terms", [
    [(1, 9.81, 0.0, 0.0)],
    [(2, 0.3, 0.5, 0.5)],
    [(3, 0.025, 0.01, 0.0)],
    [(1, 9.81, 0.0, 0.0), (2, 0.25, 0.5, 0.5), (3, 0.025, 0.004, 0.0), (2, -1.5, 0.0, 1.0)],
])
def test_header_force_functions_match_reference(reference, host_forces, tmp_path, terms):
    x, v, f0 = points()
    n = len(x)
    mass = np.float32(0.0123)
    inp = tmp_path / "in.bin"
    term_rec = np.zeros(len(terms), dtype=[("k", "<i4"), ("a", "<f4"), ("b", "<f4"), ("c", "<f4")])
    for i, t in enumerate(terms):
        term_rec[i] = t
    with open(inp, "wb") as fh:
        fh.write(np.uint64(n).tobytes() + np.uint64(len(terms)).tobytes() + mass.tobytes())
        fh.write(term_rec.tobytes())
        fh.write(x.tobytes() + v.tobytes() + f0.tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([host_forces, str(inp), str(out)], check=True)
    got = np.fromfile(out, np.float32).reshape(n, 2)

    L = reference.L
    L.ref_accumulate_forces.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_size_t, ctypes.c_float] + [ctypes.c_void_p] * 3
    kinds = np.array([t[0] for t in terms], np.int32)
    args = np.array([t[1:] for t in terms], np.float32)
    want = f0.copy()
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    L.ref_accumulate_forces(ptr(kinds), ptr(args), len(terms), n, mass, ptr(want), ptr(x), ptr(v))
    assert_bitwise(got, want, "forces %r" % (terms,))


def test_reference_gravity_term_equals_default_forces(reference):
    """The harness's term list with one gravity term is the reference's
    default_gravity_forces (the pin the GPU force tests rest on)."""
    import emerald_b200 as E
    from cpu_checkers import RefParams
    sc = E.BlockScene(24, dx=np.float32(1 / 48), seed=4, time_per_step_flicks=1411200,
                      sub_steps=4)
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=d["mass_per_particle"],
              pressure_correction_denom_override=d["pressure_correction_denom"])
    a = reference.sim(rp, sc.solid, sc.fluid, None, sc.solid_volumes)
    b = reference.sim(rp, sc.solid, sc.fluid, None, sc.solid_volumes)
    b.set_forces([(1, d["gravity"])])
    a.frame("dfsph_p")
    b.frame("dfsph_p")
    for u, w in zip(a.state(), b.state()):
        assert_bitwise(u, w, "state")
