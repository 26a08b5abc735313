"""The C++ drop-in header: a caller written against the reference's step API
(tests/cpp/step_dropin.cpp) gives the same frames as the C ABI, which
test_gpu_parity.py pins to the reference's default dam break."""
import os
import subprocess

import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "step_dropin")
    lib = os.path.join(ROOT, "emerald_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "step_dropin.cpp"), "-L", lib, "-lemerald_b200",
                    "-Wl,-rpath," + lib, "-o", out], check=True)
    return out


@pytest.mark.parametrize("method", [("dfsph_p", 4), ("iisph", 1), ("pcisph", 0)])
def test_dropin_header_frames(driver, tmp_path, method):
    import emerald_b200 as E
    name, mid = method
    path = str(tmp_path / "out.bin")
    subprocess.run([driver, str(mid), "2", path], check=True)
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    body = np.frombuffer(raw[8:], np.float32)
    x = body[:2 * n].reshape(n, 2)
    v = body[2 * n:4 * n].reshape(n, 2)
    colors = body[4 * n:8 * n].reshape(n, 4)

    p = E.default_params()
    solid = E.world_walls(p)
    fluid = E.dam_break(p, solid)
    sim = E.Simulation(p, solid, fluid)
    for _ in range(2):
        sim.frame(name)
    gx, gv = sim.state()
    assert_bitwise(x, gx, "%s positions" % name)
    assert_bitwise(v, gv, "%s velocities" % name)
    rho = sim.array("densities")
    c = np.clip(np.float32(1.0) - rho / (np.float32(1.1) * np.float32(p.target_density)),
                np.float32(0.0), np.float32(1.0)).astype(np.float32)
    assert_bitwise(colors[:, 0], c, "%s colours" % name)
    assert np.all(colors[:, 2] == 1.0) and np.all(colors[:, 3] == 1.0)


@pytest.mark.parametrize("method", [("dfsph_p", 4), ("iisph", 1)])
def test_dropin_moving_wall(driver, tmp_path, method):
    """A caller that moves the left wall between step calls: the header
    passes the changed boundary on (emerald_sim_set_solid), and the frames
    equal the C ABI run with the same boundary per frame."""
    import emerald_b200 as E
    name, mid = method
    path = str(tmp_path / "out.bin")
    subprocess.run([driver, str(mid), "2", path, "-2.0"], check=True)
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    body = np.frombuffer(raw[8:], np.float32)
    x = body[:2 * n].reshape(n, 2)

    p = E.default_params()
    walls0 = E.world_walls(p)
    fluid = E.dam_break(p, walls0)
    left = walls0[:, 0] < 0
    step = np.float32(-2.0 * 0.002)
    v = np.zeros_like(walls0)
    v[left, 0] = np.float32(-2.0)
    sim = None
    for f in range(1, 3):
        xy = walls0.copy()
        xy[left, 0] = walls0[left, 0] + np.float32(f) * step
        if sim is None:
            sim = E.Simulation(p, xy, fluid)
            sim.set_solid(None, v, None)
        else:
            sim.set_solid(xy, v, None)
        sim.frame(name)
    assert left.any()
    assert_bitwise(x, sim.state()[0], "%s positions with a moving wall" % name)
    sim.close()
