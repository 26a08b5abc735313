"""External forces against the compiled reference.

The reference computes external forces once per sub-step through
compute_all_external_forces (emerald/sph2d_box/forces.cpp:11-33) with the
caller's User_forces_function, at the start of the sub-step under IISPH,
IISPH_AP, IISPH_PSEUDO_AP and PCISPH and after the divergence solve under
DFSPH_P (dfsph_p.cpp:350). Here forces are either device terms (the
reference's gravity, pole-attraction and drag functions) or a host callback;
both must give the reference's frames bit for bit."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
METHODS = ["dfsph_p", "iisph", "iisph_ap", "iisph_pseudo_ap", "pcisph"]


def scene_pair(E, reference, seed=5):
    from cpu_checkers import RefParams
    sc = E.BlockScene(40, dx=F(1 / 80), seed=seed, time_per_step_flicks=1411200, sub_steps=4)
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=d["mass_per_particle"],
              pressure_correction_denom_override=d["pressure_correction_denom"])
    ref = reference.sim(rp, sc.solid, sc.fluid, None, sc.solid_volumes)
    sim = E.Simulation.from_block_scene(sc)
    return sc, sim, ref


def terms_for(E, sc):
    """Gravity, a pull to the tank's centre of a quarter of gravity (the
    reference's commented-out example, forces.cpp:24-28) and a drag."""
    g = F(sc.params.gravity)
    mass = F(sc.params.mass_per_particle)
    return [(E.FORCE_GRAVITY, g), (E.FORCE_POLE, F(0.25) * g * mass, 0.5, 0.5),
            (E.FORCE_DRAG, 0.025, F(sc.params.support))]


def compare(sim, ref, name, what):
    x, v = sim.state()
    rx, rv = ref.state()
    assert_bitwise(x, rx, "%s positions %s" % (name, what))
    assert_bitwise(v, rv, "%s velocities %s" % (name, what))


@pytest.mark.parametrize("method", METHODS)
def test_force_terms_match_reference(method):
    import emerald_b200 as E
    from cpu_checkers import Reference
    reference = Reference()
    sc, sim, ref = scene_pair(E, reference)
    terms = terms_for(E, sc)
    sim.set_forces(terms)
    ref.set_forces(terms)
    for f in range(2):
        sim.frame(method)
        ref.frame(method)
        compare(sim, ref, method, "after frame %d with gravity, pole and drag" % f)
    sim.close()


def test_no_force_terms_and_gravity_only():
    """No external force at all, then gravity alone from a term (the
    default scene's own force), frame by frame."""
    import emerald_b200 as E
    from cpu_checkers import Reference
    reference = Reference()
    sc, sim, ref = scene_pair(E, reference, seed=6)
    sim.set_forces([])
    ref.set_forces([])
    sim.frame("dfsph_p")
    ref.frame("dfsph_p")
    compare(sim, ref, "dfsph_p", "with no external force")
    sim.set_forces([(E.FORCE_GRAVITY, F(sc.params.gravity))])
    ref.set_forces([(1, F(sc.params.gravity))])
    sim.frame("dfsph_p")
    ref.frame("dfsph_p")
    compare(sim, ref, "dfsph_p", "with gravity from a term")
    sim.close()


def swirl(time, dt, mass, radius, f, x, v):
    """A host force that reads every argument: a pull to the centre growing
    with time, a drag scaled by radius / dt, and gravity."""
    f32 = np.float32
    k = f32(mass) * f32(1.0 + time)
    f[:, 0] += k * (f32(0.5) - x[:, 0]) - f32(radius) / f32(dt) * f32(1e-3) * v[:, 0]
    f[:, 1] += k * (f32(0.5) - x[:, 1]) - f32(mass) * f32(9.81)


def ref_callback(fn):
    import emerald_b200 as E

    def tramp(user, count, time, dt, mass, radius, f, x, v):
        view = lambda p: np.ctypeslib.as_array(p, shape=(count, 2))
        fn(time, dt, mass, radius, view(f), view(x), view(v))
    return E.FORCES_FN(tramp)


@pytest.mark.parametrize("method", ["dfsph_p", "iisph", "pcisph"])
def test_host_force_callback_matches_reference(method):
    import emerald_b200 as E
    from cpu_checkers import Reference
    reference = Reference()
    sc, sim, ref = scene_pair(E, reference, seed=7)
    calls = []

    def fn(time, dt, mass, radius, f, x, v):
        calls.append((time, dt))
        swirl(time, dt, mass, radius, f, x, v)

    sim.set_force_callback(fn)
    cb = ref_callback(swirl)
    ref.set_force_callback(cb)
    for k in range(2):
        st = sim.frame(method)
        ref.frame(method)
        compare(sim, ref, method, "after frame %d with a host force" % k)
    assert len(calls) >= 2 and all(dt > 0 for _, dt in calls)
    # removing the callback brings back the force terms (default gravity)
    sim.set_force_callback(None)
    ref.set_forces([(1, F(sc.params.gravity))])
    sim.frame(method)
    ref.frame(method)
    compare(sim, ref, method, "after the callback is removed")
    sim.close()


def test_fixed_dt_sub_steps_pass_the_callers_time():
    """emerald_sim_sub_step passes the caller's t to the force function, as
    the reference's sub-step passes its global_time_in_seconds."""
    import emerald_b200 as E
    from cpu_checkers import Reference
    reference = Reference()
    sc, sim, ref = scene_pair(E, reference, seed=8)
    seen = []

    def fn(time, dt, mass, radius, f, x, v):
        seen.append(time)
        swirl(time, dt, mass, radius, f, x, v)

    sim.set_force_callback(fn)
    ref.set_force_callback(ref_callback(swirl))
    sim.begin_frame("iisph")
    ref.begin_frame("iisph")
    for t in (0.25, 0.5):
        sim.sub_step("iisph", F(t), F(1e-4))
        ref.sub_step("iisph", F(t), F(1e-4))
    assert seen == [0.25, 0.5]
    compare(sim, ref, "iisph", "after fixed-dt sub-steps")
    sim.close()


def test_batch_scene_forces_are_per_scene():
    """Force terms belong to one scene of a batch; each scene equals itself
    run alone with the same forces."""
    import emerald_b200 as E
    a = E.BlockScene(32, dx=F(1 / 64), seed=9, time_per_step_flicks=1411200, sub_steps=4)
    b = E.BlockScene(24, dx=F(1 / 48), seed=10, time_per_step_flicks=1411200, sub_steps=4)
    batch = E.Batch(len(a.fluid) + len(b.fluid) + 256, len(a.solid) + len(b.solid) + 256, 2)
    ia = batch.add_block_scene(a)
    ib = batch.add_block_scene(b)
    ta = terms_for(E, a)
    batch.set_forces(ia, ta)
    batch.step("dfsph_p", 6)
    alone_a = E.Simulation.from_block_scene(a)
    alone_a.set_forces(ta)
    alone_a.advance("dfsph_p", 6)
    alone_b = E.Simulation.from_block_scene(b)
    alone_b.advance("dfsph_p", 6)
    for sid, alone in ((ia, alone_a), (ib, alone_b)):
        x, v = batch.state(sid)
        ax, av = alone.state()
        assert_bitwise(x, ax, "batched positions of scene %d" % sid)
        assert_bitwise(v, av, "batched velocities of scene %d" % sid)
    batch.close()
    alone_a.close()
    alone_b.close()


def test_force_terms_are_checked():
    import emerald_b200 as E
    sc = E.BlockScene(16, dx=F(1 / 32), seed=11)
    sim = E.Simulation.from_block_scene(sc)
    for bad in ([(7, 1.0)], [(E.FORCE_GRAVITY, float("nan"))], [(E.FORCE_GRAVITY, 1.0)] * 5):
        arr = E.force_terms(bad)
        rc = E.lib.emerald_sim_set_forces(sim._h, ctypes.cast(arr, ctypes.c_void_p), len(bad))
        assert rc == 22, bad
    sim.close()


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("forces") / "step_dropin")
    lib = os.path.join(ROOT, "emerald_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "step_dropin.cpp"), "-L", lib, "-lemerald_b200",
                    "-Wl,-rpath," + lib, "-o", out], check=True)
    return out


@pytest.mark.parametrize("mode", ["host", "device"])
@pytest.mark.parametrize("method", [("dfsph_p", 4), ("iisph", 1)])
def test_dropin_forces_match_reference(driver, tmp_path, mode, method):
    """A caller of the C++ drop-in with a pole force beside gravity, as a
    host lambda over the reference's accumulate functions or as device
    terms, against the compiled reference running the reference's own
    force functions on its default dam break."""
    from cpu_checkers import Reference
    name, mid = method
    path = str(tmp_path / "out.bin")
    subprocess.run([driver, str(mid), "2", path, "0", mode], check=True)
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    body = np.frombuffer(raw[8:], np.float32)
    x = body[:2 * n].reshape(n, 2)
    v = body[2 * n:4 * n].reshape(n, 2)
    reference = Reference()
    rp = reference.default_params()
    rp.update(mass_per_particle_override=0.0, pressure_correction_denom_override=0.0)
    ref = reference.sim(rp)
    g = F(rp["gravity"])
    mass = F(reference.config(rp)["mass_per_particle"])
    ref.set_forces([(1, g), (2, F(0.25) * g * mass, 0.5, 0.5)])
    for _ in range(2):
        ref.frame(name)
    rx, rv = ref.state()
    assert_bitwise(x, rx, "%s %s positions" % (name, mode))
    assert_bitwise(v, rv, "%s %s velocities" % (name, mode))
