"""The bench's reference arm builds its scene through the reference harness
alone (oracle/_ref), with no code of this library loaded. These CPU tests pin
that scene to the GPU arm's one bit for bit, and pin the harness's windowed
frame loop to the reference's whole frames, so that both arms time the same
sub-steps of the same trajectory."""
import numpy as np
import pytest

import bench
from conftest import assert_bitwise


@pytest.fixture(autouse=True)
def small_scene():
    bench.configure_scene(48)
    yield
    bench.configure_scene(512)


def test_reference_scene_equals_gpu_arm_scene(reference):
    import emerald_b200 as E
    rp, fluid, solid, volumes = bench.reference_scene(reference)
    scene = E.BlockScene(bench.N_SIDE, **bench.scene_kwargs())
    assert_bitwise(fluid, scene.fluid, "fluid positions")
    assert_bitwise(solid, scene.solid, "boundary positions")
    assert_bitwise(volumes, scene.solid_volumes, "boundary volumes")
    p = scene.params.as_dict()
    assert np.float32(rp["mass_per_particle_override"]).view(np.uint32) == \
        np.float32(p["mass_per_particle"]).view(np.uint32)
    assert np.float32(rp["pressure_correction_denom_override"]).view(np.uint32) == \
        np.float32(p["pressure_correction_denom"]).view(np.uint32)
    for k in rp:
        if k in p:
            a, b = rp[k], p[k]
            if isinstance(a, float) or isinstance(b, float):
                assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32), k
            else:
                assert a == b, k


def test_window_runs_the_reference_frame_loop(reference, oracle):
    """Sub-steps [2, k) of the windowed loop, k the sub-steps of two frames
    (counted by the C oracle's adaptive frames), leave the state the
    reference's own frame call leaves after two frames; a window that ends
    inside a frame runs no sub-step past it."""
    rp, fluid, solid, volumes = bench.reference_scene(reference)
    whole = reference.sim(rp, solid, fluid, None, volumes)
    whole.frame("dfsph_p")
    whole.frame("dfsph_p")
    op = {k: rp[k] for k in rp if k not in ("seed", "length", "mass_per_particle_override",
                                            "pressure_correction_denom_override")}
    op.update(mass_per_particle=rp["mass_per_particle_override"],
              pressure_correction_denom=rp["pressure_correction_denom_override"],
              seconds_per_sub_step=reference.config(rp)["seconds_per_sub_step"])
    osim = oracle.sim(op, solid, volumes, fluid)
    k = osim.frame("dfsph_p") + osim.frame("dfsph_p")
    assert k > 3
    win = reference.sim(rp, solid, fluid, None, volumes)
    timed, seconds = win.run_window("dfsph_p", 2, k - 2)
    assert timed == k - 2 and seconds > 0.0
    for a, b, name in zip(win.state(), whole.state(), ("positions", "velocities")):
        assert_bitwise(a, b, name)
    # one sub-step short of two frames: the last sub-step of frame 2 is not run
    short = reference.sim(rp, solid, fluid, None, volumes)
    timed, _ = short.run_window("dfsph_p", 0, k - 1)
    assert timed == k - 1
    assert not np.array_equal(short.state()[0], whole.state()[0])
