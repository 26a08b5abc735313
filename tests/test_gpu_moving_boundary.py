"""Moving boundaries: the boundary replaced between frames, against the
reference run the same way.

The reference's step functions take the Solid_state by const reference on
every call, so a caller moves a wall by passing a new one: positions and
velocities through compute_neighbor_data_and_volumes
(emerald/sph2d_box/solids.cpp:76-137). The reference harness does exactly
that between frames; the GPU takes the same positions, velocities and
volumes through emerald_sim_set_solid. Every frame's fluid state, and the
recomputed boundary volumes, must be bit-identical."""
import numpy as np
import pytest

from conftest import assert_bitwise
from cpu_checkers import RefParams
from scenes import F

pytestmark = pytest.mark.gpu

METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def scene(E):
    return E.BlockScene(20, dx=F(1 / 40), seed=5, time_per_step_flicks=1411200, sub_steps=4,
                        iisph_max_pressure_iterations=50,
                        iisph_error_average_threshold=F(0.001),
                        dfsph_divergence_error_average_threshold=F(0.001),
                        dfsph_density_error_average_threshold=F(0.0005))


def reference_sim(reference, sc):
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=d["mass_per_particle"],
              pressure_correction_denom_override=d["pressure_correction_denom"])
    return reference.sim(rp, sc.solid, sc.fluid, None, sc.solid_volumes)


def piston(sc, frame, speed):
    """The left wall (x < 0) moved by `speed` * 2 ms per frame along x, with
    that velocity; the other boundary particles at rest. At -2 m/s the wall
    retracts from the fluid and its outer rows cross into the next cell
    column within four frames."""
    xy = sc.solid.copy()
    v = np.zeros_like(xy)
    left = xy[:, 0] < 0
    step = F(speed * 0.002)
    xy[left, 0] = xy[left, 0] + F(frame) * step
    v[left, 0] = F(speed)
    return xy, v


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("recompute", [True, False])
def test_piston_frames_equal_reference(E, reference, method, recompute):
    sc = scene(E)
    sim = E.Simulation.from_block_scene(sc)
    ref = reference_sim(reference, sc)
    for f in range(1, 5):
        xy, v = piston(sc, f, -2.0)
        vols = None if recompute else sc.solid_volumes
        ref.set_solid(xy, v, vols)
        sim.set_solid(xy, v, vols)
        assert_bitwise(sim.solid()[0], ref.solid()[0], "%s boundary positions %d" % (method, f))
        assert_bitwise(sim.solid()[1], ref.solid()[1], "%s boundary volumes %d" % (method, f))
        ref.frame(method)
        sim.frame(method)
        x, vv = sim.state()
        rx, rv = ref.state()
        assert_bitwise(x, rx, "%s x after frame %d" % (method, f))
        assert_bitwise(vv, rv, "%s v after frame %d" % (method, f))
    sim.close()


@pytest.mark.parametrize("method", ["iisph", "dfsph_p"])
def test_conveyor_velocities_only(E, reference, method):
    """Boundary velocities alone (a floor sliding at 0.3 m/s, positions
    unchanged) enter the divergence and density terms as in the reference."""
    sc = scene(E)
    sim = E.Simulation.from_block_scene(sc)
    ref = reference_sim(reference, sc)
    v = np.zeros_like(sc.solid)
    v[sc.solid[:, 1] < 0, 0] = F(0.3)
    ref.set_solid(None, v, None)
    sim.set_solid(None, v, None)
    assert_bitwise(sim.solid()[1], ref.solid()[1], "volumes kept")
    for f in range(3):
        ref.frame(method)
        sim.frame(method)
    assert_bitwise(sim.state()[0], ref.state()[0], "x")
    assert_bitwise(sim.state()[1], ref.state()[1], "v")
    # the sliding floor drags the fluid above it
    still = E.Simulation.from_block_scene(sc)
    for f in range(3):
        still.frame(method)
    assert not np.array_equal(still.state()[1], sim.state()[1])
    still.close()
    sim.close()


def test_batch_set_solid_equals_single(E):
    """A moved boundary in one scene of a batch gives that scene the bits it
    gives alone and leaves the other scene's bits alone."""
    sa, sb = scene(E), E.BlockScene(16, dx=F(1 / 32), seed=9, time_per_step_flicks=1411200,
                                    sub_steps=4)
    b = E.Batch(len(sa.fluid) + len(sb.fluid) + 256, len(sa.solid) + len(sb.solid) + 256, 2)
    ia = b.add_block_scene(sa)
    ib = b.add_block_scene(sb)
    alone_a = E.Simulation.from_block_scene(sa)
    alone_b = E.Simulation.from_block_scene(sb)
    for f in range(1, 3):
        xy, v = piston(sa, f, -2.0)
        b.set_solid(ia, xy, v)
        alone_a.set_solid(xy, v)
        b.step("dfsph_p", 3)
        alone_a.advance("dfsph_p", 3)
        alone_b.advance("dfsph_p", 3)
    b.synchronize()
    assert_bitwise(b.state(ia)[0], alone_a.state()[0], "moved scene x")
    assert_bitwise(b.state(ib)[0], alone_b.state()[0], "other scene x")
    alone_a.close()
    alone_b.close()
    b.close()


def test_set_solid_keeps_count_and_rejects_bad_scene(E):
    sc = scene(E)
    sim = E.Simulation.from_block_scene(sc)
    xy0, vol0 = sim.solid()
    sim.set_solid(None, None, None)
    assert_bitwise(sim.solid()[0], xy0, "unchanged positions")
    assert_bitwise(sim.solid()[1], vol0, "unchanged volumes")
    b = E.Batch(1024, 1024, 1)
    with pytest.raises(E.EmeraldError):
        b.set_solid(3, sc.solid)
    b.close()
    sim.close()
