"""Failure handling and resumption on the host side of the GPU path.

The reference's only failure handling is EMLD_ASSERT, which aborts
(emerald/util/assert.h:14-26), and it has no checkpoint: a run's state is
State + Temp_data (emerald/sph2d_box/state.h:13-69). Here:
* non-finite positions or velocities handed to set_state / advance_host are
  refused with EMERALD_EINVAL and the simulation is left as it was;
* a snapshot taken between sub-steps (mid-frame, with the DFSPH kappas of
  the frame's warm starts) restores into the same or a new simulation, and
  the sub-steps after it are bit-identical to those after the snapshot;
* a request of the request loop can be cancelled while queued or resident,
  and the other requests' results stay bit-identical to their scenes alone.
Every failure here is made on the host; nothing faults a GPU."""
import time

import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def scene(E, n=24, seed=3, **kw):
    return E.BlockScene(n, dx=F(1 / (2 * n)), seed=seed, time_per_step_flicks=1411200, sub_steps=4,
                        dfsph_divergence_error_average_threshold=F(0.001),
                        dfsph_density_error_average_threshold=F(0.0005), **kw)


def test_set_state_refuses_non_finite_values(E):
    sim = E.Simulation.from_block_scene(scene(E))
    sim.advance("dfsph_p", 2)
    x0, v0 = sim.state()
    bad = x0.copy()
    bad[7, 1] = np.nan
    with pytest.raises(E.EmeraldError) as e:
        sim.set_state(bad, v0)
    assert e.value.code == 22
    badv = v0.copy()
    badv[3, 0] = -np.inf
    with pytest.raises(E.EmeraldError):
        sim.set_state(None, badv)
    x1, v1 = sim.state()
    assert_bitwise(x1, x0, "positions after a refused set_state")
    assert_bitwise(v1, v0, "velocities after a refused set_state")
    sim.close()


def test_advance_host_refuses_non_finite_input_without_stepping(E):
    sim = E.Simulation.from_block_scene(scene(E, seed=4))
    sim.advance("dfsph_p", 1)
    t0 = sim.time()
    x0, v0 = sim.state()
    xi = x0.copy()
    xi[0, 0] = np.inf
    with pytest.raises(E.EmeraldError) as e:
        sim.advance_host("dfsph_p", 3, xi, v0.copy())
    assert e.value.code == 22
    assert sim.time() == t0
    x1, v1 = sim.state()
    assert_bitwise(x1, x0, "positions")
    assert_bitwise(v1, v0, "velocities")
    sim.close()


@pytest.mark.parametrize("method", ["dfsph_p", "iisph", "pcisph"])
@pytest.mark.parametrize("precision", [0, 1])
def test_snapshot_restore_resumes_bit_for_bit(E, method, precision):
    """A snapshot after 3 sub-steps (inside the first frame: the DFSPH kappas
    of the frame are live), restored into a new simulation and into the
    original one after it ran on: 5 more sub-steps give the uninterrupted
    run's state, statistics and clock."""
    sc = scene(E, seed=5, precision=precision)
    a = E.Simulation.from_block_scene(sc)
    a.advance(method, 3)
    snap = a.snapshot()
    st_a = a.advance(method, 5)
    xa, va = a.state()
    ta = a.time()
    b = E.Simulation.from_block_scene(sc)
    b.restore(snap)
    st_b = b.advance(method, 5)
    assert b.time() == ta
    assert_bitwise(b.state()[0], xa, "%s positions after restore" % method)
    assert_bitwise(b.state()[1], va, "%s velocities after restore" % method)
    for k in ("pressure_iterations", "divergence_iterations", "dt", "error_average"):
        assert st_b[k] == st_a[k], (k, st_b[k], st_a[k])
    a.restore(snap)  # rewind the original
    a.advance(method, 5)
    assert_bitwise(a.state()[0], xa, "%s positions after rewinding" % method)
    a.close()
    b.close()


def test_snapshot_carries_a_moved_boundary(E):
    sc = scene(E, seed=6)
    a = E.Simulation.from_block_scene(sc)
    xy, vol = a.solid()
    moved = xy.copy()
    left = moved[:, 0] < 0
    moved[left, 0] -= F(0.002)
    vel = np.zeros_like(moved)
    vel[left, 0] = F(-1.0)
    a.set_solid(moved, vel, None)
    a.advance("dfsph_p", 2)
    snap = a.snapshot()
    a.advance("dfsph_p", 4)
    b = E.Simulation.from_block_scene(sc)
    b.restore(snap)
    b.advance("dfsph_p", 4)
    assert_bitwise(b.state()[0], a.state()[0], "positions with the moved boundary")
    assert_bitwise(b.solid()[0], a.solid()[0], "boundary positions")
    a.close()
    b.close()


def test_restore_refuses_foreign_or_damaged_snapshots(E):
    a = E.Simulation.from_block_scene(scene(E, n=24, seed=7))
    snap = a.snapshot()
    other = E.Simulation.from_block_scene(scene(E, n=20, seed=7))
    with pytest.raises(E.EmeraldError) as e:
        other.restore(snap)
    assert e.value.code == 22
    with pytest.raises(E.EmeraldError):
        a.restore(b"EMSNAPxx" + snap[8:])
    with pytest.raises(E.EmeraldError):
        a.restore(snap[:-4])
    comp = E.Simulation.from_block_scene(scene(E, n=24, seed=7, precision=1))
    with pytest.raises(E.EmeraldError):
        comp.restore(snap)
    for s in (a, other, comp):
        s.close()


def test_cancelled_requests_leave_the_others_unchanged(E):
    """Eight requests through a two-lane loop too small for all of them: one
    is cancelled while queued, one (a long one) once it is resident; both
    report EMERALD_ECANCELED and every other result equals its scene run
    alone."""
    srv = E.Server(3 << 20, "dfsph_p", max_scenes=8, max_substeps_per_launch=2, lanes=2)
    jobs = [(12, 3, 7), (16, 4, 3000), (14, 5, 6), (16, 6, 9), (10, 7, 5), (12, 8, 8),
            (14, 9, 4), (18, 10, 6)]
    scenes = [scene(E, n, seed) for n, seed, _ in jobs]
    ids = [srv.submit_block_scene(sc, steps) for sc, (_, _, steps) in zip(scenes, jobs)]
    srv.cancel(ids[7])  # the last one is still queued behind the others
    deadline = time.time() + 60
    while srv.stats()["resident"] == 0 and time.time() < deadline:
        time.sleep(0.01)
    time.sleep(0.05)
    srv.cancel(ids[1])  # 3000 sub-steps: resident now, far from done
    for k in (1, 7):
        with pytest.raises(E.EmeraldError) as e:
            srv.wait(ids[k], 60000)
        assert e.value.code == E.Server.ECANCELED
    results = {k: srv.wait(ids[k], 120000) for k in range(len(jobs)) if k not in (1, 7)}
    st = srv.stats()
    srv.close()
    assert st["cancelled"] == 2 and st["status"] == 0, st
    assert st["completed"] == len(jobs) - 2, st
    for k, out in results.items():
        sim = E.Simulation.from_block_scene(scenes[k])
        sim.advance("dfsph_p", jobs[k][2])
        x, v = sim.state()
        sim.close()
        assert_bitwise(out[0], x, "request %d positions" % k)
        assert_bitwise(out[1], v, "request %d velocities" % k)
