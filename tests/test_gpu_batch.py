"""Batches of scenes: every scene of a batch gives the bits it gives alone.

A batch runs each kernel of a sub-step once over all active scenes, with
per-scene time steps, frames and solver convergence. The reference runs one
scene per simulation object (emerald/sph2d_box/simulation.h:24-44), so the
oracle for a scene in a batch is the same scene run by itself; the single
scene path is pinned to the oracle and the reference in test_gpu_parity.py."""
import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu

METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def scenes(E, sizes, **kw):
    out = []
    for k, n in enumerate(sizes):
        out.append(E.BlockScene(n, dx=F(1.0 / (2 * n)), seed=11 + k, time_per_step_flicks=1411200,
                                sub_steps=4, iisph_max_pressure_iterations=50,
                                iisph_error_average_threshold=F(0.001),
                                dfsph_divergence_error_average_threshold=F(0.001),
                                dfsph_density_error_average_threshold=F(0.0005), **kw))
    return out


def alone(E, scene, method, n):
    sim = E.Simulation.from_block_scene(scene)
    st = sim.advance(method, n)
    x, v = sim.state()
    sim.close()
    return x, v, st


@pytest.mark.parametrize("method", METHODS)
def test_batch_equals_alone(E, method):
    """Four scenes of different sizes (and so different time steps and
    iteration counts) advanced together for 9 sub-steps."""
    sc = scenes(E, [12, 20, 31, 24])
    total = sum(len(s.fluid) for s in sc)
    total_s = sum(len(s.solid) for s in sc)
    b = E.Batch(total + 4 * 128, total_s + 4 * 128, 4)
    ids = [b.add_block_scene(s) for s in sc]
    b.step(method, 9)
    b.synchronize()
    for sid, s in zip(ids, sc):
        x, v, st = alone(E, s, method, 9)
        bx, bv = b.state(sid)
        bst = b.stats(sid)
        assert_bitwise(bx, x, "%s scene %d x" % (method, sid))
        assert_bitwise(bv, v, "%s scene %d v" % (method, sid))
        for k in ("sub_steps", "pressure_iterations", "divergence_iterations", "dt",
                  "time_seconds", "error_flags"):
            assert bst[k] == st[k], (method, sid, k, bst[k], st[k])
    b.close()


def test_continuous_batching(E):
    """Scenes join and leave a running batch between sub-steps without
    changing the others' results: A runs 10 sub-steps, B joins after 3 and
    leaves after 4 more, C takes B's room after that."""
    sa, sb, sc = scenes(E, [16, 20, 20])
    cap = len(sa.fluid) + len(sb.fluid) + 256
    cap_s = len(sa.solid) + len(sb.solid) + 256
    b = E.Batch(cap, cap_s, 2)
    a = b.add_block_scene(sa)
    b.step("dfsph_p", 3)
    bid = b.add_block_scene(sb)
    assert b.add_block_scene(sc) is None  # both scene slots are taken
    b.step("dfsph_p", 4)
    bx, bv = b.state(bid)
    x, v, _ = alone(E, sb, "dfsph_p", 4)
    assert_bitwise(bx, x, "B x")
    assert_bitwise(bv, v, "B v")
    b.remove_scene(bid)
    cid = b.add_block_scene(sc)
    assert cid is not None
    b.step("dfsph_p", 3)
    for sid, s, n in ((a, sa, 10), (cid, sc, 3)):
        x, v, st = alone(E, s, "dfsph_p", n)
        bx, bv = b.state(sid)
        assert_bitwise(bx, x, "scene %d x" % sid)
        assert_bitwise(bv, v, "scene %d v" % sid)
        assert b.stats(sid)["sub_steps"] == n
    b.close()


def test_inactive_scene_is_frozen(E):
    sa, sb = scenes(E, [12, 14])
    b = E.Batch(4096, 4096, 2)
    a = b.add_block_scene(sa)
    c = b.add_block_scene(sb, active=False)
    x0, v0 = b.state(c)
    b.step("iisph", 5)
    x1, v1 = b.state(c)
    assert_bitwise(x1, x0, "inactive x")
    assert_bitwise(v1, v0, "inactive v")
    b.set_active(c, True)
    b.step("iisph", 2)
    x, v, _ = alone(E, sb, "iisph", 2)
    assert_bitwise(b.state(c)[0], x, "late scene x")
    x, v, _ = alone(E, sa, "iisph", 7)
    assert_bitwise(b.state(a)[0], x, "first scene x")
    b.close()


def test_batch_launches_do_not_grow_with_scenes(E):
    """One batch sub-step launches the same kernels for 1 scene as for 16."""
    counts = []
    for k in (1, 16):
        sc = scenes(E, [10] * k)
        b = E.Batch(k * 256, k * 1024, k)
        for s in sc:
            b.add_block_scene(s)
        b.step("dfsph_p", 1)
        b.synchronize()
        n0 = b.kernel_launches()
        b.step("dfsph_p", 1)
        b.synchronize()
        counts.append(b.kernel_launches() - n0)
        b.close()
    # Loop bodies run once per solver iteration of the slowest scene, so
    # the counts may differ by whole iterations; the fixed part may not.
    assert counts[1] <= counts[0] + 40, counts
