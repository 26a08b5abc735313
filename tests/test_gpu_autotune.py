"""Autotuning of the gather kernels' load chunks and list prefetch: it picks
among variants that give the same bits, so a run that tunes midway equals
one that does not; it leaves the simulation's state as it found it; and
every candidate, pinned, gives the same bits."""
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def scene(E, n, seed):
    return E.BlockScene(n, dx=F(1.0 / (2 * n)), seed=seed, time_per_step_flicks=1411200,
                        sub_steps=4, iisph_max_pressure_iterations=50,
                        iisph_error_average_threshold=F(0.001),
                        dfsph_divergence_error_average_threshold=F(0.001),
                        dfsph_density_error_average_threshold=F(0.0005))


@pytest.mark.parametrize("method", ["dfsph_p", "iisph"])
def test_tuning_keeps_results(E, method):
    sc = scene(E, 40, 3)
    a = E.Simulation.from_block_scene(sc)
    b = E.Simulation.from_block_scene(sc)
    a.advance(method, 3)
    b.advance(method, 3)
    x0, v0 = b.state()
    t = b.autotune(method)
    print(method, t)
    x1, v1 = b.state()
    assert_bitwise(x1, x0, "state kept x")
    assert_bitwise(v1, v0, "state kept v")
    for k in ("apply", "divergence", "iisph_sum", "iisph_beta"):
        assert t["chunks"][k] in (1, 4, 8)
    sa = a.advance(method, 6)
    sb = b.advance(method, 6)
    assert sa["pressure_iterations"] == sb["pressure_iterations"]
    assert_bitwise(b.state()[0], a.state()[0], "x after tuning")
    assert_bitwise(b.state()[1], a.state()[1], "v after tuning")


def test_batch_tuning(E):
    scs = [scene(E, n, 7 + n) for n in (16, 24, 30)]
    b = E.Batch(4096, 4096, 3)
    ids = [b.add_block_scene(s) for s in scs]
    b.step("iisph", 2)
    t = b.autotune("iisph")
    # a batch chooses among the persistent-warp kernels of the loop families
    # (prefetch modes 2 to 5), whose loop walks skip converged scenes
    assert len(t["candidates"]) == 6 and all(c["ms_per_substep"] > 0 for c in t["candidates"])
    assert all(2 <= c["prefetch"][f] <= 5 for c in t["candidates"]
               for f in ("iisph_sum", "iisph_beta"))
    b.step("iisph", 4)
    for sid, s in zip(ids, scs):
        sim = E.Simulation.from_block_scene(s)
        sim.advance("iisph", 6)
        assert_bitwise(b.state(sid)[0], sim.state()[0], "scene %d x" % sid)


def test_tuning_needs_a_substep_of_the_method(E):
    sim = E.Simulation.from_block_scene(scene(E, 12, 1))
    with pytest.raises(E.EmeraldError):
        sim.autotune("dfsph_p")
    sim.advance("iisph", 1)
    with pytest.raises(E.EmeraldError):
        sim.autotune("dfsph_p")
    sim.autotune("iisph")


@pytest.mark.parametrize("method", ["dfsph_p", "iisph"])
def test_every_candidate_gives_the_same_bits(E, method):
    sc = scene(E, 40, 5)
    ref = E.Simulation.from_block_scene(sc)
    ref.advance(method, 8)
    probe = E.Simulation.from_block_scene(sc)
    probe.advance(method, 1)
    cands = probe.autotune(method)["candidates"]
    assert any(any(c["prefetch"].values()) for c in cands)
    # the persistent-warp kernels, in both block sizes, and with the exit
    # test fused into the loop's final kernel, are among the candidates
    fam = "apply" if method == "dfsph_p" else "iisph_sum"
    last = "apply" if method == "dfsph_p" else "iisph_beta"
    assert {c["prefetch"][fam] for c in cands} >= {2, 3}
    assert {c["prefetch"][last] for c in cands} >= {4, 5}
    for c in cands:
        sim = E.Simulation.from_block_scene(sc)
        sim.set_tuning(c["chunks"], c["prefetch"])
        sim.advance(method, 8)
        assert_bitwise(sim.state()[0], ref.state()[0], "x with %r" % c)
        assert_bitwise(sim.state()[1], ref.state()[1], "v with %r" % c)
        sim.close()


def test_set_tuning_rejects_bad_values(E):
    sim = E.Simulation.from_block_scene(scene(E, 12, 1))
    with pytest.raises(E.EmeraldError):
        sim.set_tuning({"apply": 3, "divergence": 4, "iisph_sum": 4, "iisph_beta": 4})
    with pytest.raises(E.EmeraldError):
        sim.set_tuning({"apply": 4, "divergence": 4, "iisph_sum": 4, "iisph_beta": 4},
                       {"apply": 6})
    sim.set_tuning({"apply": 4, "divergence": 8, "iisph_sum": 4, "iisph_beta": 4},
                   {"apply": 2, "divergence": 2})
    sim.set_tuning()
    sim.close()
