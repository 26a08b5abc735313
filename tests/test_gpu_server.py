"""The request loop: every request's result equals its scene run alone.

Requests arrive from another thread while earlier ones are on the GPU; the
arena (sized from a device-memory budget) holds only a few at a time, so
later requests wait in the queue and join the running batch as earlier ones
finish. Results are compared bit for bit with the single-scene path, which
test_gpu_parity.py pins to the oracle and the reference."""
import threading
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


def scene(E, n, seed, ny=None):
    side = max(n, ny or n)
    return E.BlockScene(n, ny=ny, dx=F(1.0 / (2 * side)), seed=seed, time_per_step_flicks=1411200,
                        sub_steps=4, dfsph_divergence_error_average_threshold=F(0.001),
                        dfsph_density_error_average_threshold=F(0.0005))


def alone(E, sc, n):
    sim = E.Simulation.from_block_scene(sc)
    st = sim.advance("dfsph_p", n)
    x, v = sim.state()
    sim.close()
    return x, v, st


@pytest.mark.parametrize("order", ["arrival", "largest_first"])
def test_requests_equal_alone_under_continuous_batching(E, order):
    srv = E.Server(3 << 20, "dfsph_p", max_scenes=8, max_substeps_per_launch=3, lanes=2,
                   order=order)
    cap = srv.stats()["fluid_capacity"]  # of one lane
    assert cap >= 512, cap
    jobs = [(12, None, 3, 7), (16, None, 4, 11), (20, 10, 5, 4), (14, None, 6, 9),
            (10, 18, 7, 5), (16, None, 8, 6), (12, 12, 9, 10), (18, None, 10, 5)]
    scenes = [scene(E, n, seed, ny) for n, ny, seed, _ in jobs]
    assert max(len(s.fluid) for s in scenes) <= cap
    assert sum(len(s.fluid) for s in scenes) > 2 * cap  # not all fit at once
    ids = [None] * len(jobs)

    def client():
        for k, (sc, job) in enumerate(zip(scenes, jobs)):
            ids[k] = srv.submit_block_scene(sc, job[3])
            time.sleep(0.002)

    th = threading.Thread(target=client)
    th.start()
    th.join()
    results = [srv.wait(rid, 60000) for rid in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(jobs) and st["status"] == 0, st
    assert st["resident_peak"] >= 2, st            # requests overlapped on the device
    assert st["device_bytes"] <= (3 << 20), st      # the arena kept to its budget
    for k, (sc, job) in enumerate(zip(scenes, jobs)):
        x, v, stats, timing = results[k]
        ax, av, ast = alone(E, sc, job[3])
        assert_bitwise(x, ax, "request %d x" % k)
        assert_bitwise(v, av, "request %d v" % k)
        assert stats["sub_steps"] == job[3]
        for key in ("pressure_iterations", "divergence_iterations", "dt", "time_seconds"):
            assert stats[key] == ast[key], (k, key, stats[key], ast[key])
        assert timing["total_ms"] >= timing["run_ms"] >= 0.0


def test_server_rejects_and_times_out(E):
    srv = E.Server(4 << 20, "iisph", max_scenes=4, lanes=1)
    cap = srv.stats()["fluid_capacity"]
    big = scene(E, int(np.ceil(np.sqrt(cap))) + 8, 1)
    assert len(big.fluid) > cap
    assert srv.submit_block_scene(big, 5) is None
    assert srv.stats()["rejected"] == 1
    sc = scene(E, 12, 2)
    rid = srv.submit_block_scene(sc, 400)
    assert srv.wait(rid, 0) is None                 # not done within 0 ms
    out = srv.wait(rid, 120000)
    assert out is not None and out[2]["sub_steps"] == 400
    with pytest.raises(E.EmeraldError):
        srv.wait(rid, 0)                             # already collected
    srv.close()


def test_server_footprint_matches_allocation(E):
    import torch
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    srv = E.Server(256 << 20, "dfsph_p", max_scenes=16)
    free1, _ = torch.cuda.mem_get_info()
    st = srv.stats()
    srv.close()
    used = free0 - free1
    assert st["device_bytes"] <= (256 << 20)
    # allocation granularity and the loop's stream and events on top
    assert st["device_bytes"] <= used <= st["device_bytes"] + (64 << 20), (used, st)
