"""The benchmark scene over a long run, bit for bit: 120 frames (about 1,500
CFL-adaptive DFSPH_P sub-steps) of the 512 x 512 dam break at dx = 1/1024,
support = dx, through emerald_sim_frame (one graph launch per frame), with
the state's SHA-256 after every 5th frame equal to the compiled reference's
(tests/golden/long_run_dfsph_262k.npz, made by
tests/golden/make_long_run.py through the reference's own frame loop).

The run covers the collapse of the dam, the splash on the far wall and,
near frame 105, the ejection of a single particle at about 2,600 m/s that
this small-support scene shows in the reference itself: equal digests
before and after it mean the ejection is the reference's trajectory, not
a fault of the GPU path. The energy drift and the largest speed stored
beside the digests state the same."""
import hashlib
import os

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "long_run_dfsph_262k.npz")


def test_long_run_digests_match_reference():
    import emerald_b200 as E
    g = np.load(GOLDEN)
    want = dict(zip(g["frames"].tolist(), g["digests"].tolist()))
    flicks = dict(zip(g["frames"].tolist(), g["flicks"].tolist()))
    sim = E.Simulation.from_block_scene(E.BlockScene(bench.N_SIDE, **bench.scene_kwargs()))
    assert bench.N_SIDE == 512
    last = int(g["frames"].max())
    for f in range(1, last + 1):
        sim.frame("dfsph_p")
        if f in want:
            x, v = sim.state()
            got = hashlib.sha256(x.tobytes() + v.tobytes()).hexdigest()
            assert got == want[f], "frame %d: state differs from the reference's" % f
            assert sim.time() == flicks[f], f
    # the stored run does contain the ejection it is kept for
    assert g["max_speed"].max() > 1000.0 and g["max_speed"][0] < 10.0
    sim.close()
