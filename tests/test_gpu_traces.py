"""1000-sub-step density-error and kinetic-energy traces of the CUDA path
against the reference's own run (tests/golden/trace_<method>.npz, made by
tests/golden/make_traces.py from the compiled reference).

Scene and sub-steps are those of tests/traces.py: the 128 x 128 (16,384
particle) IISPH dam-break block at dx = 1/256, every solver, 1000 fixed-dt
sub-steps from rest.

Stated tolerances, checked at every one of the 1000 sub-steps:
* kinetic energy (FP64 sum of the FP32 velocities): relative 1e-5;
* average density error (the reference's metric): absolute 1e-6, one
  thousandth of the 0.1% solver tolerance;
* max density error: absolute 1e-6.
Positions and velocities are also compared bit for bit (SHA-256 of their
FP32 bytes) after sub-steps 1, 10, 100 and 1000; the CUDA path reproduces
the reference's sub-step exactly, so the traces agree with zero error and
the tolerances above are the claim, not the measured gap.
"""
import os

import numpy as np
import pytest

import traces as T
from scenes import F

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KE_RTOL = 1e-5
ERROR_ATOL = 1e-6

_runs = {}


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def _scene():
    return dict(np.load(os.path.join(GOLDEN, "trace_scene.npz")))


def _params(E, g):
    return E.default_params(support=g["dx"], time_per_step_flicks=1411200, sub_steps=4,
                            iisph_max_pressure_iterations=50,
                            iisph_error_average_threshold=F(0.001),
                            dfsph_divergence_error_average_threshold=F(0.001),
                            dfsph_density_error_average_threshold=F(0.0005),
                            mass_per_particle=g["mass"], pressure_correction_denom=g["denom"])


def _run(E, method):
    if method not in _runs:
        g = _scene()
        sim = E.Simulation(_params(E, g), g["solid"], g["fluid"], None, g["solid_volumes"])
        try:
            _runs[method] = T.run_trace(sim, method, g["mass"])
        finally:
            sim.close()
    return _runs[method]


@pytest.mark.parametrize("method", T.METHODS)
def test_trace_within_tolerance(E, method):
    ref = np.load(os.path.join(GOLDEN, "trace_%s.npz" % method))
    assert float(ref["dt"]) == float(T.method_dt(method))
    tr = _run(E, method)
    ke, ke_ref = tr["kinetic_energy"], ref["kinetic_energy"]
    rel = np.abs(ke - ke_ref) / np.maximum(np.abs(ke_ref), 1e-30)
    worst = int(np.argmax(rel))
    assert rel[worst] <= KE_RTOL, "%s kinetic energy off by %.3g relative at sub-step %d" % (
        method, rel[worst], worst + 1)
    for key in ("avg_error", "max_error"):
        d = np.abs(tr[key] - ref[key])
        worst = int(np.argmax(d))
        assert d[worst] <= ERROR_ATOL, "%s %s off by %.3g at sub-step %d" % (
            method, key, d[worst], worst + 1)


@pytest.mark.parametrize("method", T.METHODS)
def test_trace_state_bit_identical(E, method):
    ref = np.load(os.path.join(GOLDEN, "trace_%s.npz" % method))
    tr = _run(E, method)
    for s, h in zip(ref["digest_steps"], ref["digests"]):
        assert tr["digests"][int(s)] == str(h), "%s state differs after sub-step %d" % (method, s)
    for key in ("kinetic_energy", "avg_error", "max_error", "exact_error"):
        assert np.array_equal(tr[key], ref[key]), (method, key)
