"""Density-error and kinetic-energy traces of long fixed-dt runs (test side).

The same functions read the compiled reference's run (tests/golden/make_traces.py)
and the CUDA path's run (tests/test_gpu_traces.py), so both traces are
computed identically from each sub-step's velocities and densities.

Scene: the IISPH dam-break shape of the plain 16,384-particle configuration,
a 128 x 128 fluid block at dx = 1/256 jittered +/- 0.01 dx from seed 1, three
wall rows, support = dx (the literal support 2 dx is unstable in the reference
itself), rest density 1000, gravity -9.81. Each method runs 1000 fixed-dt
sub-steps from rest: 1e-4 s for the pressure-solve methods and 5e-4 s for
PCISPH, whose precomputed denominator bakes its sub-step.
"""
import hashlib

import numpy as np

F = np.float32
SIDE = 128
DX = F(1.0 / 256)
STEPS = 1000
CHECKPOINTS = (1, 10, 100, 1000)
METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]
PCISPH_DT = F(352800 / 705600000.0)


def method_dt(method):
    return PCISPH_DT if method == "pcisph" else F(1e-4)


def density_error(rho, rho0=1000.0):
    """(average, max, exact mean) of max(0, rho - rho0) / rho0.

    The average is the reference's metric: sum of int64(err * 1000) over
    particles divided by 1000 n in double
    (emerald/sph_common/common.h:209-232); the max is in FP32 as the solvers
    keep it; the exact mean is the FP64 mean of the same per-particle errors."""
    rho0 = F(rho0)
    err = np.maximum(F(0.0), (rho.astype(F) - rho0)) / rho0
    err = err.astype(F)
    n = len(err)
    if n == 0:
        return 0.0, 0.0, 0.0
    ints = (err * F(1000.0)).astype(np.int64)
    avg = float(F(float(ints.sum()) / float(1000 * n)))
    return avg, float(err.max()), float(err.astype(np.float64).mean())


def kinetic_energy(v, mass):
    """0.5 m sum |v|^2 in FP64, summed in particle order."""
    v = v.astype(np.float64)
    return 0.5 * float(mass) * float(np.sum(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]))


def digest(x, v):
    """SHA-256 of the FP32 bytes of positions and velocities."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(x, F).tobytes())
    h.update(np.ascontiguousarray(v, F).tobytes())
    return h.hexdigest()


def run_trace(sim, method, mass, steps=STEPS):
    """Advance `sim` (reference or CUDA Simulation; both expose begin_frame,
    sub_step, state and array) `steps` fixed-dt sub-steps and return the
    trace arrays and the digests at CHECKPOINTS."""
    dt = method_dt(method)
    sim.begin_frame(method)
    avg = np.zeros(steps, np.float64)
    mx = np.zeros(steps, np.float64)
    exact = np.zeros(steps, np.float64)
    ke = np.zeros(steps, np.float64)
    digests = {}
    for s in range(steps):
        sim.sub_step(method, F(s * dt), dt)
        x, v = sim.state()
        avg[s], mx[s], exact[s] = density_error(sim.array("densities"))
        ke[s] = kinetic_energy(v, mass)
        if s + 1 in CHECKPOINTS:
            digests[s + 1] = digest(x, v)
    return {"avg_error": avg, "max_error": mx, "exact_error": exact, "kinetic_energy": ke,
            "digests": digests}
