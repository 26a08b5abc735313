"""Error of the FP32 results of every solver against the FP64 GPU oracle.

The FP32 run (the CUDA path, in either precision mode) advances its
sub-steps (CFL-adaptive, or PCISPH's fixed ones); the FP64 oracle repeats
each sub-step with the same dt, frame boundaries and iteration counts (and
the same relaxation omega, viscosity and PCISPH denominator), so the two
differ only in arithmetic precision. Reported per checkpoint: per-particle density error (relative,
L_inf and RMS), position error (in units of the particle spacing, max and
RMS), the kinetic-energy difference, and the drift of the total mechanical
energy (kinetic plus gravitational, m g y summed) from its initial value in
both runs."""
import numpy as np

from cpu_checkers import FP64Oracle

# Speed (m/s) above which a particle counts as ejected: the dam break's
# bulk flow stays below 10 m/s.
FAST = 50.0


def dfsph_scene(E, n_side, precision, seed=1):
    return E.BlockScene(n_side, dx=np.float32(1.0 / (2 * n_side)), seed=seed,
                        time_per_step_flicks=1411200, sub_steps=4,
                        dfsph_max_correction_iterations=100,
                        dfsph_divergence_error_average_threshold=np.float32(0.001),
                        dfsph_density_error_average_threshold=np.float32(0.0005),
                        precision=precision)


def iisph_scene(E, n_side, precision, seed=1):
    return E.BlockScene(n_side, dx=np.float32(1.0 / (2 * n_side)), seed=seed,
                        time_per_step_flicks=1411200, sub_steps=4,
                        iisph_max_pressure_iterations=50,
                        iisph_error_average_threshold=np.float32(0.001),
                        precision=precision)


def compare(E, n_side, steps, checkpoints, precision, seed=1, offset=0.0, method="dfsph_p"):
    """Rows of error statistics at the given sub-steps of `method` ("dfsph_p",
    "iisph", "iisph_ap", "iisph_pseudo_ap" or "pcisph"). `offset` moves the
    whole scene (fluid and walls) by (offset, offset) metres, rounded to
    float, before either run starts."""
    make = dfsph_scene if method == "dfsph_p" else iisph_scene
    scene = make(E, n_side, precision, seed)
    p = scene.params
    off = np.float32(offset)
    fluid = (scene.fluid + off).astype(np.float32)
    solid = (scene.solid + off).astype(np.float32)
    sim = E.Simulation(p, solid, fluid, None, scene.solid_volumes)
    ref = FP64Oracle().sim(p.support, p.target_density, p.mass_per_particle, p.gravity,
                           solid, scene.solid_volumes, fluid)
    mass = float(p.mass_per_particle)
    g = float(p.gravity)
    dx = float(scene.dx)
    e0 = mass * g * float(np.sum(fluid[:, 1].astype(np.float64)))
    tps = int(p.time_per_step_flicks)
    rows = []
    for step in range(1, steps + 1):
        new_frame = sim.time() % tps == 0
        st = sim.advance(method, 1)
        dt = float(np.float32(st["dt"]))
        if method == "dfsph_p":
            ref.sub_step(dt, new_frame, st["divergence_iterations"], st["pressure_iterations"])
        elif method == "iisph":
            ref.sub_step_iisph(dt, st["pressure_iterations"], float(p.iisph_omega))
        elif method in ("iisph_ap", "iisph_pseudo_ap"):
            ref.sub_step_ap(dt, st["pressure_iterations"], float(p.iisph_omega),
                            method == "iisph_pseudo_ap")
        else:
            ref.sub_step_pcisph(dt, st["pressure_iterations"], float(p.viscosity),
                                float(p.pressure_correction_denom))
        if step in checkpoints:
            x, v = sim.state()
            rho = sim.array("densities").astype(np.float64)
            x64 = ref.get("x")
            v64 = ref.get("v")
            rho64 = ref.get("densities")
            drel = np.abs(rho - rho64) / np.abs(rho64)
            dpos = np.hypot(*(x.astype(np.float64) - x64).T) / dx
            ke = 0.5 * mass * float(np.sum(v.astype(np.float64) ** 2))
            ke64 = 0.5 * mass * float(np.sum(v64 ** 2))
            e32 = ke + mass * g * float(np.sum(x[:, 1].astype(np.float64)))
            e64 = ke64 + mass * g * float(np.sum(x64[:, 1]))
            extra = {}
            if method in ("iisph", "iisph_ap", "iisph_pseudo_ap"):
                pr = sim.array("pressures").astype(np.float64)
                pr64 = ref.get("pressures")
                scale = float(np.abs(pr64).max()) or 1.0
                extra = dict(pressure_linf=float(np.abs(pr - pr64).max()) / scale,
                             pressure_rms=float(np.sqrt(np.mean((pr - pr64) ** 2))) / scale)
            vscale = float(np.abs(v64).max()) or 1.0
            rows.append(dict(step=step, density_linf=float(drel.max()),
                             velocity_linf_rel=float(np.abs(v.astype(np.float64) - v64).max())
                             / vscale,
                             density_rms=float(np.sqrt(np.mean(drel ** 2))),
                             position_max_dx=float(dpos.max()),
                             position_rms_dx=float(np.sqrt(np.mean(dpos ** 2))),
                             position_p99_dx=float(np.percentile(dpos, 99)),
                             fast_fp32=int(np.sum(np.hypot(*v.astype(np.float64).T) > FAST)),
                             fast_fp64=int(np.sum(np.hypot(*v64.T) > FAST)),
                             kinetic_energy=ke, kinetic_energy_fp64=ke64,
                             energy_rel_diff=abs(ke - ke64) / ke64 if ke64 else 0.0,
                             energy_drift=(e32 - e0) / abs(e0) if e0 else 0.0,
                             energy_drift_fp64=(e64 - e0) / abs(e0) if e0 else 0.0,
                             iterations=st["pressure_iterations"], **extra))
    ref.close()
    sim.close()
    return rows
