"""Seeded synthetic scene sets for the batched and served forms of the step.

Every scene is a dam break: an nx-by-ny fluid block at spacing dx in the
corner of a [0, 1]^2 tank with three boundary rows on the floor and side
walls (see BlockScene). Scene sets are drawn from numpy's PCG64 with a fixed
seed, so every process that asks for the same set gets the same scenes.
"""
import math

import numpy as np

from . import BlockScene

# DFSPH frame: 2e-3 s per frame, sub-steps between tps/60 and tps/4 = 5e-4 s.
TPS_FLICKS = 1411200


def block_shape(n, aspect):
    """nx * ny close to n with nx / ny close to `aspect` (both at least 4)."""
    nx = max(4, int(round(math.sqrt(n * aspect))))
    ny = max(4, int(round(n / nx)))
    return nx, ny


def scene_for(nx, ny, seed, viscosity=0.01, **overrides):
    """A dam-break block of nx-by-ny particles; dx fits the longer side of the
    block into half the tank, as in the 512x512 dx=1/1024 scene. DFSPH may
    take up to 100 correction iterations (the reference's default cap of 15
    leaves these scenes above 0.1% average density error)."""
    dx = np.float32(1.0 / (2 * max(nx, ny)))
    kw = dict(time_per_step_flicks=TPS_FLICKS, sub_steps=4,
              iisph_max_pressure_iterations=50,
              iisph_error_average_threshold=np.float32(0.001),
              dfsph_divergence_error_average_threshold=np.float32(0.001),
              dfsph_density_error_average_threshold=np.float32(0.0005),
              dfsph_max_correction_iterations=100,
              viscosity=np.float32(viscosity))
    kw.update(overrides)
    return BlockScene(nx, dx=dx, ny=ny, seed=seed, **kw)


def batched_specs(count=512, lo=1024, hi=65536, seed=2024):
    """Scene descriptions of the batched workload: fluid count log-uniform in
    [lo, hi], block aspect ratio uniform in [0.25, 4], viscosity uniform in
    [0.001, 0.05]. Returns dicts with nx, ny, seed, viscosity."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    aspect = rng.uniform(0.25, 4.0, count)
    visc = rng.uniform(0.001, 0.05, count)
    out = []
    for k in range(count):
        nx, ny = block_shape(n[k], aspect[k])
        out.append(dict(nx=nx, ny=ny, seed=int(seed * 1000 + k), viscosity=float(visc[k])))
    return out


def serving_requests(count, rate=200.0, lo=2048, hi=262144, steps_lo=50, steps_hi=500, seed=77):
    """Request stream of the served workload: Poisson arrivals at `rate` per
    second, fluid count log-uniform in [lo, hi], sub-step count uniform in
    [steps_lo, steps_hi], square blocks. Returns dicts with arrival (s), nx,
    ny, seed, substeps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate, count)
    arrival = np.cumsum(gaps) - gaps[0]
    n = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    steps = rng.integers(steps_lo, steps_hi + 1, count)
    out = []
    for k in range(count):
        side = max(4, int(round(math.sqrt(n[k]))))
        out.append(dict(arrival=float(arrival[k]), nx=side, ny=side, seed=int(seed * 1000 + k),
                        substeps=int(steps[k])))
    return out


def assign_scenes(sizes, world):
    """Greedy longest-first bin-pack of scenes onto `world` GPUs by particle
    count: returns a list of scene-index lists, one per rank. Deterministic
    (ties go to the lower rank, equal sizes keep index order)."""
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    load = [0] * world
    out = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda j: (load[j], j))
        out[r].append(k)
        load[r] += int(sizes[k])
    for lst in out:
        lst.sort()
    return out


def route_requests(requests, world):
    """Routes a request stream (serving_requests dicts, in arrival order) to
    `world` GPUs, each with its own request loop: every request goes, as it
    arrives, to the rank with the least work routed so far (fluid particles
    x sub-steps; ties to the lower rank). Returns a list of request-index
    lists, one per rank, each in arrival order. Deterministic, so every
    process computes the same routing without exchanging anything."""
    load = [0] * world
    out = [[] for _ in range(world)]
    for k, r in enumerate(requests):
        j = min(range(world), key=lambda q: (load[q], q))
        out[j].append(k)
        load[j] += int(r["nx"]) * int(r["ny"]) * int(r["substeps"])
    return out
