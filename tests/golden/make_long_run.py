"""Regenerates tests/golden/long_run_dfsph_262k.npz (and, with side 1024,
long_run_dfsph_1m.npz) from the reference.

Runs the unmodified emerald sources compiled against the project's shims
(oracle/_ref/libemerald_ref.so, built by oracle/build_oracle.py) on the
benchmark scene (bench.reference_scene: the side x side DFSPH_P dam break,
dx = 1/(2 side), support = dx, built by the reference harness alone) through the
reference's own CFL-adaptive frame loop, and stores every `every` frames the
SHA-256 of positions and velocities, the total mechanical energy drift
(kinetic plus m g y, relative to the initial potential energy) and the
largest speed. The run covers the dam's collapse, the splash on the far wall
and the ejection of single particles at high speed that this small-support
scene shows: at side 512 one particle near frame 105 (of 2 ms, about 1,300
sub-steps); at side 1024 a few near frame 84 (about 1,400 sub-steps), then a
spreading cascade from frame 88 on.

Usage: python tests/golden/make_long_run.py [frames] [every] [side]
       (default 120 5 512; the 1,048,576-particle fixture: 95 5 1024)
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from cpu_checkers import Reference, ensure_built  # noqa: E402

import bench  # noqa: E402



def out_path(side):
    return os.path.join(HERE, "long_run_dfsph_%s.npz" % ({512: "262k", 1024: "1m"}[side]))


def digest(x, v):
    return hashlib.sha256(np.ascontiguousarray(x).tobytes() +
                          np.ascontiguousarray(v).tobytes()).hexdigest()


def energy_drift(x, v, mass, g, e0):
    ke = 0.5 * mass * float(np.sum(v.astype(np.float64) ** 2))
    return (ke + mass * g * float(np.sum(x[:, 1].astype(np.float64))) - e0) / abs(e0)


def main(frames, every, side):
    ensure_built()
    R = Reference()
    R.set_threads(os.cpu_count() or 1)
    bench.configure_scene(side)
    rp, fluid, solid, volumes = bench.reference_scene(R)
    sim = R.sim(rp, solid, fluid, None, volumes)
    mass = float(rp["mass_per_particle_override"])
    g = float(rp["gravity"])
    e0 = mass * g * float(np.sum(fluid[:, 1].astype(np.float64)))
    rows = []
    t0 = time.time()
    for f in range(1, frames + 1):
        sim.frame("dfsph_p")
        if f % every:
            continue
        x, v = sim.state()
        vmax = float(np.sqrt(np.max(np.sum(v.astype(np.float64) ** 2, axis=1))))
        rows.append((f, digest(x, v), energy_drift(x, v, mass, g, e0), vmax, sim.time()))
        print("frame %d: drift %.3e, max speed %.3f, %.0f s" % (f, rows[-1][2], vmax,
                                                              time.time() - t0), flush=True)
    np.savez_compressed(out_path(side), frames=np.array([r[0] for r in rows], np.int64),
                        digests=np.array([r[1] for r in rows]),
                        energy_drift=np.array([r[2] for r in rows], np.float64),
                        max_speed=np.array([r[3] for r in rows], np.float64),
                        flicks=np.array([r[4] for r in rows], np.int64))


if __name__ == "__main__":
    a = sys.argv[1:]
    main(int(a[0]) if a else 120, int(a[1]) if len(a) > 1 else 5,
         int(a[2]) if len(a) > 2 else 512)
