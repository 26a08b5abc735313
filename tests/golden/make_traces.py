"""Regenerates the 1000-sub-step trace fixtures in tests/golden/ from the reference.

Runs the unmodified emerald sources compiled against the project's shims
(oracle/_ref/libemerald_ref.so, built by oracle/build_oracle.py from the
reference's sources) on the scene described in tests/traces.py and stores, for
each solver, trace_<method>.npz: the per-sub-step density error (the
reference's average metric, max and exact mean) and kinetic energy, and the
SHA-256 of positions and velocities after sub-steps 1, 10, 100 and 1000.
The scene inputs (fluid, walls, volumes, mass, PCISPH denominator) go to
trace_scene.npz, so the GPU test replays exactly these.

Usage: python tests/golden/make_traces.py [method ...]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from cpu_checkers import Reference, ensure_built  # noqa: E402
from scenes import walls  # noqa: E402
import traces as T  # noqa: E402
from make_golden import block_params  # noqa: E402


def main(methods):
    ensure_built()
    import emerald_b200 as E
    R = Reference()
    R.set_threads(os.cpu_count() or 1)
    dx = T.DX
    mass, denom = E.lattice_config(E.default_params(support=dx), dx, T.PCISPH_DT)
    xy = R.block_scene(T.SIDE, T.SIDE, dx)
    w = walls(dx)
    vol = np.full(len(w), T.F(mass) / T.F(1000.0), np.float32)
    np.savez_compressed(os.path.join(HERE, "trace_scene.npz"), fluid=xy, solid=w,
                        solid_volumes=vol, mass=mass, denom=denom, dx=dx)
    for m in methods:
        t0 = time.time()
        sim = R.sim(block_params(R, dx, mass, denom), w, xy, None, vol)
        tr = T.run_trace(sim, m, mass)
        steps = np.array(sorted(tr["digests"]), np.int64)
        np.savez_compressed(os.path.join(HERE, "trace_%s.npz" % m),
                            dt=T.method_dt(m), avg_error=tr["avg_error"],
                            max_error=tr["max_error"], exact_error=tr["exact_error"],
                            kinetic_energy=tr["kinetic_energy"], digest_steps=steps,
                            digests=np.array([tr["digests"][int(s)] for s in steps]))
        print("%s: %d sub-steps in %.1f s, final KE %.6g, avg error %.4g" % (
            m, T.STEPS, time.time() - t0, tr["kinetic_energy"][-1], tr["avg_error"][-1]))


if __name__ == "__main__":
    main(sys.argv[1:] or T.METHODS)
