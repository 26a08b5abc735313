"""Regenerates the golden fixtures in tests/golden/ from the reference.

Runs the unmodified emerald sources compiled against the project's shims
(oracle/_ref/libemerald_ref.so, built by oracle/build_oracle.py from the
reference's sources) and stores small inputs and outputs as .npz files:

* uniform_7927.npz: the 7927-point fixture of the reference's own tests
  (emerald/sph_common/tests/test_neighborhood.cpp:18-31: std::mt19937_64{17272},
  U(-100, 100)), with the reference's sort products and neighbour lists for
  cell size 2.1 (test_neighborhood.cpp:177-292).
* run_<method>.npz: a 24x24 block scene (dx = 1/48, support = dx) advanced
  six fixed-dt sub-steps by each solver; positions, velocities and densities
  after every sub-step.
* frames_default.npz: the reference's default scene (world walls, hex dam
  break) advanced two frames by DFSPH_P and IISPH.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from cpu_checkers import Reference, ensure_built  # noqa: E402
from scenes import F, walls  # noqa: E402

METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]


def block_params(R, dx, mass, denom):
    rp = R.default_params()
    rp.update(support=dx, iisph_max_pressure_iterations=50, iisph_error_average_threshold=0.001,
              dfsph_divergence_error_average_threshold=0.001,
              dfsph_density_error_average_threshold=0.0005, time_per_step_flicks=1411200,
              sub_steps=4, mass_per_particle_override=mass,
              pressure_correction_denom_override=denom)
    return rp


def main():
    ensure_built()
    R = Reference()
    R.set_threads(1)
    pts = R.uniform_points(7927, 17272, -100.0, 100.0)
    nb = R.self_neighborhoods(pts, 2.1)
    keep = ("grid_coords", "z_indices", "pair_index", "block_indices", "counts", "idx")
    np.savez_compressed(os.path.join(HERE, "uniform_7927.npz"), xy=pts,
                        **{k: nb[k] for k in keep})

    n = 24
    dx = F(1.0 / 48)
    # lattice mass and PCISPH denominator of the square template, as computed by
    # the product (checked against tests/scenes.py in the CPU tests)
    import emerald_b200 as E
    mass, denom = E.lattice_config(E.default_params(support=dx), dx, F(352800 / 705600000.0))
    xy = R.block_scene(n, n, dx)
    w = walls(dx)
    vol = np.full(len(w), F(mass) / F(1000.0), np.float32)
    for m in METHODS:
        rp = block_params(R, dx, mass, denom)
        dt = F(352800 / 705600000.0) if m == "pcisph" else F(1e-4)
        sim = R.sim(rp, w, xy, None, vol)
        sim.begin_frame(m)
        xs, vs, ds = [], [], []
        for s in range(6):
            sim.sub_step(m, F(s * dt), dt)
            x, v = sim.state()
            xs.append(x)
            vs.append(v)
            ds.append(sim.array("densities"))
        np.savez_compressed(os.path.join(HERE, "run_%s.npz" % m), fluid=xy, solid=w,
                            solid_volumes=vol, mass=mass, denom=denom, dx=dx, dt=dt,
                            x=np.array(xs), v=np.array(vs), rho=np.array(ds))

    rp = R.default_params()
    out = {}
    for m in ["dfsph_p", "iisph"]:
        sim = R.sim(rp)
        sx, svol = sim.solid()
        x0, _ = sim.state()
        out["solid"] = sx
        out["solid_volumes"] = svol
        out["fluid"] = x0
        for f in range(2):
            sim.frame(m)
            x, v = sim.state()
            out["%s_x%d" % (m, f)] = x
            out["%s_v%d" % (m, f)] = v
    np.savez_compressed(os.path.join(HERE, "frames_default.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
