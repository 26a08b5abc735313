"""The CUDA path against the oracle and the reference's golden runs.

Every comparison is bit-exact: positions, velocities, densities, neighbour
lists and sort products of the GPU sub-step must equal the reference's."""
import os

import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def golden_params(E, g):
    return E.default_params(support=g["dx"], time_per_step_flicks=1411200, sub_steps=4,
                            iisph_max_pressure_iterations=50,
                            iisph_error_average_threshold=F(0.001),
                            dfsph_divergence_error_average_threshold=F(0.001),
                            dfsph_density_error_average_threshold=F(0.0005),
                            mass_per_particle=g["mass"], pressure_correction_denom=g["denom"])


def oracle_params(E, p):
    d = p.as_dict()
    cfg = E.config(p)
    out = {k: d[k] for k in d if k not in ("seed", "length")}
    out.update(mass_per_particle=cfg["mass_per_particle"],
               pressure_correction_denom=cfg["pressure_correction_denom"],
               seconds_per_sub_step=cfg["seconds_per_sub_step"])
    return out


@pytest.mark.parametrize("method", METHODS)
def test_golden_runs(E, method):
    """Six fixed-dt sub-steps of each solver equal the reference's run."""
    g = dict(np.load(os.path.join(GOLDEN, "run_%s.npz" % method)))
    sim = E.Simulation(golden_params(E, g), g["solid"], g["fluid"], None, g["solid_volumes"])
    sim.begin_frame(method)
    dt = g["dt"]
    for s in range(len(g["x"])):
        sim.sub_step(method, F(s * dt), dt)
        x, v = sim.state()
        assert_bitwise(x, g["x"][s], "%s x after sub-step %d" % (method, s))
        assert_bitwise(v, g["v"][s], "%s v after sub-step %d" % (method, s))
        assert_bitwise(sim.array("densities"), g["rho"][s], "%s densities %d" % (method, s))


@pytest.mark.parametrize("method", METHODS)
def test_substeps_match_oracle(E, oracle, method):
    """Ten sub-steps of a jittered 48x48 block with every solver temporary,
    the neighbour lists and the iteration counts compared."""
    scene = E.BlockScene(48, dx=F(1 / 96), seed=5, dt=F(352800 / 705600000.0),
                         iisph_max_pressure_iterations=50,
                         iisph_error_average_threshold=F(0.001),
                         time_per_step_flicks=1411200, sub_steps=4)
    sim = E.Simulation.from_block_scene(scene)
    osim = oracle.sim(oracle_params(E, scene.params), scene.solid, scene.solid_volumes,
                      scene.fluid)
    dt = F(352800 / 705600000.0) if method == "pcisph" else F(2e-4)
    sim.begin_frame(method)
    osim.begin_frame(method)
    for s in range(10):
        st = sim.sub_step(method, F(s * dt), dt)
        ost = osim.sub_step(method, F(s * dt), dt)
        assert st["pressure_iterations"] == ost["pressure_iterations"], (s, st, ost)
        if method == "dfsph_p":
            assert st["divergence_iterations"] == ost["divergence_iterations"], (s, st, ost)
        x, v = sim.state()
        ox, ov = osim.state()
        assert_bitwise(x, ox, "%s x %d" % (method, s))
        assert_bitwise(v, ov, "%s v %d" % (method, s))
    names = {"pcisph": ["densities", "pressures", "pressure_forces", "position_stars",
                        "velocity_stars", "velocity_external_forces"],
             "iisph": ["densities", "pressures", "density_stars", "aiis", "diis", "sum_dij_pjs"],
             "iisph_ap": ["densities", "pressures", "density_stars", "aiis",
                          "pressure_accelerations"],
             "iisph_pseudo_ap": ["densities", "pressures", "density_stars", "aiis",
                                 "pressure_accelerations"],
             "dfsph_p": ["densities", "density_stars", "alphas", "divergence_kappas",
                         "density_kappas"]}[method]
    for name in names:
        assert_bitwise(sim.array(name), osim.array(name), "%s %s" % (method, name))
    for solid in (False, True):
        c1, i1, w1, g1 = sim.neighbors(solid)
        c2, i2, w2, g2 = osim.neighbors(solid)
        assert_bitwise(c1, c2, "counts")
        assert_bitwise(i1, i2, "indices")
        if method != "pcisph":
            assert_bitwise(w1, w2, "W")
            assert_bitwise(g1, g2, "grad W")


@pytest.mark.parametrize("method", ["dfsph_p", "iisph", "pcisph", "iisph_pseudo_ap"])
def test_adaptive_frames_match_oracle(E, oracle, method):
    scene = E.BlockScene(40, dx=F(1 / 80), seed=2, dt=F(352800 / 705600000.0),
                         time_per_step_flicks=1411200, sub_steps=4)
    sim = E.Simulation.from_block_scene(scene)
    osim = oracle.sim(oracle_params(E, scene.params), scene.solid, scene.solid_volumes,
                      scene.fluid)
    for f in range(3):
        st = sim.frame(method)
        k = osim.frame(method)
        assert st["sub_steps"] == k
        assert sim.time() == osim.time()
        x, v = sim.state()
        ox, ov = osim.state()
        assert_bitwise(x, ox, "%s frame %d x" % (method, f))
        assert_bitwise(v, ov, "%s frame %d v" % (method, f))


def test_advance_equals_frames(E):
    scene = E.BlockScene(32, dx=F(1 / 64), seed=4, time_per_step_flicks=1411200, sub_steps=4)
    a = E.Simulation.from_block_scene(scene)
    b = E.Simulation.from_block_scene(scene)
    n = 0
    for _ in range(3):
        n += a.frame("dfsph_p")["sub_steps"]
    b.advance("dfsph_p", n)
    assert_bitwise(a.state()[0], b.state()[0], "x")
    assert a.time() == b.time()


def test_advance_host_equals_separate_calls(E):
    """One emerald_sim_advance_host call per sub-step (state in, advance,
    state out) equals set_state, advance and get_state."""
    scene = E.BlockScene(24, dx=F(1 / 48), seed=6, time_per_step_flicks=1411200, sub_steps=4)
    a = E.Simulation.from_block_scene(scene)
    b = E.Simulation.from_block_scene(scene)
    x, v = a.state()
    for _ in range(4):
        a.set_state(x, v)
        a.advance("dfsph_p", 1)
        x, v = a.state()
    xb, vb = b.state()
    for _ in range(4):
        b.advance_host("dfsph_p", 1, xb, vb)
    assert_bitwise(xb, x, "x")
    assert_bitwise(vb, v, "v")
    assert a.time() == b.time()


def test_default_scene_frames(E):
    """The reference's own dam break (hex lattice, world walls with 16 blocks,
    boundary volumes 1.7/sum W computed on the GPU)."""
    g = dict(np.load(os.path.join(GOLDEN, "frames_default.npz")))
    p = E.default_params()
    for m in ["dfsph_p", "iisph"]:
        sim = E.Simulation(p, g["solid"], g["fluid"])
        _, vol = sim.solid()
        assert_bitwise(vol, g["solid_volumes"], "boundary volumes")
        for f in range(2):
            sim.frame(m)
            x, v = sim.state()
            assert_bitwise(x, g["%s_x%d" % (m, f)], "%s frame %d x" % (m, f))
            assert_bitwise(v, g["%s_v%d" % (m, f)], "%s frame %d v" % (m, f))


def test_fixture_neighbors_and_sort(E):
    """The reference test fixture (7927 points in [-100, 100]^2, cell 2.1):
    negative cells exercise the full 64-bit key range, including the key of
    cell (-1, -1), which equals the table's empty marker."""
    g = dict(np.load(os.path.join(GOLDEN, "uniform_7927.npz")))
    p = E.default_params(support=F(1.05))
    far = np.array([[1e4, 1e4]], np.float32)
    sim = E.Simulation(p, far, g["xy"], None, np.ones(1, np.float32))
    sim.sub_step("pcisph", 0.0, F(1e-6))
    counts, idx, _, _ = sim.neighbors()
    assert_bitwise(counts, g["counts"], "counts")
    assert_bitwise(idx, g["idx"], "indices")
    s = sim.sort()
    assert_bitwise(s["grid_coords"], g["grid_coords"], "grid coords")
    assert_bitwise(s["z_indices"], g["z_indices"], "z")
    assert_bitwise(s["pair_index"], g["pair_index"], "pair index")
    assert_bitwise(s["block_indices"], g["block_indices"], "block indices")
    assert np.all(np.diff(s["pair_z"].astype(np.float64)) >= 0) or np.all(
        s["pair_z"][1:] >= s["pair_z"][:-1])


def test_sort_products_match_oracle(E, oracle):
    scene = E.BlockScene(64, dx=F(1 / 128), seed=9)
    sim = E.Simulation.from_block_scene(scene)
    x0 = scene.fluid
    sim.sub_step("dfsph_p", 0.0, F(1e-4))
    for solid, pts in ((False, x0), (True, scene.solid)):
        s = sim.sort(solid)
        o = oracle.sort(pts, F(2 * scene.support))
        for k in ("grid_coords", "z_indices", "pair_z", "pair_index", "block_indices", "blocks"):
            assert_bitwise(s[k], o[k].astype(s[k].dtype), "%s %s" % ("solid" if solid else "fluid", k))


def test_large_scene_matches_oracle(E, oracle):
    """The 512x512 (262144-particle) dam break of the DFSPH benchmark, two
    adaptive sub-steps against the oracle."""
    scene = E.BlockScene(512, dx=F(1 / 1024), seed=1, time_per_step_flicks=1411200, sub_steps=4,
                         dfsph_divergence_error_average_threshold=F(0.001),
                         dfsph_density_error_average_threshold=F(0.0005))
    sim = E.Simulation.from_block_scene(scene)
    osim = oracle.sim(oracle_params(E, scene.params), scene.solid, scene.solid_volumes,
                      scene.fluid)
    oracle.set_threads(os.cpu_count() or 1)
    sim.begin_frame("dfsph_p")
    osim.begin_frame("dfsph_p")
    try:
        for s in range(2):
            osim.sub_step("dfsph_p", F(s * 2e-4), F(2e-4))
            sim.sub_step("dfsph_p", F(s * 2e-4), F(2e-4))
    finally:
        oracle.set_threads(1)
    assert_bitwise(sim.state()[0], osim.state()[0], "x")
    assert_bitwise(sim.state()[1], osim.state()[1], "v")
    counts, idx, _, _ = sim.neighbors()
    c2, i2, _, _ = osim.neighbors()
    assert_bitwise(counts, c2, "counts")
    assert_bitwise(idx, i2, "indices")


@pytest.mark.parametrize("method", METHODS)
def test_graph_and_eager_modes_agree(E, method):
    """A sub-step as one CUDA graph (solver loops as conditional nodes, three
    iterations per body launch) and as host-driven kernel launches (one exit
    test on the host per iteration) give the same bits and iteration counts."""
    scene = E.BlockScene(32, dx=F(1 / 64), seed=8, time_per_step_flicks=1411200, sub_steps=4,
                         iisph_max_pressure_iterations=50,
                         iisph_error_average_threshold=F(0.001))
    a = E.Simulation.from_block_scene(scene)
    b = E.Simulation.from_block_scene(scene)
    b.set_graphs(False)
    for f in range(2):
        sa = a.frame(method)
        sb = b.frame(method)
        assert sa["sub_steps"] == sb["sub_steps"]
        assert sa["pressure_iterations"] == sb["pressure_iterations"]
        assert_bitwise(a.state()[0], b.state()[0], "x")
        assert_bitwise(a.state()[1], b.state()[1], "v")
    # a graph's loop body runs several iterations; kernels of iterations past
    # convergence launch and return at once, so graphs launch at least as many
    assert a.kernel_launches() >= b.kernel_launches()


def test_dense_cells_take_the_fallback_path(E, oracle):
    """A lattice with dense clusters: a cell with 50 members (more than a
    warp), a 3x3 block with more than 128 candidates, and a particle with
    more than 64 neighbours inside the radius (the reference keeps the first
    64 in scan order). Fluid and boundary lists equal the oracle's."""
    rng = np.random.Generator(np.random.PCG64(4))
    dx = F(1 / 80)
    g = (np.arange(40, dtype=np.float32) + F(0.5)) * dx
    lattice = np.stack(np.meshgrid(g, g), -1).reshape(-1, 2).astype(np.float32)
    cell = F(2 * dx)
    c1 = (F(0.2) + rng.uniform(0.0, 0.9, (50, 2)).astype(np.float32) * cell).astype(np.float32)
    c2 = (F(0.6) + rng.uniform(-1.4, 1.4, (150, 2)).astype(np.float32) * cell).astype(np.float32)
    c3 = (F(0.35) + rng.uniform(-0.3, 0.3, (80, 2)).astype(np.float32) * cell).astype(np.float32)
    fluid = np.concatenate([lattice, c1, c2, c3]).astype(np.float32)
    solid = np.concatenate([
        np.stack([g, np.full_like(g, -dx / 2)], -1),
        (F(0.5) + rng.uniform(-1.2, 1.2, (140, 2)).astype(np.float32) * cell) * np.float32([1, 0]) +
        np.float32([0, -dx]),
    ]).astype(np.float32)
    p = E.default_params(support=dx)
    sim = E.Simulation(p, solid, fluid, None, np.full(len(solid), F(1e-4), np.float32))
    sim.sub_step("dfsph_p", 0.0, F(1e-6))
    for is_solid, other in ((False, fluid), (True, solid)):
        counts, idx, _, _ = sim.neighbors(is_solid)
        oc, oi, _, _ = oracle.neighborhoods(fluid, other, not is_solid, cell)
        assert counts.max() == 64 or is_solid
        assert_bitwise(counts, oc, "%s counts" % ("solid" if is_solid else "fluid"))
        mask = np.arange(64)[None, :] < oc[:, None]
        assert_bitwise(np.where(mask, idx, 0), np.where(mask, oi, 0),
                       "%s indices" % ("solid" if is_solid else "fluid"))


def test_pcisph_literal_support_matches_reference(E, reference):
    """PCISPH at the configs' literal support h = 2 dx (about 45 neighbours
    per particle, so every list takes the 64-entry path) against the
    compiled reference, frame by frame."""
    from cpu_checkers import RefParams
    sc = E.BlockScene(48, dx=F(1 / 96), seed=3, support_ratio=2.0, time_per_step_flicks=1411200,
                      sub_steps=4)
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=d["mass_per_particle"],
              pressure_correction_denom_override=d["pressure_correction_denom"])
    ref = reference.sim(rp, sc.solid, sc.fluid, None, sc.solid_volumes)
    sim = E.Simulation.from_block_scene(sc)
    for f in range(3):
        ref.frame("pcisph")
        sim.frame("pcisph")
        assert_bitwise(sim.state()[0], ref.state()[0], "x after frame %d" % f)
        assert_bitwise(sim.state()[1], ref.state()[1], "v after frame %d" % f)
    counts = sim.neighbors(False)[0]
    assert counts.mean() > 30, counts.mean()
    assert_bitwise(counts, ref.neighbors()[0], "neighbour counts")
    sim.close()


def spray_fluid(sc):
    """The block plus particles in the air, all farther than 2h from one
    another and from the block: ten lone droplets (no neighbours), two pairs
    h/2 apart, and two particles at the same position (distance 0, so W(0)
    and a zero gradient) on a cell corner (x = 7 cells, y = 12 cells of
    2h = 1/16 m, exact in float)."""
    h = float(sc.params.support)
    drops = [(x, y) for y in (0.8, 0.9) for x in (0.1, 0.3, 0.5, 0.7, 0.9)]
    pairs = [(0.2, 0.7), (0.2 + 0.5 * h, 0.7), (0.6, 0.7), (0.6 + 0.5 * h, 0.7)]
    same = [(0.4375, 0.75), (0.4375, 0.75)]
    extra = np.array(drops + pairs + same, np.float32)
    return np.concatenate([sc.fluid, extra]).astype(np.float32), len(extra)


@pytest.mark.parametrize("method", METHODS)
def test_spray_scene_matches_reference(E, reference, method):
    """Zero-neighbour particles, two-particle clusters and coincident
    particles take the empty-list and zero-gradient branches of every
    solver (dii, aii and alpha of 0, pressures left as they were); two
    frames equal the compiled reference bit for bit."""
    from cpu_checkers import RefParams
    sc = E.BlockScene(16, dx=F(1 / 32), seed=12, time_per_step_flicks=1411200, sub_steps=4,
                      iisph_max_pressure_iterations=50,
                      iisph_error_average_threshold=F(0.001))
    fluid, n_extra = spray_fluid(sc)
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=d["mass_per_particle"],
              pressure_correction_denom_override=d["pressure_correction_denom"])
    ref = reference.sim(rp, sc.solid, fluid, None, sc.solid_volumes)
    sim = E.Simulation(sc.params, sc.solid, fluid, None, sc.solid_volumes)
    for f in range(2):
        ref.frame(method)
        sim.frame(method)
        assert_bitwise(sim.state()[0], ref.state()[0], "%s x after frame %d" % (method, f))
        assert_bitwise(sim.state()[1], ref.state()[1], "%s v after frame %d" % (method, f))
    counts = sim.neighbors(False)[0]
    assert np.all(counts[-n_extra:-6] == 0)
    assert np.all(counts[-6:] == 1)
    x = sim.state()[0]
    assert np.array_equal(x[-1], x[-2])
    sim.close()


@pytest.mark.parametrize("method", METHODS)
def test_empty_fluid_scene_steps(E, method):
    """A scene with walls and no fluid particles frames without error and
    returns empty state arrays."""
    sc = E.BlockScene(16, dx=F(1 / 32), seed=12, time_per_step_flicks=1411200, sub_steps=4)
    sim = E.Simulation(sc.params, sc.solid, np.zeros((0, 2), np.float32), None,
                       sc.solid_volumes)
    st = sim.frame(method)
    assert st["sub_steps"] >= 1
    x, v = sim.state()
    assert x.shape == (0, 2) and v.shape == (0, 2)
    sim.close()


def test_bench_arms_share_the_trajectory(E, reference):
    """The bench's reference arm (sub-steps [W, W + K) of the reference's own
    frame loop, scene built by the harness alone) and its GPU arm (W
    sub-steps of warm-up, then K) end on the same state bit for bit, so both
    time the same work."""
    import bench
    bench.configure_scene(48)
    try:
        rp, fluid, solid, volumes = bench.reference_scene(reference)
        ref = reference.sim(rp, solid, fluid, None, volumes)
        timed, _ = ref.run_window("dfsph_p", 5, 7)
        assert timed == 7
        sim = E.Simulation.from_block_scene(E.BlockScene(bench.N_SIDE, **bench.scene_kwargs()))
        sim.advance("dfsph_p", 5, stats=False)
        sim.advance("dfsph_p", 7, stats=False)
        x, v = sim.state()
        rx, rv = ref.state()
        assert_bitwise(x, rx, "positions after the bench window")
        assert_bitwise(v, rv, "velocities after the bench window")
        sim.close()
    finally:
        bench.configure_scene(512)


@pytest.mark.parametrize("method", ["dfsph_p", "iisph", "pcisph"])
def test_frame_is_one_graph_launch(E, oracle, method):
    """emerald_sim_frame runs a frame as one graph launch (a conditional
    while node around the sub-step) and waits on the host once: after the
    first frame (which captures the graphs), every frame costs one host
    wait, runs the oracle's sub-step count and ends on its state bit for
    bit. Frames alternate between two graphs, one that re-sorts the
    particles' storage order first and one that does not, so the first two
    frames capture. A frame begun by emerald_sim_advance is finished, not
    restarted."""
    scene = E.BlockScene(40, dx=F(1 / 80), seed=13, time_per_step_flicks=1411200, sub_steps=4,
                         dfsph_divergence_error_average_threshold=F(0.001),
                         dfsph_density_error_average_threshold=F(0.0005))
    sim = E.Simulation.from_block_scene(scene)
    osim = oracle.sim(oracle_params(E, scene.params), scene.solid, scene.solid_volumes,
                      scene.fluid)
    for _ in range(2):
        sim.frame(method)
        osim.frame(method)
    waits = []
    for _ in range(3):
        w0 = sim.host_waits()
        st = sim.frame(method)
        waits.append(sim.host_waits() - w0)
        assert st["sub_steps"] == osim.frame(method)
    assert waits == [1, 1, 1], waits
    assert_bitwise(sim.state()[0], osim.state()[0], "%s positions after 5 frames" % method)
    assert_bitwise(sim.state()[1], osim.state()[1], "%s velocities after 5 frames" % method)
    # two sub-steps into the sixth frame, then the frame call finishes it
    sim.advance(method, 2, stats=False)
    st = sim.frame(method)
    k = osim.frame(method)
    assert st["sub_steps"] == k - 2, (st["sub_steps"], k)
    assert_bitwise(sim.state()[0], osim.state()[0], "%s positions after a split frame" % method)
    sim.close()
