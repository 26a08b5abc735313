"""The CPU oracle (oracle/sph_oracle.c) against the reference's known
answers, its test fixture and golden runs of the reference itself."""
import os

import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
METHODS = ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"]


def spread_reference(v, bits=32):
    """Single_axis_index<2, BIT>::encode (emerald/z_index/z_index.h:11-24)."""
    out = 0
    for b in range(bits):
        out |= ((v >> b) & 1) << (2 * b)
    return out


# Known answers of emerald/z_index/tests/test_z_index.cpp:11-70.
Z_ENCODE_KATS = [
    (0b111, 0b111, 0b0011_1111),
    (0xFFFF, 0xFFFF, 0xFFFF_FFFF),
    (0, 0xFFFF, 0b1010_1010_1010_1010_1010_1010_1010_1010),
    (0xFFFF_FFFF, 0xFFFF_FFFF, 0xFFFF_FFFF_FFFF_FFFF),
]


@pytest.mark.parametrize("x,y,z", Z_ENCODE_KATS)
def test_z_index_known_answers(oracle, x, y, z):
    assert oracle.z_index(x, y) == z


@pytest.mark.parametrize("v", [21430205, 0b111, 0xFFFF, 0xFF00, 0xFFFF_FFFF, 0x8000_0001])
def test_z_index_single_axis(oracle, v):
    assert oracle.z_index(v, 0) == spread_reference(v)
    assert oracle.z_index(0, v) == spread_reference(v) << 1


def test_spread_known_answers():
    assert spread_reference(0b111) == 0b10101
    assert spread_reference(0xFFFF) == 0x5555_5555
    assert spread_reference(0xFF00) == 0x5555_0000


# emerald/sph_common/tests/test_common.cpp:42-63
@pytest.mark.parametrize("p,cell,expected", [
    ((-2.4, 9.11), 2.95, (-1, 3)),
    ((4.1, 5.9), 1.0, (4, 5)),
    ((-4.1, -5.9), 1.0, (-5, -6)),
])
def test_grid_coord_known_answers(oracle, p, cell, expected):
    s = oracle.sort(np.array([p], np.float32), F(cell))
    assert tuple(s["grid_coords"][0]) == expected


@pytest.fixture(scope="module")
def fixture7927():
    return dict(np.load(os.path.join(GOLDEN, "uniform_7927.npz")))


def test_fixture_sort_matches_reference(oracle, fixture7927):
    xy = fixture7927["xy"]
    s = oracle.sort(xy, F(2.1))
    assert_bitwise(s["grid_coords"], fixture7927["grid_coords"], "grid coords")
    assert_bitwise(s["z_indices"], fixture7927["z_indices"], "z")
    assert_bitwise(s["pair_index"], fixture7927["pair_index"], "sorted pair indices")
    assert_bitwise(s["block_indices"], fixture7927["block_indices"], "block indices")
    # the sort is the lexicographic order of (z, index), as std::sort
    order = np.lexsort((np.arange(len(xy)), s["z_indices"]))
    assert np.array_equal(order, s["pair_index"])
    # blocks: unique keys, ranges cover all pairs (test_neighborhood.cpp:90-175)
    assert len(s["blocks"]) == len(np.unique(s["z_indices"]))
    assert s["blocks"][0][0] == 0 and s["blocks"][-1][1] == len(xy)
    assert np.all(s["blocks"][1:, 0] == s["blocks"][:-1, 1])


def test_reference_sort_functions_match_fixture(reference, oracle, fixture7927):
    """The harness's per-function wrappers around the reference's own
    compute_index_pairs, sort_index_pairs, compute_block_indices,
    fill_blocks, create_block_map and create_regular_neighborhoods (the
    checkers of the device versions) reproduce the fixture's sort products
    and lists, with the grid at the origin."""
    from cpu_checkers import ptr
    xy = np.ascontiguousarray(fixture7927["xy"], np.float32)
    n = len(xy)
    L = reference.L
    gc = np.zeros((n, 2), np.int32)
    L.ref_common_grid_coords(n, F(2.1), F(0.0), F(0.0), ptr(gc), ptr(xy))
    assert_bitwise(gc, fixture7927["grid_coords"], "grid coords")
    z = np.zeros(n, np.uint64)
    L.ref_common_z_indices(n, ptr(z), ptr(gc))
    pairs = np.zeros((n, 2), np.uint64)
    L.ref_common_index_pairs(n, ptr(pairs), ptr(z))
    assert_bitwise(pairs[:, 1], np.arange(n, dtype=np.uint64), "unsorted pair indices")
    L.ref_common_sort_index_pairs(n, ptr(pairs))
    assert_bitwise(pairs[:, 1], fixture7927["pair_index"].astype(np.uint64), "sorted pairs")
    bi = np.zeros(n, np.uint32)
    L.ref_common_block_indices(n, ptr(bi), ptr(pairs))
    assert_bitwise(bi, fixture7927["block_indices"], "block indices")
    nb = int(bi[-1]) + 1
    blocks = np.zeros((nb, 2), np.uint64)
    L.ref_common_fill_blocks(n, nb, ptr(blocks), ptr(bi))
    assert_bitwise(blocks, oracle.sort(xy, F(2.1))["blocks"].astype(np.uint64), "blocks")
    counts = np.zeros(n, np.uint8)
    idx = np.zeros((n, 64), np.uint64)
    dist = np.zeros((n, 64), np.float32)
    vec = np.zeros((n, 64, 2), np.float32)
    L.ref_common_regular_neighborhoods(n, n, F(2.1), ptr(counts), ptr(idx), ptr(dist), ptr(vec),
                                       ptr(xy), ptr(gc), ptr(xy), 1, n, ptr(pairs), nb,
                                       ptr(blocks))
    assert_bitwise(counts, fixture7927["counts"], "counts")
    live = np.arange(64)[None, :] < counts[:, None]
    assert_bitwise(np.where(live, idx, 0), np.where(live, fixture7927["idx"], 0).astype(np.uint64),
                   "indices")


def test_fixture_neighbors_match_reference(oracle, fixture7927):
    xy = fixture7927["xy"]
    counts, idx, dist, vec = oracle.neighborhoods(xy, xy, True, F(2.1))
    assert_bitwise(counts, fixture7927["counts"], "counts")
    assert_bitwise(idx, fixture7927["idx"], "indices")


def test_fixture_neighbors_brute_force(oracle, fixture7927):
    """Completeness and exactness of the lists against an O(N^2) search, as
    emerald/sph_common/tests/test_neighborhood.cpp:177-292 checks them."""
    xy = fixture7927["xy"]
    cell = F(2.1)
    counts, idx, dist, vec = oracle.neighborhoods(xy, xy, True, cell)
    n = len(xy)
    for lo in range(0, n, 1024):
        d = xy[None, :, :] - xy[lo:lo + 1024, None, :]  # float32 (pj - pi)
        l2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]
        r = np.sqrt(l2.astype(np.float32))
        for k in range(d.shape[0]):
            i = lo + k
            near = np.nonzero((r[k] < cell) & (np.arange(n) != i))[0]
            assert counts[i] == len(near)
            got = idx[i, :counts[i]]
            assert set(got.tolist()) == set(near.tolist())
            pos = {j: a for a, j in enumerate(got.tolist())}
            for j in near:
                a = pos[j]
                assert vec[i, a, 0] == d[k, j, 0] and vec[i, a, 1] == d[k, j, 1]
                assert dist[i, a] == r[k, j]
            key = list(zip(dist[i, :counts[i]].tolist(), got.tolist()))
            assert key == sorted(key)


def test_kernel_shape(oracle):
    h = F(0.5)
    w0 = oracle.kernel_w(0.0, h)
    assert w0 > 0 and oracle.kernel_w(float(2 * h), h) == 0.0
    assert oracle.kernel_w(float(2 * h) + 1e-3, h) == 0.0
    g = oracle.kernel_grad_w(0.0, 0.0, h)
    assert g[0] == 0.0 and g[1] == 0.0


def _golden_sim(oracle, m):
    g = dict(np.load(os.path.join(GOLDEN, "run_%s.npz" % m)))
    p = dict(time_per_step_flicks=1411200, sub_steps=4, support=g["dx"], gravity=F(9.81),
             viscosity=F(0.01), target_density=F(1000.0), iisph_max_pressure_iterations=50,
             iisph_error_average_threshold=F(0.001), iisph_error_max_threshold=F(0.05),
             iisph_omega=F(0.5), dfsph_max_correction_iterations=15,
             dfsph_density_error_average_threshold=F(0.0005),
             dfsph_density_error_max_threshold=F(0.03),
             dfsph_divergence_error_average_threshold=F(0.001),
             dfsph_divergence_error_max_threshold=F(0.03), mass_per_particle=g["mass"],
             pressure_correction_denom=g["denom"], seconds_per_sub_step=F(352800 / 705600000.0))
    return g, p


@pytest.mark.parametrize("method", METHODS)
def test_oracle_golden_runs(oracle, method):
    g, p = _golden_sim(oracle, method)
    sim = oracle.sim(p, g["solid"], g["solid_volumes"], g["fluid"])
    sim.begin_frame(method)
    dt = g["dt"]
    for s in range(len(g["x"])):
        sim.sub_step(method, F(s * dt), dt)
        x, v = sim.state()
        assert_bitwise(x, g["x"][s], "%s x step %d" % (method, s))
        assert_bitwise(v, g["v"][s], "%s v step %d" % (method, s))
        assert_bitwise(sim.array("densities"), g["rho"][s], "%s rho step %d" % (method, s))


def test_oracle_default_scene_frames(oracle, reference):
    g = dict(np.load(os.path.join(GOLDEN, "frames_default.npz")))
    rp = reference.default_params()
    cfg = reference.config(rp)
    vol = oracle.solid_volumes(g["solid"], rp["support"], 1.7)
    assert_bitwise(vol, g["solid_volumes"], "boundary volumes")
    p = {k: rp[k] for k in ["time_per_step_flicks", "sub_steps", "support", "gravity", "viscosity",
                            "target_density", "iisph_max_pressure_iterations",
                            "iisph_error_average_threshold", "iisph_error_max_threshold",
                            "iisph_omega", "dfsph_max_correction_iterations",
                            "dfsph_density_error_average_threshold",
                            "dfsph_density_error_max_threshold",
                            "dfsph_divergence_error_average_threshold",
                            "dfsph_divergence_error_max_threshold"]}
    p.update(mass_per_particle=cfg["mass_per_particle"],
             pressure_correction_denom=cfg["pressure_correction_denom"],
             seconds_per_sub_step=cfg["seconds_per_sub_step"])
    for m in ["dfsph_p", "iisph"]:
        sim = oracle.sim(p, g["solid"], None, g["fluid"])
        for f in range(2):
            sim.frame(m)
            x, v = sim.state()
            assert_bitwise(x, g["%s_x%d" % (m, f)], "%s frame %d x" % (m, f))
            assert_bitwise(v, g["%s_v%d" % (m, f)], "%s frame %d v" % (m, f))


@pytest.mark.parametrize("method", METHODS)
def test_oracle_matches_reference_live(oracle, reference, method):
    """Twelve sub-steps of a 40x40 scene, the reference run live."""
    import emerald_b200 as E
    from scenes import walls
    dx = F(1.0 / 80)
    dt = F(352800 / 705600000.0) if method == "pcisph" else F(2e-4)
    mass, denom = E.lattice_config(E.default_params(support=dx), dx, F(352800 / 705600000.0))
    xy = reference.block_scene(40, 40, dx, 0.0, 0.0, 0.01, 3)
    w = walls(dx)
    vol = np.full(len(w), F(mass) / F(1000.0), np.float32)
    rp = reference.default_params()
    rp.update(support=dx, time_per_step_flicks=1411200, sub_steps=4,
              mass_per_particle_override=mass, pressure_correction_denom_override=denom)
    rs = reference.sim(rp, w, xy, None, vol)
    cfg = reference.config(rp)
    p = {k: rp[k] for k in rp if k not in ("seed", "length", "mass_per_particle_override",
                                          "pressure_correction_denom_override")}
    p.update(mass_per_particle=cfg["mass_per_particle"],
             pressure_correction_denom=cfg["pressure_correction_denom"],
             seconds_per_sub_step=cfg["seconds_per_sub_step"])
    os_ = oracle.sim(p, w, vol, xy)
    rs.begin_frame(method)
    os_.begin_frame(method)
    for s in range(12):
        rs.sub_step(method, F(s * dt), dt)
        os_.sub_step(method, F(s * dt), dt)
    assert_bitwise(os_.state()[0], rs.state()[0], "x")
    assert_bitwise(os_.state()[1], rs.state()[1], "v")
    c1, i1, w1, g1 = rs.neighbors()
    c2, i2, w2, g2 = os_.neighbors()
    assert_bitwise(c2, c1, "counts")
    assert_bitwise(i2, i1, "indices")
    if method != "pcisph":
        assert_bitwise(w2, w1, "W")
        assert_bitwise(g2, g1, "grad W")


def test_oracle_thread_count_invariance(oracle):
    g, p = _golden_sim(oracle, "dfsph_p")
    outs = []
    for t in (1, 4):
        oracle.set_threads(t)
        sim = oracle.sim(p, g["solid"], g["solid_volumes"], g["fluid"])
        sim.begin_frame("dfsph_p")
        for s in range(3):
            sim.sub_step("dfsph_p", F(s * 1e-4), F(1e-4))
        outs.append(sim.state()[0])
    oracle.set_threads(1)
    assert_bitwise(outs[0], outs[1], "x")


def test_literal_h2dx_scene_is_unstable_in_the_reference(reference):
    """The configs' literal kernel radius (support h = 2 dx) with the
    reference's own mass per particle and boundary volumes (compute_volumes,
    1.7 / sum W) blows up within the first DFSPH frame in the compiled
    reference itself, which is why the benchmark scenes use support = dx."""
    import emerald_b200 as E
    from cpu_checkers import RefParams
    dx = F(1 / 128)
    sc = E.BlockScene(64, dx=dx, seed=1, support_ratio=2.0, time_per_step_flicks=1411200,
                      sub_steps=4, dfsph_max_correction_iterations=100,
                      dfsph_divergence_error_average_threshold=F(0.001),
                      dfsph_density_error_average_threshold=F(0.0005))
    d = sc.params.as_dict()
    rp = {k: d[k] for k, _ in RefParams._fields_ if k in d}
    rp.update(mass_per_particle_override=0.0, pressure_correction_denom_override=0.0)
    ref = reference.sim(rp, sc.solid, sc.fluid, None, None)
    ref.frame("dfsph_p")
    v = ref.state()[1].astype(np.float64)
    assert np.sqrt((v * v).sum(1)).max() > 100.0


@pytest.mark.parametrize("method", METHODS)
def test_oracle_traces_match_reference(oracle, method):
    """All 1000 fixed-dt sub-steps of the reference's trace fixtures
    (tests/golden/trace_<method>.npz; the 128 x 128 dam-break block of
    tests/traces.py): density-error and kinetic-energy traces equal at every
    sub-step, positions and velocities bit-identical after sub-steps 1, 10,
    100 and 1000. About 12 s per solver on 8 host threads."""
    import traces as T
    g = dict(np.load(os.path.join(GOLDEN, "trace_scene.npz")))
    ref = np.load(os.path.join(GOLDEN, "trace_%s.npz" % method))
    p = dict(_golden_sim(oracle, method)[1])
    p.update(support=g["dx"], mass_per_particle=g["mass"], pressure_correction_denom=g["denom"],
             seconds_per_sub_step=T.PCISPH_DT)
    oracle.set_threads(os.cpu_count() or 1)
    try:
        sim = oracle.sim(p, g["solid"], g["solid_volumes"], g["fluid"])
        tr = T.run_trace(sim, method, g["mass"])
    finally:
        oracle.set_threads(1)
    for key in ("kinetic_energy", "avg_error", "max_error", "exact_error"):
        assert np.array_equal(tr[key], ref[key]), (method, key)
    for s, h in zip(ref["digest_steps"], ref["digests"]):
        assert tr["digests"][int(s)] == str(h), (method, int(s))
