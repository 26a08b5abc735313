"""Precision modes of every solver against the FP64 GPU oracle.

REFERENCE mode is the reference's FP32 arithmetic (bit-exact with it, see
test_gpu_parity.py); COMPENSATED mode uses Kahan-compensated neighbour sums,
exact FP64 error averages and FP64 position accumulators. Both are compared
with the FP64 oracle run with the same sub-step sizes and iteration counts;
the errors are stated by these tests (run with -s to see them)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


def test_fp64_oracle_first_step_agrees(E):
    """After one sub-step both FP32 modes agree with double precision to
    FP32 rounding: densities within 1e-5 relative, positions within 1e-5 dx."""
    from precision import compare
    for mode in (E.PRECISION_REFERENCE, E.PRECISION_COMPENSATED):
        r = compare(E, 48, 1, {1}, mode)[0]
        print("mode", mode, r)
        assert r["density_linf"] < 1e-5, r
        assert r["position_max_dx"] < 1e-5, r


def test_compensated_sums_are_closer_on_the_first_step(E):
    """From the same initial state, the compensated neighbour sums give
    densities closer to double precision than the reference's FP32 sums."""
    from precision import compare
    for n_side in (48, 96):
        ref = compare(E, n_side, 1, {1}, E.PRECISION_REFERENCE)[0]
        comp = compare(E, n_side, 1, {1}, E.PRECISION_COMPENSATED)[0]
        print("n_side", n_side, "reference", ref, "compensated", comp)
        assert comp["density_linf"] <= ref["density_linf"]
        assert comp["density_rms"] <= ref["density_rms"]


def test_double_positions_do_not_accumulate_rounding(E):
    """A scene 16 m from the origin, where a float position carries about
    2e-6 m of rounding: FP32 accumulation loses part of every sub-step's
    increment, the FP64 accumulators only round once. Over 10 sub-steps
    (before chaotic growth dominates) the compensated positions stay well
    closer to the FP64 oracle."""
    from precision import compare
    ref = compare(E, 48, 10, {10}, E.PRECISION_REFERENCE, offset=16.0)[0]
    comp = compare(E, 48, 10, {10}, E.PRECISION_COMPENSATED, offset=16.0)[0]
    print("offset 16 m: reference", ref, "compensated", comp)
    assert comp["position_rms_dx"] < 0.7 * ref["position_rms_dx"], (ref, comp)


def test_compensated_mode_meets_tolerance(E):
    """The compensated mode keeps the solver's exit test: every sub-step ends
    at or below the 0.05% average density error (or at the cap)."""
    from precision import dfsph_scene
    sim = E.Simulation.from_block_scene(dfsph_scene(E, 64, E.PRECISION_COMPENSATED))
    for _ in range(30):
        st = sim.advance("dfsph_p", 1)
        assert st["error_average"] <= 0.0005 or st["pressure_iterations"] == 100, st


def test_iisph_fp64_oracle_first_step_agrees(E):
    """IISPH after one sub-step: densities within 1e-5 relative of double
    precision, positions within 1e-4 dx, and the pressures the FP32 solve
    ends with within 1e-3 of the largest FP64 pressure."""
    from precision import compare
    for mode in (E.PRECISION_REFERENCE, E.PRECISION_COMPENSATED):
        r = compare(E, 48, 1, {1}, mode, method="iisph")[0]
        print("iisph mode", mode, r)
        assert r["iterations"] >= 2, r
        assert r["density_linf"] < 1e-5, r
        assert r["position_max_dx"] < 1e-4, r
        assert r["pressure_linf"] < 1e-3, r


def test_iisph_fp64_oracle_ten_steps(E):
    """Ten IISPH sub-steps of a 96x96 block: the FP32 run stays close to the
    FP64 oracle (RMS position error below 1e-3 dx, kinetic energy within
    1%), in both precision modes."""
    from precision import compare
    for mode in (E.PRECISION_REFERENCE, E.PRECISION_COMPENSATED):
        r = compare(E, 96, 10, {10}, mode, method="iisph")[0]
        print("iisph 10 sub-steps, mode", mode, r)
        assert r["position_rms_dx"] < 1e-3, r
        assert r["energy_rel_diff"] < 1e-2, r
        assert r["density_linf"] < 1e-3, r


@pytest.mark.parametrize("method", ["pcisph", "iisph", "iisph_ap", "iisph_pseudo_ap", "dfsph_p"])
def test_compensated_positions_follow_every_method(E, method):
    """A compensated scene keeps its FP64 positions (which the neighbour
    search reads) current under every method: ten sub-steps in compensated
    mode stay within rounding of the same ten in reference mode (RMS
    position difference below 1e-3 dx; a stale FP64 copy would leave the
    neighbour vectors at the initial positions and differ by far more)."""
    from precision import dfsph_scene, iisph_scene
    make = dfsph_scene if method == "dfsph_p" else iisph_scene
    out = []
    for mode in (E.PRECISION_REFERENCE, E.PRECISION_COMPENSATED):
        sc = make(E, 48, mode)
        sim = E.Simulation.from_block_scene(sc)
        for _ in range(10):
            sim.advance(method, 1)
        out.append(sim.state()[0].astype(np.float64))
        sim.close()
    dx = float(sc.dx)
    d = np.hypot(*(out[1] - out[0]).T) / dx
    print(method, "compensated vs reference after 10 sub-steps: RMS %.3e dx, max %.3e dx" % (
        float(np.sqrt(np.mean(d ** 2))), float(d.max())))
    assert np.all(np.isfinite(out[1]))
    assert float(np.sqrt(np.mean(d ** 2))) < 1e-3


@pytest.mark.parametrize("method", ["iisph_ap", "iisph_pseudo_ap", "pcisph"])
def test_fp64_oracle_first_step_every_solver(E, method):
    """IISPH_AP, IISPH_PSEUDO_AP and PCISPH after one sub-step of a 48x48
    block: densities within 1e-5 relative of double precision and velocities
    within 1e-4 of the largest FP64 speed (AP: about 2e-5 measured), 1e-3 for
    PCISPH (1.1e-4 measured: its artificial viscosity acts only on pairs
    with v_ij . x_ij < 0, and for pairs near zero FP32 and FP64 take
    different branches). A term missing from either side shows as 1e-2 or
    more. Both precision modes."""
    from precision import compare
    vtol = 1e-3 if method == "pcisph" else 1e-4
    for mode in (E.PRECISION_REFERENCE, E.PRECISION_COMPENSATED):
        r = compare(E, 48, 1, {1}, mode, method=method)[0]
        print(method, "mode", mode, r)
        assert r["iterations"] >= 2, r
        assert r["density_linf"] < 1e-5, r
        assert r["velocity_linf_rel"] < vtol, r
        if method != "pcisph":
            assert r["pressure_linf"] < 1e-3, r


@pytest.mark.parametrize("method", ["iisph_ap", "iisph_pseudo_ap", "pcisph"])
def test_fp64_oracle_ten_steps_every_solver(E, method):
    """Ten sub-steps of a 96x96 block: kinetic energy within 1% of the FP64
    oracle and densities within 1e-3 relative, in reference mode."""
    from precision import compare
    r = compare(E, 96, 10, {10}, E.PRECISION_REFERENCE, method=method)[0]
    print(method, "10 sub-steps", r)
    assert r["energy_rel_diff"] < 1e-2, r
    assert r["density_linf"] < 1e-3, r
