"""The solver operator functions (iisph_ops, dfsph_p_ops, pcisph_ops,
iisph_ap_ops, iisph_pseudo_ap_ops) on device memory against the
reference's own functions, compiled from its sources, on the same inputs:
every output bit for bit, the iteration functions' (average, max) error
pairs included.

Inputs: the block of device_ops.make_case with some neighbour counts
cleared (particles with no fluid neighbours, no boundary neighbours, or
neither), some densities zero and one denormal a_ii, so that every
safe-divide fallback and early return of the reference is taken. Each
function's inputs are the reference's outputs of the functions before it."""
import ctypes

import numpy as np
import pytest

from conftest import assert_bitwise
from cpu_checkers import ptr
from device_ops import Keep, check, dev, host, lists, make_case, nbhd, reference_kernels
from scenes import F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def E():
    import emerald_b200
    return emerald_b200


@pytest.fixture(scope="module")
def case(E, oracle, reference):
    c = make_case(E, oracle)
    n = c["n"]
    c["fc"] = c["fc"].copy()
    c["sc"] = c["sc"].copy()
    c["fc"][::37] = 0          # isolated: neither list
    c["sc"][::37] = 0
    c["fc"][11::59] = 0        # boundary neighbours only, where it has any
    c["sc"][5::53] = 0         # fluid neighbours only
    c["fw"], c["fgw"] = reference_kernels(reference, c, c["fc"], c["fd"], c["fv"])
    c["sw"], c["sgw"] = reference_kernels(reference, c, c["sc"], c["sd"], c["sv"])
    rng = np.random.Generator(np.random.PCG64(17))
    c["rho_z"] = c["rho"].copy()
    c["rho_z"][3::41] = 0.0     # unsafe divisions by rho^2
    c["div"] = rng.normal(0, 50, n).astype(np.float32)
    c["div"][::9] = 0.0
    assert (c["fc"] == 0).any() and ((c["fc"] == 0) & (c["sc"] > 0)).any()
    return c


class HostNb:
    """A neighbour set for the reference harness: six host pointers in the
    emerald_neighborhood layout, held alive with their arrays."""

    def __init__(self, E, c, which):
        if which == "f":
            arrays = (c["fc"], c["fi"], c["fd"], c["fv"], c["fw"], c["fgw"])
        else:
            arrays = (c["sc"], c["si"], c["sd"], c["sv"], c["sw"], c["sgw"])
        self.arrays = [np.ascontiguousarray(a) for a in arrays]
        self.nb = E.Neighborhood(*[a.ctypes.data for a in self.arrays])

    @property
    def p(self):
        return ctypes.c_void_p(ctypes.addressof(self.nb))


def dev_lists(E, c):
    """Device neighbour sets with distances and vectors (PCISPH reads them)."""
    d = {k: dev(c[k]) for k in ("fc", "fi", "fd", "fv", "fw", "fgw", "sc", "si", "sd", "sv",
                                "sw", "sgw")}
    f = nbhd(E, d["fc"], d["fi"], d["fd"], d["fv"], d["fw"], d["fgw"])
    s = nbhd(E, d["sc"], d["si"], d["sd"], d["sv"], d["sw"], d["sgw"])
    return f, s


def zeros(*shape):
    return dev(np.zeros(shape, np.float32))


def result_buffer():
    return zeros(4)


def reference_iisph(R, c, dt, f, s):
    """The reference's IISPH operator chain on the case, host arrays."""
    n, ns = c["n"], c["ns"]
    out = {}
    out["diis"] = np.zeros((n, 2), np.float32)
    R.ref_ops_iisph_diis(n, dt, c["rho0"], ptr(out["diis"]), ptr(c["rho_z"]), ptr(c["fvol"]),
                         f.p, ptr(c["svol"]), s.p)
    out["aiis"] = np.zeros(n, np.float32)
    out["stars"] = np.zeros(n, np.float32)
    R.ref_ops_iisph_aiis_stars(n, dt, c["rho0"], ptr(out["aiis"]), ptr(out["stars"]),
                               ptr(out["diis"]), ptr(c["rho_z"]), ptr(c["fvol"]), ptr(c["vel"]),
                               f.p, ptr(c["svol"]), ptr(c["svel"]), ns, s.p)
    out["sdp"] = np.zeros((n, 2), np.float32)
    R.ref_ops_iisph_sum_dij_pjs(n, dt, c["rho0"], ptr(out["sdp"]), ptr(c["fvol"]),
                                ptr(c["rho_z"]), ptr(c["p"]), f.p)
    out["betas"] = np.zeros(n, np.float32)
    R.ref_ops_iisph_betas(n, dt, c["rho0"], ptr(out["betas"]), ptr(c["rho_z"]), ptr(c["p"]),
                          ptr(out["diis"]), ptr(out["sdp"]), ptr(c["fvol"]), f.p,
                          ptr(c["svol"]), s.p)
    alphas = out["aiis"].copy()
    alphas[7] = np.float32(1e-40)   # |a_ii| / FLT_MIN below |numerator|: unsafe
    out["alphas"] = alphas
    out["new_p"] = out["betas"].copy()
    out["new_p_err"] = np.zeros(2, np.float32)
    R.ref_ops_iisph_new_pressures(n, F(0.5), c["rho0"], ptr(out["new_p"]), ptr(c["p"]),
                                  ptr(alphas), ptr(out["stars"]), ptr(out["new_p_err"]))
    return out


def test_iisph_ops(E, reference, case):
    K = Keep()
    c = case
    n = c["n"]
    dt = F(3e-4)
    hf, hs = HostNb(E, c, "f"), HostNb(E, c, "s")
    ref = reference_iisph(reference.L, c, dt, hf, hs)
    f, s = dev_lists(E, c)
    diis = zeros(n, 2)
    check(E.lib.emerald_iisph_compute_diis(n, dt, c["rho0"], diis.data_ptr(), K(c["rho_z"]),
                                           K(c["fvol"]), f, K(c["svol"]), s, None))
    assert_bitwise(host(diis), ref["diis"], "d_ii")
    aiis, stars = zeros(n), zeros(n)
    check(E.lib.emerald_iisph_compute_aiis_and_density_stars(
        n, dt, c["rho0"], aiis.data_ptr(), stars.data_ptr(), K(ref["diis"]), K(c["rho_z"]),
        K(c["fvol"]), K(c["vel"]), f, K(c["svol"]), K(c["svel"]), s, None))
    assert_bitwise(host(aiis), ref["aiis"], "a_ii")
    assert_bitwise(host(stars), ref["stars"], "density stars")
    sdp = zeros(n, 2)
    check(E.lib.emerald_iisph_compute_sum_dij_pjs(n, dt, c["rho0"], sdp.data_ptr(), K(c["fvol"]),
                                                  K(c["rho_z"]), K(c["p"]), f, None))
    assert_bitwise(host(sdp), ref["sdp"], "sum d_ij p_j")
    betas = zeros(n)
    check(E.lib.emerald_iisph_compute_betas(n, dt, c["rho0"], betas.data_ptr(), K(c["rho_z"]),
                                            K(c["p"]), K(ref["diis"]), K(ref["sdp"]),
                                            K(c["fvol"]), f, K(c["svol"]), s, None))
    assert_bitwise(host(betas), ref["betas"], "betas")
    io = dev(ref["betas"])
    res = result_buffer()
    check(E.lib.emerald_iisph_compute_new_pressures(n, F(0.5), c["rho0"], io.data_ptr(),
                                                    K(c["p"]), K(ref["alphas"]),
                                                    K(ref["stars"]), res.data_ptr(), None))
    assert_bitwise(host(io), ref["new_p"], "new pressures")
    assert_bitwise(host(res)[:2], ref["new_p_err"], "new pressures (average, max) error")
    assert ref["new_p_err"][1] > 0


def test_dfsph_ops(E, reference, case):
    K = Keep()
    c = case
    n = c["n"]
    hf, hs = HostNb(E, c, "f"), HostNb(E, c, "s")
    coeffs_ref = np.zeros(n, np.float32)
    reference.L.ref_ops_dfsph_shared_coeffs(n, c["rho0"], ptr(coeffs_ref), ptr(c["rho_z"]),
                                            ptr(c["fvol"]), hf.p, ptr(c["svol"]), hs.p)
    f, s = dev_lists(E, c)
    coeffs = zeros(n)
    check(E.lib.emerald_dfsph_p_compute_shared_coeffs(n, c["rho0"], coeffs.data_ptr(),
                                                      K(c["rho_z"]), K(c["fvol"]), f,
                                                      K(c["svol"]), s, None))
    assert_bitwise(host(coeffs), coeffs_ref, "shared coefficients (alpha)")
    for dt in (F(3e-4), F(0.0)):
        dpp_ref, vpp_ref = np.zeros(n, np.float32), np.zeros(n, np.float32)
        reference.L.ref_ops_dfsph_pseudo_pressures(n, dt, c["rho0"], ptr(dpp_ref), ptr(vpp_ref),
                                                   ptr(c["rho"]), ptr(c["div"]),
                                                   ptr(coeffs_ref))
        dpp, vpp = zeros(n), zeros(n)
        check(E.lib.emerald_dfsph_p_compute_density_pseudo_pressures(
            n, dt, c["rho0"], dpp.data_ptr(), K(c["rho"]), K(coeffs_ref), None))
        check(E.lib.emerald_dfsph_p_compute_divergence_pseudo_pressures(
            n, dt, c["rho0"], vpp.data_ptr(), K(c["div"]), K(coeffs_ref), None))
        assert_bitwise(host(dpp), dpp_ref, "density pseudo-pressures dt=%g" % dt)
        assert_bitwise(host(vpp), vpp_ref, "divergence pseudo-pressures dt=%g" % dt)


def test_pcisph_ops(E, reference, case):
    K = Keep()
    c = case
    n = c["n"]
    hf, hs = HostNb(E, c, "f"), HostNb(E, c, "s")
    mass, visc, denom = F(0.42), F(0.05), F(-3.5e-3)
    rho_ref = np.zeros(n, np.float32)
    reference.L.ref_ops_pcisph_densities(n, mass, c["support"], c["rho0"], ptr(rho_ref), hf.p,
                                         ptr(c["svol"]), hs.p)
    f, s = dev_lists(E, c)
    rho = zeros(n)
    check(E.lib.emerald_pcisph_compute_densities(n, mass, c["support"], rho.data_ptr(),
                                                 K(c["fc"]), K(c["fw"]), None))
    check(E.lib.emerald_pcisph_accumulate_density_from_solids(
        n, c["rho0"], rho.data_ptr(), K(c["svol"]), K(c["sc"]), K(c["si"]), K(c["sw"]), None))
    assert_bitwise(host(rho), rho_ref, "PCISPH densities")
    # Pressures from densities around the target (the update's max(., 0)
    # clamps half of them).
    dens = (c["rho0"] + np.random.Generator(np.random.PCG64(3)).normal(0, 5, n)).astype(
        np.float32)
    p_ref = c["p"].copy()
    reference.L.ref_ops_pcisph_update_pressures(n, c["rho0"], denom, ptr(p_ref), ptr(dens))
    p = dev(c["p"])
    check(E.lib.emerald_pcisph_update_pressures(n, c["rho0"], denom, p.data_ptr(), K(dens),
                                                None))
    assert_bitwise(host(p), p_ref, "PCISPH pressures")
    f0 = (np.random.Generator(np.random.PCG64(4)).normal(0, 1e-3, (n, 2))).astype(np.float32)
    fo_ref = f0.copy()
    reference.L.ref_ops_pcisph_forces(n, mass, c["support"], visc, c["rho0"], ptr(fo_ref), hf.p,
                                      ptr(c["vel"]), ptr(p_ref), ptr(c["rho"]), ptr(c["svol"]),
                                      hs.p)
    fo = dev(f0)
    check(E.lib.emerald_pcisph_accumulate_pressure_forces(
        n, mass, c["support"], visc, fo.data_ptr(), K(c["fc"]), K(c["fi"]), K(c["fd"]),
        K(c["fv"]), K(c["fgw"]), K(c["vel"]), K(p_ref), K(c["rho"]), None))
    check(E.lib.emerald_pcisph_accumulate_pressure_forces_from_solids(
        n, mass, c["rho0"], fo.data_ptr(), K(c["svol"]), K(c["sc"]), K(c["si"]), K(c["sgw"]),
        K(p_ref), K(c["rho"]), None))
    assert_bitwise(host(fo), fo_ref, "PCISPH pressure and viscosity forces")


@pytest.mark.parametrize("pseudo", [0, 1])
def test_iisph_ap_family_ops(E, reference, case, pseudo):
    K = Keep()
    c = case
    n, ns = c["n"], c["ns"]
    dt = F(2.5e-4)
    hf, hs = HostNb(E, c, "f"), HostNb(E, c, "s")
    R = reference.L
    stars_ref, diag_ref = np.zeros(n, np.float32), np.zeros(n, np.float32)
    R.ref_ops_ap_stars_diagonals(pseudo, n, dt, c["rho0"], ptr(stars_ref), ptr(diag_ref),
                                 ptr(c["rho_z"]), ptr(c["fvol"]), ptr(c["vel"]), hf.p,
                                 ptr(c["svol"]), ptr(c["svel"]), ns, hs.p)
    f, s = dev_lists(E, c)
    stars, diag = zeros(n), zeros(n)
    fn = (E.lib.emerald_iisph_pseudo_ap_density_stars_and_pseudo_diagonals if pseudo
          else E.lib.emerald_iisph_ap_density_stars_and_diagonals)
    check(fn(n, dt, c["rho0"], stars.data_ptr(), diag.data_ptr(), K(c["rho_z"]), K(c["fvol"]),
             K(c["vel"]), f, K(c["svol"]), K(c["svel"]), s, None))
    assert_bitwise(host(stars), stars_ref, "density stars")
    assert_bitwise(host(diag), diag_ref, "diagonals")
    assert (diag_ref == 0).any() and (diag_ref != 0).any()
    res = result_buffer()
    err_ref = np.zeros(2, np.float32)
    if not pseudo:
        acc = c["acc"]
        p_ref = c["p"].copy()
        R.ref_ops_ap_iterate(n, dt, c["rho0"], F(0.5), ptr(p_ref), ptr(stars_ref), ptr(acc),
                             ptr(diag_ref), ptr(c["fvol"]), hf.p, ptr(c["svol"]), hs.p,
                             ptr(err_ref))
        p = dev(c["p"])
        check(E.lib.emerald_iisph_ap_iterate_pressures_in_place(
            n, dt, c["rho0"], F(0.5), p.data_ptr(), K(stars_ref), K(acc), K(diag_ref),
            K(c["fvol"]), f, K(c["svol"]), s, res.data_ptr(), None))
        assert_bitwise(host(p), p_ref, "IISPH_AP pressures")
    else:
        pp0 = (c["p"] * F(1e-6)).astype(np.float32)
        disp_ref = np.zeros((n, 2), np.float32)
        R.ref_ops_pseudo_displacements(n, c["rho0"], ptr(disp_ref), ptr(pp0), ptr(c["rho_z"]),
                                       ptr(c["fvol"]), hf.p, ptr(c["svol"]), hs.p)
        disp = zeros(n, 2)
        check(E.lib.emerald_iisph_pseudo_ap_compute_pseudo_pressure_displacements(
            n, c["rho0"], disp.data_ptr(), K(pp0), K(c["rho_z"]), K(c["fvol"]), f, K(c["svol"]),
            s, None))
        assert_bitwise(host(disp), disp_ref, "pseudo-pressure displacements")
        pp_ref = pp0.copy()
        R.ref_ops_pseudo_iterate(n, c["rho0"], F(0.5), ptr(pp_ref), ptr(stars_ref),
                                 ptr(disp_ref), ptr(diag_ref), ptr(c["fvol"]), hf.p,
                                 ptr(c["svol"]), hs.p, ptr(err_ref))
        pp = dev(pp0)
        check(E.lib.emerald_iisph_pseudo_ap_iterate_pseudo_pressures_in_place(
            n, c["rho0"], F(0.5), pp.data_ptr(), K(stars_ref), K(disp_ref), K(diag_ref),
            K(c["fvol"]), f, K(c["svol"]), s, res.data_ptr(), None))
        assert_bitwise(host(pp), pp_ref, "pseudo-pressures")
        for dt_i in (dt, F(0.0)):
            v_ref, x_ref = c["vel"].copy(), c["fluid"].copy()
            R.ref_ops_pseudo_integrate(n, dt_i, ptr(v_ref), ptr(x_ref), ptr(disp_ref))
            v, x = dev(c["vel"]), dev(c["fluid"])
            check(E.lib.emerald_iisph_pseudo_ap_integrate_velocities_and_positions_in_place(
                n, dt_i, v.data_ptr(), x.data_ptr(), K(disp_ref), None))
            assert_bitwise(host(v), v_ref, "velocities dt=%g" % dt_i)
            assert_bitwise(host(x), x_ref, "positions dt=%g" % dt_i)
    assert_bitwise(host(res)[:2], err_ref, "iteration (average, max) error")
    assert err_ref[1] > 0


def test_iteration_results_empty_and_invalid(E):
    """n = 0 gives the reference's {0, 0}; a misaligned or missing result
    buffer and missing inputs are EINVAL."""
    res = dev(np.full(4, 7.0, np.float32))
    check(E.lib.emerald_iisph_compute_new_pressures(0, F(0.5), F(1000), None, None, None, None,
                                                    res.data_ptr(), None))
    assert list(host(res)[:2]) == [0.0, 0.0]
    assert E.lib.emerald_iisph_compute_new_pressures(0, F(0.5), F(1000), None, None, None, None,
                                                     res.data_ptr() + 4, None) == 22
    assert E.lib.emerald_iisph_ap_iterate_pressures_in_place(
        4, F(1e-3), F(1000), F(0.5), None, None, None, None, None, E.Neighborhood(), None,
        E.Neighborhood(), res.data_ptr(), None) == 22
    assert E.lib.emerald_dfsph_p_compute_shared_coeffs(4, F(1000), None, None, None,
                                                       E.Neighborhood(), None, E.Neighborhood(),
                                                       None) == 22
