"""The sph_common free functions on device memory against the reference's
own functions (compiled from its sources), on the same inputs: every output
bit for bit.

Inputs: a jittered 24x24 block with its tank walls, neighbour lists from the
oracle's search (equal to the reference's), and seeded velocities, pressures,
densities and per-particle volumes."""
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
def case(E, oracle):
    return make_case(E, oracle)


def test_grid_coords_and_z_indices(E, reference, case):
    K = Keep()
    n = case["n"]
    x = dev(case["fluid"])
    gc = dev(np.zeros((n, 2), np.int32))
    check(E.lib.emerald_compute_grid_coords(n, case["cell"], F(-0.1), F(-0.05), gc.data_ptr(),
                                            x.data_ptr(), None))
    ref = np.zeros((n, 2), np.int32)
    reference.L.ref_common_grid_coords(n, case["cell"], F(-0.1), F(-0.05), ptr(ref),
                                       ptr(case["fluid"]))
    assert_bitwise(host(gc), ref, "grid coords")
    z = dev(np.zeros(n, np.uint64))
    check(E.lib.emerald_compute_z_indices(n, z.data_ptr(), gc.data_ptr(), None))
    rz = np.zeros(n, np.uint64)
    reference.L.ref_common_z_indices(n, ptr(rz), ptr(ref))
    assert_bitwise(host(z), rz, "z indices")


def test_neighbor_geometry_and_kernels(E, reference, case):
    K = Keep()
    n, ns = case["n"], case["ns"]
    for counts, idx, other in ((case["fc"], case["fi"], case["fluid"]),
                               (case["sc"], case["si"], case["solid"])):
        dist = dev(np.zeros((n, 64), np.float32))
        vec = dev(np.zeros((n, 64, 2), np.float32))
        check(E.lib.emerald_compute_neighbor_distances_and_vectors_to(
            n, dist.data_ptr(), vec.data_ptr(), K(case["fluid"]),
            K(other), K(counts), K(idx), None))
        rd = np.zeros((n, 64), np.float32)
        rv = np.zeros((n, 64, 2), np.float32)
        reference.L.ref_common_distances_vectors(n, len(other), ptr(rd), ptr(rv),
                                                 ptr(case["fluid"]), ptr(other), ptr(counts),
                                                 ptr(idx))
        mask = np.arange(64)[None, :] < counts[:, None]
        assert_bitwise(np.where(mask, host(dist), 0), np.where(mask, rd, 0), "distances")
        assert_bitwise(np.where(mask[..., None], host(vec), 0), np.where(mask[..., None], rv, 0),
                       "vectors_to")
        w = dev(np.zeros((n, 64), np.float32))
        gw = dev(np.zeros((n, 64, 2), np.float32))
        c_d = dev(counts)
        check(E.lib.emerald_compute_neighbor_kernels(n, case["support"], w.data_ptr(),
                                                     c_d.data_ptr(), dist.data_ptr(), None))
        check(E.lib.emerald_compute_neighbor_kernel_gradients(n, case["support"], gw.data_ptr(),
                                                              c_d.data_ptr(), vec.data_ptr(),
                                                              None))
        rw = np.zeros((n, 64), np.float32)
        rgw = np.zeros((n, 64, 2), np.float32)
        reference.L.ref_common_kernels(n, case["support"], ptr(rw), ptr(rgw), ptr(counts),
                                       ptr(rd), ptr(rv))
        assert_bitwise(np.where(mask, host(w), 0), np.where(mask, rw, 0), "kernels")
        assert_bitwise(np.where(mask[..., None], host(gw), 0), np.where(mask[..., None], rgw, 0),
                       "kernel gradients")
    case["fw"], case["fgw"] = reference_kernels(reference, case, case["fc"], case["fd"], case["fv"])
    case["sw"], case["sgw"] = reference_kernels(reference, case, case["sc"], case["sd"], case["sv"])


def test_densities_divergences_and_stars(E, reference, case):
    K = Keep()
    n, ns = case["n"], case["ns"]
    f, s = lists(E, reference, case)
    fvol, svol = dev(case["fvol"]), dev(case["svol"])
    rho = dev(np.zeros(n, np.float32))
    check(E.lib.emerald_compute_densities(n, case["support"], case["rho0"], rho.data_ptr(),
                                          fvol.data_ptr(), f, svol.data_ptr(), s, None))
    rr = np.zeros(n, np.float32)
    reference.L.ref_common_densities(n, case["support"], case["rho0"], ptr(rr), ptr(case["fvol"]),
                                     ptr(case["fc"]), ptr(case["fi"]), ptr(case["fw"]),
                                     ptr(case["svol"]), ptr(case["sc"]), ptr(case["si"]),
                                     ptr(case["sw"]))
    assert_bitwise(host(rho), rr, "densities")
    vel, svel = dev(case["vel"]), dev(case["svel"])
    div = dev(np.zeros(n, np.float32))
    check(E.lib.emerald_compute_divergences(n, case["rho0"], div.data_ptr(), fvol.data_ptr(),
                                            vel.data_ptr(), f, svol.data_ptr(), svel.data_ptr(),
                                            s, None))
    rd = np.zeros(n, np.float32)
    reference.L.ref_common_divergences(n, case["rho0"], ptr(rd), ptr(case["fvol"]),
                                       ptr(case["vel"]), ptr(case["fc"]), ptr(case["fi"]),
                                       ptr(case["fgw"]), ptr(case["svol"]), ptr(case["svel"]), ns,
                                       ptr(case["sc"]), ptr(case["si"]), ptr(case["sgw"]))
    assert_bitwise(host(div), rd, "divergences")
    stars = dev(np.zeros(n, np.float32))
    dt = F(3e-4)
    check(E.lib.emerald_predict_density_stars(n, dt, case["rho0"], stars.data_ptr(),
                                              K(case["rho"]), fvol.data_ptr(),
                                              vel.data_ptr(), f, svol.data_ptr(),
                                              svel.data_ptr(), s, None))
    rs = np.zeros(n, np.float32)
    reference.L.ref_common_density_stars(n, dt, case["rho0"], ptr(rs), ptr(case["rho"]),
                                         ptr(case["fvol"]), ptr(case["vel"]), ptr(case["fc"]),
                                         ptr(case["fi"]), ptr(case["fgw"]), ptr(case["svol"]),
                                         ptr(case["svel"]), ns, ptr(case["sc"]), ptr(case["si"]),
                                         ptr(case["sgw"]))
    assert_bitwise(host(stars), rs, "density stars")


def test_pressure_terms(E, reference, case):
    K = Keep()
    n = case["n"]
    f, s = lists(E, reference, case)
    fvol, svol = dev(case["fvol"]), dev(case["svol"])
    rho, p = dev(case["rho"]), dev(case["p"])
    vel = dev(case["vel"])
    dt = F(2.5e-4)
    check(E.lib.emerald_apply_pressures_in_place(n, dt, case["rho0"], vel.data_ptr(),
                                                 rho.data_ptr(), p.data_ptr(), fvol.data_ptr(), f,
                                                 svol.data_ptr(), s, None))
    rv = case["vel"].copy()
    reference.L.ref_common_apply_pressures(n, dt, case["rho0"], ptr(rv), ptr(case["rho"]),
                                           ptr(case["p"]), ptr(case["fvol"]), ptr(case["fc"]),
                                           ptr(case["fi"]), ptr(case["fgw"]), ptr(case["svol"]),
                                           ptr(case["sc"]), ptr(case["si"]), ptr(case["sgw"]))
    assert_bitwise(host(vel), rv, "velocities after apply_pressures_in_place")
    acc = dev(np.zeros((n, 2), np.float32))
    check(E.lib.emerald_compute_pressure_accelerations(n, case["rho0"], acc.data_ptr(),
                                                       p.data_ptr(), rho.data_ptr(),
                                                       fvol.data_ptr(), f, svol.data_ptr(), s,
                                                       None))
    ra = np.zeros((n, 2), np.float32)
    reference.L.ref_common_pressure_accelerations(n, case["rho0"], ptr(ra), ptr(case["p"]),
                                                  ptr(case["rho"]), ptr(case["fvol"]),
                                                  ptr(case["fc"]), ptr(case["fi"]),
                                                  ptr(case["fgw"]), ptr(case["svol"]),
                                                  ptr(case["sc"]), ptr(case["si"]),
                                                  ptr(case["sgw"]))
    assert_bitwise(host(acc), ra, "pressure accelerations")


def test_integration_volumes_and_reductions(E, reference, case):
    K = Keep()
    n = case["n"]
    dt = F(4e-4)
    vf, va, x = dev(case["vel"]), dev(case["vel"]), dev(case["fluid"])
    check(E.lib.emerald_integrate_velocities_with_forces(n, dt, case["rho0"], vf.data_ptr(),
                                                         K(case["fvol"]),
                                                         K(case["forces"]), None))
    check(E.lib.emerald_integrate_velocities(n, dt, va.data_ptr(), K(case["acc"]),
                                             None))
    check(E.lib.emerald_integrate_positions(n, dt, x.data_ptr(), K(case["vel"]),
                                            None))
    rvf, rva, rx = case["vel"].copy(), case["vel"].copy(), case["fluid"].copy()
    reference.L.ref_common_integrate(n, dt, case["rho0"], ptr(rvf), ptr(rva), ptr(rx),
                                     ptr(case["fvol"]), ptr(case["forces"]), ptr(case["acc"]),
                                     ptr(case["vel"]))
    assert_bitwise(host(vf), rvf, "velocities from forces")
    assert_bitwise(host(va), rva, "velocities from accelerations")
    assert_bitwise(host(x), rx, "positions")
    vol = dev(np.zeros(n, np.float32))
    check(E.lib.emerald_compute_constant_volumes(n, case["rho0"], F(0.37), vol.data_ptr(), None))
    rvol = np.zeros(n, np.float32)
    reference.L.ref_common_constant_volumes(n, case["rho0"], F(0.37), ptr(rvol))
    assert_bitwise(host(vol), rvol, "constant volumes")
    out = dev(np.zeros(1, np.float32))
    check(E.lib.emerald_max_vector_squared_magnitude(n, out.data_ptr(),
                                                     K(case["vel"]), None))
    assert host(out)[0] == reference.L.ref_max_vector_squared_magnitude(n, ptr(case["vel"]))
    check(E.lib.emerald_max_density_error(n, case["rho0"], out.data_ptr(),
                                          K(case["rho"]), None))
    assert host(out)[0] == reference.L.ref_max_density_error(n, case["rho0"], ptr(case["rho"]))
    fl = dev(np.zeros(1, np.int64))
    for factor in (F(0.4), F(0.2)):
        check(E.lib.emerald_cfl_maximum_time_step(n, case["support"], factor, fl.data_ptr(),
                                                  K(case["vel"]), None))
        assert host(fl)[0] == reference.L.ref_cfl_maximum_time_step(n, case["support"], factor,
                                                                    ptr(case["vel"]))
    zeros = dev(np.zeros((n, 2), np.float32))
    check(E.lib.emerald_cfl_maximum_time_step(n, case["support"], F(0.4), fl.data_ptr(),
                                              zeros.data_ptr(), None))
    assert host(fl)[0] == reference.L.ref_cfl_maximum_time_step(
        n, case["support"], F(0.4), ptr(np.zeros((n, 2), np.float32)))
    vals = np.random.Generator(np.random.PCG64(9)).normal(0, 0.01, n).astype(np.float32)
    am = dev(np.zeros(2, np.float32))
    for disc in (F(1000.0), F(37.0)):
        check(E.lib.emerald_scalar_average_and_max(n, disc, am.data_ptr(), K(vals),
                                                   None))
        ram = np.zeros(2, np.float32)
        reference.L.ref_common_average_and_max(n, disc, ptr(vals), ptr(ram))
        assert_bitwise(host(am), ram, "average and max")


def test_empty_and_invalid(E):
    K = Keep()
    assert E.lib.emerald_compute_densities(0, F(0.01), F(1000), None, None, E.Neighborhood(),
                                           None, E.Neighborhood(), None) == 0
    assert E.lib.emerald_compute_neighbor_kernels(10, F(0.0), None, None, None, None) == 22


# ---------------------------------------------- z-order sort and the search

def workspace(E, n):
    import ctypes
    b = ctypes.c_size_t()
    check(E.lib.emerald_index_pairs_workspace(n, ctypes.byref(b)))
    import torch
    return torch.empty(max(b.value, 1), dtype=torch.uint8, device="cuda")


def device_sort(E, pairs):
    """emerald_sort_index_pairs on a copy of the interleaved (z, index) pairs."""
    n = len(pairs)
    d = dev(pairs)
    ws = workspace(E, n)
    check(E.lib.emerald_sort_index_pairs(n, d.data_ptr(), ws.data_ptr(), ws.numel(), None))
    return host(d)


def reference_sort(reference, pairs):
    out = np.ascontiguousarray(pairs.copy())
    reference.L.ref_common_sort_index_pairs(len(out), ptr(out))
    return out


def sorted_set(E, reference, xy, cell):
    """The reference's chain (neighborhoods_from_state.cpp:15-44) for one
    point set with the grid at the origin, through the device functions:
    grid coords, z keys, sorted pairs, block indices, blocks, the block map.
    Each product is compared with the reference's on the way."""
    n = len(xy)
    K = Keep()
    gc = dev(np.zeros((n, 2), np.int32))
    check(E.lib.emerald_compute_grid_coords(n, cell, F(0.0), F(0.0), gc.data_ptr(), K(xy), None))
    z = dev(np.zeros(n, np.uint64))
    check(E.lib.emerald_compute_z_indices(n, z.data_ptr(), gc.data_ptr(), None))
    pairs = dev(np.zeros((n, 2), np.uint64))
    check(E.lib.emerald_compute_index_pairs(n, pairs.data_ptr(), z.data_ptr(), None))
    rpairs = np.zeros((n, 2), np.uint64)
    reference.L.ref_common_index_pairs(n, ptr(rpairs), ptr(host(z)))
    assert_bitwise(host(pairs), rpairs, "index pairs")
    ws = workspace(E, n)
    check(E.lib.emerald_sort_index_pairs(n, pairs.data_ptr(), ws.data_ptr(), ws.numel(), None))
    reference.L.ref_common_sort_index_pairs(n, ptr(rpairs))
    assert_bitwise(host(pairs), rpairs, "sorted pairs")
    bi = dev(np.zeros(n, np.uint32))
    check(E.lib.emerald_compute_block_indices(n, bi.data_ptr(), pairs.data_ptr(), ws.data_ptr(),
                                              ws.numel(), None))
    rbi = np.zeros(n, np.uint32)
    reference.L.ref_common_block_indices(n, ptr(rbi), ptr(rpairs))
    assert_bitwise(host(bi), rbi, "block indices")
    nb = int(rbi[-1]) + 1
    blocks = dev(np.zeros((nb, 2), np.uint64))
    check(E.lib.emerald_fill_blocks(n, blocks.data_ptr(), bi.data_ptr(), None))
    rblocks = np.zeros((nb, 2), np.uint64)
    reference.L.ref_common_fill_blocks(n, nb, ptr(rblocks), ptr(rbi))
    assert_bitwise(host(blocks), rblocks, "blocks")
    return dict(n=n, xy=xy, gc=gc, pairs=pairs, rpairs=rpairs, blocks=blocks, rblocks=rblocks,
                nb=nb, keep=K)


def compare_search(E, reference, self_set, other_set, cell, bmap, what):
    import ctypes
    n = self_set["n"]
    same = other_set is self_set
    x = dev(self_set["xy"])
    ox = x if same else dev(other_set["xy"])
    check(E.lib.emerald_create_block_map(other_set["nb"], bmap, other_set["blocks"].data_ptr(),
                                         other_set["pairs"].data_ptr(), None))
    counts = dev(np.full(n, 255, np.uint8))
    idx = dev(np.zeros((n, 64), np.uint64))
    dist = dev(np.zeros((n, 64), np.float32))
    vec = dev(np.zeros((n, 64, 2), np.float32))
    check(E.lib.emerald_create_regular_neighborhoods(
        n, cell, counts.data_ptr(), idx.data_ptr(), dist.data_ptr(), vec.data_ptr(), x.data_ptr(),
        self_set["gc"].data_ptr(), ox.data_ptr(), other_set["pairs"].data_ptr(), bmap, None))
    rc = np.zeros(n, np.uint8)
    ri = np.zeros((n, 64), np.uint64)
    rd = np.zeros((n, 64), np.float32)
    rv = np.zeros((n, 64, 2), np.float32)
    reference.L.ref_common_regular_neighborhoods(
        n, other_set["n"], cell, ptr(rc), ptr(ri), ptr(rd), ptr(rv), ptr(self_set["xy"]),
        ptr(host(self_set["gc"])), ptr(other_set["xy"]), 1 if same else 0, other_set["n"],
        ptr(other_set["rpairs"]), other_set["nb"], ptr(other_set["rblocks"]))
    c = host(counts)
    assert_bitwise(c, rc, "%s counts" % what)
    live = np.arange(64)[None, :] < c[:, None]
    assert_bitwise(np.where(live, host(idx), 0), ri, "%s indices" % what)
    assert_bitwise(np.where(live, host(dist), 0), rd, "%s distances" % what)
    assert_bitwise(np.where(live[..., None], host(vec), 0), rv, "%s vectors_to" % what)
    return c


@pytest.fixture()
def block_map(E):
    import ctypes
    m = ctypes.c_void_p()
    check(E.lib.emerald_block_map_create(ctypes.byref(m)))
    yield m.value
    check(E.lib.emerald_block_map_destroy(m.value))


def test_index_pair_sort_matches_reference(E, reference):
    """Random pairs with many equal z keys, indices out of order and equal
    pairs, the all-ones z key of cell (-1, -1), and 2^20 pairs: the device
    sort gives std::sort's order."""
    rng = np.random.Generator(np.random.PCG64(17))
    for n, zmax, imax in ((2, 3, 2), (37, 4, 10), (5000, 300, 1 << 40), (1 << 20, 1 << 30, 1 << 20)):
        z = rng.integers(0, zmax, n, dtype=np.uint64)
        z[rng.integers(0, n, max(1, n // 50))] = np.uint64(0xFFFFFFFFFFFFFFFF)
        pairs = np.stack([z, rng.integers(0, imax, n, dtype=np.uint64)], axis=1)
        assert_bitwise(device_sort(E, pairs), reference_sort(reference, pairs),
                       "sorted pairs n=%d" % n)
    # nothing to do for 0 or 1 pair (neighborhood.cpp:20)
    one = np.array([[5, 9]], np.uint64)
    assert_bitwise(device_sort(E, one), one, "one pair")
    assert E.lib.emerald_sort_index_pairs(0, None, None, 0, None) == 0


def test_sort_products_and_search_match_reference(E, reference, case, block_map):
    """The tank case (fluid against itself and against its walls, whose
    cells reach negative coordinates and cell (-1, -1)) through the device
    chain, every product against the reference's."""
    cell = case["cell"]
    fluid = sorted_set(E, reference, case["fluid"], cell)
    solid = sorted_set(E, reference, case["solid"], cell)
    assert (host(solid["gc"]) < 0).any()
    assert np.uint64(0xFFFFFFFFFFFFFFFF) in host(solid["pairs"])[:, 0]
    cf = compare_search(E, reference, fluid, fluid, cell, block_map, "fluid")
    cs = compare_search(E, reference, fluid, solid, cell, block_map, "boundary")
    assert cf.max() > 10 and cs.max() > 0


def test_search_caps_dense_cells_like_the_reference(E, reference, block_map):
    """Cells holding far more than 64 candidates: the search keeps the first
    64 accepted in the reference's visiting order and sorts those, so the
    lists equal the reference's, not the 64 nearest. The map is refilled with
    more blocks afterwards (its table grows)."""
    rng = np.random.Generator(np.random.PCG64(23))
    cell = F(0.05)
    dense = rng.uniform(0.0, 0.1, (900, 2)).astype(np.float32)
    sparse = rng.uniform(-0.5, 1.5, (3000, 2)).astype(np.float32)
    xy = np.concatenate([dense, sparse]).astype(np.float32)
    s = sorted_set(E, reference, xy, cell)
    c = compare_search(E, reference, s, s, cell, block_map, "dense")
    assert (c == 64).sum() > 100
    big = rng.uniform(-2.0, 2.0, (20000, 2)).astype(np.float32)
    b = sorted_set(E, reference, big, F(0.01))
    assert b["nb"] > 4 * s["nb"]
    compare_search(E, reference, b, b, F(0.01), block_map, "after growing")
    # a map of no blocks finds nothing
    check(E.lib.emerald_create_block_map(0, block_map, None, None, None))
    counts = dev(np.full(4, 7, np.uint8))
    K = Keep()
    check(E.lib.emerald_create_regular_neighborhoods(
        4, cell, counts.data_ptr(), K(np.zeros((4, 64), np.uint64)),
        K(np.zeros((4, 64), np.float32)), K(np.zeros((4, 64, 2), np.float32)), K(xy[:4]),
        K(np.zeros((4, 2), np.int32)), K(xy[:4]), K(np.zeros((1, 2), np.uint64)), block_map,
        None))
    assert (host(counts) == 0).all()
