"""Inputs and device plumbing shared by the tests of the device free
functions: a jittered 24x24 block with its tank walls, neighbour lists from
the oracle's search (equal to the reference's) in the reference's row-major
64-entry layout, and seeded velocities, pressures, densities and volumes."""
import numpy as np

from cpu_checkers import ptr
from scenes import F


def make_case(E, oracle):
    scene = E.BlockScene(24, dx=F(1 / 48), seed=21)
    fluid = scene.fluid.astype(np.float32)
    solid = scene.solid.astype(np.float32)
    cell = F(2 * scene.support)
    fc, fi, fd, fv = oracle.neighborhoods(fluid, fluid, True, cell)
    sc, si, sd, sv = oracle.neighborhoods(fluid, solid, False, cell)
    rng = np.random.Generator(np.random.PCG64(5))
    n, ns = len(fluid), len(solid)
    c = dict(
        n=n, ns=ns, support=np.float32(scene.support), cell=cell, rho0=F(1000.0),
        fluid=fluid, solid=solid,
        fc=fc, fi=fi.astype(np.uint64), fd=fd, fv=np.ascontiguousarray(fv),
        sc=sc, si=si.astype(np.uint64), sd=sd, sv=np.ascontiguousarray(sv),
        fvol=(F(1 / 48) ** 2 * (1 + rng.uniform(-0.05, 0.05, n))).astype(np.float32),
        svol=(F(1 / 48) ** 2 * (1 + rng.uniform(-0.05, 0.05, ns))).astype(np.float32),
        vel=rng.normal(0, 0.3, (n, 2)).astype(np.float32),
        svel=rng.normal(0, 0.05, (ns, 2)).astype(np.float32),
        rho=(1000 + rng.normal(0, 20, n)).astype(np.float32),
        p=np.abs(rng.normal(0, 500, n)).astype(np.float32),
        acc=rng.normal(0, 2, (n, 2)).astype(np.float32),
        forces=rng.normal(0, 1e-3, (n, 2)).astype(np.float32),
    )
    c["p"][::7] = 0.0
    return c


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class Keep:
    """Device copies that stay alive until the test ends (a temporary
    tensor's memory may be reused before an asynchronous kernel reads it)."""

    def __init__(self):
        self.held = []

    def __call__(self, a):
        t = dev(a)
        self.held.append(t)
        return t.data_ptr()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def nbhd(E, counts, idx=None, dist=None, vec=None, w=None, gw=None):
    keep = [x for x in (counts, idx, dist, vec, w, gw) if x is not None]
    nb = E.Neighborhood(*[None if x is None else x.data_ptr() for x in
                          (counts, idx, dist, vec, w, gw)])
    nb._keep = keep
    return nb


def check(rc):
    assert rc == 0, rc


def reference_kernels(reference, case, counts, dist, vec):
    n = case["n"]
    rw = np.zeros((n, 64), np.float32)
    rgw = np.zeros((n, 64, 2), np.float32)
    reference.L.ref_common_kernels(n, case["support"], ptr(rw), ptr(rgw), ptr(counts),
                                   ptr(np.ascontiguousarray(dist)), ptr(vec))
    return rw, rgw


def lists(E, reference, case):
    if "fw" not in case:
        case["fw"], case["fgw"] = reference_kernels(reference, case, case["fc"], case["fd"],
                                                    case["fv"])
        case["sw"], case["sgw"] = reference_kernels(reference, case, case["sc"], case["sd"],
                                                    case["sv"])
    d = {k: dev(case[k]) for k in ("fc", "fi", "fw", "fgw", "sc", "si", "sw", "sgw")}
    f = nbhd(E, d["fc"], d["fi"], None, None, d["fw"], d["fgw"])
    s = nbhd(E, d["sc"], d["si"], None, None, d["sw"], d["sgw"])
    return f, s
