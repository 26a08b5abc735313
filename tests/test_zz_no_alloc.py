"""The allocation-free neighbour build, emerald_neighbors_static.

Callers that cannot allocate device memory (hosts that own every device
allocation through their own allocator, per-frame loops that must not stall
on cudaMalloc/cudaFree) pass positions and output buffers; the call's scratch
is a static device array. Its lists must equal the simulation's own fluid
neighbour build bit for bit, on consecutive calls that reuse the array.

This file sorts last so that a run stopping at the first failure has run
every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import assert_bitwise
from scenes import F

pytestmark = pytest.mark.gpu


def reference_lists(E, scene):
    """Fluid lists from the simulation path (built at the start of a sub-step
    from the initial positions)."""
    sim = E.Simulation.from_block_scene(scene)
    sim.sub_step("dfsph_p", 0.0, F(1e-4))
    return sim.neighbors(False)


def static_lists(E, torch, xy, support):
    n = len(xy)
    stride = n + 37
    d_xy = torch.from_numpy(np.ascontiguousarray(xy)).cuda()
    d_cnt = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
    d_idx = torch.zeros((64, stride), dtype=torch.int32, device="cuda")
    d_w = torch.zeros((64, stride), dtype=torch.float32, device="cuda")
    d_gw = torch.zeros((64, stride, 2), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    E.neighbors_static(d_xy.data_ptr(), n, float(support), d_cnt.data_ptr(), d_idx.data_ptr(),
                       d_w.data_ptr(), d_gw.data_ptr(), stride)
    torch.cuda.synchronize()
    counts = d_cnt.cpu().numpy()
    idx = d_idx.cpu().numpy().view(np.uint32)[:, :n].T.copy()
    w = d_w.cpu().numpy()[:, :n].T.copy()
    gw = d_gw.cpu().numpy()[:, :n, :].transpose(1, 0, 2).copy()
    live = np.arange(64)[None, :] < counts[:, None]
    idx[~live] = 0
    w[~live] = 0.0
    gw[~live] = 0.0
    return counts, idx, w, gw


def test_static_build_matches_simulation_on_two_calls():
    import torch

    import emerald_b200 as E
    big = E.BlockScene(160, dx=F(1 / 320), seed=21)      # 25600 points
    small = E.BlockScene(96, ny=64, dx=F(1 / 192), seed=22)  # 6144 points, after the big one
    for scene in (big, small):
        want = reference_lists(E, scene)
        got = static_lists(E, torch, scene.fluid, scene.support)
        for name, a, b in zip(("counts", "indices", "W", "grad W"), got, want):
            assert_bitwise(a, b, name)


def test_static_build_at_the_size_limit():
    """Exactly EMERALD_STATIC_MAX_POINTS points (a 256 x 256 block): the last
    tile of the static arena and the fullest cell table it can hold."""
    import torch

    import emerald_b200 as E
    scene = E.BlockScene(256, dx=F(1 / 512), seed=23)
    assert len(scene.fluid) == E.STATIC_MAX_POINTS
    want = reference_lists(E, scene)
    got = static_lists(E, torch, scene.fluid, scene.support)
    for name, a, b in zip(("counts", "indices", "W", "grad W"), got, want):
        assert_bitwise(a, b, name)


def call_static(E, xy, n, cnt, idx, w, gw, stride):
    rc = E.lib.emerald_neighbors_static(ctypes.c_void_p(xy), n, 0.01, ctypes.c_void_p(cnt),
                                        ctypes.c_void_p(idx), ctypes.c_void_p(w),
                                        ctypes.c_void_p(gw), stride, None)
    return rc, E.lib.emerald_last_error().decode()


def test_static_build_rejects_oversize():
    import emerald_b200 as E
    n = E.STATIC_MAX_POINTS + 1
    rc, msg = call_static(E, 256, n, 256, 256, 256, 256, n)
    assert rc == 22 and "EMERALD_STATIC_MAX_POINTS" in msg


def test_static_build_rejects_misaligned_buffers():
    """float2 positions and gradients need 8-byte alignment, the 32-bit lists
    4-byte; the call returns EMERALD_EINVAL before it enqueues anything (the
    pointers here are never dereferenced)."""
    import emerald_b200 as E
    rc, msg = call_static(E, 260, 16, 256, 256, 256, 256, 16)
    assert rc == 22 and "8-byte" in msg
    rc, msg = call_static(E, 256, 16, 256, 256, 256, 260, 16)
    assert rc == 22 and "8-byte" in msg
    rc, msg = call_static(E, 256, 16, 256, 258, 256, 256, 16)
    assert rc == 22 and "4-byte" in msg
