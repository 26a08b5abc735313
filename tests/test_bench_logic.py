"""Host-side logic of bench.py that feeds its JSON line: which committed ncu
capture supplies a kernel's DRAM traffic, the algorithmic-byte model, and
the 0.1% density-error bar as the solvers hold it (FP32 0.001f)."""
import numpy as np
import pytest

import bench


@pytest.fixture
def side():
    """Restores the default workload after a test changes it."""
    yield
    bench.configure_scene(512)


def test_traffic_comes_from_captures_of_the_same_workload(side):
    bench.configure_scene(512)
    assert bench.traffic_from_profile("apply_pressures") == 40127488.0
    assert bench.traffic_from_profile("neighbors_fluid") is not None
    bench.configure_scene(1024)
    assert bench.traffic_from_profile("apply_pressures") == 168200000.0
    assert bench.traffic_from_profile("neighbors_fluid") is None
    bench.configure_scene(256)
    assert bench.traffic_from_profile("apply_pressures") is None


def test_algorithmic_bytes_follow_the_csr_model():
    n, nnz_f, nnz_s, n_s = 1000, 10000.0, 500.0, 300
    # 12 B per list entry, 4 B per boundary volume, 22 B per particle
    assert bench.algorithmic_bytes("apply_pressures", n, nnz_f, nnz_s, n_s) == \
        12.0 * (nnz_f + nnz_s) + 4.0 * n_s + 22.0 * n
    # the neighbour build writes 16 B per entry (index, W, gradient)
    assert bench.algorithmic_bytes("neighbors_fluid", n, nnz_f, nnz_s, n_s) == \
        16.0 * nnz_f + 13.0 * n
    assert bench.algorithmic_bytes("no_such_kernel", n, nnz_f, nnz_s, n_s) is None


def test_tolerance_is_the_solvers_fp32_bar():
    # an average of exactly 0.001f meets the solvers' exit test (<= 0.001f)
    at_bar = float(np.float32(0.001))
    assert at_bar > 0.001
    assert not at_bar > bench.TOL_0_1
    assert float(np.nextafter(np.float32(0.001), np.float32(1.0))) > bench.TOL_0_1
