import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def oracle():
    from cpu_checkers import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from cpu_checkers import Reference
    if not Reference.available:
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return Reference()


def bits(a):
    import numpy as np
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_bitwise(a, b, what=""):
    import numpy as np
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    ba, bb = bits(a), bits(b)
    if not np.array_equal(ba, bb):
        diff = np.argwhere(ba != bb)
        first = tuple(diff[0])
        raise AssertionError("%s differs at %d entries, first %s: %r vs %r (max |d| %g)" % (
            what, len(diff), first, a[first], b[first],
            float(np.nanmax(np.abs(a.astype(np.float64) - b.astype(np.float64))))))
