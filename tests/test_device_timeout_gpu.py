"""Failure detection without a GPU fault: every wait inside the staged SpMV
kernel is bounded.  A test hook makes the warp that owns tile 0 withhold that
tile's copies, so its wait runs into the (here 50 ms) limit; the kernel records
the error, drains its copies and returns, the host reports
HBDIA_ERR_DEVICE_TIMEOUT at the next synchronize, and the context stays
usable for the next, correct SpMV."""
import time

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu


def test_staged_wait_timeout_is_reported_and_recoverable(lib, orc):
    n = 32 ** 3
    rows, cols, vals = lib.generate_stencil27(32, 32, 32, 26.0, -1.0, 0.01, 0.1, 1.0, 4)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    m.setKernel(lib.KERNEL_STAGED)
    m.setWaitTimeout(50_000_000)
    x = np.random.default_rng(2).uniform(-1, 1, n)
    xv, yv = lib.HBDIAVector(x), lib.HBDIAVector(np.zeros(n))
    assert m.selectedKernel(xv.getDeviceDataPtr()) == lib.KERNEL_STAGED
    m.testSkipTile(0)
    t = time.time()
    lib.hbdiaSpMV(m, xv, yv, True, False)
    with pytest.raises(lib.HBDIADeviceTimeout):
        m.synchronize()
    assert time.time() - t < 10.0
    assert m.deviceStatus() == 0          # reported once, then cleared
    m.testSkipTile(-1)
    lib.hbdiaSpMV(m, xv, yv, True, False)
    m.synchronize()
    yref = orc.convert(rows, cols, vals, n, n, 32, 2).spmv(x)
    assert bits_equal(yv.toHost(), yref)
