"""hbdia_spmv_host_noalloc: the host-buffer SpMV through the library's fixed
per-device array.  Two calls in a row must give exactly what hbdia_spmv_host
gives for the same inputs (same kernels, tolerance 0); no call, the first
(set-up) one included, may add to the library's allocation counter
(hbdia_allocation_count, which every cudaMalloc / cudaMallocHost of the
library goes through); the calls after the first must not change the
device's free memory, and the first may grow it by at most the 32 MiB array
(loaded with its module on first use); sizes beyond the array are rejected.
Kept in the last-collected file so it also runs after the rest of the suite
has used the device; the set-up check runs in a fresh process."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu

MAX_ELEMS = 1 << 21


def _matrix(lib, dtype):
    rows, cols, vals = lib.generate_stencil27(40, 40, 40, extra_fraction=0.01, seed=3)
    n = 40 ** 3
    m = lib.HBDIA(rows, cols, vals.astype(dtype), n, n, dtype=dtype)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(lib.STORE_NATIVE)
    assert m.info().numCoo > 0
    return m, n


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_matches_spmv_host_twice(lib, dtype):
    import torch
    torch.cuda.init()
    m, n = _matrix(lib, dtype)
    rng = np.random.default_rng(5)
    x1 = rng.uniform(-1, 1, n).astype(dtype)
    x2 = rng.uniform(-1, 1, n).astype(dtype)
    y1 = np.full(n, np.nan, dtype)
    y2 = np.full(n, np.nan, dtype)
    a0 = lib.allocation_count()
    lib.spmv_host_noalloc(m, x1, y1)  # first call on this device may do the set-up
    free0, _ = torch.cuda.mem_get_info()
    lib.spmv_host_noalloc(m, x2, y2)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert lib.allocation_count() == a0
    r1 = np.zeros(n, dtype)
    r2 = np.zeros(n, dtype)
    lib.spmv_host(m, x1, r1)
    lib.spmv_host(m, x2, r2)
    assert bits_equal(y1, r1)
    assert bits_equal(y2, r2)
    assert not bits_equal(y1, y2)


def test_noalloc_fresh_matrix_allocates_nothing(lib):
    import torch
    m0, n0 = _matrix(lib, np.float64)
    lib.spmv_host_noalloc(m0, np.ones(n0), np.zeros(n0))  # set-up done
    m, n = _matrix(lib, np.float64)
    x = np.random.default_rng(9).uniform(-1, 1, n)
    y = np.zeros(n)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    a0 = lib.allocation_count()
    lib.spmv_host_noalloc(m, x, y)
    lib.spmv_host_noalloc(m, x, y)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert lib.allocation_count() == a0
    r = np.zeros(n)
    lib.spmv_host(m, x, r)
    assert bits_equal(y, r)


def test_noalloc_rejects_oversize_and_host_only(lib):
    n = MAX_ELEMS + 32
    i = np.arange(n, dtype=np.int32)
    m = lib.HBDIA(i, i, np.ones(n), n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(lib.STORE_NATIVE)
    with pytest.raises(ValueError, match=str(MAX_ELEMS)):
        lib.spmv_host_noalloc(m, np.ones(n), np.zeros(n))
    k = 1000
    j = np.arange(k, dtype=np.int32)
    h = lib.HBDIA(j, j, np.ones(k), k, k)
    h.convertToHBDIAFormat(32, 2, upload=False)
    with pytest.raises(RuntimeError, match="prepare_gpu"):
        lib.spmv_host_noalloc(h, np.ones(k), np.zeros(k))


_FRESH = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import hbdia_b200 as lib
import torch
torch.cuda.init()
rows, cols, vals = lib.generate_stencil27(40, 40, 40, extra_fraction=0.01, seed=3)
n = 40 ** 3
m = lib.HBDIA(rows, cols, vals, n, n)
m.convertToHBDIAFormat(32, 2, upload=False)
m.prepareForGPU(lib.STORE_NATIVE)
x = np.random.default_rng(4).uniform(-1, 1, n)
y = np.zeros(n)
torch.cuda.synchronize()
a0 = lib.allocation_count()
free0, _ = torch.cuda.mem_get_info()
lib.spmv_host_noalloc(m, x, y)   # the set-up call
free1, _ = torch.cuda.mem_get_info()
a1 = lib.allocation_count()
lib.spmv_host_noalloc(m, x, y)
free2, _ = torch.cuda.mem_get_info()
a2 = lib.allocation_count()
r = np.zeros(n)
lib.spmv_host(m, x, r)
print(a0 == a1 == a2, free0 - free1, free1 - free2, bool(np.array_equal(y.view(np.uint64), r.view(np.uint64))))
"""


def test_noalloc_setup_call_in_fresh_process(lib):
    """The first call on a device, in a process that has not called it yet:
    it allocates nothing through the library, and the device memory it
    commits is the array itself (its module is loaded on first use)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    same, grew_setup, grew_after, exact = r.stdout.split()[-4:]
    assert same == "True" and exact == "True", r.stdout
    assert 0 <= int(grew_setup) <= 34 * (1 << 20), r.stdout  # the 32 MiB array, page-rounded
    assert int(grew_after) == 0, r.stdout
