"""Reduced-precision value storage with FP64 accumulation.

The blocked-DIA values are stored as FP32, or as BF16 with one FP32 scale per
block, and widened to FP64 inside the kernel; x, y, the COO remainder and all
arithmetic stay FP64.  Each result is checked two ways:
  * bit-exact against the oracle's FP64 SpMV run on the same rounded values
    (so the kernels are exact for what they store), and
  * against the plain FP64 oracle, scaled per row by sum_j |a_ij x_j|:
    FP32 storage <= 2^-24 (one rounding of each value), BF16 <= 2^-8.
The workload is the banded matrix of the precision configuration (offsets
0, +-1, +-2, +-64, +-4096; off-diagonals U(0.5, 1.5) dropped with p = 0.3;
centre = row |sum| + 1; 0.2% scattered entries), at n = 2^18 for every kernel
and at the configuration's own n = 8M (2^23) for the default kernel.
"""
import numpy as np
import pytest

import oracle
from conftest import bits_equal

pytestmark = pytest.mark.gpu

OFFSETS = [0, 1, -1, 2, -2, 64, -64, 4096, -4096]


def _scaled_err(y, yref, rows, cols, vals, x):
    scale = np.zeros(len(y))
    np.add.at(scale, rows, np.abs(vals * x[cols]))
    return float(np.max(np.abs(y - yref) / np.maximum(scale, np.finfo(float).tiny)))


@pytest.fixture(scope="module")
def banded(lib):
    n = 1 << 18
    rows, cols, vals = lib.generate_banded(n, OFFSETS, 0.5, 1.5, 0.3, 0.002, 2)
    x = np.random.default_rng(2).uniform(-1, 1, n)
    return n, rows, cols, vals, x


@pytest.mark.parametrize("kernel", [4, 5, 3, 2, 1], ids=["pipe", "quad", "staged", "warp", "rowwise"])
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_reduced_storage(lib, orc, banded, storage, kernel):
    n, rows, cols, vals, x = banded
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(lib.STORE_F32 if storage == "f32" else lib.STORE_BF16_SCALED)
    m.setKernel(kernel)
    assert m.info().storage == (1 if storage == "f32" else 2)
    yv = lib.HBDIAVector(np.zeros(n))
    lib.hbdiaSpMV(m, lib.HBDIAVector(x), yv, True, False)
    m.synchronize()
    y = yv.toHost()
    om = orc.convert(rows, cols, vals, n, n, 32, 2)
    L = om.layout()
    if storage == "f32":
        stored = L.data.astype(np.float32).astype(np.float64)
        bound = 2.0 ** -24
    else:
        stored = oracle.bf16_block_scaled(L.data, L.block_start, 32)
        bound = 2.0 ** -8
    assert bits_equal(y, om.spmv_with_values(stored, x))
    err = _scaled_err(y, om.spmv(x), rows, cols, vals, x)
    assert err <= bound, err


def test_storage_bytes_model(lib, banded):
    n, rows, cols, vals, x = banded
    sizes = {}
    for st in (lib.STORE_NATIVE, lib.STORE_F32, lib.STORE_BF16_SCALED):
        m = lib.HBDIA(rows, cols, vals, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(st)
        sizes[st] = (m.bytesPerSpmv(), m.info().numSlots, m.info().numBlocks)
    slots, blocks = sizes[lib.STORE_NATIVE][1], sizes[lib.STORE_NATIVE][2]
    assert sizes[lib.STORE_NATIVE][0] - sizes[lib.STORE_F32][0] == 4 * slots
    assert sizes[lib.STORE_NATIVE][0] - sizes[lib.STORE_BF16_SCALED][0] == 6 * slots - 4 * blocks


def test_config3a_full_size(lib, orc):
    """The precision configuration at its own size, n = 8M: the default
    kernel with FP32 and BF16-scaled storage, bit-exact for the stored values
    and within one rounding of them against the FP64 SpMV."""
    n = 1 << 23
    rows, cols, vals = lib.generate_banded(n, OFFSETS, 0.5, 1.5, 0.3, 0.002, 2)
    x = lib.fill_uniform(n, -1.0, 1.0, 2)
    om = orc.convert(rows, cols, vals, n, n, 32, 2)
    L = om.layout()
    y64 = om.spmv(x)
    scale = np.maximum(np.bincount(rows, weights=np.abs(vals * x[cols]), minlength=n), np.finfo(float).tiny)
    for storage, st, bound in (("f32", lib.STORE_F32, 2.0 ** -24), ("bf16", lib.STORE_BF16_SCALED, 2.0 ** -8)):
        m = lib.HBDIA(rows, cols, vals, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(st)
        yv = lib.HBDIAVector(np.zeros(n))
        lib.hbdiaSpMV(m, lib.HBDIAVector(x), yv, True, False)
        m.synchronize()
        y = yv.toHost()
        stored = (L.data.astype(np.float32).astype(np.float64) if storage == "f32"
                  else oracle.bf16_block_scaled(L.data, L.block_start, 32))
        assert bits_equal(y, om.spmv_with_values(stored, x)), storage
        err = float(np.max(np.abs(y - y64) / scale))
        assert err <= bound, (storage, err)
        del m
