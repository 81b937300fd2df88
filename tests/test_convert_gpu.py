"""GPU converter (hbdia_matrix_convert_on_device): the device-built layout --
offsets, block starts, values, COO remainder, its row pointer, histograms,
numberDiagonals -- equals the host converter's bit for bit (which
tests/test_convert.py pins to the oracle and to the reference), and SpMVs
on it equal the oracle's."""
import numpy as np
import pytest

from conftest import bits_equal, random_coo

pytestmark = pytest.mark.gpu


def _pair(lib, rows, cols, vals, nr, nc, bw, thr, max_coo=10**9, dtype=np.float64):
    host = lib.HBDIA(rows, cols, vals.astype(dtype), nr, nc, dtype=dtype)
    host.convertToHBDIAFormat(bw, thr, max_coo, upload=False)
    dev = lib.HBDIA(rows, cols, vals.astype(dtype), nr, nc, dtype=dtype)
    dev.convertOnDevice(bw, thr, max_coo)
    return host, dev


def _same_layout(host, dev):
    hi, di = host.info(), dev.info()
    for f in ("numBlocks", "numberDiagonals", "totalOffsets", "numSlots", "numCoo", "histogramLength"):
        assert getattr(hi, f) == getattr(di, f), f
    a, b = host.layout(), dev.layout()
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
            if a[k].dtype.kind == "f":
                assert bits_equal(a[k], b[k]), k
            else:
                assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], k


def _sorted(rng, nr, nc, nnz, zero_frac=0.05):
    return random_coo(rng, nr, nc, nnz, sort=True, zero_frac=zero_frac)


@pytest.mark.parametrize("bw", [32, 16, 8, 64, 3])
@pytest.mark.parametrize("thr", [1, 2, 3])
def test_layout_equals_host(lib, bw, thr):
    rng = np.random.default_rng(100 + bw * 7 + thr)
    n = 1500
    rows, cols, vals = _sorted(rng, n, n, 12000)
    # a band so that offsets are kept, plus duplicates of some entries
    i = np.arange(n, dtype=np.int32)
    band = [(i[:-1], i[1:]), (i, i), (i[1:], i[:-1])]
    br = np.concatenate([b[0] for b in band] + [rows])
    bc = np.concatenate([b[1] for b in band] + [cols])
    bv = rng.standard_normal(len(br))
    dup = rng.integers(0, len(br), 800)
    br, bc, bv = np.concatenate([br, br[dup]]), np.concatenate([bc, bc[dup]]), np.concatenate([bv, -bv[dup]])
    o = np.argsort(br, kind="stable")
    host, dev = _pair(lib, br[o], bc[o], bv[o], n, n, bw, thr)
    _same_layout(host, dev)


@pytest.mark.parametrize("max_coo", [0, 1, 50, 400, 10**9])
def test_max_coo_cutoff(lib, max_coo):
    rng = np.random.default_rng(7)
    rows, cols, vals = _sorted(rng, 900, 900, 9000)
    host, dev = _pair(lib, rows, cols, vals, 900, 900, 32, 3, max_coo)
    _same_layout(host, dev)


@pytest.mark.parametrize("shape", [(700, 1000), (1000, 700), (33, 2000), (2000, 33)])
def test_rectangular_and_tail_blocks(lib, shape):
    nr, nc = shape
    rng = np.random.default_rng(nr + nc)
    rows, cols, vals = _sorted(rng, nr, nc, 8000)
    host, dev = _pair(lib, rows, cols, vals, nr, nc, 32, 2)
    _same_layout(host, dev)


def test_block_larger_than_shared_sort(lib):
    """Block 0 holds 32 rows x 200 entries (6400 > 4096): the global-memory path."""
    rng = np.random.default_rng(3)
    nr, nc = 200, 5000
    rows = np.repeat(np.arange(32, dtype=np.int32), 200)
    cols = np.concatenate([np.sort(rng.choice(nc, 200, replace=False)) for _ in range(32)]).astype(np.int32)
    r2, c2, v2 = _sorted(rng, nr, nc, 3000)
    keep = r2 >= 32
    rows = np.concatenate([rows, r2[keep]])
    cols = np.concatenate([cols, c2[keep]])
    vals = rng.standard_normal(len(rows))
    host, dev = _pair(lib, rows, cols, vals, nr, nc, 32, 2)
    _same_layout(host, dev)


def test_stencil_float32_and_spmv(lib, orc):
    import torch
    rows, cols, vals = lib.generate_stencil27(20, 20, 20, extra_fraction=0.01, seed=5)
    n = 8000
    for dt in (np.float64, np.float32):
        host, dev = _pair(lib, rows, cols, vals, n, n, 32, 2, dtype=dt)
        _same_layout(host, dev)
    dev = lib.HBDIA(rows, cols, vals, n, n)
    dev.convertOnDevice(32, 2)
    x = np.random.default_rng(2).uniform(-1, 1, n)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros(n, dtype=torch.float64, device="cuda")
    for kern in (lib.KERNEL_PIPE, lib.KERNEL_QUAD, lib.KERNEL_WARP, lib.KERNEL_ROWWISE, lib.KERNEL_STAGED):
        dev.setKernel(kern)
        lib.spmv_device(dev, xt.data_ptr(), yt.data_ptr(), 0)
        torch.cuda.synchronize()
        assert bits_equal(yt.cpu().numpy(), orc.convert(rows, cols, vals, n, n, 32, 2).spmv(x))


@pytest.mark.parametrize("storage", [1, 2])
def test_reduced_storage_equals_host_built(lib, storage):
    import torch
    rows, cols, vals = lib.generate_stencil27(18, 18, 18, extra_fraction=0.01, seed=6)
    n = 18 ** 3
    host = lib.HBDIA(rows, cols, vals, n, n)
    host.convertToHBDIAFormat(32, 2, upload=False)
    host.prepareForGPU(storage)
    dev = lib.HBDIA(rows, cols, vals, n, n)
    dev.convertOnDevice(32, 2, storage=storage)
    assert dev.info().storage == storage and dev.info().deviceBytes > 0
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, n)).cuda()
    y1 = torch.zeros(n, dtype=torch.float64, device="cuda")
    y2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    lib.spmv_device(host, x.data_ptr(), y1.data_ptr(), 0)
    lib.spmv_device(dev, x.data_ptr(), y2.data_ptr(), 0)
    torch.cuda.synchronize()
    assert bits_equal(y1.cpu().numpy(), y2.cpu().numpy())
    with pytest.raises(NotImplementedError):
        dev.layout()  # no exact values to export from reduced storage


def test_unsorted_rejected_and_noops(lib):
    rows = np.array([3, 1, 2], np.int32)
    cols = np.array([0, 1, 2], np.int32)
    m = lib.HBDIA(rows, cols, np.ones(3), 4, 4)
    with pytest.raises(NotImplementedError, match="row-sorted"):
        m.convertOnDevice(32, 1)
    e = lib.HBDIA(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0), 4, 4)
    e.convertOnDevice(32, 1)  # empty matrix: no-op, like the reference
    assert not e.getHasHBDIA()
    rows, cols, vals = lib.generate_stencil7(6, 6, 6, 6.0, -1.0)
    m = lib.HBDIA(rows, cols, vals, 216, 216)
    m.convertOnDevice(32, 2)
    before = m.info().deviceBytes
    m.convertOnDevice(16, 1)  # converted already: no-op
    assert m.getBlockWidth() == 32 and m.info().deviceBytes == before
