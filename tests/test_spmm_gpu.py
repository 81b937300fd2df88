"""Multi-RHS SpMM: Y = A X on k right-hand sides.  Column j of Y must equal
the SpMV of column j bit for bit (same arithmetic order), for every RHS tile
width, block width, storage and X layout; the autotuner only ever changes
speed."""
import numpy as np
import pytest

from conftest import bits_equal, random_coo

pytestmark = pytest.mark.gpu


def _spmm(lib, m, X, k, ldx=None, ldy=None, offset=0):
    import torch
    n = m.getNumRows()
    ldx = ldx or k
    ldy = ldy or k
    Xt = torch.zeros(n * ldx + offset, dtype=torch.float64, device="cuda")
    Xt[offset:offset + n * ldx].view(n, ldx)[:, :k] = torch.from_numpy(X).cuda()
    Yt = torch.full((n * ldy,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib.spmm_device(m, Xt.data_ptr() + 8 * offset, ldx, Yt.data_ptr(), ldy, k)
    m.synchronize()
    return Yt.view(n, ldy)[:, :k].cpu().numpy()


def _expected(orc, rows, cols, vals, n, bw, thr, X):
    om = orc.convert(rows, cols, vals, n, n, bw, thr)
    return np.stack([om.spmv(np.ascontiguousarray(X[:, j])) for j in range(X.shape[1])], axis=1)


@pytest.mark.parametrize("tile", [2, 4, 8, 16, 32])
@pytest.mark.parametrize("k", [1, 3, 4, 9, 16, 33])
def test_spmm_columns_equal_spmv(lib, orc, tile, k):
    rng = np.random.default_rng(300 + k)
    n = 3000
    rows, cols, vals = random_coo(rng, n, n, 30000)
    X = rng.uniform(-1, 1, (n, k))
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    m.setTuning(lib.TUNE_SPMM_TILE, tile)
    Y = _spmm(lib, m, X, k)
    assert bits_equal(np.ascontiguousarray(Y), _expected(orc, rows, cols, vals, n, 32, 2, X))


@pytest.mark.parametrize("bw", [8, 32])
def test_spmm_layouts(lib, orc, bw):
    """padded leading dimensions and an X that is not 16-byte aligned"""
    rng = np.random.default_rng(41)
    n = 20 * 21 * 22
    rows, cols, vals = lib.generate_stencil27(20, 21, 22, 26.0, -1.0, 0.01, 0.1, 1.0, 9)
    k = 6
    X = rng.uniform(-1, 1, (n, k))
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(bw, 2)
    want = _expected(orc, rows, cols, vals, n, bw, 2, X)
    for ldx, ldy, off in ((6, 6, 0), (8, 7, 0), (7, 6, 1), (6, 9, 1)):
        Y = _spmm(lib, m, X, k, ldx, ldy, off)
        assert bits_equal(np.ascontiguousarray(Y), want), (ldx, ldy, off)


def test_spmm_f32_storage(lib, orc):
    import oracle  # noqa: F401
    rng = np.random.default_rng(44)
    n = 16 ** 3
    rows, cols, vals = lib.generate_stencil27(16, 16, 16, 26.0, -1.0, 0.02, 0.1, 1.0, 3)
    k = 4
    X = rng.uniform(-1, 1, (n, k))
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(lib.STORE_F32)
    Y = _spmm(lib, m, X, k)
    om = orc.convert(rows, cols, vals, n, n, 32, 2)
    stored = om.layout().data.astype(np.float32).astype(np.float64)
    want = np.stack([om.spmv_with_values(stored, np.ascontiguousarray(X[:, j])) for j in range(k)], axis=1)
    assert bits_equal(np.ascontiguousarray(Y), want)


def test_autotune_spmv_and_spmm(lib, orc):
    import torch
    lib.autotune_clear()
    n = 48 ** 3
    rows, cols, vals = lib.generate_stencil27(48, 48, 48, 26.0, -1.0, 0.01, 0.1, 1.0, 2)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    x = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, n)).cuda()
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = m.autotune(x.data_ptr(), y.data_ptr(), k=1)
    assert r.kernel in (lib.KERNEL_PIPE, lib.KERNEL_WARP, lib.KERNEL_STAGED) and r.fromCache == 0
    assert r.msPerCall > 0
    # a second matrix of the same class takes the cached choice
    m2 = lib.HBDIA(rows, cols, vals, n, n)
    m2.convertToHBDIAFormat(32, 2)
    r2 = m2.autotune(x.data_ptr(), y.data_ptr(), k=1)
    assert r2.fromCache == 1 and r2.kernel == r.kernel and r2.unroll == r.unroll
    lib.spmv_device(m2, x.data_ptr(), y.data_ptr())
    m2.synchronize()
    xn = x.cpu().numpy()
    assert bits_equal(y.cpu().numpy(), orc.convert(rows, cols, vals, n, n, 32, 2).spmv(xn))
    k = 8
    X = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, (n, k))).cuda().contiguous()
    Y = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    r3 = m.autotune(X.data_ptr(), Y.data_ptr(), k=k)
    assert r3.spmmTile in (2, 4, 8, 16, 32)
    lib.spmm_device(m, X.data_ptr(), k, Y.data_ptr(), k, k)
    m.synchronize()
    want = _expected(orc, rows, cols, vals, n, 32, 2, X.cpu().numpy()[:, :2])
    assert bits_equal(np.ascontiguousarray(Y.cpu().numpy()[:, :2]), want)


@pytest.mark.parametrize("bw", [32, 16])
@pytest.mark.parametrize("tile", [2, 4, 16])
@pytest.mark.parametrize("k", [1, 5, 17])
def test_spmm_colmajor_equals_spmv(lib, orc, bw, tile, k):
    """Column-major blocks (each right-hand side a contiguous vector, leading
    dimension larger than n): column j equals the SpMV of vector j."""
    import torch
    rng = np.random.default_rng(900 + k + bw)
    n = 2500
    rows, cols, vals = random_coo(rng, n, n, 26000)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(bw, 2)
    m.setTuning(lib.TUNE_SPMM_TILE, tile)
    ld = n + 37
    X = rng.uniform(-1, 1, (k, n))
    Xt = torch.zeros((k, ld), dtype=torch.float64, device="cuda")
    Xt[:, :n] = torch.from_numpy(X).cuda()
    Yt = torch.full((k, ld + 3), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib.spmm_device_colmajor(m, Xt.data_ptr(), ld, Yt.data_ptr(), ld + 3, k)
    m.synchronize()
    Y = Yt.cpu().numpy()
    om = orc.convert(rows, cols, vals, n, n, bw, 2)
    for j in range(k):
        assert bits_equal(Y[j, :n], om.spmv(np.ascontiguousarray(X[j])))
    assert np.isnan(Y[:, n:]).all()  # nothing outside the columns written
    with pytest.raises(ValueError):
        lib.spmm_device_colmajor(m, Xt.data_ptr(), n - 1, Yt.data_ptr(), ld, k)


@pytest.mark.parametrize("storage", [0, 1, 2])
@pytest.mark.parametrize("k", [1, 3, 8, 13, 32, 45])
def test_spmv_list_equals_spmv(lib, k, storage):
    """Separate device vectors (scattered allocations) through the
    vector-list SpMM: each y_j equals its own SpMV bit for bit, for every
    value storage, k past one launch's 32, and tile widths forced."""
    import torch
    rng = np.random.default_rng(700 + k)
    n = 2500
    rows, cols, vals = random_coo(rng, n, n, 25000)
    i = np.arange(n, dtype=np.int32)
    rows = np.concatenate([rows, i, i[1:]]).astype(np.int32)
    cols = np.concatenate([cols, i, i[:-1]]).astype(np.int32)
    vals = np.concatenate([vals, rng.uniform(-1, 1, 2 * n - 1)])
    o = np.argsort(rows, kind="stable")
    m = lib.HBDIA(rows[o], cols[o], vals[o], n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(storage)
    xs = [torch.from_numpy(rng.uniform(-1, 1, n)).cuda() for _ in range(k)]
    pad = [torch.empty(int(rng.integers(1, 100)), dtype=torch.float64, device="cuda") for _ in range(k)]
    ys = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(k)]
    ref = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(k)]
    for x, r in zip(xs, ref):
        lib.spmv_device(m, x.data_ptr(), r.data_ptr(), 0)
    for tile in (0, 2, 4, 16):
        m.setTuning(lib.TUNE_SPMM_TILE, tile)
        for y in ys:
            y.fill_(float("nan"))
        lib.spmv_list_device(m, [x.data_ptr() for x in xs], [y.data_ptr() for y in ys], 0)
        torch.cuda.synchronize()
        for y, r in zip(ys, ref):
            assert bits_equal(y.cpu().numpy(), r.cpu().numpy()), tile
    del pad


def test_spmv_list_other_block_widths_and_errors(lib, orc):
    import torch
    rng = np.random.default_rng(9)
    n = 900
    rows, cols, vals = random_coo(rng, n, n, 9000)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(16, 1)
    xs = [rng.uniform(-1, 1, n) for _ in range(5)]
    tx = [torch.from_numpy(x).cuda() for x in xs]
    ty = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in xs]
    lib.spmv_list_device(m, [t.data_ptr() for t in tx], [t.data_ptr() for t in ty], 0)
    torch.cuda.synchronize()
    om = orc.convert(rows, cols, vals, n, n, 16, 1)
    for x, y in zip(xs, ty):
        assert bits_equal(y.cpu().numpy(), om.spmv(x))
    with pytest.raises(ValueError):
        lib.spmv_list_device(m, [tx[0].data_ptr(), 0], [ty[0].data_ptr(), ty[1].data_ptr()], 0)
    lib.spmv_list_device(m, [], [], 0)  # nothing to do
