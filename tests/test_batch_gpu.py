"""Batched persistent launch (hbdia_batch_*): every matrix's y equals the
single-matrix entry point's y bit for bit (which the SpMV tests pin to the
oracle and to the reference), for every configuration, mixed right-hand-side
counts, rebinding under graph replay, each value storage and both value
types."""
import numpy as np
import pytest

from conftest import bits_equal, random_coo

pytestmark = pytest.mark.gpu


def _matrices(lib, dtype=np.float64, storage=0):
    rng = np.random.default_rng(17)
    srcs = []
    for e in (5, 9, 16, 23):
        r, c, v = lib.generate_stencil27(e, e, e, extra_fraction=0.01, seed=e)
        srcs.append((r, c, v, e ** 3, e ** 3))
    r, c, v = lib.generate_stencil7(12, 12, 12, 6.0, -1.0)
    srcs.append((r, c, v, 1728, 1728))
    r, c, v = lib.generate_banded(3000, [0, 1, -1, 700, -2100], 0.5, 1.5, 0.2, 0.01, 4)
    srcs.append((r, c, v, 3000, 3000))
    r, c, v = random_coo(rng, 777, 777, 9000)
    srcs.append((r, c, v, 777, 777))
    r, c, v = random_coo(rng, 500, 700, 4000)  # rectangular
    srcs.append((r, c, v, 500, 700))
    srcs.append((np.array([0], np.int32), np.array([0], np.int32), np.array([2.5]), 1, 1))
    mats = []
    for r, c, v, nr, nc in srcs:
        m = lib.HBDIA(r, c, v.astype(dtype), nr, nc, dtype=dtype)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(storage)
        mats.append(m)
    return mats


def _vectors(mats, dtype, k=None, seed=3):
    import torch
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    for i, m in enumerate(mats):
        inf = m.info()
        rows = max(inf.numRows, inf.numCols)
        ki = 1 if k is None else k[i]
        cols = max(ki, 1)
        xs.append(torch.from_numpy(rng.uniform(-1, 1, (rows, cols)).astype(dtype)).cuda())
        ys.append(torch.full((rows, cols), float("nan"), dtype=tdt, device="cuda"))
    return xs, ys


def _single(lib, m, x, k):
    """What the single-matrix entry points give."""
    import torch
    y = torch.zeros_like(x)
    if k == 1:
        lib.spmv_device(m, x.data_ptr(), y.data_ptr(), 0)
    else:
        lib.spmm_device(m, x.data_ptr(), x.shape[1], y.data_ptr(), y.shape[1], k, 0)
    torch.cuda.synchronize()
    return y


def _check_all(lib, mats, xs, ys, k=None):
    import torch
    torch.cuda.synchronize()
    for i, m in enumerate(mats):
        ki = 1 if k is None else k[i]
        n = m.info().numRows
        if ki == 0:
            assert torch.isnan(ys[i]).all()
            continue
        ref = _single(lib, m, xs[i], ki)
        assert bits_equal(ys[i][:n].cpu().numpy(), ref[:n].cpu().numpy()), f"matrix {i}"


def _bind(b, xs, ys, k=None):
    if k is None:
        b.bind([x.data_ptr() for x in xs], [y.data_ptr() for y in ys])
    else:
        b.bind([x.data_ptr() for x in xs], [y.data_ptr() for y in ys], k=k,
               ldx=[x.shape[1] for x in xs], ldy=[y.shape[1] for y in ys])


def test_batch_matches_single_matrix(lib, orc):
    mats = _matrices(lib)
    xs, ys = _vectors(mats, np.float64)
    b = lib.Batch(mats)
    _bind(b, xs, ys)
    b.run(0)
    _check_all(lib, mats, xs, ys)
    # one matrix straight against the oracle as well
    r, c, v = lib.generate_stencil27(16, 16, 16, extra_fraction=0.01, seed=16)
    o = orc.convert(r, c, v, 4096, 4096, 32, 2)
    assert bits_equal(ys[2][:, 0].cpu().numpy(), o.spmv(xs[2][:, 0].cpu().numpy()))
    count, tiles, nbytes = b.info()
    assert count == len(mats)
    assert tiles == sum((m.info().numRows + 31) // 32 for m in mats)
    assert nbytes == sum(m.info().bytesPerSpmv for m in mats)


@pytest.mark.parametrize("threads", [128, 256, 512])
@pytest.mark.parametrize("grab", [1, 3, 8])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_queue_configs_identical(lib, threads, grab, graph):
    mats = _matrices(lib)
    xs, ys = _vectors(mats, np.float64)
    b = lib.Batch(mats)
    b.set_config(lib.BATCH_QUEUE, None, threads, grab, 8, graph)
    _bind(b, xs, ys)
    b.run(0)
    b.run(0)  # replay
    _check_all(lib, mats, xs, ys)


@pytest.mark.parametrize("streams", [1, 3, 16, 64])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_concurrent_configs_identical(lib, streams, graph):
    mats = _matrices(lib)
    xs, ys = _vectors(mats, np.float64)
    b = lib.Batch(mats)
    b.set_config(lib.BATCH_CONCURRENT, streams, graph=graph)
    _bind(b, xs, ys)
    b.run(0)
    b.run(0)  # replay
    _check_all(lib, mats, xs, ys)


@pytest.mark.parametrize("schedule,tile", [(0, 8), (1, 4), (1, 8), (1, 16)])
def test_batch_mixed_rhs(lib, schedule, tile):
    mats = _matrices(lib)
    k = [1, 3, 8, 0, 2, 17, 1, 5, 1]
    xs, ys = _vectors(mats, np.float64, k)
    b = lib.Batch(mats)
    b.set_config(schedule, None, 256, 2, tile, True)
    _bind(b, xs, ys, k)
    b.run(0)
    _check_all(lib, mats, xs, ys, k)


def test_batch_strided_rhs(lib):
    """Leading dimensions larger than k (column windows of wider blocks)."""
    import torch
    mats = _matrices(lib)[:4]
    rng = np.random.default_rng(8)
    k = [3, 5, 4, 2]
    X, Y = [], []
    for m in mats:
        rows = m.info().numRows
        X.append(torch.from_numpy(rng.uniform(-1, 1, (rows, 7))).cuda())
        Y.append(torch.zeros((rows, 9), dtype=torch.float64, device="cuda"))
    b = lib.Batch(mats)
    b.bind([x[:, 1:].data_ptr() for x in X], [y[:, 2:].data_ptr() for y in Y], k=k,
           ldx=[7] * 4, ldy=[9] * 4)
    b.run(0)
    torch.cuda.synchronize()
    for m, ki, x, y in zip(mats, k, X, Y):
        for j in range(ki):
            ref = _single(lib, m, x[:, 1 + j].contiguous(), 1)
            assert bits_equal(y[:, 2 + j].cpu().numpy(), ref.cpu().numpy())
        assert (y[:, :2] == 0).all() and (y[:, 2 + ki:] == 0).all()


@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_rebind_under_graph(lib, schedule):
    """New pointers and a switch between single-vector and multi-RHS bindings
    replay the right graph."""
    mats = _matrices(lib)
    b = lib.Batch(mats)
    b.set_config(schedule)
    for seed, k in ((1, None), (2, [1, 2, 1, 1, 3, 1, 1, 1, 1]), (3, None), (4, [2] * 9)):
        xs, ys = _vectors(mats, np.float64, k, seed=seed)
        _bind(b, xs, ys, k)
        b.run(0)
        _check_all(lib, mats, xs, ys, k)


@pytest.mark.parametrize("dtype,storage", [(np.float64, 1), (np.float64, 2), (np.float32, 0)])
@pytest.mark.parametrize("multi", [False, True])
@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_storage_and_dtype(lib, dtype, storage, multi, schedule):
    mats = _matrices(lib, dtype, storage)
    k = [1, 2, 1, 1, 6, 1, 1, 3, 1] if multi else [1, 1, 0, 1, 1, 1, 1, 1, 1]
    xs, ys = _vectors(mats, dtype, k)
    b = lib.Batch(mats)
    b.set_config(schedule)
    _bind(b, xs, ys, k)
    b.run(0)
    _check_all(lib, mats, xs, ys, k)


def test_batch_autotune_keeps_results(lib):
    mats = _matrices(lib)
    k = [1, 4, 1, 1, 1, 1, 2, 1, 1]
    xs, ys = _vectors(mats, np.float64, k)
    b = lib.Batch(mats)
    _bind(b, xs, ys, k)
    ms, n = b.autotune(0)
    assert ms > 0 and n == 3 + 3 * 5 * 3  # 3 stream counts + threads x grab x RHS tile
    c = b.config()
    assert c.schedule in (0, 1) and c.streams in (4, 9, 16, 64)
    assert c.threadsPerBlock in (128, 256, 512) and c.tilesPerGrab in (1, 2, 4, 8, 16) and c.rhsTile in (4, 8, 16)
    for y in ys:
        y.fill_(float("nan"))
    b.run(0)
    _check_all(lib, mats, xs, ys, k)


def test_batch_autotune_single_vector(lib):
    mats = _matrices(lib)
    xs, ys = _vectors(mats, np.float64)
    b = lib.Batch(mats)
    _bind(b, xs, ys)
    ms, n = b.autotune(0)
    assert ms > 0 and n == 3 + 3 * 5  # 3 stream counts + threads x grab
    for y in ys:
        y.fill_(float("nan"))
    b.run(0)
    _check_all(lib, mats, xs, ys)


def test_batch_rejections(lib):
    import torch
    mats = _matrices(lib)[:2]
    b = lib.Batch(mats)
    with pytest.raises(ValueError):
        b.run(0)  # nothing bound
    with pytest.raises(ValueError):
        b.set_config(lib.BATCH_QUEUE, None, 192, 2, 8, True)
    with pytest.raises(ValueError):
        b.set_config(lib.BATCH_CONCURRENT, 65)
    with pytest.raises(ValueError):
        b.set_config(7)
    with pytest.raises(ValueError):
        b.bind([0, 0], [0, 0])
    r, c, v = lib.generate_stencil7(6, 6, 6, 6.0, -1.0)
    f32 = lib.HBDIA(r, c, v, 216, 216)
    f32.convertToHBDIAFormat(32, 2, upload=False)
    f32.prepareForGPU(lib.STORE_F32)
    with pytest.raises(ValueError):
        lib.Batch([mats[0], f32])
    w16 = lib.HBDIA(r, c, v, 216, 216)
    w16.convertToHBDIAFormat(16, 2)
    with pytest.raises(NotImplementedError):
        lib.Batch([w16])
    host = lib.HBDIA(r, c, v, 216, 216)
    host.convertToHBDIAFormat(32, 2, upload=False)
    with pytest.raises(RuntimeError):
        lib.Batch([host])
    x = torch.zeros(216, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        b.bind([x.data_ptr()] * 2, [x.data_ptr()] * 2, k=[2, 1], ldx=[1, 1], ldy=[2, 1])
    with pytest.raises(ValueError, match="contiguous"):
        b.bind([x.data_ptr()] * 2, [x.data_ptr()] * 2, k=[1, 1], ldx=[7, 1], ldy=[1, 1])


@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_many_segments(lib, schedule):
    """330 matrices: three queue segments (each its own kernel node), or 330
    concurrent launches; rebound and replayed."""
    rng = np.random.default_rng(29)
    mats = []
    for i in range(330):
        e = int(rng.integers(3, 9))
        r, c, v = lib.generate_stencil7(e, e, e, 6.0, -1.0 - i * 1e-3)
        m = lib.HBDIA(r, c, v, e ** 3, e ** 3)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(0)
        mats.append(m)
    b = lib.Batch(mats)
    b.set_config(schedule)
    for seed, k in ((5, None), (6, [int(rng.integers(0, 4)) for _ in range(330)])):
        xs, ys = _vectors(mats, np.float64, k, seed=seed)
        _bind(b, xs, ys, k)
        b.run(0)
        _check_all(lib, mats, xs, ys, k)
