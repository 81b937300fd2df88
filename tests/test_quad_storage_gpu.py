"""Quad-interleaved value storage (HBDIA_STORE_F32_QUAD / HBDIA_STORE_BF16_QUAD):
the values of every uniform quad (four consecutive blocks with one list of at
most 32 offsets) stored [offset][lane][block] so that the quad kernel loads a
lane's four values of an offset at once.  The y must equal the plain FP32 /
BF16-scaled storage's bit for bit -- on matrices whose quads are all uniform
(banded), mixed with non-uniform and boundary quads and a partial last quad
(stencil with a dense COO corner and an odd row count), and mostly non-uniform
(random) -- for every group size of the quad kernel; the CG solver and the
server give the same solutions on it; products other than the SpMV refuse it."""
import numpy as np
import pytest

from conftest import bits_equal, random_coo

pytestmark = pytest.mark.gpu


def _stencil_with_corner(lib):
    n = 40 * 41 * 40 + 7
    r, c, v = lib.generate_stencil27(40, 41, 40, 26.0, -1.0, 0.02, 0.1, 1.0, 9)
    extra_r = np.repeat(np.arange(96, 101, dtype=np.int32), 14)
    extra_c = (np.arange(70, dtype=np.int32) * 977 + 5) % n
    rows = np.concatenate([r, extra_r])
    cols = np.concatenate([c, extra_c])
    vals = np.concatenate([v, np.random.default_rng(5).uniform(0.1, 1.0, 70)])
    o = np.argsort(rows, kind="stable")
    return rows[o], cols[o], vals[o], n


def _cases(lib):
    n = 1 << 18
    r, c, v = lib.generate_banded(n, [0, 1, -1, 2, -2, 64, -64, 4096, -4096], 0.5, 1.5, 0.3, 0.002, 2)
    yield "banded", r, c, v, n
    yield ("stencil",) + _stencil_with_corner(lib)
    rr, cc, vv = random_coo(np.random.default_rng(11), 5000, 5000, 60000)
    o = np.argsort(rr, kind="stable")
    yield "random", rr[o], cc[o], vv[o], 5000


def _spmv(lib, m, x):
    yv = lib.HBDIAVector(np.full(len(x), np.nan))
    lib.hbdiaSpMV(m, lib.HBDIAVector(x), yv, True, False)
    m.synchronize()
    return yv.toHost()


@pytest.mark.parametrize("pair", [("STORE_F32", "STORE_F32_QUAD"), ("STORE_BF16_SCALED", "STORE_BF16_QUAD")],
                         ids=["f32", "bf16"])
def test_quad_storage_equals_narrow_storage(lib, pair):
    plain, quad = getattr(lib, pair[0]), getattr(lib, pair[1])
    for name, rows, cols, vals, n in _cases(lib):
        x = np.random.default_rng(3).uniform(-1, 1, n)
        ref = lib.HBDIA(rows, cols, vals, n, n)
        ref.convertToHBDIAFormat(32, 2, upload=False)
        ref.prepareForGPU(plain)
        ref.setKernel(lib.KERNEL_PIPE)
        yref = _spmv(lib, ref, x)
        m = lib.HBDIA(rows, cols, vals, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(quad)
        assert m.info().storage == quad
        m.setKernel(lib.KERNEL_PIPE)  # the layout runs the quad kernel whatever is set
        xv = lib.HBDIAVector(x)
        assert m.selectedKernel(xv.getDeviceDataPtr()) == lib.KERNEL_QUAD
        for g in (0, 1, 2, 4, 8):
            m.setTuning(lib.TUNE_QUAD_GROUP, g)
            assert bits_equal(_spmv(lib, m, x), yref), (name, g)
        assert m.bytesPerSpmv() == ref.bytesPerSpmv()


def test_quad_storage_refuses_other_products(lib):
    import torch
    n = 4096
    rows, cols, vals = lib.generate_stencil27(16, 16, 16, 26.0, -1.0, 0.01, 0.1, 1.0, 1)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(lib.STORE_F32_QUAD)
    X = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    Y = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(NotImplementedError):
        lib.spmm_device(m, X.data_ptr(), 4, Y.data_ptr(), 4, 4)
    with pytest.raises(NotImplementedError):
        lib.Batch([m])
    with pytest.raises(NotImplementedError):  # blockWidth other than 32
        m8 = lib.HBDIA(rows, cols, vals, n, n)
        m8.convertToHBDIAFormat(8, 2, upload=False)
        m8.prepareForGPU(lib.STORE_F32_QUAD)


def test_cg_and_server_on_quad_storage(lib):
    """CG iterating on the quad-interleaved FP32 values gives the FP32
    storage's solution bit for bit (same iterations), alone and in a server."""
    import torch
    g = 24
    n = g ** 3
    rows, cols, vals = lib.generate_stencil27_spd(g, g, g, 1e-3, 7)
    b = lib.fill_uniform(n, -1.0, 1.0, 11)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    bt = torch.from_numpy(b).cuda()
    sol = {}
    for st in (lib.STORE_F32, lib.STORE_F32_QUAD):
        xt = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = lib.cg_solve(m, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=st)
        assert r.converged == 1
        sol[st] = (r.iterations, xt.cpu().numpy())
    assert sol[lib.STORE_F32][0] == sol[lib.STORE_F32_QUAD][0]
    assert bits_equal(sol[lib.STORE_F32][1], sol[lib.STORE_F32_QUAD][1])
    for group in (1, 4):
        srv = lib.Server(cgIterStorage=lib.STORE_F32_QUAD, cgMaxGroup=group, cgWorkers=1)
        mid = srv.add_matrix(m)
        srv.pause(True)
        ys = [np.full(n, np.nan) for _ in range(3)]
        ts = [srv.submit(mid, lib.REQ_CG, b, y) for y in ys]
        srv.pause(False)
        infos = [srv.wait(t) for t in ts]
        srv.close()
        for info, y in zip(infos, ys):
            assert info.status == 0 and info.cgIterations == sol[lib.STORE_F32][0]
            assert bits_equal(y, sol[lib.STORE_F32][1])


def test_quad_iteration_storage_falls_back(lib):
    """CG's default iteration storage is quad-interleaved FP32; a layout that
    cannot take it (blockWidth 8) iterates on the per-block FP32 values,
    which give the same iterates: same solution, bit for bit."""
    import torch
    g = 16
    n = g ** 3
    rows, cols, vals = lib.generate_stencil27_spd(g, g, g, 1e-3, 7)
    b = lib.fill_uniform(n, -1.0, 1.0, 11)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(8, 2)
    bt = torch.from_numpy(b).cuda()
    out = []
    for st in (lib.STORE_F32_QUAD, lib.STORE_F32):
        xt = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = lib.cg_solve(m, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=st)
        assert r.converged == 1
        out.append((r.iterations, xt.cpu().numpy()))
    assert out[0][0] == out[1][0] and bits_equal(out[0][1], out[1][1])
    srv = lib.Server()  # default cgIterStorage: the quad-interleaved FP32 values
    y = np.full(n, np.nan)
    info = srv.wait(srv.submit(srv.add_matrix(m), lib.REQ_CG, b, y))
    srv.close()
    assert info.status == 0 and bits_equal(y, out[1][1])


def test_quad_storage_other_builders_refuse(lib):
    """The GPU converter and plans over a caller's layout build per-block
    layouts only: both refuse the quad-interleaved storage codes."""
    n = 4096
    rows, cols, vals = lib.generate_stencil27(16, 16, 16, 26.0, -1.0, 0.01, 0.1, 1.0, 1)
    for st in (lib.STORE_F32_QUAD, lib.STORE_BF16_QUAD):
        m = lib.HBDIA(rows, cols, vals, n, n)
        with pytest.raises(ValueError):
            m.convertOnDevice(32, 2, storage=st)
        with pytest.raises(ValueError):  # refused on the host: no array is read
            lib.LayoutPlan(storage=st, numRows=n, numCols=n, blockWidth=32, numBlocks=128, totalOffsets=1,
                           numCoo=0, values=0, offsets=0, blockStart=0)
