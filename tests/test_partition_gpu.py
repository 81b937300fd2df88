"""Row-partitioned SpMV on the GPU.  One GPU stands in for P ranks without any
kernel waiting on another: each rank's partial matrix gets its own plan and x
window, the halo ranges move between the windows through the library's
halo-copy kernel (pack from the owner's window, unpack into the reader's),
and each rank's fused SpMV runs over its window alone -- everything outside
the exchanged ranges is NaN, so a read outside them would show.  The rows of
y equal the oracle's partial-matrix SpMV bit for bit, and the whole-matrix
SpMV bit for bit when the partitions are whole blocks."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _segments(rng, src_len, dst_len, nseg):
    so, do, ln = [], [], []
    d = 0
    for _ in range(nseg):
        k = int(rng.integers(0, 40))
        if d + k > dst_len:
            break
        s = int(rng.integers(0, src_len - k + 1))
        so.append(s), do.append(d), ln.append(k)
        d += k + int(rng.integers(0, 3))
    return so, do, ln


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_halo_copy_kernel(lib, dtype):
    import torch
    from hbdia_b200.distributed import _HaloPlan
    rng = np.random.default_rng(4)
    src_len, dst_len = 5000, 20000
    so, do, ln = _segments(rng, src_len, dst_len, 600)
    src = rng.standard_normal(src_len).astype(dtype)
    dst0 = rng.standard_normal(dst_len).astype(dtype)
    exp = dst0.copy()
    for s, d, k in zip(so, do, ln):
        exp[d:d + k] = src[s:s + k]
    plan = _HaloPlan(so, do, ln, src_len, dst_len, np.dtype(dtype).itemsize, torch.device("cuda"))
    ts = torch.from_numpy(src).cuda()
    td = torch.from_numpy(dst0).cuda()
    plan(ts, td)
    torch.cuda.synchronize()
    assert bits_equal(td.cpu().numpy(), exp)
    with pytest.raises(IndexError):
        _HaloPlan([src_len - 2], [0], [3], src_len, dst_len, 8, torch.device("cuda"))


def _stencil(lib, nx, ny, nz, noise, it):
    m = lib.HBDIA()
    m.create3DStencil27Point(nx, ny, nz, noise, it)
    return m.getRowIndices(), m.getColIndices(), m.getValues(), nx * ny * nz


def _emulated(lib, rows, cols, vals, n, P, bw, thr, x, kernel=None, storage=None):
    """P ranks on one GPU: returns the concatenated y and the per-rank oracle y."""
    import torch
    from hbdia_b200.distributed import _HaloPlan
    g = lib.HBDIA(rows, cols, vals, n, n)
    ranks = []
    for p in range(P):
        m = g.partition(P, p)
        m.convertToHBDIAFormat(bw, thr, upload=storage is None)
        if storage is not None and m.getHasHBDIA():
            m.prepareForGPU(storage)
        if kernel is not None and m.getHasHBDIA():
            m.setKernel(kernel)
        w0, wl = m.window()
        win = torch.full((wl,), float("nan"), dtype=torch.float64, device="cuda")
        rb, nl = m.getGlobalRowIndex(0), m.getNumRows()
        win[rb - w0:rb - w0 + nl] = torch.from_numpy(x[rb:rb + nl]).cuda()
        ranks.append((m, w0, win, rb, nl))
    # exchange: rank p reads each of its processDataRanges from the owner q
    for p, (m, w0, win, rb, nl) in enumerate(ranks):
        for q, segs in enumerate(m.getPartialMatrixMetadata()["processDataRanges"]):
            if q == p or not segs:
                continue
            mq, wq0, winq = ranks[q][0], ranks[q][1], ranks[q][2]
            total = sum(e - s for s, e in segs)
            buf = torch.empty(total, dtype=torch.float64, device="cuda")
            off = np.cumsum([0] + [e - s for s, e in segs])[:-1]
            pack = _HaloPlan([s - wq0 for s, _ in segs], off, [e - s for s, e in segs], winq.numel(), total, 8,
                             torch.device("cuda"))
            unpack = _HaloPlan(off, [s - w0 for s, _ in segs], [e - s for s, e in segs], total, win.numel(), 8,
                               torch.device("cuda"))
            pack(winq, buf)
            unpack(buf, win)
    ys = []
    for m, w0, win, rb, nl in ranks:
        y = torch.zeros(nl, dtype=torch.float64, device="cuda")
        if m.getHasHBDIA():
            lib.spmv_device(m, win.data_ptr(), y.data_ptr(), 0)
        ys.append(y)
    torch.cuda.synchronize()
    return [y.cpu().numpy() for y in ys], ranks


@pytest.mark.parametrize("P,bw,thr,grid", [(2, 32, 2, (16, 16, 16)), (4, 32, 1, (16, 16, 16)), (3, 32, 2, (16, 16, 16)),
                                            (8, 32, 2, (16, 32, 16)), (5, 16, 1, (12, 12, 12))])
def test_emulated_ranks_equal_oracle(lib, orc, P, bw, thr, grid):
    rows, cols, vals, n = _stencil(lib, *grid, 0.01, 2)
    x = np.random.default_rng(P).uniform(-1, 1, n)
    kernels = [None, lib.KERNEL_QUAD, lib.KERNEL_WARP, lib.KERNEL_ROWWISE, lib.KERNEL_STAGED] if bw == 32 else [None]
    whole = orc.convert(rows, cols, vals, n, n, bw, thr).spmv(x)
    for kern in kernels:
        ys, ranks = _emulated(lib, rows, cols, vals, n, P, bw, thr, x, kern)
        for y, (m, w0, win, rb, nl) in zip(ys, ranks):
            r, c, v = m.coo()
            exp = orc.convert_partial(r, c, v, nl, n, rb, bw, thr).spmv_partial(x)
            assert bits_equal(y, exp), (kern, rb)
        y = np.concatenate(ys)
        if n % P == 0 and (n // P) % bw == 0:
            assert bits_equal(y, whole)
        sc = orc.coo_spmv(rows, cols, np.abs(vals), np.abs(x), n)
        assert np.all(np.abs(y - whole) <= 1e-12 * sc)


def test_emulated_ranks_quad_storage(lib):
    """A rank's partial matrix (x read through its column window) with the
    quad-interleaved FP32 / BF16 values gives the per-block storage's y, bit
    for bit, on every rank."""
    rows, cols, vals, n = _stencil(lib, 16, 32, 16, 0.01, 2)
    x = np.random.default_rng(9).uniform(-1, 1, n)
    for plain, quad in ((lib.STORE_F32, lib.STORE_F32_QUAD), (lib.STORE_BF16_SCALED, lib.STORE_BF16_QUAD)):
        ya, ranks = _emulated(lib, rows, cols, vals, n, 4, 32, 2, x, storage=plain)
        yb, ranks_q = _emulated(lib, rows, cols, vals, n, 4, 32, 2, x, storage=quad)
        for a, b, (m, *_rest) in zip(ya, yb, ranks_q):
            assert m.info().storage == quad
            assert bits_equal(a, b)


def test_emulated_ranks_random_extras_and_empty_rank(lib, orc):
    """Random columns all over x (many short halo ranges) and a rank whose
    rows hold no entries."""
    rng = np.random.default_rng(11)
    n = 4096
    r = np.concatenate([np.arange(3000), rng.integers(0, 3000, 20000)]).astype(np.int32)
    c = np.concatenate([np.arange(3000), rng.integers(0, n, 20000)]).astype(np.int32)
    o = np.argsort(r, kind="stable")
    r, c = r[o], c[o]
    v = rng.uniform(-1, 1, len(r))
    x = rng.uniform(-1, 1, n)
    ys, ranks = _emulated(lib, r, c, v, n, 4, 32, 2, x)
    assert not ranks[3][0].getHasHBDIA() and np.all(ys[3] == 0)
    whole = orc.convert(r, c, v, n, n, 32, 2).spmv(x)
    assert bits_equal(np.concatenate(ys), whole)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _nccl_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        import oracle
        import hbdia_b200 as lib
        from hbdia_b200.distributed import Distributor, PartialVector
        D = Distributor(blockWidth=32, threshold=2)
        rows, cols, vals, n = _stencil(lib, 16, 16, 16, 0.01, 0)
        local = D.scatterMatrix(lib.HBDIA(rows, cols, vals, n, n))
        x = np.random.default_rng(3).uniform(-1, 1, n)
        vec = PartialVector(D.scatterVector(x), local, device="cuda")
        y = torch.zeros(local.getNumRows(), dtype=torch.float64, device="cuda")
        D.spmv(local, vec, y)
        got = D.gatherVector(y)
        exp = oracle.Restated().convert(rows, cols, vals, n, n, 32, 2).spmv(x)
        out[rank] = bool(bits_equal(got, exp))
    finally:
        dist.destroy_process_group()


def test_distributor_single_rank_nccl(lib):
    """The Distributor's NCCL path end to end on one rank (no peers)."""
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_nccl_rank, args=(1, port, out), nprocs=1, join=True, start_method="spawn")
        assert dict(out) == {0: True}
