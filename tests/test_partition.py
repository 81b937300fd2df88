"""Row-partitioned distribution on CPU: partitions, partial-matrix layouts and
their metadata (data ranges, per-process ranges, buffer sizes) against the
reference's own BasicExtractor / partial conversion / analyzeDataRanges /
extractPartialMatrixMetadata (oracle/_ref), and the N>1 exchange path as gloo
ranks: every halo entry arrives (the reference's verifyDataExchange check)
and the gathered y -- each rank's rows computed by the oracle over nothing but
its x window -- equals the whole-matrix SpMV."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import bits_equal

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
QUIET = {"noise": 0.0}


def _stencil(ref_or_lib, nx, ny, nz, noise, it):
    m = ref_or_lib.HBDIA()
    m.create3DStencil27Point(nx, ny, nz, noise, it)
    r, c, v = m.getRowIndices(), m.getColIndices(), m.getValues()
    return r, c, v, nx * ny * nz


def _banded(n, seed):
    rng = np.random.default_rng(seed)
    offs = [-40, -3, -1, 0, 1, 2, 33]
    rows, cols = [], []
    for o in offs:
        r = np.arange(max(0, -o), min(n, n - o))
        keep = rng.random(len(r)) > 0.2
        rows.append(r[keep]), cols.append(r[keep] + o)
    extra = rng.integers(0, n, (n // 10, 2))
    rows.append(extra[:, 0]), cols.append(extra[:, 1])
    r = np.concatenate(rows).astype(np.int32)
    c = np.concatenate(cols).astype(np.int32)
    o = np.argsort(r, kind="stable")
    return r[o], c[o], rng.uniform(-1, 1, len(r)), n


def _data_ranges(part_coo_cols, layout, bw, row_base, n_local, n_global):
    """analyzeDataRanges restated: COO columns and every kept offset's lane
    columns of existing rows, merged into [start, end) ranges."""
    mark = np.zeros(n_global + 1, bool)
    mark[part_coo_cols] = True
    bs, off = layout["block_start"], layout["offsets"]
    for b in range(len(bs) - 1):
        lanes = min(bw, n_local - b * bw)
        for k in range(bs[b], bs[b + 1]):
            g0 = row_base + b * bw + off[k]
            lo, hi = max(g0, 0), min(g0 + lanes, n_global)
            if lo < hi:
                mark[lo:hi] = True
    d = np.diff(np.concatenate([[0], mark[:n_global].astype(np.int8), [0]]))
    return np.stack([np.flatnonzero(d == 1), np.flatnonzero(d == -1)], axis=1).astype(np.int32)


def _process_ranges(meta):
    return np.array([(q, s, e) for q, rs in enumerate(meta["processDataRanges"]) for s, e in rs],
                    np.int32).reshape(-1, 3)


CASES = [  # (matrix, P, blockWidth, threshold); n / P a multiple of bw where the reference is compared whole
    ("stencil", 2, 32, 1), ("stencil", 4, 32, 2), ("stencil", 8, 32, 1), ("stencil", 4, 16, 1),
    ("banded", 2, 32, 1), ("banded", 4, 32, 2), ("banded", 3, 32, 1), ("stencil", 3, 32, 1), ("stencil", 5, 8, 2),
]


def _matrix(lib, kind):
    if kind == "stencil":
        return _stencil(lib, 8, 8, 8, 0.01, 0)
    return _banded(768, 5)


@pytest.mark.parametrize("kind,P,bw,thr", CASES)
def test_partitions_match_reference(lib, ref, kind, P, bw, thr):
    rows, cols, vals, n = _matrix(lib, kind)
    g = lib.HBDIA(rows, cols, vals, n, n)
    aligned = n % P == 0 and (n // P) % bw == 0
    for part in range(P):
        R = ref.partition(rows, cols, vals, n, P, part, bw, thr)
        m = g.partition(P, part)
        assert m.isPartialMatrix() and m.getNumGlobalRows() == n and m.getNumGlobalNonZeros() == len(vals)
        r, c, v = m.coo()
        assert np.array_equal(r, R["rows"]) and np.array_equal(c, R["cols"]) and bits_equal(v, R["vals"])
        assert m.getGlobalRowIndex(0) == R["row_start"] and m.getNumRows() == R["num_local_rows"]
        m.convertToHBDIAFormat(bw, thr, upload=False)
        L, RL = m.layout(), R["layout"]
        for k in ("offsets", "block_start", "coo_row", "coo_col", "coo_row_ptr", "hist_blocks", "hist_nnz"):
            assert np.array_equal(L[k], getattr(RL, k)), k
        assert bits_equal(L["data"], RL.data) and bits_equal(L["coo_val"], RL.coo_val)
        assert m.getNumberDiagonals() == RL.number_diagonals
        meta = m.getPartialMatrixMetadata()
        dr = np.array(meta["dataRanges"], np.int32).reshape(-1, 2)
        rb = m.getGlobalRowIndex(0)
        # the reference reads its row mapping past the end for a partial last
        # block's missing lanes; only whole blocks have a defined answer there
        assert np.array_equal(dr, _data_ranges(c, L, bw, rb, m.getNumRows(), n))
        if aligned:
            assert np.array_equal(dr, R["data_ranges"])
            assert np.array_equal(_process_ranges(meta), R["process_ranges"])
            assert meta["totalBufferSize"] == R["total_buffer_size"]
        # HBDIAVector(localData, matrix, rank, size) buffer sizes
        pr = _process_ranges(meta)
        i = m.partialInfo()
        assert i.leftBufferSize == int(np.sum((pr[:, 2] - pr[:, 1])[pr[:, 0] < part]))
        assert i.rightBufferSize == int(np.sum((pr[:, 2] - pr[:, 1])[pr[:, 0] > part]))
        # the window holds the rank's rows and every data range
        w0, wl = m.window()
        assert w0 <= rb and rb + m.getNumRows() <= w0 + wl
        assert len(dr) == 0 or (dr[0, 0] >= w0 and dr[-1, 1] <= w0 + wl)


def test_partitions_reassemble_and_spmv_is_window_local(lib, orc):
    """Every entry lands in exactly one partition in input order; each
    partition's oracle rows of y need only its window (x NaN elsewhere); the
    concatenation equals the whole-matrix SpMV -- bit for bit when the
    partitions are whole blocks, within rounding otherwise."""
    rows, cols, vals, n = _stencil(lib, 12, 12, 12, 0.02, 3)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    for P, bw, thr in ((4, 16, 2), (3, 32, 2), (6, 32, 1)):
        g = lib.HBDIA(rows, cols, vals, n, n)
        whole = orc.convert(rows, cols, vals, n, n, bw, thr).spmv(x)
        ys, rr = [], []
        for part in range(P):
            m = g.partition(P, part)
            r, c, v = m.coo()
            rb = m.getGlobalRowIndex(0)
            rr.append(r + rb)
            m.convertToHBDIAFormat(bw, thr, upload=False)
            w0, wl = m.window()
            xw = np.full(n, np.nan)
            xw[w0:w0 + wl] = x[w0:w0 + wl]
            y = orc.convert_partial(r, c, v, m.getNumRows(), n, rb, bw, thr).spmv_partial(xw)
            assert not np.any(np.isnan(y))
            ys.append(y)
        assert np.array_equal(np.concatenate(rr), rows)
        y = np.concatenate(ys)
        if n % P == 0 and (n // P) % bw == 0:
            assert bits_equal(y, whole)
        scale = orc.coo_spmv(rows, cols, np.abs(vals), np.abs(x), n)
        assert np.all(np.abs(y - whole) <= 1e-12 * scale)


def test_partial_errors(lib):
    r = np.array([0, 1], np.int32)
    c = np.array([0, 5], np.int32)
    v = np.ones(2)
    with pytest.raises(NotImplementedError):
        lib.HBDIA.partial(r, c, v, 2, 8, [3, 5], True, 8, 8, 2, 0, 2)
    with pytest.raises(NotImplementedError):  # square matrices only
        lib.HBDIA.partial(r, c, v, 2, 8, [0, 1], True, 6, 8, 2, 0, 2)
    with pytest.raises(IndexError):  # local rows past the global matrix
        lib.HBDIA.partial(r, c, v, 2, 8, [7, 8], True, 8, 8, 2, 1, 2)
    with pytest.raises(IndexError):  # a column outside the global matrix
        lib.HBDIA.partial(r, np.array([0, 8], np.int32), v, 2, 8, [0, 1], True, 8, 8, 2, 0, 2)
    with pytest.raises(ValueError):
        lib.HBDIA.partial(r, c, v, 2, 8, [0, 1], True, 8, 8, 2, 2, 2)
    g = lib.HBDIA(r, c, v, 8, 8)
    with pytest.raises(ValueError):
        g.partition(9, 0)  # more processes than rows
    with pytest.raises(ValueError):
        g.partition(2, 2)
    with pytest.raises(NotImplementedError):
        lib.HBDIA(r, c, v, 8, 10).partition(2, 0)
    p = g.partition(2, 1)  # rows 4..7 hold no entries: nothing to convert
    p.convertToHBDIAFormat(32, 1, upload=False)
    assert not p.getHasHBDIA() and p.window() == (4, 4) and p.getDataRanges() == []
    with pytest.raises(NotImplementedError):
        p.partition(2, 0)
    q = g.partition(2, 0)
    q.convertToHBDIAFormat(32, 1, upload=False)  # both offsets kept: every lane of block 0 reads
    assert q.getDataRanges() == [(0, 8)] and q.window() == (0, 8)
    q = g.partition(2, 0)
    q.convertToHBDIAFormat(32, 2, upload=False)  # both entries in COO: only their columns
    assert q.getDataRanges() == [(0, 1), (5, 6)] and q.window() == (0, 6)
    meta = q.getPartialMatrixMetadata()
    assert meta["processDataRanges"] == [[(0, 1)], [(5, 6)]] and meta["totalBufferSize"] == 2


# ---------------------------------------------------------------- gloo ranks
def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, case, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import oracle
        import hbdia_b200 as lib
        from hbdia_b200.distributed import Distributor, PartialVector
        kind, bw, thr = case
        D = Distributor(blockWidth=bw, threshold=thr)
        if D.isRootProcess():
            if kind == "stencil":
                rows, cols, vals, n = _stencil(lib, 8, 16, 8, 0.02, 1)
            elif kind == "banded":
                rows, cols, vals, n = _banded(700, 9)
            else:  # the last rank's rows hold no entries
                n = 96
                rows = np.repeat(np.arange(40, dtype=np.int32), 2)
                cols = np.stack([np.arange(40), (np.arange(40) * 7 + 50) % n], 1).ravel().astype(np.int32)
                vals = np.linspace(-1, 1, len(rows))
            g = lib.HBDIA(rows, cols, vals, n, n)
            local = D.scatterMatrix(g)
            xg = np.arange(n, dtype=np.float64)
            xl = D.scatterVector(xg)
        else:
            local = D.receiveMatrix()
            xl = D.receiveVector()
        assert local.getNumRows() == len(xl) and local.isPartialMatrix()
        vec = PartialVector(xl, local, rank, world)
        assert vec.getTotalSize() == vec.getLocalSize() + vec.leftSize + vec.rightSize
        D.exchangeData(local, vec)
        ok_verify = D.verifyDataExchange(local, vec)
        orc = oracle.Restated()
        r, c, v = local.coo()
        rb = local.getGlobalRowIndex(0)
        n = local.getNumGlobalRows()
        ys = []
        for scale in (1.0, -0.5):  # a second exchange reuses the agreed ranges
            vec.local.copy_(vec.local * scale) if scale != 1.0 else None
            D.exchangeData(local, vec)
            xw = np.full(n, np.nan)
            w0, wl = local.window()
            xw[w0:w0 + wl] = vec.window.numpy()
            if local.getHasHBDIA():
                y = orc.convert_partial(r, c, v, local.getNumRows(), n, rb, bw, thr).spmv_partial(xw)
            else:
                y = np.zeros(local.getNumRows())
            ys.append(D.gatherVector(y))
        if D.isRootProcess():
            whole = orc.convert(rows, cols, vals, n, n, bw, thr)
            exp = [whole.spmv(xg), whole.spmv(xg * -0.5)]
            aligned = n % world == 0 and (n // world) % bw == 0
            res = []
            for y, e in zip(ys, exp):
                sc = orc.coo_spmv(rows, cols, np.abs(vals), np.abs(xg), n) + 1e-300
                res.append((bool(bits_equal(y, e)) if aligned else True, float(np.max(np.abs(y - e) / sc))))
            out[rank] = (ok_verify, res)
        else:
            out[rank] = (ok_verify, None)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [(2, ("stencil", 32, 1)), (4, ("stencil", 16, 2)), (3, ("banded", 32, 1)),
                                        (2, ("banded", 8, 2)), (3, ("empty_last", 32, 1))])
def test_gloo_ranks_exchange_and_spmv(lib, world, case):
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, port, case, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert all(res[r][0] for r in range(world)), "verifyDataExchange failed"
    for exact, err in res[0][1]:
        assert exact and err <= 1e-12
