"""Plans over a device layout the caller owns (hbdia_plan_create): the HBDIA
arrays as prepareForGPU leaves them on the device -- here uploaded from the
reference's own conversions (tests/golden) and from this library's layouts --
run through the fused kernels with results bit-identical to the oracle and to
the matrix entry points; malformed layouts are refused before any SpMV."""
import glob
import os

import numpy as np
import pytest

from conftest import bits_equal, random_coo

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _plan(lib, L, nr, nc, bw, dtype=np.float64, storage=0, values=None, scales=None):
    vals = _dev(L["data"] if values is None else values)
    arrs = {"values": vals, "offsets": _dev(L["offsets"].astype(np.int32)),
            "blockStart": _dev(L["block_start"].astype(np.int32))}
    ncoo = len(L["coo_row"])
    if ncoo:
        arrs.update(cooRow=_dev(L["coo_row"].astype(np.int32)), cooCol=_dev(L["coo_col"].astype(np.int32)),
                    cooVal=_dev(L["coo_val"]), cooRowPtr=_dev(L["coo_row_ptr"].astype(np.int32)))
    if scales is not None:
        arrs["scales"] = _dev(scales.astype(np.float32))
    ptrs = {k: v.data_ptr() for k, v in arrs.items()}
    return lib.LayoutPlan(dtype=dtype, storage=storage, numRows=nr, numCols=nc, blockWidth=bw,
                          numBlocks=len(L["block_start"]) - 1, totalOffsets=int(L["block_start"][-1]),
                          numCoo=ncoo, keep=arrs, **ptrs)


def _run(plan, x, n, dtype=np.float64):
    import torch
    xt = _dev(x)
    y = torch.full((n,), float("nan"), dtype=torch.float64 if dtype == np.float64 else torch.float32, device="cuda")
    plan.spmv(xt.data_ptr(), y.data_ptr(), 0)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_reference_layouts(lib, orc):
    """The reference's own converted layouts (golden fixtures, written from
    its convertToHBDIAFormat): y equals the oracle's bit for bit."""
    seen = 0
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        d = np.load(f)
        if "block_start" not in d or not bool(d["has_hbdia"]):
            continue
        nr, nc, bw, thr = (int(v) for v in d["params"][:4])
        dtype = d["data"].dtype.type
        L = {k: d[k] for k in ("offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr")}
        x = np.random.default_rng(3).uniform(-1, 1, max(nr, nc)).astype(dtype)
        sorted_coo = len(L["coo_row"]) < 2 or bool(np.all(np.diff(L["coo_row"]) >= 0))
        if not sorted_coo:  # the reference's row pointer assumes row-sorted COO
            with pytest.raises(ValueError, match="row-sorted|cooRowPtr"):
                _plan(lib, L, nr, nc, bw, dtype)
            continue
        plan = _plan(lib, L, nr, nc, bw, dtype)
        exp = orc.convert(d["rows"], d["cols"], d["vals"], nr, nc, bw, thr, int(d["params"][4])).spmv(x)[:nr]
        assert bits_equal(_run(plan, x, nr, dtype), exp), f
        seen += 1
    assert seen >= 5


@pytest.mark.parametrize("storage", [0, 1, 2])
@pytest.mark.parametrize("bw", [32, 8])
def test_own_layouts_equal_matrix_entry_points(lib, storage, bw):
    import torch
    rng = np.random.default_rng(5 + bw)
    n = 20000
    rows, cols, vals = random_coo(rng, n, n, 200000)
    i = np.arange(n, dtype=np.int32)
    rows = np.concatenate([rows, i, i[1:], i[:-1]]).astype(np.int32)
    cols = np.concatenate([cols, i, i[:-1], i[1:]]).astype(np.int32)
    vals = np.concatenate([vals, rng.uniform(-1, 1, 3 * n - 2)])
    o = np.argsort(rows, kind="stable")
    m = lib.HBDIA(rows[o], cols[o], vals[o], n, n)
    m.convertToHBDIAFormat(bw, 2, upload=False)
    m.prepareForGPU(storage)
    L = m.layout()
    values, scales = L["data"], None
    if storage == 1:
        values = L["data"].astype(np.float32)
    elif storage == 2:  # bfloat16 of v / block max |v|, one float scale per block
        bs = L["block_start"]
        scales = np.ones(len(bs) - 1)
        q = np.zeros(len(values), np.float32)
        for b in range(len(bs) - 1):
            s0, s1 = bs[b] * bw, bs[b + 1] * bw
            mx = np.max(np.abs(values[s0:s1])) if s1 > s0 else 0.0
            scales[b] = mx if mx > 0 else 1.0
            q[s0:s1] = (values[s0:s1] / scales[b]).astype(np.float32)
        values = torch.from_numpy(q).to(torch.bfloat16).view(torch.int16).numpy()
    plan = _plan(lib, L, n, n, bw, storage=storage, values=values, scales=scales)
    x = rng.uniform(-1, 1, n)
    xt = _dev(x)
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    lib.spmv_device(m, xt.data_ptr(), y.data_ptr(), 0)
    torch.cuda.synchronize()
    assert bits_equal(_run(plan, x, n), y.cpu().numpy())
    # SpMM on the plan
    k = 6
    X = _dev(rng.uniform(-1, 1, (n, k)))
    Y1 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    Y2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    lib.spmm_device(m, X.data_ptr(), k, Y1.data_ptr(), k, k)
    plan.spmm(X.data_ptr(), k, Y2.data_ptr(), k, k, 0)
    torch.cuda.synchronize()
    assert torch.equal(Y1.view(torch.int64), Y2.view(torch.int64))


def test_malformed_layouts_refused(lib):
    rng = np.random.default_rng(2)
    n = 3000
    rows, cols, vals = random_coo(rng, n, n, 20000)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    L = m.layout()
    assert len(L["coo_row"]) > 0
    bad = dict(L, block_start=L["block_start"].copy())
    bad["block_start"][5] = bad["block_start"][6] + 1
    with pytest.raises(ValueError, match="blockStart"):
        _plan(lib, bad, n, n, 32)
    bad = dict(L, coo_row_ptr=L["coo_row_ptr"].copy())
    bad["coo_row_ptr"][-1] += 1
    with pytest.raises(ValueError, match="cooRowPtr"):
        _plan(lib, bad, n, n, 32)
    bad = dict(L, coo_col=L["coo_col"].copy())
    bad["coo_col"][3] = n
    with pytest.raises(IndexError):
        _plan(lib, bad, n, n, 32)
    bad = dict(L, coo_row=L["coo_row"].copy())
    bad["coo_row"][0], bad["coo_row"][-1] = bad["coo_row"][-1], bad["coo_row"][0]
    with pytest.raises(ValueError, match="row-sorted"):
        _plan(lib, bad, n, n, 32)
    with pytest.raises(ValueError):  # more blocks than the matrix has
        lib.LayoutPlan(numRows=n, numCols=n, blockWidth=32, numBlocks=n, totalOffsets=0, numCoo=0, values=0,
                       offsets=0, blockStart=1)
    # a good plan still works afterwards
    plan = _plan(lib, L, n, n, 32)
    x = rng.uniform(-1, 1, n)
    assert np.all(np.isfinite(_run(plan, x, n)))


@pytest.mark.parametrize("case", ["stencil", "random"])
def test_reference_device_arrays(lib, ref, case):
    """The reference converts on the GPU (its prepareForGPU allocates and fills
    its device arrays); a plan over THOSE arrays, no copy, gives the same y as
    the reference's own hbdiaSpMV on them, bit for bit."""
    rng = np.random.default_rng(8)
    if case == "stencil":
        rows, cols, vals, nr, nc = ref.stencil27(16, 16, 16, 0.01, 2)
    else:
        nr = nc = 5000
        rows, cols, vals = random_coo(rng, nr, nc, 60000)
    g = ref.gpu_matrix(rows, cols, vals, nr, nc, 32, 2)
    a = g.arrays()
    assert a["numCoo"] > 0 and a["values"] and a["cooRowPtr"]
    plan = lib.LayoutPlan(numRows=nr, numCols=nc, blockWidth=32, keep=g, **a)
    x = rng.uniform(-1, 1, max(nr, nc))
    assert bits_equal(_run(plan, x, nr), g.spmv(x))
    del plan
