"""Serving engine (hbdia_server_*): a request's result is the same whether it
is served alone or batched with others (bit for bit), SpMV results equal the
single-matrix entry points on the same value storage, CG results reach the
FP64 tolerance (checked on the host) and equal hbdia_cg_solve, and admission
keeps the device memory the server holds within its budget."""
import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu


def _spd(lib, e, seed):
    rows, cols, vals = lib.generate_stencil27_spd(e, e, e, 1e-3, seed, extra_fraction=0.005)
    n = e ** 3
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    return m, (rows, cols, vals), n


@pytest.fixture(scope="module")
def mats(lib):
    return [_spd(lib, e, 5 + e) for e in (10, 14, 18)]


def _host_residual(rcv, x, b):
    rows, cols, vals = rcv
    ax = np.zeros(len(b))
    np.add.at(ax, rows, vals * x[cols])
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


def _pinned(n, rng=None):
    import torch
    t = torch.empty(n, dtype=torch.float64).pin_memory()
    a = t.numpy()
    if rng is not None:
        a[:] = rng.uniform(-1, 1, n)
    else:
        a[:] = np.nan
    return t, a


@pytest.mark.parametrize("batching", [1, 0])
def test_same_alone_and_in_mix(lib, mats, batching):
    srv = lib.Server(batching=batching)
    ids = [srv.add_matrix(m) for m, _, _ in mats]
    rng = np.random.default_rng(1)
    keep = []
    # alone: one SpMV and one CG per matrix, each waited for before the next
    alone = []
    for mid, (m, rcv, n) in zip(ids, mats):
        tx, x = _pinned(n, rng)
        ty, y = _pinned(n)
        info = srv.wait(srv.submit(mid, lib.REQ_SPMV, x, y))
        assert info.status == 0 and info.batchRhs == 1
        tb, b = _pinned(n, rng)
        tc, c = _pinned(n)
        info = srv.wait(srv.submit(mid, lib.REQ_CG, b, c))
        assert info.status == 0 and info.cgRelResidual <= 1e-10
        assert _host_residual(rcv, c, b) <= 2e-10
        keep += [tx, ty, tb, tc]
        alone.append((x.copy(), y.copy(), b.copy(), c.copy()))
    # mix: a burst of SpMVs on every matrix (the alone x among them) and CGs,
    # queued while the server is paused so that they are served together
    srv.pause(True)
    pending = []
    for rep in range(8):
        for j, (mid, (m, rcv, n)) in enumerate(zip(ids, mats)):
            x0, y0, b0, c0 = alone[j]
            tx, x = _pinned(n, rng)
            if rep in (2, 5):
                x[:] = x0
            ty, y = _pinned(n)
            keep += [tx, ty]
            pending.append(("spmv", j, rep, x, y, srv.submit(mid, lib.REQ_SPMV, x, y)))
            if rep == 3:
                tb, b = _pinned(n)
                b[:] = b0
                tc, c = _pinned(n)
                keep += [tb, tc]
                pending.append(("cg", j, rep, b, c, srv.submit(mid, lib.REQ_CG, b, c)))
    with pytest.raises(RuntimeError, match="paused"):
        srv.wait(pending[0][-1])
    srv.pause(False)
    widest = 1
    for kind, j, rep, x, y, t in pending:
        info = srv.wait(t)
        assert info.status == 0
        x0, y0, b0, c0 = alone[j]
        if kind == "spmv":
            widest = max(widest, info.batchRhs)
            if rep in (2, 5):
                assert bits_equal(y, y0)
            if batching == 0:
                assert info.batchRhs == 1
        else:
            assert bits_equal(y, c0)
    if batching:
        assert widest == 8  # each matrix's 8 queued SpMVs went as one SpMM
    st = srv.stats()
    assert st.completed == len(pending) + 2 * len(mats) and st.matrices == 3
    srv.close()


def test_cg_group_equals_lone_solves(lib, mats):
    """CG requests queued together on one matrix are solved as one lockstep
    group (one SpMM per iteration); each result equals its lone cg_solve bit
    for bit, whatever the group's other members -- including a zero right-hand
    side (done before the first iteration) and a smooth one that converges at
    its own iteration count."""
    import torch
    m, rcv, n = mats[2]
    rows, cols, vals = rcv
    rng = np.random.default_rng(21)
    bs = [rng.uniform(-1, 1, n), np.zeros(n), np.cos(np.arange(n) * 0.001), rng.uniform(-1, 1, n) * 1e3,
          rng.uniform(0, 1, n)]
    srv = lib.Server(cgWorkers=1, cgMaxGroup=8)
    mid = srv.add_matrix(m)
    srv.pause(True)
    keep, pending = [], []
    for b0 in bs:
        tb, b = _pinned(n)
        b[:] = b0
        tc, c = _pinned(n)
        keep += [tb, tc]
        pending.append((b0, c, srv.submit(mid, lib.REQ_CG, b, c)))
    srv.pause(False)
    infos = [srv.wait(t) for _, _, t in pending]
    st = srv.stats()
    srv.close()
    assert all(i.status == 0 for i in infos)
    assert max(i.batchRhs for i in infos) == len(bs)  # all five went as one group
    assert st.cgGroups == 1
    ref = lib.HBDIA(rows, cols, vals, n, n)
    ref.convertToHBDIAFormat(32, 2)
    iters = set()
    for (b0, c, _), info in zip(pending, infos):
        bt = torch.from_numpy(b0).cuda()
        xt = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = lib.cg_solve(ref, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=lib.STORE_F32)
        assert r.iterations == info.cgIterations and r.updates == info.cgUpdates
        assert bits_equal(xt.cpu().numpy(), c)
        iters.add(info.cgIterations)
    assert len(iters) > 1  # the members left the group at different iterations


def test_spmv_matches_entry_points_and_fp64(lib, mats):
    import torch
    m, rcv, n = mats[1]
    rows, cols, vals = rcv
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, n)
    res = {}
    for storage in (lib.STORE_F32, lib.STORE_NATIVE):
        srv = lib.Server(spmvStorage=storage)
        mid = srv.add_matrix(m)
        y = np.full(n, np.nan)
        assert srv.wait(srv.submit(mid, lib.REQ_SPMV, x, y)).status == 0
        srv.close()
        ref = lib.HBDIA(rows, cols, vals, n, n)
        ref.convertToHBDIAFormat(32, 2, upload=False)
        ref.prepareForGPU(storage)
        xt = torch.from_numpy(x).cuda()
        yt = torch.zeros(n, dtype=torch.float64, device="cuda")
        lib.spmv_device(ref, xt.data_ptr(), yt.data_ptr(), 0)
        torch.cuda.synchronize()
        assert bits_equal(y, yt.cpu().numpy())
        res[storage] = y
    scale = np.zeros(n)
    np.add.at(scale, rows, np.abs(vals * x[cols]))
    assert np.max(np.abs(res[lib.STORE_F32] - res[lib.STORE_NATIVE]) / scale) <= 1e-6


def test_cg_matches_cg_solve(lib, mats):
    import torch
    m, rcv, n = mats[0]
    rows, cols, vals = rcv
    b = np.random.default_rng(9).uniform(-1, 1, n)
    srv = lib.Server()
    mid = srv.add_matrix(m)
    y = np.zeros(n)
    info = srv.wait(srv.submit(mid, lib.REQ_CG, b, y))
    srv.close()
    assert info.status == 0 and info.cgUpdates >= 1
    ref = lib.HBDIA(rows, cols, vals, n, n)
    ref.convertToHBDIAFormat(32, 2)
    bt = torch.from_numpy(b).cuda()
    xt = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = lib.cg_solve(ref, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=lib.STORE_F32)
    assert r.iterations == info.cgIterations and r.updates == info.cgUpdates
    assert bits_equal(xt.cpu().numpy(), y)


def test_admission_budget(lib, mats):
    m0, _, _ = mats[0]
    with pytest.raises(MemoryError, match="admission"):
        lib.Server(memoryBudget=1 << 16).add_matrix(m0)  # the 1000-row matrix needs about 1 MB
    big = lib.Server()
    big.add_matrix(m0)
    need1 = big.stats().deviceBytes  # plans, staging and the CG workspaces' share
    big.add_matrix(m0)
    need2 = big.stats().deviceBytes  # a second copy adds no CG workspace growth
    big.close()
    per = need2 - need1
    assert 0 < per < need1
    budget = need2 + per // 2  # two copies fit, not three
    srv = lib.Server(memoryBudget=budget)
    srv.add_matrix(m0)
    srv.add_matrix(m0)
    with pytest.raises(MemoryError):
        srv.add_matrix(m0)
    assert srv.stats().deviceBytes <= budget
    srv.close()


def test_server_rejections(lib, mats):
    m0, _, n = mats[0]
    srv = lib.Server()
    mid = srv.add_matrix(m0)
    x, y = np.zeros(n), np.zeros(n)
    with pytest.raises(IndexError):
        srv.submit(mid + 5, lib.REQ_SPMV, x, y)
    with pytest.raises(ValueError):
        srv.submit(mid, 7, x, y)
    t = srv.submit(mid, lib.REQ_SPMV, x, y)
    srv.wait(t)
    with pytest.raises(ValueError):
        srv.wait(t)  # collected already
    with pytest.raises(TypeError):
        lib.Server(noSuchOption=1)
    with pytest.raises(ValueError):
        lib.Server(maxRhs=0)
    host_only = lib.HBDIA(np.array([0], np.int32), np.array([0], np.int32), np.array([1.0]), 1, 1)
    with pytest.raises(RuntimeError):
        srv.add_matrix(host_only)  # not converted
    srv.close()


def test_burst_over_many_matrices(lib):
    """A burst over 20 matrices, queued while paused, is issued in one
    scheduler pass (each matrix's two requests as one batch on its own
    stream) and gives the bits of the requests served alone."""
    srv = lib.Server()
    rng = np.random.default_rng(12)
    mats = []
    for i in range(20):
        m, rcv, n = _spd(lib, 4 + i % 4, 30 + i)
        mats.append((srv.add_matrix(m), n))
    alone = []
    for mid, n in mats:
        x = rng.uniform(-1, 1, n)
        y = np.full(n, np.nan)
        srv.wait(srv.submit(mid, lib.REQ_SPMV, x, y))
        alone.append((x, y))
    srv.pause(True)
    pend = []
    for (mid, n), (x, y0) in zip(mats, alone):
        for _ in range(2):
            y = np.full(n, np.nan)
            pend.append((srv.submit(mid, lib.REQ_SPMV, x, y), y, y0))
    srv.pause(False)
    for t, y, y0 in pend:
        info = srv.wait(t)
        assert info.status == 0 and info.batchRhs == 2
        assert bits_equal(y, y0)
    assert srv.stats().spmvSteps == 21  # 20 alone + one pass for the whole burst
    srv.close()


def test_device_requests_equal_host_requests(lib, mats):
    """Requests on device buffers (read and written in place) give the same
    bits as the same requests on host buffers, batched or alone, mixed with
    host requests in one step; device CG equals host CG."""
    import torch
    srv = lib.Server()
    ids = [srv.add_matrix(m) for m, _, _ in mats]
    rng = np.random.default_rng(3)
    keep, host_y, dev = [], {}, []
    # reference results: host requests served one at a time
    for j, (mid, (m, rcv, n)) in enumerate(zip(ids, mats)):
        for rep in range(3):
            tx, x = _pinned(n, rng)
            ty, y = _pinned(n)
            keep += [tx, ty]
            assert srv.wait(srv.submit(mid, lib.REQ_SPMV, x, y)).status == 0
            host_y[(j, rep)] = (x.copy(), y.copy())
        tb, b = _pinned(n, rng)
        tc, c = _pinned(n)
        keep += [tb, tc]
        assert srv.wait(srv.submit(mid, lib.REQ_CG, b, c)).status == 0
        host_y[(j, "cg")] = (b.copy(), c.copy())
    # the same inputs as device requests, queued together with host requests
    srv.pause(True)
    pending = []
    for rep in range(12):
        for j, (mid, (m, rcv, n)) in enumerate(zip(ids, mats)):
            x0, y0 = host_y[(j, rep % 3)]
            xd = torch.from_numpy(x0).cuda()
            yd = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
            pending.append((y0, yd, srv.submit_device(mid, lib.REQ_SPMV, xd, yd)))
            keep.append(xd)
            if rep % 4 == 1:  # a host request in the same step
                tx, x = _pinned(n)
                x[:] = x0
                ty, y = _pinned(n)
                keep += [tx, ty]
                pending.append((y0, y, srv.submit(mid, lib.REQ_SPMV, x, y)))
            if rep == 5:
                b0, c0 = host_y[(j, "cg")]
                bd = torch.from_numpy(b0).cuda()
                cd = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
                keep.append(bd)
                pending.append((c0, cd, srv.submit_device(mid, lib.REQ_CG, bd, cd)))
    srv.pause(False)
    widest = 0
    for exp, got, t in pending:
        info = srv.wait(t)
        assert info.status == 0
        widest = max(widest, info.batchRhs)
        g = got.cpu().numpy() if hasattr(got, "is_cuda") else got
        assert bits_equal(g, exp)
    assert widest >= 12  # the paused backlog formed vector-list batches
    with pytest.raises(ValueError):
        srv.submit_device(ids[0], lib.REQ_SPMV, torch.zeros(4), torch.zeros(4))
    srv.close()
