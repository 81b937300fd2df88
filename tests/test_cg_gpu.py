"""Mixed-precision CG: FP64 refinement around FP32-storage inner CG reaches
the FP64 residual target; the final residual is recomputed independently on
the host from the COO triplets.  Plain FP64 CG (inner storage FP64) is the
comparison point; runs are bit-reproducible."""
import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu


def _host_residual(rows, cols, vals, x, b):
    ax = np.zeros(len(b))
    np.add.at(ax, rows, vals * x[cols])
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def spd(lib):
    g = 40
    n = g ** 3
    rows, cols, vals = lib.generate_stencil27_spd(g, g, g, 1e-3, 7)
    b = lib.fill_uniform(n, -1.0, 1.0, 11)
    return n, rows, cols, vals, b




@pytest.mark.parametrize("inner", ["f32", "f64"])
def test_cg_reaches_fp64_tolerance(lib, spd, inner):
    import torch
    n, rows, cols, vals, b = spd
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    bt = torch.from_numpy(b).cuda()
    xt = torch.zeros(n, dtype=torch.float64, device="cuda")
    st = lib.STORE_F32 if inner == "f32" else lib.STORE_NATIVE
    r = lib.cg_solve(m, bt.data_ptr(), xt.data_ptr(), tol=1e-10, inner_storage=st, inner_tol=1e-6 if inner == "f32" else 1e-11)
    assert r.converged == 1 and r.relResidual <= 1e-10
    assert _host_residual(rows, cols, vals, xt.cpu().numpy(), b) <= 2e-10
    if inner == "f32":
        assert r.outerIterations >= 2  # FP32-stored values need refinement
    # bit-reproducible
    x2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    r2 = lib.cg_solve(m, bt.data_ptr(), x2.data_ptr(), tol=1e-10, inner_storage=st,
                      inner_tol=1e-6 if inner == "f32" else 1e-11)
    assert r2.innerIterations == r.innerIterations
    assert bits_equal(x2.cpu().numpy(), xt.cpu().numpy())


def test_cg_rejects_bad_input(lib, spd):
    n, rows, cols, vals, b = spd
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    with pytest.raises(ValueError):
        lib.cg_solve(m, 0, 0)
    m32 = lib.HBDIA(rows, cols, vals.astype(np.float32), n, n, dtype=np.float32)
    m32.convertToHBDIAFormat(32, 2)
    import torch
    t = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(NotImplementedError):
        lib.cg_solve(m32, t.data_ptr(), t.data_ptr())
