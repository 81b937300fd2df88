"""Seeded workload generators (host code, no GPU)."""
import numpy as np
import pytest


@pytest.mark.parametrize("extra", [0.0, 0.01, 0.05])
def test_spd_generator_symmetric_dominant(lib, extra):
    nx, ny, nz = 6, 7, 5
    rows, cols, vals = lib.generate_stencil27_spd(nx, ny, nz, 1e-3, 7, extra_fraction=extra)
    n = nx * ny * nz
    stencil = (3 * nx - 2) * (3 * ny - 2) * (3 * nz - 2)
    assert len(vals) == stencil + 2 * int(np.floor(extra * stencil / 2))
    # row-sorted, ascending distinct columns in each row
    key = rows.astype(np.int64) * n + cols
    assert np.all(np.diff(key) > 0)
    d = {(r, c): v for r, c, v in zip(rows.tolist(), cols.tolist(), vals.tolist())}
    assert all(d[(c, r)] == v for (r, c), v in d.items())
    diag = np.array([d[(i, i)] for i in range(n)])
    off = np.zeros(n)
    np.add.at(off, rows[rows != cols], np.abs(vals[rows != cols]))
    assert np.allclose(diag, (1 + 1e-3) * off)
    # extras lie outside the 27-point pattern
    def coord(i):
        return np.stack([i % nx, (i // nx) % ny, i // (nx * ny)], axis=1)
    far = np.abs(coord(rows) - coord(cols)).max(axis=1) > 1
    assert far.sum() == len(vals) - stencil
    # same seed, same matrix; another seed, another one
    r2, c2, v2 = lib.generate_stencil27_spd(nx, ny, nz, 1e-3, 7, extra_fraction=extra)
    assert np.array_equal(c2, cols) and np.array_equal(v2, vals)


def test_spd_generator_rejects(lib):
    with pytest.raises(ValueError):
        lib.generate_stencil27_spd(3, 3, 3, 1e-3, 7, extra_fraction=1.0)  # 171 pairs; 193 exist off-pattern
    with pytest.raises(ValueError):
        lib.generate_stencil27_spd(4, 4, 4, -1.0, 7)
