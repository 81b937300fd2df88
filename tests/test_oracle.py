"""The oracle is pinned before it is trusted: the C restatement must reproduce
the golden fixtures recorded from the reference's own code
(tests/golden/make_golden.py), and -- where oracle/_ref is built -- agree with
the reference on fresh random inputs."""
import glob
import os

import numpy as np
import pytest

from conftest import bits_equal, random_coo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LAYOUT_KEYS = ("offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
               "hist_blocks", "hist_nnz")


def layout_fixtures():
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if os.path.basename(p) not in ("cpu_coo_spmv.npz", "spmv_reference_gpu.npz", "dia_reference.npz"))


def assert_layout_equal(L, d):
    assert int(L.num_blocks) == int(d["num_blocks"])
    assert int(L.number_diagonals) == int(d["number_diagonals"])
    for k in LAYOUT_KEYS:
        a, b = getattr(L, k), d[k]
        assert a.shape == b.shape, k
        assert a.dtype == b.dtype, k
        if a.dtype.kind == "f":
            assert bits_equal(a, b), k
        else:
            assert np.array_equal(a, b), k


@pytest.mark.parametrize("path", layout_fixtures(), ids=lambda p: os.path.basename(p))
def test_restated_oracle_matches_golden(orc, path):
    d = np.load(path)
    nr, nc, bw, thr, mc = [int(v) for v in d["params"]]
    L = orc.convert(d["rows"], d["cols"], d["vals"], nr, nc, bw, thr, mc).layout()
    assert_layout_equal(L, d)


def test_print_test_20x20_known_answer():
    """Known answer of the reference's own print test (bw 8, threshold 3):
    three row blocks with offsets {-1,0,1,2}, {-1,0,1,2}, {-1,0,1}; the
    remainder holds the four scattered 0.3 entries that share no kept
    diagonal; (18,19) is a duplicate of the super-diagonal and wins its slot."""
    d = np.load(os.path.join(GOLDEN, "print_test_20x20.npz"))
    bs = d["block_start"]
    per_block = [d["offsets"][bs[b]:bs[b + 1]].tolist() for b in range(int(d["num_blocks"]))]
    assert per_block == [[-1, 0, 1, 2], [-1, 0, 1, 2], [-1, 0, 1]]
    assert list(zip(d["coo_row"].tolist(), d["coo_col"].tolist())) == [(2, 15), (5, 18), (10, 3), (15, 8)]
    # slot of (18,19): block 2, offset +1 (index 2), lane 2
    assert d["data"][(int(bs[2]) + 2) * 8 + 2] == 0.3


def test_restated_coo_spmv_matches_reference_golden(orc):
    d = np.load(os.path.join(GOLDEN, "cpu_coo_spmv.npz"))
    y = orc.coo_spmv(d["rows"], d["cols"], d["vals"], d["x"], len(d["x"]))
    assert bits_equal(y, d["y"])


def test_restated_spmv_matches_reference_gpu_golden(orc):
    """y of the reference's full hbdiaSpMV (recorded on a B200 by
    make_golden.py --gpu) equals the restated oracle's y bit for bit."""
    p = os.path.join(GOLDEN, "spmv_reference_gpu.npz")
    if not os.path.exists(p):
        pytest.skip("reference GPU fixture not recorded yet")
    d = np.load(p)
    for k in range(int(d["ncase"])):
        nr, nc, bw, thr = [int(v) for v in d[f"c{k}_params"]]
        y = orc.convert(d[f"c{k}_rows"], d[f"c{k}_cols"], d[f"c{k}_vals"], nr, nc, bw, thr).spmv(d[f"c{k}_x"])
        assert bits_equal(y, d[f"c{k}_y"]), k


def test_restated_vs_reference_random(orc, ref):
    rng = np.random.default_rng(77)
    for trial in range(60):
        nr = int(rng.integers(1, 120))
        nc = int(rng.integers(1, 120)) if trial % 4 == 0 else nr
        rows, cols, vals = random_coo(rng, nr, nc, int(rng.integers(0, 700)), sort=trial % 3 != 0)
        bw = int(rng.choice([1, 3, 4, 8, 32, 64]))
        thr = int(rng.integers(-1, 5))
        mc = int(rng.choice([0, 2, 20, 10 ** 9]))
        for dt in (np.float64, np.float32):
            a = ref.convert(rows, cols, vals.astype(dt), nr, nc, bw, thr, mc)
            if not a.has_hbdia:
                continue
            b = orc.convert(rows, cols, vals.astype(dt), nr, nc, bw, thr, mc).layout()
            for k in LAYOUT_KEYS:
                x, y = getattr(a, k), getattr(b, k)
                assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), (trial, k)
            assert a.number_diagonals == b.number_diagonals


def test_reference_coo_kernel_vs_restated_sorted(orc, ref):
    rng = np.random.default_rng(78)
    n = 3000
    rows, cols, vals = random_coo(rng, n, n, 20000)
    x = rng.standard_normal(n)
    y_ref = ref.cpu_coo(rows, cols, vals).spmv(x, n)
    y_orc = orc.coo_spmv(rows, cols, vals, x, n)
    assert bits_equal(y_ref, y_orc)


@pytest.mark.parametrize("grid,frac,seed", [((16, 16, 16), 0.01, 1), ((20, 12, 9), 0.02, 3), ((33, 8, 5), 0.0, 0)])
def test_workload_generator_restated(orc, grid, frac, seed):
    """The oracle's restated bench-workload generator (used by the reference
    arm of bench.py, which must not load the product library) builds exactly
    the product generator's matrix and x."""
    import hbdia_b200 as hb
    a = orc.workload_stencil27(*grid, 26.0, -1.0, frac, 0.1, 1.0, seed)
    b = hb.generate_stencil27(*grid, 26.0, -1.0, frac, 0.1, 1.0, seed)
    for u, v in zip(a, b):
        assert u.dtype == v.dtype and np.array_equal(u.view(np.uint8), v.view(np.uint8))
    n = grid[0] * grid[1] * grid[2]
    assert np.array_equal(orc.fill_uniform(n, -1.0, 1.0, seed).view(np.uint64),
                          hb.fill_uniform(n, -1.0, 1.0, seed).view(np.uint64))
