"""The library's host converter and drop-in API (no GPU): bit-exact layout
against the golden fixtures and the oracle, the reference's error behaviour,
and the reference's matrix sources (stencil generator, Matrix Market)."""
import glob
import os

import numpy as np
import pytest

from conftest import bits_equal, random_coo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr", "hist_blocks",
        "hist_nnz")


def _layout_equal(L, other, get=lambda o, k: o[k]):
    for k in KEYS:
        a, b = L[k], get(other, k)
        if a.shape != b.shape or not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
            return k
    return None


@pytest.mark.parametrize("path", sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                                        if os.path.basename(p) not in ("cpu_coo_spmv.npz",
                                                                       "spmv_reference_gpu.npz",
                                                                       "dia_reference.npz")),
                         ids=os.path.basename)
def test_library_converter_matches_golden(lib, path):
    d = np.load(path)
    nr, nc, bw, thr, mc = [int(v) for v in d["params"]]
    m = lib.HBDIA(d["rows"], d["cols"], d["vals"], nr, nc, dtype=d["vals"].dtype)
    m.convertToHBDIAFormat(bw, thr, mc, upload=False)
    L = m.layout()
    assert L["num_blocks"] == int(d["num_blocks"])
    assert L["number_diagonals"] == int(d["number_diagonals"])
    assert _layout_equal(L, d) is None
    assert m.getNumBlocks() == int(d["num_blocks"])
    assert m.getOffsetsPerBlock() == [d["offsets"][d["block_start"][b]:d["block_start"][b + 1]].tolist()
                                      for b in range(int(d["num_blocks"]))]


def test_library_vs_oracle_random(lib, orc):
    rng = np.random.default_rng(5)
    for trial in range(150):
        nr = int(rng.integers(1, 150))
        nc = int(rng.integers(1, 150)) if trial % 3 == 0 else nr
        rows, cols, vals = random_coo(rng, nr, nc, int(rng.integers(1, 900)), sort=trial % 2 == 0)
        bw = int(rng.choice([1, 2, 3, 4, 7, 8, 16, 32, 64, 128]))
        thr = int(rng.integers(-1, 6))
        mc = int(rng.choice([0, 1, 3, 10, 10 ** 9]))
        for dt in (np.float64, np.float32):
            m = lib.HBDIA(rows, cols, vals.astype(dt), nr, nc, dtype=dt)
            m.convertToHBDIAFormat(bw, thr, mc, upload=False)
            L = m.layout()
            o = orc.convert(rows, cols, vals.astype(dt), nr, nc, bw, thr, mc).layout()
            assert L["number_diagonals"] == o.number_diagonals
            assert _layout_equal(L, o, get=getattr) is None, trial


def test_config1_layout_matches_oracle(lib, orc):
    """64^3 stencil + 0.5% extras (seed 0), bw 32, thr 2: the benchmark-config
    layout is bit-exact and has the expected shape."""
    n = 64 ** 3
    rows, cols, vals = lib.generate_stencil27(64, 64, 64, 26.0, -1.0, 0.005, 0.1, 1.0, 0)
    assert len(vals) == 6_859_000 + int(0.005 * 6_859_000)
    m = lib.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    L = m.layout()
    o = orc.convert(rows, cols, vals, n, n, 32, 2).layout()
    assert _layout_equal(L, o, get=getattr) is None
    assert L["num_blocks"] == 8192
    assert len(L["offsets"]) >= 216_600          # 7688*27 + 496*18 + 8*12 from the stencil
    assert len(L["coo_row"]) > 0.99 * int(0.005 * 6_859_000)


def test_reference_generator_golden(lib):
    for name, args in (("stencil8_example.npz", (8, 8, 8, 0.0, 0)), ("stencil6_noise.npz", (6, 6, 6, 0.05, 1))):
        d = np.load(os.path.join(GOLDEN, name))
        m = lib.HBDIA()
        m.create3DStencil27Point(*args)
        assert np.array_equal(m.getRowIndices(), d["rows"])
        assert np.array_equal(m.getColIndices(), d["cols"])
        assert bits_equal(m.getValues(), d["vals"])
        assert m.getNumRows() == m.getNumCols() == args[0] * args[1] * args[2]


def test_reference_generator_vs_reference(lib, ref):
    for args in ((5, 5, 5, 0.3, 2), (4, 6, 4, 0.1, 0), (10, 10, 10, 0.01, 3)):
        r, c, v, nr, nc = ref.stencil27(*args)
        m = lib.HBDIA()
        m.create3DStencil27Point(*args)
        assert np.array_equal(m.getRowIndices(), r) and np.array_equal(m.getColIndices(), c)
        assert bits_equal(m.getValues(), v) and m.getNumRows() == nr
        assert np.array_equal(m.getNnzPerRow(), np.bincount(r, minlength=nr))


def test_reference_generator_rejects_out_of_range_grids(lib):
    # nx != nz makes the reference's generator index outside the matrix
    with pytest.raises(NotImplementedError, match="nx == nz"):
        lib.HBDIA().create3DStencil27Point(4, 6, 3, 0.1, 0)


def _write_mtx(path, header, entries, dims, symmetric=False, pattern=False):
    with open(path, "w") as f:
        kind = "pattern" if pattern else "real"
        f.write(f"%%MatrixMarket matrix coordinate {kind} {'symmetric' if symmetric else 'general'}\n")
        f.write("% generated test matrix\n")
        f.write(f"{dims[0]} {dims[1]} {len(entries)}\n")
        for e in entries:
            f.write(" ".join(str(t) for t in e) + "\n")


def test_load_mtx_matches_reference(lib, ref, tmp_path):
    rng = np.random.default_rng(9)
    for k, (sym, pat) in enumerate(((False, False), (True, False), (False, True))):
        n = 40
        ents = []
        for _ in range(150):
            i, j = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
            if sym and j > i:
                i, j = j, i
            ents.append((i, j) if pat else (i, j, float(np.round(rng.standard_normal(), 6))))
        p = str(tmp_path / f"m{k}.mtx")
        _write_mtx(p, None, ents, (n, n), symmetric=sym, pattern=pat)
        ok, r, c, v, nr, nc = ref.load_mtx(p)
        m = lib.HBDIA()
        assert m.loadMTX(p) == ok
        assert np.array_equal(m.getRowIndices(), r) and np.array_equal(m.getColIndices(), c)
        assert bits_equal(m.getValues(), v)
        assert (m.getNumRows(), m.getNumCols()) == (nr, nc)
    m = lib.HBDIA()
    assert m.loadMTX(str(tmp_path / "missing.mtx")) is False


def test_load_mtx_sized_out_of_range(lib, tmp_path):
    p = str(tmp_path / "s.mtx")
    _write_mtx(p, None, [(1, 1, 2.0), (5, 2, 1.0)], (5, 5))
    m = lib.HBDIA()
    assert m.loadMTX(p, 10, 10) is True
    assert m.getNumRows() == 10
    with pytest.raises(IndexError, match="out of range"):
        lib.HBDIA().loadMTX(p, 4, 4)


def test_constructor_errors(lib):
    # src/Format/HBDIA.cpp:58-79
    with pytest.raises(ValueError, match="same size"):
        lib.HBDIA([0, 1], [0], [1.0, 2.0], 2, 2)
    with pytest.raises(ValueError, match="positive"):
        lib.HBDIA([0], [0], [1.0], 0, 2)
    with pytest.raises(IndexError, match="Row index 5 is out of range"):
        lib.HBDIA([5], [0], [1.0], 3, 3)
    with pytest.raises(IndexError, match="Column index 3 is out of range"):
        lib.HBDIA([0], [3], [1.0], 3, 3)
    # dims-inferring constructor (src/Format/HBDIA.cpp:23-49)
    m = lib.HBDIA([0, 4], [7, 1], [1.0, 2.0])
    assert (m.getNumRows(), m.getNumCols()) == (5, 8)


def test_convert_noops_and_guards(lib):
    # empty matrix: the reference returns without converting (HBDIA.cpp:521-524)
    m = lib.HBDIA(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0), 4, 4)
    m.convertToHBDIAFormat(4, 1, upload=False)
    assert not m.isHBDIAFormat()
    # second conversion is a no-op (HBDIA.cpp:511-514)
    m = lib.HBDIA([0, 1, 2], [0, 1, 2], [1.0, 2.0, 3.0], 3, 3)
    m.convertToHBDIAFormat(2, 1, upload=False)
    first = m.layout()
    m.convertToHBDIAFormat(1, 5, upload=False)
    assert m.getBlockWidth() == 2 and _layout_equal(m.layout(), first) is None
    with pytest.raises(ValueError):
        lib.HBDIA([0], [0], [1.0], 1, 1).convertToHBDIAFormat(0, 1, upload=False)


def test_workload_generators(lib):
    r, c, v = lib.generate_stencil27(4, 5, 6)
    assert len(v) == (3 * 4 - 2) * (3 * 5 - 2) * (3 * 6 - 2)
    assert np.all(np.diff(r) >= 0)
    n = 4 * 5 * 6
    d = {(a, b): x for a, b, x in zip(r, c, v)}
    assert len(d) == len(v)
    assert all(d[(i, i)] == 26.0 for i in range(n))
    r2, c2, v2 = lib.generate_stencil27(16, 16, 16, 26.0, -1.0, 0.01, 0.1, 1.0, 7)
    extras = len(v2) - (46 ** 3)
    assert extras == int(0.01 * 46 ** 3)
    ext = v2[v2 > 0][v2[v2 > 0] != 26.0]
    assert np.all((ext >= 0.1) & (ext < 1.0))
    assert len(set(zip(r2.tolist(), c2.tolist()))) == len(v2)      # no repeats
    # deterministic
    r3, c3, v3 = lib.generate_stencil27(16, 16, 16, 26.0, -1.0, 0.01, 0.1, 1.0, 7)
    assert np.array_equal(c2, c3) and bits_equal(v2, v3)
    r7, c7, v7 = lib.generate_stencil7(3, 3, 3)
    assert len(v7) == 27 + 2 * 3 * (2 * 9)
    rb, cb, vb = lib.generate_banded(5000, [0, 1, -1, 2, -2, 64, -64, 4096, -4096], 0.5, 1.5, 0.3, 0.002, 2)
    assert np.all(np.diff(rb) >= 0)
    diag = vb[rb == cb]
    assert len(diag) == 5000 and np.all(diag >= 1.0)
    x = lib.fill_uniform(1000, -1.0, 1.0, 1)
    assert np.all((x >= -1) & (x < 1)) and bits_equal(x, lib.fill_uniform(1000, -1.0, 1.0, 1))
