"""DIA format (convertToDIAFormat, removeCOODuplicates) against the
reference's own outputs (tests/golden/dia_reference.npz, written by
tests/golden/make_golden.py from the reference's code, and the compiled
reference itself where it is built), and the storage-cost figures of the
reference's benchmark."""
import os

import numpy as np
import pytest

from conftest import bits_equal, random_coo

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "dia_reference.npz")


def _ours(lib, r, c, v, nr, nc, unique, first):
    m = lib.HBDIA(r, c, v, nr, nc)
    if first:
        m.removeCOODuplicates()
    m.convertToDIAFormat(COOisUnique=unique)
    return m


def _check(m, off, diag, out, nnz):
    assert m.isDIAFormat()
    assert np.array_equal(m.getOffsets(), off)
    d = m.getDiagonals()
    assert d.shape == diag.shape and bits_equal(d, diag)
    r, c, v = m.coo()
    assert np.array_equal(r, out[0]) and np.array_equal(c, out[1]) and bits_equal(v, out[2])
    assert m.getNumNonZeros() == nnz


def test_golden_dia(lib):
    g = np.load(GOLDEN)
    for k in range(int(g["ncase"])):
        nr, nc, uniq, first, nnz = (int(x) for x in g[f"c{k}_params"])
        m = _ours(lib, g[f"c{k}_rows"], g[f"c{k}_cols"], g[f"c{k}_vals"], nr, nc, bool(uniq), bool(first))
        _check(m, g[f"c{k}_offsets"], g[f"c{k}_diag"],
               (g[f"c{k}_out_rows"], g[f"c{k}_out_cols"], g[f"c{k}_out_vals"]), nnz)


@pytest.mark.parametrize("seed", range(6))
def test_dia_against_reference(lib, ref, seed):
    rng = np.random.default_rng(900 + seed)
    nr, nc = int(rng.integers(5, 80)), int(rng.integers(5, 80))
    r, c, v = random_coo(rng, nr, nc, int(rng.integers(1, 400)), sort=bool(seed % 2), zero_frac=0.1)
    dup = rng.integers(0, len(r), 10)
    r, c, v = np.concatenate([r, r[dup]]), np.concatenate([c, c[dup]]), np.concatenate([v, -v[dup]])
    for uniq in (False, True):
        off, diag, out, nnz = ref.dia(r, c, v, nr, nc, coo_unique=uniq)
        _check(_ours(lib, r, c, v, nr, nc, uniq, False), off, diag, out, nnz)


def test_dia_noops_and_then_hbdia(lib):
    e = lib.HBDIA(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0), 4, 4)
    e.convertToDIAFormat()
    assert e.isDIAFormat() and len(e.getOffsets()) == 0
    r = np.array([0, 1, 1, 1], np.int32)
    c = np.array([0, 1, 1, 0], np.int32)
    m = lib.HBDIA(r, c, np.array([1.0, 2.0, 3.0, 4.0]), 2, 2)
    m.convertToDIAFormat()
    assert m.getNumNonZeros() == 3  # duplicates consolidated, as the reference does
    m.convertToDIAFormat(COOisUnique=True)  # converted already: no-op
    assert m.getNumNonZeros() == 3
    m.convertToHBDIAFormat(32, 1, upload=False)  # the conversion sees the consolidated COO
    d = m.layout()["data"]  # offsets -1 then 0, 32 lanes each
    assert d[:2].tolist() == [0.0, 4.0] and d[32:34].tolist() == [1.0, 5.0]


def test_storage_costs(lib, orc):
    import oracle
    cases = []
    m = lib.HBDIA()
    m.create3DStencil27Point(8, 8, 8, 0.02, 0)  # records nnz per row (SELL)
    m.convertToHBDIAFormat(32, 1, upload=False)
    cases.append(m)
    rng = np.random.default_rng(3)
    r, c, v = random_coo(rng, 300, 200, 3000)
    m2 = lib.HBDIA(r, c, v, 300, 200)
    m2.convertToHBDIAFormat(16, 2, upload=False)
    cases.append(m2)
    for m in cases:
        i = m.info()
        lay = m.layout()
        npr = np.zeros(i.numRows, np.int32)
        lib._lib.load().hbdia_matrix_export_nnz_per_row(m.handle, npr.ctypes.data)
        if m is cases[1]:
            npr = np.zeros(0, np.int32)  # only the stencil generator records them
        want = oracle.storage_costs(8, i.numRows, i.numCols, i.numNonZeros, i.numberDiagonals, i.numBlocks,
                                    i.blockWidth, i.numSlots, i.numCoo, lay["hist_blocks"], npr)
        assert m.storageCosts() == want
    # by hand: the reference print test's 3x3 matrix, blockWidth 4, threshold 2
    r = np.array([0, 0, 1, 1, 1, 2, 2], np.int32)
    c = np.array([0, 2, 0, 1, 2, 1, 2], np.int32)
    m3 = lib.HBDIA(r, c, np.arange(1.0, 8.0), 3, 3)
    m3.convertToHBDIAFormat(4, 2, upload=False)
    i = m3.info()
    # values + block pointer + one int per stored offset + COO (row, col, value)
    hb = i.numSlots * 8 + (i.numBlocks + 1) * 4 + i.totalOffsets * 4 + i.numCoo * (4 + 4 + 8)
    assert m3.storageCosts() == {
        "hbdia": hb, "coo": 7 * (4 + 4 + 8), "dia": i.numberDiagonals * (3 * 8 + 4),
        "sell": 4,  # no per-row counts: only the slice pointer
        "csr": 7 * (8 + 4) + (3 + 1) * 4}


def test_storage_report_csv(lib, tmp_path):
    m = lib.HBDIA()
    m.create3DStencil27Point(6, 6, 6, 0.0, 0)
    m.convertToHBDIAFormat(32, 2, upload=False)
    lib.write_storage_report(m, str(tmp_path), "3D27Stencil", 6, 6, 6, 0.0)
    import csv
    with open(tmp_path / "matrix_info.csv") as f:
        rows = list(csv.reader(f))
    assert rows[0][:5] == ["name", "nx", "ny", "nz", "noise"] and len(rows[0]) == 30
    info = dict(zip(rows[0], rows[1]))
    assert int(info["coo_cost_bytes"]) == m.storageCosts()["coo"]
    with open(tmp_path / "histogram.csv") as f:
        h = list(csv.reader(f))
    assert h[0] == ["diagonal_count", "blocks_with_diagonals", "nnz_in_blocks"] and len(h) > 1
