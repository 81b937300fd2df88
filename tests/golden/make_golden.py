"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Runs only where the reference tree exists: it builds oracle/_ref from the
reference sources (oracle/Makefile) and records, for small fixed inputs, the
exact outputs of the reference's convertToHBDIAFormat
(src/Format/HBDIA.cpp:507-718), convertToDIAFormat and removeCOODuplicates
(src/Format/HBDIA.cpp:372-505), create3DStencil27Point
(src/Format/HBDIA.cpp:1416-1607) and cpu_coo_spmv_kernel
(src/Operations/HBDIASpMV.cpp:36-99).  With --gpu (on a CUDA machine) it also
records the reference's full hbdiaSpMV result (its blocked-DIA kernel,
src/Operations/HBDIASpMV.cu:7-74, recompiled for sm_100a, plus the CPU COO
path and vector_add) into spmv_reference_gpu.npz.

Inputs are either the reference's own test matrices (the print test's 3x3 and
20x20 examples, tests/run_HBDIA_print_test.cpp:12-104; the single-GPU example's
8^3 stencil, simple_hbdia_example.cpp:17-27) or seeded random matrices defined
here.

    python tests/golden/make_golden.py [--gpu]
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

LAYOUT_KEYS = ("offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
               "hist_blocks", "hist_nnz")


def print_test_3x3():
    rows = np.array([0, 0, 1, 1, 1, 2, 2], np.int32)
    cols = np.array([0, 2, 0, 1, 2, 1, 2], np.int32)
    vals = np.arange(1.0, 8.0)
    return rows, cols, vals


def print_test_20x20():
    """tests/run_HBDIA_print_test.cpp:55-92, entry order as built there."""
    r, c, v = [], [], []
    for i in range(20):
        r.append(i); c.append(i); v.append(5.0 + i * 0.1)
    for i in range(19):
        r.append(i); c.append(i + 1); v.append(2.0 + i * 0.05)
    for i in range(1, 20):
        r.append(i); c.append(i - 1); v.append(1.0 + i * 0.05)
    for i in range(0, 18, 3):
        r.append(i); c.append(i + 2); v.append(0.5 + i * 0.02)
    for a, b in ((2, 15), (5, 18), (10, 3), (15, 8), (18, 19)):
        r.append(a); c.append(b); v.append(0.3)
    return np.array(r, np.int32), np.array(c, np.int32), np.array(v)


def random_cases():
    rng = np.random.default_rng(20240601)
    cases = []
    specs = [
        # (numRows, numCols, nnz, sorted, bw, thr, max_coo)
        (50, 50, 300, True, 8, 2, 10 ** 9),
        (50, 50, 300, False, 8, 2, 10 ** 9),     # unsorted input
        (70, 40, 350, True, 16, 2, 10 ** 9),     # more rows than columns
        (40, 70, 350, True, 16, 2, 10 ** 9),     # more columns than rows
        (64, 64, 500, True, 32, 3, 5),           # max_coo cut-off
        (33, 33, 200, True, 32, 1, 10 ** 9),     # rows not a multiple of bw
        (45, 45, 260, True, 5, 2, 0),            # max_coo 0: everything kept
        (30, 30, 150, True, 4, -1, 10 ** 9),     # threshold <= 0
    ]
    for k, (nr, nc, nnz, srt, bw, thr, mc) in enumerate(specs):
        rows = rng.integers(0, nr, nnz).astype(np.int32)
        cols = rng.integers(0, nc, nnz).astype(np.int32)
        if srt:
            o = np.argsort(rows, kind="stable")
            rows, cols = rows[o], cols[o]
        vals = rng.standard_normal(nnz)
        vals[rng.random(nnz) < 0.05] = 0.0
        # duplicates of earlier entries with new values (last-wins in DIA)
        d = rng.integers(0, nnz, 20)
        rows = np.concatenate([rows, rows[d]])
        cols = np.concatenate([cols, cols[d]])
        vals = np.concatenate([vals, rng.standard_normal(20)])
        if srt:
            o = np.argsort(rows, kind="stable")
            rows, cols, vals = rows[o], cols[o], vals[o]
        cases.append((f"random{k}", rows, cols, vals, nr, nc, bw, thr, mc))
    return cases


def save_layout(path, rows, cols, vals, nr, nc, bw, thr, mc, L: oracle.Layout, **extra):
    np.savez_compressed(path, rows=rows, cols=cols, vals=vals,
                        params=np.array([nr, nc, bw, thr, mc], np.int64),
                        num_blocks=L.num_blocks, number_diagonals=L.number_diagonals,
                        has_hbdia=int(L.has_hbdia), **{k: getattr(L, k) for k in LAYOUT_KEYS}, **extra)


def dia_cases():
    """Inputs of the DIA fixtures: (rows, cols, vals, numRows, numCols,
    COOisUnique, removeCOODuplicates first)."""
    rng = np.random.default_rng(42)
    out = []
    r, c, v = print_test_3x3()
    out.append((r, c, v, 3, 3, False, False))
    for nr, nc, nnz in ((40, 30, 300), (30, 45, 260)):
        r = np.sort(rng.integers(0, nr, nnz)).astype(np.int32)
        c = rng.integers(0, nc, nnz).astype(np.int32)
        v = rng.standard_normal(nnz)
        dup = rng.integers(0, nnz, 40)  # repeated positions with other values
        r = np.concatenate([r, r[dup]])
        c = np.concatenate([c, c[dup]])
        v = np.concatenate([v, rng.standard_normal(40)])
        v[rng.random(len(v)) < 0.05] = -0.0
        out.append((r, c, v, nr, nc, False, False))
        out.append((r, c, v, nr, nc, True, False))   # duplicates kept: last one wins in DIA
        out.append((r, c, v, nr, nc, False, True))   # removeCOODuplicates, then the conversion
    return out


def save_dia(path, R):
    out = {}
    cases = dia_cases()
    r, c, v, nr, nc = R.stencil27(6, 6, 6, 0.05, 1)
    cases.append((r, c, v, nr, nc, False, False))
    for k, (r, c, v, nr, nc, uniq, first) in enumerate(cases):
        off, diag, (orr, occ, ovv), nnz = R.dia(r, c, v, nr, nc, coo_unique=uniq, remove_first=first)
        out.update({f"c{k}_rows": r, f"c{k}_cols": c, f"c{k}_vals": v,
                    f"c{k}_params": np.array([nr, nc, int(uniq), int(first), nnz], np.int64),
                    f"c{k}_offsets": off, f"c{k}_diag": diag, f"c{k}_out_rows": orr, f"c{k}_out_cols": occ,
                    f"c{k}_out_vals": ovv})
    np.savez_compressed(path, ncase=len(cases), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--dia-only", action="store_true", help="write dia_reference.npz only")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not oracle.Reference.available():
        oracle.build()
    R = oracle.Reference()
    # the reference's convertToDIAFormat / removeCOODuplicates (src/Format/HBDIA.cpp:372-505)
    save_dia(os.path.join(a.out, "dia_reference.npz"), R)
    if a.dia_only:
        print("golden fixtures written to", a.out)
        return

    r, c, v = print_test_3x3()
    save_layout(os.path.join(a.out, "print_test_3x3.npz"), r, c, v, 3, 3, 4, 2, 10 ** 9,
                R.convert(r, c, v, 3, 3, 4, 2))
    r, c, v = print_test_20x20()
    save_layout(os.path.join(a.out, "print_test_20x20.npz"), r, c, v, 20, 20, 8, 3, 10 ** 9,
                R.convert(r, c, v, 20, 20, 8, 3))
    # single-GPU example: create3DStencil27Point(8,8,8,0.0), convertToHBDIAFormat(32,2)
    r, c, v, nr, nc = R.stencil27(8, 8, 8, 0.0, 0)
    save_layout(os.path.join(a.out, "stencil8_example.npz"), r, c, v, nr, nc, 32, 2, 10 ** 9,
                R.convert(r, c, v, nr, nc, 32, 2))
    # the generator with noise (unstable sort inside rows, RNG draws)
    r, c, v, nr, nc = R.stencil27(6, 6, 6, 0.05, 1)
    save_layout(os.path.join(a.out, "stencil6_noise.npz"), r, c, v, nr, nc, 8, 2, 10 ** 9,
                R.convert(r, c, v, nr, nc, 8, 2), stencil_args=np.array([6, 6, 6, 1], np.int64),
                noise=0.05)
    for name, r, c, v, nr, nc, bw, thr, mc in random_cases():
        save_layout(os.path.join(a.out, f"{name}.npz"), r, c, v, nr, nc, bw, thr, mc,
                    R.convert(r, c, v, nr, nc, bw, thr, mc))
    # float32 conversion
    r, c, v = print_test_20x20()
    v32 = v.astype(np.float32)
    save_layout(os.path.join(a.out, "print_test_20x20_f32.npz"), r, c, v32, 20, 20, 8, 3, 10 ** 9,
                R.convert(r, c, v32, 20, 20, 8, 3))
    # the reference's CPU COO SpMV (cpu_coo_spmv_kernel) on the 6^3 noisy stencil
    r, c, v, nr, nc = R.stencil27(6, 6, 6, 0.05, 1)
    x = np.linspace(-1.0, 1.0, nr)
    y = R.cpu_coo(r, c, v).spmv(x, nr)
    np.savez_compressed(os.path.join(a.out, "cpu_coo_spmv.npz"), rows=r, cols=c, vals=v, x=x, y=y)

    if a.gpu:
        out = {}
        for k, (nx, bw, thr, xs) in enumerate(((8, 32, 2, "iota"), (12, 8, 2, "rand"), (16, 32, 3, "rand"))):
            r, c, v, nr, nc = R.stencil27(nx, nx, nx, 0.02, k)
            x = np.arange(1.0, nr + 1.0) if xs == "iota" else np.random.default_rng(k).uniform(-1, 1, nr)
            y = R.gpu_spmv(r, c, v, nr, nc, bw, thr, x, exec_cpu=True, exec_gpu=False)
            out.update({f"c{k}_rows": r, f"c{k}_cols": c, f"c{k}_vals": v, f"c{k}_x": x, f"c{k}_y": y,
                        f"c{k}_params": np.array([nr, nc, bw, thr], np.int64)})
        np.savez_compressed(os.path.join(a.out, "spmv_reference_gpu.npz"), ncase=3, **out)
    print("golden fixtures written to", a.out)


if __name__ == "__main__":
    main()
