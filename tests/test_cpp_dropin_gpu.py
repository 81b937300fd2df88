"""The C++ drop-in API (include/hbdia/, in the shape of the reference's
include/) used the way the reference's own programs use theirs.

* tests/cpp/test_dropin.cpp: this repository's checks of every drop-in member.
* The reference's own callers, compiled unchanged where they lie against the
  drop-in by oracle/Makefile's `dropin` target (prebuilt under oracle/_ref/dropin,
  which needs the reference tree at build time): benchmarking/benchHBDIA.cpp
  driven by tests/cpp/bench_hbdia_main.cpp, and the single-GPU main of
  tests/run_HBDIA_cusparse_comparison.cpp, whose own check compares the
  fused SpMV with cuSPARSE (its reference implementation) at 1e-6.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def _prebuilt(name):
    p = os.path.join(DROPIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (oracle/_ref/dropin is built where the reference tree is present)")
    return p


def test_cpp_dropin_program(lib):
    from hbdia_b200 import build
    exe = build.build_cpp_tests()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout


def test_reference_benchhbdia_unchanged(lib, orc, tmp_path):
    """benchmarking/benchHBDIA.cpp (the reference's) on the drop-in: both of
    its vector modes give the reference arithmetic's y bit for bit, and that y
    equals the oracle's restated HBDIA SpMV of the same matrix."""
    import hbdia_b200 as hb
    exe = _prebuilt("bench_hbdia")
    out = tmp_path / "y.bin"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout
    y = np.fromfile(out, dtype=np.float64)
    m = hb.HBDIA(dtype=np.float64)
    m.create3DStencil27Point(32, 32, 32, 0.01, 0)
    rows, cols, vals = m.getRowIndices(), m.getColIndices(), m.getValues()
    n = 32 ** 3
    x = np.arange(1, n + 1, dtype=np.float64)
    yref = orc.convert(rows, cols, vals, n, n, 32, 2).spmv(x)
    assert np.array_equal(y.view(np.uint64), yref.view(np.uint64))


def test_reference_cusparse_comparison_unchanged(lib):
    """The single-GPU main of tests/run_HBDIA_cusparse_comparison.cpp (the
    reference's): 128^3 stencil, 20 drop-in SpMVs, its cuSPARSE COO SpMV as
    the reference result, its own 1e-6 accuracy verdict."""
    exe = _prebuilt("cusparse_comparison")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    print(r.stdout[-2000:])
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr
    assert "ACCURACY TEST PASSED" in r.stdout
    assert "Error count:   0/" in r.stdout
