import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger inputs")


@pytest.fixture(scope="session")
def lib():
    """The product library, built in-tree if needed (no fallback)."""
    from hbdia_b200 import build as _build
    _build.build()
    import hbdia_b200
    hbdia_b200._lib.load()
    return hbdia_b200


@pytest.fixture(scope="session")
def orc():
    """The oracle (test infrastructure): the C restatement."""
    import oracle
    if not os.path.exists(oracle._ORACLE_SO):
        oracle.build()
    return oracle.Restated()


@pytest.fixture(scope="session")
def ref():
    """The reference's own code compiled by oracle/Makefile, when present."""
    import oracle
    if not oracle.Reference.available():
        oracle.build()  # builds oracle/_ref where the reference tree is present (oracle/Makefile)
        if not oracle.Reference.available():
            pytest.skip("oracle/_ref/libhbdia_ref.so not built on this machine")
    return oracle.Reference()


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def bits_equal(a: np.ndarray, b: np.ndarray) -> bool:
    """Bitwise equality of float arrays (distinguishes -0.0 / +0.0, NaN payloads)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    u = np.uint64 if a.dtype == np.float64 else np.uint32
    return bool(np.array_equal(a.view(u), b.view(u)))


def random_coo(rng, nr, nc, nnz, sort=True, zero_frac=0.05):
    rows = rng.integers(0, nr, nnz).astype(np.int32)
    cols = rng.integers(0, nc, nnz).astype(np.int32)
    if sort:
        o = np.argsort(rows, kind="stable")
        rows, cols = rows[o], cols[o]
    vals = rng.standard_normal(nnz)
    vals[rng.random(nnz) < zero_frac] = 0.0
    return rows, cols, vals
