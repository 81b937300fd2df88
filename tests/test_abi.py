"""The C ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(hbdia_[a-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"hbdia_matrix_create", "hbdia_matrix_convert", "hbdia_spmv", "hbdia_vector_create",
            "hbdia_spmv_device", "hbdia_spmv_host"} <= names


def test_library_exports_every_declared_symbol(lib):
    so = ctypes.CDLL(lib.library_path())
    missing = [n for n in sorted(declared_functions()) if not hasattr(so, n)]
    assert not missing, missing


def test_python_binding_covers_header(lib):
    from hbdia_b200 import _lib
    assert declared_functions() <= set(_lib.EXPORTED)


def test_status_strings_and_errors_without_gpu(lib):
    so = lib._lib.load()
    assert so.hbdia_status_string(-3) == b"HBDIA_ERR_RUNTIME"
    assert so.hbdia_version().startswith(b"hbdia_b200")
    # a failing call sets a message and returns a code (no exit, no exception)
    h = ctypes.c_void_p()
    rc = so.hbdia_matrix_create(0, None, None, None, 1, 4, 4, ctypes.byref(h))
    assert rc == -1 and b"null" in so.hbdia_last_error()


def test_server_option_validation_without_gpu(lib):
    """Server options are checked before any CUDA call: SpMV batches are SpMMs,
    so the quad-interleaved storages (SpMV only) are refused for them; an
    unknown CG iteration storage is refused too."""
    import pytest
    for bad in ({"spmvStorage": lib.STORE_F32_QUAD}, {"spmvStorage": lib.STORE_BF16_QUAD},
                {"cgIterStorage": 5}, {"cgIterStorage": -1}, {"cgMaxGroup": 17}):
        with pytest.raises(ValueError):
            lib.Server(**bad)
    o = lib._lib.ServerOptions()
    lib._lib.load().hbdia_server_default_options(ctypes.byref(o))
    assert o.spmvStorage == lib.STORE_F32 and o.cgIterStorage == lib.STORE_F32_QUAD and o.cgMaxGroup == 1
