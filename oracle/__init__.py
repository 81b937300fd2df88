"""Test infrastructure only: the ORACLE for the HBDIA hot path.

Two checkers live here, both CPU-only:

* ``restated`` -- ``hbdia_oracle.c``, a plain-C restatement of the reference's
  ``convertToHBDIAFormat`` (src/Format/HBDIA.cpp:507-718) and ``hbdiaSpMV``
  arithmetic (src/Operations/HBDIASpMV.cu:7-88, src/Operations/HBDIASpMV.cpp:36-99).
* ``reference`` -- the reference's own sources compiled by ``oracle/Makefile``
  into ``oracle/_ref/libhbdia_ref.so`` (present whenever it was built where the
  reference tree exists; the built file travels with the repository snapshot).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU baseline
and its ``--impl reference`` arm) import this package, and only to check or to
time the CPU baseline.  The product package ``hbdia_b200`` never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "_build", "libhbdia_oracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libhbdia_ref.so")

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p


def build(quiet: bool = True) -> None:
    """Compile both oracles (the reference part only where its tree exists)."""
    out = subprocess.run(["make", "-C", _HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


@dataclass
class Layout:
    """The HBDIA host layout, field for field what the reference's getters
    return (src/Format/HBDIA.hpp:88-114), with offsetsPerBlock flattened into
    ``offsets`` + ``block_start`` (the form of prepareForGPU,
    src/Format/HBDIA.cpp:733-760)."""

    has_hbdia: bool
    num_rows: int
    num_cols: int
    num_blocks: int
    offsets: np.ndarray        # int32[total kept offsets]
    block_start: np.ndarray    # int32[num_blocks + 1]
    data: np.ndarray           # T[slots]
    coo_row: np.ndarray        # int32[nCoo]
    coo_col: np.ndarray        # int32[nCoo]
    coo_val: np.ndarray        # T[nCoo]
    coo_row_ptr: np.ndarray    # int32[numRows + 1]
    number_diagonals: int
    hist_blocks: np.ndarray
    hist_nnz: np.ndarray

    def offsets_per_block(self):
        bs = self.block_start
        return [self.offsets[bs[b]:bs[b + 1]].tolist() for b in range(self.num_blocks)]


def _alloc_layout(sizes, dtype):
    nb, tot, slots, nc, nd, hl, has, nr, ncol, rpl = [int(s) for s in sizes]
    return dict(
        nb=nb, nd=nd, has=bool(has), nr=nr, ncol=ncol,
        offsets=np.zeros(max(tot, 0), np.int32),
        block_start=np.zeros(nb + 1 if has else 0, np.int32),
        data=np.zeros(slots, dtype),
        coo_row=np.zeros(nc, np.int32), coo_col=np.zeros(nc, np.int32),
        coo_val=np.zeros(nc, dtype), coo_row_ptr=np.zeros(rpl, np.int32),
        hist_blocks=np.zeros(hl, np.int32), hist_nnz=np.zeros(hl, np.int32),
    )


def _to_layout(a) -> Layout:
    return Layout(a["has"], a["nr"], a["ncol"], a["nb"] if a["has"] else 0, a["offsets"],
                  a["block_start"], a["data"], a["coo_row"], a["coo_col"], a["coo_val"],
                  a["coo_row_ptr"], a["nd"], a["hist_blocks"], a["hist_nnz"])


# --------------------------------------------------------------------------- restated
class Restated:
    """ctypes front of oracle/hbdia_oracle.c."""

    def __init__(self, path: str = _ORACLE_SO):
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.orc_convert.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int64, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int64, ctypes.POINTER(_vp)]
        lib.orc_convert.restype = ctypes.c_int
        lib.orc_convert_partial.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int64, ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int64, ctypes.POINTER(_vp)]
        lib.orc_convert_partial.restype = ctypes.c_int
        lib.orc_spmv_partial_f64.argtypes = [_vp, ctypes.c_int32, _vp, _vp]
        lib.orc_sizes.argtypes = [_vp, _i64p]
        lib.orc_export.argtypes = [_vp] * 10
        lib.orc_destroy.argtypes = [_vp]
        lib.orc_spmv_f64.argtypes = [_vp, _vp, _vp]
        lib.orc_spmv_f32.argtypes = [_vp, _vp, _vp]
        lib.orc_spmv_f64_values.argtypes = [_vp, _vp, _vp, _vp]
        lib.orc_coo_spmv_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int64, _vp, ctypes.c_int32, _vp]
        lib.orc_fill_uniform.argtypes = [_vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_uint64]
        lib.orc_workload_stencil27.argtypes = [ctypes.c_int32] * 3 + [ctypes.c_double] * 5 + [ctypes.c_uint64, _i64p,
                                                                                               _vp, _vp, _vp]
        lib.orc_workload_stencil27.restype = ctypes.c_int
        self.lib = lib

    def fill_uniform(self, n, lo, hi, seed):
        """x[i] = lo + (hi - lo) * U[0, 1), MT19937-64(seed): the bench's x."""
        out = np.empty(n, np.float64)
        self.lib.orc_fill_uniform(_ptr(out), n, lo, hi, seed)
        return out

    def workload_stencil27(self, nx, ny, nz, center, neighbor, frac, lo, hi, seed):
        """The bench's 27-point stencil with extra off-pattern entries
        (rows, cols, vals), built by the oracle's own restatement."""
        nnz = ctypes.c_int64()
        if self.lib.orc_workload_stencil27(nx, ny, nz, center, neighbor, frac, lo, hi, seed, ctypes.byref(nnz),
                                           None, None, None) != 0:
            raise ValueError("bad stencil arguments")
        rows = np.empty(nnz.value, np.int32)
        cols = np.empty(nnz.value, np.int32)
        vals = np.empty(nnz.value, np.float64)
        if self.lib.orc_workload_stencil27(nx, ny, nz, center, neighbor, frac, lo, hi, seed, ctypes.byref(nnz),
                                           _ptr(rows), _ptr(cols), _ptr(vals)) != 0:
            raise MemoryError("stencil workload")
        return rows, cols, vals

    def convert(self, rows, cols, vals, num_rows, num_cols, bw=32, thr=1, max_coo=1_000_000_000):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals)
        assert vals.dtype in (np.float64, np.float32)
        h = _vp()
        rc = self.lib.orc_convert(_ptr(rows), _ptr(cols), _ptr(vals), int(vals.dtype == np.float32),
                                  len(vals), num_rows, num_cols, bw, thr, max_coo, ctypes.byref(h))
        if rc != 0:
            if h:
                self.lib.orc_destroy(h)
            raise RuntimeError(f"orc_convert failed with {rc}")
        return _OracleMatrix(self, h, vals.dtype)

    def convert_partial(self, rows, cols, vals, num_rows, num_cols, row_base, bw=32, thr=1,
                        max_coo=1_000_000_000):
        """A partial matrix (local rows, global columns, global row = row_base +
        local row) converted as the reference's partial-matrix constructor
        does (offsets col - globalRow)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        h = _vp()
        rc = self.lib.orc_convert_partial(_ptr(rows), _ptr(cols), _ptr(vals), 0, len(vals), num_rows, num_cols,
                                          row_base, bw, thr, max_coo, ctypes.byref(h))
        if rc != 0:
            if h:
                self.lib.orc_destroy(h)
            raise RuntimeError(f"orc_convert_partial failed with {rc}")
        m = _OracleMatrix(self, h, np.float64)
        m.num_rows = num_rows
        return m

    def coo_spmv(self, rows, cols, vals, x, num_rows, y=None):
        y = np.zeros(num_rows, np.float64) if y is None else y
        self.lib.orc_coo_spmv_f64(_ptr(rows), _ptr(cols), _ptr(vals), len(vals), _ptr(x), num_rows, _ptr(y))
        return y


class _OracleMatrix:
    def __init__(self, owner: Restated, h, dtype):
        self._o, self._h, self.dtype = owner, h, np.dtype(dtype)

    def __del__(self):
        if getattr(self, "_h", None):
            self._o.lib.orc_destroy(self._h)
            self._h = None

    def layout(self) -> Layout:
        sizes = np.zeros(10, np.int64)
        self._o.lib.orc_sizes(self._h, sizes.ctypes.data_as(_i64p))
        a = _alloc_layout(sizes, self.dtype)
        self._o.lib.orc_export(self._h, *[_ptr(a[k]) for k in (
            "offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
            "hist_blocks", "hist_nnz")])
        return _to_layout(a)

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, self.dtype)
        y = np.zeros_like(x)
        f = self._o.lib.orc_spmv_f32 if self.dtype == np.float32 else self._o.lib.orc_spmv_f64
        f(self._h, _ptr(x), _ptr(y))
        return y

    def spmv_partial(self, x_global: np.ndarray) -> np.ndarray:
        """A partial matrix's rows of y over the global x."""
        x = np.ascontiguousarray(x_global, np.float64)
        y = np.zeros(self.num_rows, np.float64)
        self._o.lib.orc_spmv_partial_f64(self._h, len(x), _ptr(x), _ptr(y))
        return y

    def spmv_with_values(self, values: np.ndarray, x: np.ndarray) -> np.ndarray:
        """Double SpMV with the blocked-DIA values replaced (reduced-precision storage)."""
        values = np.ascontiguousarray(values, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        self._o.lib.orc_spmv_f64_values(self._h, _ptr(values), _ptr(y), _ptr(x))
        return y


def bf16_block_scaled(data: np.ndarray, block_start: np.ndarray, bw: int) -> np.ndarray:
    """Values as stored with bfloat16 + one float scale per block, widened
    back to double: scale = float(max |v| of the block) (1 if all zero),
    q = bf16_round_nearest_even(float(v / scale)), value = double(q) * scale."""
    out = np.empty_like(data)
    for b in range(len(block_start) - 1):
        s0, s1 = int(block_start[b]) * bw, int(block_start[b + 1]) * bw
        if s1 == s0:
            continue
        v = data[s0:s1]
        m = float(np.max(np.abs(v)))
        s = np.float32(m) if m > 0 else np.float32(1.0)
        q = (v / np.float64(s)).astype(np.float32)
        bits = q.view(np.uint32).astype(np.uint64)
        bits = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16
        f = bits.astype(np.uint32).view(np.float32)
        out[s0:s1] = f.astype(np.float64) * np.float64(s)
    return out


# --------------------------------------------------------------------------- reference
class Reference:
    """ctypes front of oracle/_ref/libhbdia_ref.so (the reference's own code)."""

    def __init__(self, path: str = _REF_SO):
        lib = ctypes.CDLL(path)
        for t, ct in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(lib, f"ref_matrix_create_{t}")
            f.argtypes = [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            f.restype = _vp
            f = getattr(lib, f"ref_matrix_convert_{t}")
            f.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            f.restype = ctypes.c_int
            getattr(lib, f"ref_matrix_sizes_{t}").argtypes = [_vp, _i64p]
            getattr(lib, f"ref_matrix_export_{t}").argtypes = [_vp] * 10
            getattr(lib, f"ref_matrix_destroy_{t}").argtypes = [_vp]
            f = getattr(lib, f"ref_cpu_coo_create_{t}")
            f.argtypes = [_vp, _vp, _vp, ctypes.c_int64]
            f.restype = _vp
            getattr(lib, f"ref_cpu_coo_spmv_{t}").argtypes = [_vp, _vp, ctypes.c_int, _vp]
            getattr(lib, f"ref_cpu_coo_destroy_{t}").argtypes = [_vp]
        lib.ref_matrix_remove_dups_f64.argtypes = [_vp]
        lib.ref_matrix_convert_dia_f64.argtypes = [_vp, ctypes.c_int]
        lib.ref_matrix_dia_sizes_f64.argtypes = [_vp, _vp]
        lib.ref_matrix_export_dia_f64.argtypes = [_vp] * 6
        lib.ref_gpu_matrix_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int64] + [ctypes.c_int] * 4
        lib.ref_gpu_matrix_f64.restype = _vp
        lib.ref_gpu_matrix_arrays_f64.argtypes = [_vp, _i64p, _vp]
        lib.ref_gpu_matrix_spmv_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int]
        lib.ref_gpu_matrix_spmv_f64.restype = ctypes.c_int
        lib.ref_partition_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int64] + [ctypes.c_int] * 5
        lib.ref_partition_f64.restype = _vp
        lib.ref_partition_sizes.argtypes = [_vp, _i64p]
        lib.ref_partition_export.argtypes = [_vp] * 6
        lib.ref_partition_matrix.argtypes = [_vp]
        lib.ref_partition_matrix.restype = _vp
        lib.ref_partition_destroy.argtypes = [_vp]
        lib.ref_coo_sizes_f64.argtypes = [_vp, _i64p]
        lib.ref_coo_export_f64.argtypes = [_vp, _vp, _vp, _vp]
        lib.ref_stencil27_f64.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_int]
        lib.ref_stencil27_f64.restype = _vp
        lib.ref_load_mtx_f64.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        lib.ref_load_mtx_f64.restype = _vp
        lib.ref_omp_max_threads.restype = ctypes.c_int
        lib.ref_omp_set_threads.argtypes = [ctypes.c_int]
        lib.ref_gpu_spmv_f64.argtypes = [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int]
        lib.ref_gpu_spmv_f64.restype = ctypes.c_int
        self.lib = lib

    @staticmethod
    def available(path: str = _REF_SO) -> bool:
        return os.path.exists(path)

    def dia(self, rows, cols, vals, num_rows, num_cols, coo_unique=False, remove_first=False):
        """The reference's convertToDIAFormat on a float64 matrix: (offsets,
        diagonals [numDiagonals, length], (rows, cols, vals) of its COO after
        the call, numNonZeros)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        h = self.lib.ref_matrix_create_f64(_ptr(rows), _ptr(cols), _ptr(vals), len(vals), num_rows, num_cols, 1)
        if not h:
            raise ValueError("reference constructor rejected the input")
        try:
            if remove_first:
                self.lib.ref_matrix_remove_dups_f64(h)
            self.lib.ref_matrix_convert_dia_f64(h, int(bool(coo_unique)))
            s = np.zeros(5, np.int64)
            self.lib.ref_matrix_dia_sizes_f64(h, _ptr(s))
            nd, ln, nnz, ncoo = int(s[0]), int(s[1]), int(s[2]), int(s[3])
            off = np.zeros(nd, np.int32)
            diag = np.zeros((nd, ln), np.float64)
            r, c, v = np.zeros(ncoo, np.int32), np.zeros(ncoo, np.int32), np.zeros(ncoo, np.float64)
            self.lib.ref_matrix_export_dia_f64(h, _ptr(off), _ptr(diag), _ptr(r), _ptr(c), _ptr(v))
            return off, diag, (r, c, v), nnz
        finally:
            self.lib.ref_matrix_destroy_f64(h)

    # convertToHBDIAFormat through the partial-matrix constructor (no GPU needed)
    def convert(self, rows, cols, vals, num_rows, num_cols, bw=32, thr=1, max_coo=1_000_000_000,
                coo_unique=False) -> Layout:
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals)
        t = "f32" if vals.dtype == np.float32 else "f64"
        h = getattr(self.lib, f"ref_matrix_create_{t}")(_ptr(rows), _ptr(cols), _ptr(vals), len(vals),
                                                        num_rows, num_cols, 1)
        if not h:
            raise ValueError("reference constructor rejected the input")
        try:
            max_coo = int(min(max_coo, 2**31 - 1))
            getattr(self.lib, f"ref_matrix_convert_{t}")(h, bw, thr, max_coo, int(coo_unique))
            sizes = np.zeros(10, np.int64)
            getattr(self.lib, f"ref_matrix_sizes_{t}")(h, sizes.ctypes.data_as(_i64p))
            a = _alloc_layout(sizes, vals.dtype)
            if a["has"]:
                getattr(self.lib, f"ref_matrix_export_{t}")(h, *[_ptr(a[k]) for k in (
                    "offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
                    "hist_blocks", "hist_nnz")])
            return _to_layout(a)
        finally:
            getattr(self.lib, f"ref_matrix_destroy_{t}")(h)

    def gpu_matrix(self, rows, cols, vals, num_rows, num_cols, bw, thr) -> "_RefGpuMatrix":
        """A float64 matrix converted by the reference on the GPU (its
        prepareForGPU device arrays stay alive with the returned object)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        h = self.lib.ref_gpu_matrix_f64(_ptr(rows), _ptr(cols), _ptr(vals), len(vals), num_rows, num_cols, bw, thr)
        if not h:
            raise RuntimeError("reference conversion failed")
        return _RefGpuMatrix(self, h, num_rows)

    def partition(self, rows, cols, vals, n, num_processes, part, bw=32, thr=1) -> dict:
        """One rank's side of BasicDistributor::scatterMatrix / receiveMatrix
        run on the reference's own code: its partition (local COO, first
        global row), the partial matrix's HBDIA layout, dataRanges,
        processDataRanges (triples process, start, end) and totalBufferSize."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        h = self.lib.ref_partition_f64(_ptr(rows), _ptr(cols), _ptr(vals), len(vals), n, num_processes, part,
                                       bw, thr)
        if not h:
            raise ValueError("reference partitioning failed")
        try:
            s = np.zeros(6, np.int64)
            self.lib.ref_partition_sizes(h, s.ctypes.data_as(_i64p))
            nnz, nd, npr = int(s[2]), int(s[3]), int(s[4])
            r, c, v = np.zeros(nnz, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz, np.float64)
            data = np.zeros((nd, 2), np.int32)
            proc = np.zeros((npr, 3), np.int32)
            self.lib.ref_partition_export(h, _ptr(r), _ptr(c), _ptr(v), _ptr(data), _ptr(proc))
            m = self.lib.ref_partition_matrix(h)
            sizes = np.zeros(10, np.int64)
            self.lib.ref_matrix_sizes_f64(m, sizes.ctypes.data_as(_i64p))
            a = _alloc_layout(sizes, np.float64)
            if a["has"]:
                self.lib.ref_matrix_export_f64(m, *[_ptr(a[k]) for k in (
                    "offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
                    "hist_blocks", "hist_nnz")])
            return {"row_start": int(s[0]), "num_local_rows": int(s[1]), "rows": r, "cols": c, "vals": v,
                    "data_ranges": data, "process_ranges": proc, "total_buffer_size": int(s[5]),
                    "layout": _to_layout(a)}
        finally:
            self.lib.ref_partition_destroy(h)

    def _export_coo(self, h):
        s = np.zeros(3, np.int64)
        self.lib.ref_coo_sizes_f64(h, s.ctypes.data_as(_i64p))
        nnz = int(s[0])
        r, c, v = np.zeros(nnz, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz, np.float64)
        self.lib.ref_coo_export_f64(h, _ptr(r), _ptr(c), _ptr(v))
        return r, c, v, int(s[1]), int(s[2])

    def stencil27(self, nx, ny, nz, noise=0.0, iteration=0):
        """create3DStencil27Point (src/Format/HBDIA.cpp:1416-1607) -> COO arrays."""
        h = self.lib.ref_stencil27_f64(nx, ny, nz, noise, iteration)
        try:
            return self._export_coo(h)
        finally:
            self.lib.ref_matrix_destroy_f64(h)

    def load_mtx(self, path: str):
        ok = ctypes.c_int(0)
        h = self.lib.ref_load_mtx_f64(path.encode(), ctypes.byref(ok))
        try:
            return (bool(ok.value),) + self._export_coo(h)
        finally:
            self.lib.ref_matrix_destroy_f64(h)

    def cpu_coo(self, rows, cols, vals):
        return _RefCoo(self, rows, cols, vals)

    def omp_max_threads(self) -> int:
        return int(self.lib.ref_omp_max_threads())

    def gpu_spmv(self, rows, cols, vals, num_rows, num_cols, bw, thr, x, exec_cpu=True, exec_gpu=False):
        """The reference's own hbdiaSpMV on the GPU (needs a CUDA device)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(num_rows, np.float64)
        rc = self.lib.ref_gpu_spmv_f64(_ptr(rows), _ptr(cols), _ptr(vals), len(vals), num_rows, num_cols,
                                       bw, thr, _ptr(x), _ptr(y), int(exec_cpu), int(exec_gpu))
        if rc != 0:
            raise RuntimeError(f"reference hbdiaSpMV failed with {rc}")
        return y


class _RefGpuMatrix:
    def __init__(self, owner: Reference, h, n):
        self._o, self._h, self.n = owner, h, n

    def arrays(self) -> dict:
        """numBlocks, totalOffsets, numCoo and the device addresses of its
        prepareForGPU arrays (getHBDIADataDevice() ... getCpuRowPtrDevice())."""
        s = np.zeros(3, np.int64)
        p = (ctypes.c_void_p * 7)()
        self._o.lib.ref_gpu_matrix_arrays_f64(self._h, s.ctypes.data_as(_i64p), p)
        names = ("values", "offsets", "blockStart", "cooRow", "cooCol", "cooVal", "cooRowPtr")
        return {"numBlocks": int(s[0]), "totalOffsets": int(s[1]), "numCoo": int(s[2]),
                **{k: (v or 0) for k, v in zip(names, p)}}

    def spmv(self, x: np.ndarray, exec_cpu: bool = True) -> np.ndarray:
        """The reference's own hbdiaSpMV on this matrix."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.n, np.float64)
        rc = self._o.lib.ref_gpu_matrix_spmv_f64(self._h, _ptr(x), _ptr(y), int(exec_cpu))
        if rc != 0:
            raise RuntimeError(f"reference hbdiaSpMV failed ({rc})")
        return y

    def __del__(self):
        if getattr(self, "_h", None):
            self._o.lib.ref_matrix_destroy_f64(self._h)
            self._h = None


class _RefCoo:
    """The reference's cpu_coo_spmv_kernel over a COO matrix held in std::vectors."""

    def __init__(self, owner: Reference, rows, cols, vals):
        self._o = owner
        self._rows = np.ascontiguousarray(rows, np.int32)
        self._cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals)
        self.t = "f32" if vals.dtype == np.float32 else "f64"
        self.dtype = vals.dtype
        self._h = getattr(owner.lib, f"ref_cpu_coo_create_{self.t}")(
            _ptr(self._rows), _ptr(self._cols), _ptr(vals), len(vals))

    def spmv(self, x, num_rows, y: Optional[np.ndarray] = None):
        y = np.zeros(num_rows, self.dtype) if y is None else y
        getattr(self._o.lib, f"ref_cpu_coo_spmv_{self.t}")(self._h, _ptr(x), num_rows, _ptr(y))
        return y

    def __del__(self):
        if getattr(self, "_h", None):
            getattr(self._o.lib, f"ref_cpu_coo_destroy_{self.t}")(self._h)
            self._h = None


def storage_costs(value_bytes, num_rows, num_cols, nnz, number_diagonals, num_blocks, block_width, hbdia_slots,
                  coo_entries, hist_blocks, nnz_per_row):
    """The storage-cost arithmetic of the reference's benchmark
    (benchmarking/benchmark.cpp:171-215), restated: HBDIA, COO, DIA, SELL-C
    (C = block width) and CSR bytes of one matrix.  Test infrastructure."""
    sum_hist = sum(i * int(h) for i, h in enumerate(hist_blocks))
    hbdia = hbdia_slots * value_bytes + (num_blocks + 1) * 4 + sum_hist * 4 + coo_entries * 4 * 2 + coo_entries * value_bytes
    coo = nnz * 4 * 2 + nnz * value_bytes
    dia = number_diagonals * min(num_rows, num_cols) * value_bytes + number_diagonals * 4
    sell, mx = 0, 0
    for i, c in enumerate(nnz_per_row):
        if i % block_width == 0 and i > 0:
            sell += mx * block_width * value_bytes + mx * block_width * 4
            mx = 0
        mx = max(mx, int(c))
    sell += mx * block_width * value_bytes + mx * block_width * 4
    sell += ((num_rows + block_width - 1) // block_width) * 4
    csr = nnz * value_bytes + nnz * 4 + (num_rows + 1) * 4
    return {"hbdia": hbdia, "coo": coo, "dia": dia, "sell": sell, "csr": csr}
