"""hbdia_b200 -- B200-native HBDIA sparse matrix-vector product.

Python mirror of the reference's API (nrottstegge/HBDIA):

* :class:`HBDIA`        -- ``HBDIA<T>`` (include/Format/HBDIA.hpp:24-291)
* :class:`HBDIAVector`  -- ``HBDIAVector<T>`` (include/Format/HBDIAVector.hpp:23-109)
* :func:`hbdiaSpMV`     -- ``hbdiaSpMV`` (include/Operations/HBDIASpMV.hpp:8-10)

Everything runs through the C ABI of ``libhbdia_b200.so`` (include/hbdia_b200.h);
the SpMV itself is one fused sm_100a kernel launch.  There is no CPU path.
"""
from __future__ import annotations

import ctypes
from enum import IntEnum
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (BATCH_CONCURRENT, BATCH_QUEUE, REQ_CG, REQ_SPMV, KERNEL_AUTO, KERNEL_PIPE, KERNEL_QUAD, KERNEL_ROWWISE, KERNEL_STAGED, KERNEL_WARP, TUNE_PREFETCH, TUNE_QUAD_GROUP, TUNE_SPMM_TILE, TUNE_STAGES, TUNE_TAIL,
                   TUNE_UNROLL, HBDIACudaError,
                   HBDIADeviceTimeout, STORE_BF16_SCALED, STORE_F32, STORE_NATIVE, STORE_F32_QUAD, STORE_BF16_QUAD, MatrixInfo,
                   check as _check, load as _load)

__all__ = ["ExecutionMode", "HBDIA", "HBDIAVector", "hbdiaSpMV", "spmv_device", "spmm_device",
           "spmv_host", "generate_stencil27", "generate_stencil7", "generate_banded", "fill_uniform",
           "HBDIACudaError", "set_device", "STORE_NATIVE", "STORE_F32", "STORE_BF16_SCALED", "STORE_F32_QUAD",
           "STORE_BF16_QUAD", "library_path"]

DEFAULT_BLOCK_WIDTH = 32      # include/types.hpp:14
DEFAULT_THRESHOLD = 1         # include/types.hpp:15
MAX_COO_ENTRIES = 1000000000  # include/types.hpp:16


class ExecutionMode(IntEnum):
    """include/types.hpp:7-10."""
    CPU_COO = 0
    GPU_COO = 1


def library_path() -> str:
    return _lib.LIB_PATH


def set_device(device: int) -> None:
    """Select the GPU for this host thread's library calls (default 0)."""
    _check(_load().hbdia_set_device(int(device)))


def _vp(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _dtype_code(dtype) -> int:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return _lib.HBDIA_F64
    if dt == np.float32:
        return _lib.HBDIA_F32
    raise ValueError(f"unsupported value type {dt}; use float64 or float32")


class HBDIA:
    """``HBDIA<T>``: COO input, conversion to blocked-DIA + COO remainder, and
    the device layout.  ``dtype`` plays the role of the template argument."""

    def __init__(self, rowIndices: Optional[Sequence[int]] = None, colIndices: Optional[Sequence[int]] = None,
                 values: Optional[Sequence[float]] = None, numRows: Optional[int] = None,
                 numCols: Optional[int] = None, dtype=np.float64):
        lib = _load()
        self.dtype = np.dtype(dtype)
        self._h = ctypes.c_void_p()
        code = _dtype_code(self.dtype)
        if rowIndices is None and colIndices is None and values is None:
            _check(lib.hbdia_matrix_create_empty(code, ctypes.byref(self._h)))  # HBDIA()
            return
        r = np.ascontiguousarray(rowIndices, np.int32)
        c = np.ascontiguousarray(colIndices, np.int32)
        v = np.ascontiguousarray(values, self.dtype)
        if not (len(r) == len(c) == len(v)):
            # src/Format/HBDIA.cpp:27-29
            raise ValueError("Row indices, column indices, and values vectors must have the same size")
        nr = -1 if numRows is None else int(numRows)
        nc = -1 if numCols is None else int(numCols)
        if (numRows is None) != (numCols is None):
            raise ValueError("give both numRows and numCols, or neither")
        if numRows is not None and (nr <= 0 or nc <= 0):
            raise ValueError("Matrix dimensions must be positive")
        _check(lib.hbdia_matrix_create(code, _vp(r), _vp(c), _vp(v), len(v), nr, nc, ctypes.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _load().hbdia_matrix_destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # ---- matrix sources
    def create3DStencil27Point(self, nx: int, ny: int, nz: int, noise: float = 0.0, iteration: int = 0) -> None:
        _check(_load().hbdia_matrix_stencil27(self._h, nx, ny, nz, float(noise), iteration))

    def loadMTX(self, filename: str, numRows: Optional[int] = None, numCols: Optional[int] = None) -> bool:
        ok = ctypes.c_int32(0)
        _check(_load().hbdia_matrix_load_mtx(self._h, filename.encode(), numRows or 0, numCols or 0,
                                            ctypes.byref(ok)))
        return bool(ok.value)

    # ---- conversion
    def convertToHBDIAFormat(self, blockWidth: int = DEFAULT_BLOCK_WIDTH, threshold: int = DEFAULT_THRESHOLD,
                             max_coo_entries: int = MAX_COO_ENTRIES, COOisUnique: bool = False,
                             execMode: ExecutionMode = ExecutionMode.GPU_COO, upload: bool = True) -> None:
        """src/Format/HBDIA.cpp:507-718.  ``upload=False`` skips the device
        layout (the reference's partial-matrix behaviour), so it runs without a GPU."""
        _check(_load().hbdia_matrix_convert(self._h, blockWidth, threshold, int(max_coo_entries),
                                            int(bool(COOisUnique)), int(execMode), int(bool(upload))))

    def convertOnDevice(self, blockWidth: int = DEFAULT_BLOCK_WIDTH, threshold: int = DEFAULT_THRESHOLD,
                        max_coo_entries: int = MAX_COO_ENTRIES, storage: int = STORE_NATIVE) -> None:
        """convertToHBDIAFormat + prepareForGPU on the GPU (row-sorted COO)."""
        _check(_load().hbdia_matrix_convert_on_device(self._h, blockWidth, threshold, int(max_coo_entries), storage))

    def prepareForGPU(self, storage: int = STORE_NATIVE) -> None:
        _check(_load().hbdia_matrix_prepare_gpu(self._h, storage))

    def initializeCuSparse(self) -> None:
        """Kept for source compatibility (src/Format/HBDIA.cpp:919-994): the COO
        remainder runs inside the fused kernel, so there is nothing to set up."""

    # ---- getters (include/Format/HBDIA.hpp:72-115)
    def info(self) -> MatrixInfo:
        i = MatrixInfo()
        _check(_load().hbdia_matrix_get_info(self._h, ctypes.byref(i)))
        return i

    def getNumRows(self) -> int: return self.info().numRows
    def getNumCols(self) -> int: return self.info().numCols
    def getNumNonZeros(self) -> int: return self.info().numNonZeros
    def getBlockWidth(self) -> int: return self.info().blockWidth
    def getThreshold(self) -> int: return self.info().threshold
    def getMaxCooEntries(self) -> int: return self.info().maxCooEntries
    def getNumBlocks(self) -> int: return self.info().numBlocks
    def getNumberDiagonals(self) -> int: return self.info().numberDiagonals
    def getHasCOO(self) -> bool: return bool(self.info().hasCOO)
    def getHasHBDIA(self) -> bool: return bool(self.info().hasHBDIA)
    isCOOFormat = getHasCOO
    isHBDIAFormat = getHasHBDIA

    # ---- DIA format (src/Format/HBDIA.cpp:372-505)
    def removeCOODuplicates(self) -> None:
        _check(_load().hbdia_matrix_remove_duplicates(self._h))

    def convertToDIAFormat(self, COOisUnique: bool = False) -> None:
        _check(_load().hbdia_matrix_convert_dia(self._h, int(bool(COOisUnique))))

    def _dia_info(self):
        h, nd, ln = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
        _check(_load().hbdia_matrix_dia_info(self._h, ctypes.byref(h), ctypes.byref(nd), ctypes.byref(ln)))
        return bool(h.value), nd.value, ln.value

    def isDIAFormat(self) -> bool:
        return self._dia_info()[0]

    getHasDIA = isDIAFormat

    def getOffsets(self) -> np.ndarray:
        _, nd, _ = self._dia_info()
        out = np.zeros(nd, np.int32)
        _check(_load().hbdia_matrix_export_dia(self._h, _vp(out), None))
        return out

    def getDiagonals(self) -> np.ndarray:
        """[numDiagonals, min(numRows, numCols)]"""
        _, nd, ln = self._dia_info()
        out = np.zeros((nd, ln), self.dtype)
        _check(_load().hbdia_matrix_export_dia(self._h, None, _vp(out)))
        return out

    def coo(self):
        """The COO arrays (rows, cols, values) as the matrix holds them now."""
        n = self.getNumNonZeros()
        r, c, v = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, self.dtype)
        _check(_load().hbdia_matrix_export_coo(self._h, _vp(r), _vp(c), _vp(v)))
        return r, c, v

    def storageCosts(self) -> dict:
        """Bytes of HBDIA, COO, DIA, SELL and CSR storage
        (benchmarking/benchmark.cpp:171-215)."""
        s = _lib.StorageCosts()
        _check(_load().hbdia_matrix_storage_costs(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k in ("hbdia", "coo", "dia", "sell", "csr")}

    def layout(self) -> dict:
        """The host layout as numpy arrays: offsets/block_start (flattened
        offsetsPerBlock), data, coo_row/coo_col/coo_val, coo_row_ptr, hist_blocks,
        hist_nnz, number_diagonals, num_blocks."""
        i = self.info()
        if not i.hasHBDIA:
            raise RuntimeError("matrix is not in HBDIA format")
        out = dict(
            offsets=np.zeros(i.totalOffsets, np.int32), block_start=np.zeros(i.numBlocks + 1, np.int32),
            data=np.zeros(i.numSlots, self.dtype), coo_row=np.zeros(i.numCoo, np.int32),
            coo_col=np.zeros(i.numCoo, np.int32), coo_val=np.zeros(i.numCoo, self.dtype),
            coo_row_ptr=np.zeros(i.numRows + 1, np.int32), hist_blocks=np.zeros(i.histogramLength, np.int32),
            hist_nnz=np.zeros(i.histogramLength, np.int32))
        _check(_load().hbdia_matrix_export_layout(self._h, *[_vp(out[k]) for k in (
            "offsets", "block_start", "data", "coo_row", "coo_col", "coo_val", "coo_row_ptr",
            "hist_blocks", "hist_nnz")]))
        out["number_diagonals"] = i.numberDiagonals
        out["num_blocks"] = i.numBlocks
        return out

    def getHBDIAData(self) -> np.ndarray: return self.layout()["data"]
    def getCpuRowIndices(self) -> np.ndarray: return self.layout()["coo_row"]
    def getCpuColIndices(self) -> np.ndarray: return self.layout()["coo_col"]
    def getCpuValues(self) -> np.ndarray: return self.layout()["coo_val"]
    def getCpuRowPtr(self) -> np.ndarray: return self.layout()["coo_row_ptr"]
    def getHistogramBlocks(self) -> np.ndarray: return self.layout()["hist_blocks"]
    def getHistogramNnz(self) -> np.ndarray: return self.layout()["hist_nnz"]

    def getOffsetsPerBlock(self) -> List[List[int]]:
        L = self.layout()
        bs = L["block_start"]
        return [L["offsets"][bs[b]:bs[b + 1]].tolist() for b in range(L["num_blocks"])]

    def _coo(self):
        i = self.info()
        r = np.zeros(i.numNonZeros, np.int32)
        c = np.zeros(i.numNonZeros, np.int32)
        v = np.zeros(i.numNonZeros, self.dtype)
        _check(_load().hbdia_matrix_export_coo(self._h, _vp(r), _vp(c), _vp(v)))
        return r, c, v

    def getRowIndices(self) -> np.ndarray: return self._coo()[0]
    def getColIndices(self) -> np.ndarray: return self._coo()[1]
    def getValues(self) -> np.ndarray: return self._coo()[2]

    def getNnzPerRow(self) -> np.ndarray:
        out = np.zeros(self.info().numRows, np.int32)
        _check(_load().hbdia_matrix_export_nnz_per_row(self._h, _vp(out)))
        return out

    def getBDIAStream(self) -> int:
        s = ctypes.c_void_p()
        _check(_load().hbdia_matrix_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def deviceArrays(self) -> dict:
        """The device arrays of the GPU getters (include/Format/HBDIA.hpp:155-165):
        name -> device address (0 where the reference's getter returns null)."""
        a = _lib.DeviceArrays()
        _check(_load().hbdia_matrix_device_arrays(self._h, ctypes.byref(a)))
        return {name: getattr(a, name) or 0 for name, _ in a._fields_}

    def bytesPerSpmv(self) -> int:
        """Algorithmic HBM bytes of one SpMV over the device layout."""
        return self.info().bytesPerSpmv

    def synchronize(self) -> None:
        """Wait for the matrix's stream; raises HBDIADeviceTimeout when a
        bounded device-side wait ran out since the last check."""
        _check(_load().hbdia_matrix_synchronize(self._h))

    def deviceStatus(self) -> int:
        b = ctypes.c_int32(0)
        _check(_load().hbdia_matrix_device_status(self._h, ctypes.byref(b)))
        return b.value

    def setKernel(self, kernel: int) -> None:
        """KERNEL_AUTO / KERNEL_ROWWISE / KERNEL_WARP / KERNEL_STAGED."""
        _check(_load().hbdia_matrix_set_kernel(self._h, int(kernel)))

    def selectedKernel(self, x_ptr: int) -> int:
        k = ctypes.c_int32(0)
        _check(_load().hbdia_matrix_selected_kernel(self._h, ctypes.c_void_p(x_ptr), ctypes.byref(k)))
        return k.value

    def setTuning(self, key: int, value: int) -> None:
        """Kernel tuning knob (TUNE_UNROLL: 0, 9 or 27); results stay bit-identical."""
        _check(_load().hbdia_matrix_set_tuning(self._h, int(key), int(value)))

    def autotune(self, X_ptr: int, Y_ptr: int, k: int = 1, ldx: int = 0, ldy: int = 0,
                 stream: Optional[int] = None, force: bool = False) -> "_lib.TuneResult":
        """Time this matrix's SpMV (k = 1) or SpMM (k > 1) configurations on the
        given device buffers, keep the fastest (see hbdia_matrix_autotune)."""
        r = _lib.TuneResult()
        _check(_load().hbdia_matrix_autotune(self._h, ctypes.c_void_p(X_ptr), ldx or k, ctypes.c_void_p(Y_ptr),
                                             ldy or k, int(k), _stream_arg(stream), int(bool(force)),
                                             ctypes.byref(r)))
        return r

    def setWaitTimeout(self, nanoseconds: int) -> None:
        _check(_load().hbdia_matrix_set_wait_timeout(self._h, int(nanoseconds)))

    def testSkipTile(self, tile: int) -> None:
        """Test hook: the staged kernel never issues the copies of 32-row
        tile `tile`, so its bounded wait runs out (-1: off)."""
        _check(_load().hbdia_matrix_test_skip_tile(self._h, int(tile)))

    # ---- partial matrices: one rank's rows (include/Format/HBDIA.hpp:37-39, 77-79, 117-136)
    @classmethod
    def _adopt(cls, handle: ctypes.c_void_p, dtype) -> "HBDIA":
        m = cls.__new__(cls)
        m.dtype = np.dtype(dtype)
        m._h = handle
        return m

    @classmethod
    def partial(cls, rowIndices, colIndices, values, numRows: int, numCols: int, globalRowMapping,
                partialMatrix: bool = True, numGlobalRows: Optional[int] = None,
                numGlobalCols: Optional[int] = None, numGlobalNonZeros: int = 0, rank: int = 0, size: int = 1,
                dtype=np.float64) -> "HBDIA":
        """``HBDIA(rows, cols, vals, numRows, numCols, globalRowMapping, partialMatrix,
        numGlobalRows, numGlobalCols, numGlobalNonZeros, rank, size)``
        (src/Format/HBDIA.cpp:118-154): local rows, global columns.  The global
        row mapping must be contiguous (the one BasicExtractor builds)."""
        if not partialMatrix:
            return cls(rowIndices, colIndices, values, numRows, numCols, dtype=dtype)
        mapping = np.asarray(globalRowMapping, np.int64)
        if len(mapping) != numRows:
            raise ValueError("Global row mapping size must match number of rows")
        if np.any(np.diff(mapping) != 1):
            raise NotImplementedError("only contiguous global row mappings (the row-wise partition's)")
        r = np.ascontiguousarray(rowIndices, np.int32)
        c = np.ascontiguousarray(colIndices, np.int32)
        v = np.ascontiguousarray(values, np.dtype(dtype))
        if not (len(r) == len(c) == len(v)):
            raise ValueError("Row indices, column indices, and values vectors must have the same size")
        h = ctypes.c_void_p()
        _check(_load().hbdia_matrix_create_partial(
            _dtype_code(np.dtype(dtype)), _vp(r), _vp(c), _vp(v), len(v), int(numRows),
            int(numGlobalRows if numGlobalRows is not None else numCols),
            int(numGlobalCols if numGlobalCols is not None else numCols), int(numGlobalNonZeros),
            int(mapping[0]) if len(mapping) else 0, int(rank), int(size), ctypes.byref(h)))
        return cls._adopt(h, dtype)

    def partition(self, numProcesses: int, part: int) -> "HBDIA":
        """Partition ``part`` of BasicExtractor's row-wise partitioning
        (src/DataExchange/BasicExtractor.cpp:124-234) as a partial matrix."""
        h = ctypes.c_void_p()
        _check(_load().hbdia_matrix_partition(self._h, int(numProcesses), int(part), ctypes.byref(h)))
        return HBDIA._adopt(h, self.dtype)

    def partialInfo(self) -> "_lib.PartialInfo":
        i = _lib.PartialInfo()
        _check(_load().hbdia_matrix_partial_info(self._h, ctypes.byref(i)))
        return i

    def isPartialMatrix(self) -> bool: return bool(self.partialInfo().isPartial)
    def getNumGlobalRows(self) -> int: return self.partialInfo().numGlobalRows
    def getNumGlobalCols(self) -> int: return self.partialInfo().numGlobalCols
    def getNumGlobalNonZeros(self) -> int: return self.partialInfo().numGlobalNonZeros

    def getGlobalRowMapping(self) -> np.ndarray:
        i = self.partialInfo()
        if not i.isPartial:
            return np.zeros(0, np.int32)
        return np.arange(i.globalRowStart, i.globalRowStart + self.getNumRows(), dtype=np.int32)

    def getGlobalRowIndex(self, localRowIndex: int) -> int:
        i = self.partialInfo()
        return int(localRowIndex) + (i.globalRowStart if i.isPartial else 0)

    def _ranges(self):
        i = self.partialInfo()
        d = np.zeros((i.numDataRanges, 2), np.int32)
        p = np.zeros((i.numProcessRanges, 3), np.int32)
        _check(_load().hbdia_matrix_export_ranges(self._h, _vp(d), _vp(p)))
        return i, d, p

    def analyzeDataRanges(self) -> None:
        """Kept for the reference's call sequence: a partial matrix's data
        ranges are computed by convertToHBDIAFormat."""

    def getDataRanges(self) -> List[tuple]:
        """analyzeDataRanges (src/Format/HBDIA.cpp:1333-1414): merged [start, end)
        ranges of the global columns this rank's rows read."""
        return [tuple(int(v) for v in r) for r in self._ranges()[1]]

    def hasPartialMatrixMetadata(self) -> bool:
        i = self.partialInfo()
        return bool(i.isPartial and i.hasMetadata and i.totalBufferSize > 0)

    def getPartialMatrixMetadata(self) -> dict:
        """PartialMatrixMetadata (include/Format/HBDIA.hpp:18-22): dataRanges,
        processDataRanges[p] (the ranges process p provides) and totalBufferSize."""
        i, d, p = self._ranges()
        per = [[] for _ in range(max(i.size, 1))]
        for q, s, e in p:
            per[int(q)].append((int(s), int(e)))
        return {"dataRanges": [tuple(int(v) for v in r) for r in d], "processDataRanges": per,
                "totalBufferSize": int(i.totalBufferSize)}

    def window(self) -> tuple:
        """(first global column, length) of the x window the plan reads."""
        i = self.partialInfo()
        return int(i.windowStart), int(i.windowLength)


class HBDIAVector:
    """``HBDIAVector<T>`` on one GPU: a device buffer (no halos)."""

    def __init__(self, localData, dtype=None):
        lib = _load()
        data = np.ascontiguousarray(localData, dtype if dtype is not None else None)
        if data.dtype not in (np.float64, np.float32):
            data = data.astype(np.float64)
        self.dtype = data.dtype
        self._h = ctypes.c_void_p()
        _check(lib.hbdia_vector_create(_dtype_code(self.dtype), _vp(data), len(data), ctypes.byref(self._h)))
        self._n = len(data)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _load().hbdia_vector_destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def getDeviceDataPtr(self) -> int:
        p = ctypes.c_void_p()
        _check(_load().hbdia_vector_device_ptr(self._h, ctypes.byref(p)))
        return p.value or 0

    getDeviceLocalPtr = getDeviceDataPtr

    def getDeviceCOOResultsPtr(self) -> int:
        """include/Format/HBDIAVector.hpp:53: a zeroed buffer of the vector's
        length, kept for callers that clear it; the fused SpMV never uses it."""
        p = ctypes.c_void_p()
        _check(_load().hbdia_vector_coo_results_ptr(self._h, ctypes.byref(p)))
        return p.value or 0

    def getLocalSize(self) -> int:
        return self._n

    getTotalSize = getLocalSize

    def toHost(self) -> np.ndarray:
        out = np.empty(self._n, self.dtype)
        _check(_load().hbdia_vector_download(self._h, _vp(out)))
        return out

    def upload(self, data) -> None:
        d = np.ascontiguousarray(data, self.dtype)
        if len(d) != self._n:
            raise ValueError("size mismatch")
        _check(_load().hbdia_vector_upload(self._h, _vp(d)))


def hbdiaSpMV(matrix: HBDIA, inputVector: HBDIAVector, outputVector: HBDIAVector,
              execCOOCPU: bool, execCOOGPU: bool) -> bool:
    """src/Operations/HBDIASpMV.cpp:186-251: y = A x, asynchronous on the
    matrix's stream.  Raises RuntimeError("... Invalid COO execution flags")
    when the matrix has a COO remainder and both flags are False."""
    _check(_load().hbdia_spmv(matrix.handle, inputVector.handle, outputVector.handle,
                              int(bool(execCOOCPU)), int(bool(execCOOGPU))))
    return True


_CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the handle value 0 means the legacy default stream


def _stream_arg(stream: Optional[int]) -> ctypes.c_void_p:
    """None -> the matrix's own stream (NULL at the ABI); an int is a
    cudaStream_t handle, where 0 (e.g. torch's default stream) is the legacy
    default stream."""
    if stream is None:
        return ctypes.c_void_p(None)
    return ctypes.c_void_p(int(stream) or _CUDA_STREAM_LEGACY)


def spmv_device(matrix: HBDIA, x_ptr: int, y_ptr: int, stream: Optional[int] = None) -> None:
    """y = A x on raw device pointers (e.g. torch tensors' data_ptr()) on
    ``stream`` (None: the matrix's stream; torch's ``cuda_stream`` values,
    0 included, are passed as they are)."""
    _check(_load().hbdia_spmv_device(matrix.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                     _stream_arg(stream)))


def autotune_clear() -> None:
    """Forget the process-wide autotuning table."""
    _check(_load().hbdia_autotune_clear())


def spmm_device(matrix: HBDIA, X_ptr: int, ldx: int, Y_ptr: int, ldy: int, k: int,
                stream: Optional[int] = None) -> None:
    """Y = A X for k row-major right-hand sides on raw device pointers."""
    _check(_load().hbdia_spmm_device(matrix.handle, ctypes.c_void_p(X_ptr), ldx, ctypes.c_void_p(Y_ptr), ldy,
                                     k, _stream_arg(stream)))


def spmm_device_colmajor(matrix: HBDIA, X_ptr: int, ldx: int, Y_ptr: int, ldy: int, k: int,
                         stream: Optional[int] = None) -> None:
    """Y = A X for k column-major right-hand sides (vector j at X + j*ldx)."""
    _check(_load().hbdia_spmm_device_colmajor(matrix.handle, ctypes.c_void_p(X_ptr), ldx, ctypes.c_void_p(Y_ptr),
                                              ldy, k, _stream_arg(stream)))


def spmv_list_device(matrix: HBDIA, x_ptrs: Sequence[int], y_ptrs: Sequence[int],
                     stream: Optional[int] = None) -> None:
    """y_j = A x_j for separate device vectors, each stored value read once per
    32 vectors; y_j equals spmv_device(matrix, x_j, y_j) bit for bit."""
    k = len(x_ptrs)
    if len(y_ptrs) != k:
        raise ValueError("x and y lists differ in length")
    xa = (ctypes.c_void_p * max(k, 1))(*x_ptrs)
    ya = (ctypes.c_void_p * max(k, 1))(*y_ptrs)
    _check(_load().hbdia_spmv_list_device(matrix.handle, xa, ya, k, _stream_arg(stream)))


class LayoutPlan:
    """``hbdia_plan`` over HBDIA device arrays the caller owns (the arrays
    prepareForGPU leaves on the device).  Pointers are device addresses
    (ints); ``keep`` holds whatever owns them for the plan's lifetime."""

    def __init__(self, *, dtype=np.float64, storage: int = STORE_NATIVE, numRows: int, numCols: int,
                 blockWidth: int, numBlocks: int, totalOffsets: int, numCoo: int, values: int, offsets: int,
                 blockStart: int, cooRow: int = 0, cooCol: int = 0, cooVal: int = 0, cooRowPtr: int = 0,
                 scales: int = 0, keep=None):
        d = _lib.LayoutDesc(_dtype_code(dtype), storage, numRows, numCols, blockWidth, numBlocks, totalOffsets,
                            numCoo, values or None, scales or None, offsets or None, blockStart or None,
                            cooRow or None, cooCol or None, cooVal or None, cooRowPtr or None)
        self._h = ctypes.c_void_p()
        self._keep = keep
        self.numRows, self.numCols = numRows, numCols
        _check(_load().hbdia_plan_create(ctypes.byref(d), ctypes.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _load().hbdia_plan_destroy(h)
            self._h = None

    def spmv(self, x_ptr: int, y_ptr: int, stream: Optional[int] = None) -> None:
        _check(_load().hbdia_plan_spmv(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), _stream_arg(stream)))

    def spmm(self, X_ptr: int, ldx: int, Y_ptr: int, ldy: int, k: int, stream: Optional[int] = None) -> None:
        _check(_load().hbdia_plan_spmm(self._h, ctypes.c_void_p(X_ptr), ldx, ctypes.c_void_p(Y_ptr), ldy, k,
                                       _stream_arg(stream)))


def spmv_host_many(matrix: HBDIA, xs: Sequence[np.ndarray], ys: Sequence[np.ndarray]) -> None:
    """y_j = A x_j for host arrays, pipelined so that one step's upload
    overlaps another's download (page-locked arrays for the overlap)."""
    if len(xs) != len(ys):
        raise ValueError("x and y lists differ in length")
    nx = max(matrix.getNumRows(), matrix.getNumCols())
    for x, y in zip(xs, ys):
        if x.dtype != matrix.dtype or y.dtype != matrix.dtype or not x.flags.c_contiguous or not y.flags.c_contiguous \
                or x.size < nx or y.size < matrix.getNumRows():
            raise ValueError("vectors must be contiguous arrays of the matrix's type and size")
    k = len(xs)
    xa = (ctypes.c_void_p * max(k, 1))(*[x.ctypes.data for x in xs])
    ya = (ctypes.c_void_p * max(k, 1))(*[y.ctypes.data for y in ys])
    _check(_load().hbdia_spmv_host_many(matrix.handle, xa, ya, k))


def spmv_host(matrix: HBDIA, x: np.ndarray, y: np.ndarray) -> None:
    """End-to-end y = A x on host arrays (copies in, SpMV, copies out, sync)."""
    _check(_load().hbdia_spmv_host(matrix.handle, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(y.ctypes.data)))


def allocation_count() -> tuple:
    """(device, page-locked host) allocations the library has made since it
    was loaded (hbdia_allocation_count)."""
    d, h = ctypes.c_int64(), ctypes.c_int64()
    _check(_load().hbdia_allocation_count(ctypes.byref(d), ctypes.byref(h)))
    return d.value, h.value


def spmv_host_noalloc(matrix: HBDIA, x: np.ndarray, y: np.ndarray) -> None:
    """spmv_host through the library's fixed per-device array (no device
    allocation; max(numRows, numCols) <= 2^21; calls must not overlap)."""
    _check(_load().hbdia_spmv_host_noalloc(matrix.handle, ctypes.c_void_p(x.ctypes.data),
                                           ctypes.c_void_p(y.ctypes.data)))


# ---------------------------------------------------------------- workloads
def _two_call(fn, *args):
    nnz = ctypes.c_int64(0)
    _check(fn(*args, ctypes.byref(nnz), None, None, None))
    r = np.empty(nnz.value, np.int32)
    c = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value, np.float64)
    _check(fn(*args, ctypes.byref(nnz), _vp(r), _vp(c), _vp(v)))
    return r, c, v


def generate_stencil27(nx: int, ny: int, nz: int, center: float = 26.0, neighbor: float = -1.0,
                       extra_fraction: float = 0.0, extra_lo: float = 0.1, extra_hi: float = 1.0, seed: int = 0):
    """Seeded 27-point stencil (+ extra off-pattern entries), row-sorted COO."""
    return _two_call(_load().hbdia_generate_stencil27, nx, ny, nz, center, neighbor, extra_fraction,
                     extra_lo, extra_hi, seed)


def generate_stencil7(nx: int, ny: int, nz: int, center: float = 6.0, neighbor: float = -1.0):
    return _two_call(_load().hbdia_generate_stencil7, nx, ny, nz, center, neighbor)


def generate_banded(n: int, offsets: Sequence[int], lo: float = 0.5, hi: float = 1.5, drop: float = 0.3,
                    scatter: float = 0.002, seed: int = 2):
    o = np.ascontiguousarray(offsets, np.int32)
    return _two_call(_load().hbdia_generate_banded, n, _vp(o), len(o), lo, hi, drop, scatter, seed)


def generate_stencil27_spd(nx: int, ny: int, nz: int, shift: float = 1e-3, seed: int = 7,
                           extra_fraction: float = 0.0):
    """SPD symmetrised 27-point stencil (symmetric random off-diagonals -(0.5 + u),
    plus symmetric off-pattern pairs making up ``extra_fraction`` of the
    stencil's entries, diagonal (1 + shift) * row |sum|)."""
    return _two_call(_load().hbdia_generate_stencil27_spd, nx, ny, nz, float(shift), float(extra_fraction), seed)


def cg_solve(matrix: HBDIA, b_ptr: int, x_ptr: int, tol: float = 1e-10, iter_storage: int = STORE_F32_QUAD,
             update_factor: float = 0.1, max_updates: int = 100, max_iterations: int = 20000,
             check_every: int = 10, stream: Optional[int] = None) -> "_lib.CgResult":
    """CG on device buffers b, x (x: initial guess in, solution out): the
    iterations' SpMVs use the ``iter_storage`` values (STORE_F32_QUAD, the
    default, or STORE_F32: mixed precision, both giving the same iterates;
    STORE_NATIVE: plain FP64 CG), with reliable updates of the FP64 residual
    and convergence judged on it (hbdia_cg_solve)."""
    o = _lib.CgOptions(tol, update_factor, max_updates, max_iterations, iter_storage, check_every)
    r = _lib.CgResult()
    _check(_load().hbdia_cg_solve(matrix.handle, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr), ctypes.byref(o),
                                  _stream_arg(stream), ctypes.byref(r)))
    return r


class Batch:
    """Many device-resident matrices (block width 32, one value type and
    storage) computed by one persistent launch (hbdia_batch_*).  Every y is bit
    for bit what spmv_device / spmm_device give for that matrix alone.  The
    matrices must stay alive and on the device while the batch exists."""

    def __init__(self, matrices: Sequence[HBDIA]):
        self._mats = list(matrices)  # keeps the matrices alive
        arr = (ctypes.c_void_p * len(self._mats))(*[m.handle.value for m in self._mats])
        h = ctypes.c_void_p()
        _check(_load().hbdia_batch_create(arr, len(self._mats), ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            _load().hbdia_batch_destroy(h)
            self.handle = None

    def __len__(self) -> int:
        return len(self._mats)

    def bind(self, x_ptrs: Sequence[int], y_ptrs: Sequence[int], k: Optional[Sequence[int]] = None,
             ldx: Optional[Sequence[int]] = None, ldy: Optional[Sequence[int]] = None) -> None:
        """Device pointers per matrix; k[i] right-hand sides (row-major n x k
        blocks with leading dimensions ldx[i], ldy[i]); k[i] == 0 leaves
        matrix i out.  Runs already enqueued keep their old binding."""
        n = len(self._mats)
        X = (ctypes.c_void_p * n)(*[int(p) or None for p in x_ptrs])
        Y = (ctypes.c_void_p * n)(*[int(p) or None for p in y_ptrs])
        K = (ctypes.c_int32 * n)(*k) if k is not None else None
        LX = (ctypes.c_int64 * n)(*ldx) if ldx is not None else None
        LY = (ctypes.c_int64 * n)(*ldy) if ldy is not None else None
        _check(_load().hbdia_batch_bind(self.handle, X, LX, Y, LY, K))

    def run(self, stream: Optional[int] = None) -> None:
        _check(_load().hbdia_batch_run(self.handle, _stream_arg(stream)))

    def set_config(self, schedule: int = _lib.BATCH_CONCURRENT, streams: Optional[int] = None, threads: int = 256,
                   grab: int = 4, rhs_tile: int = 8, graph: bool = True) -> None:
        """schedule: BATCH_CONCURRENT (each matrix's own kernel on a ring of
        ``streams`` streams) or BATCH_QUEUE (one persistent launch per 160
        matrices, ``threads`` per CTA, ``grab`` tiles per atomic, ``rhs_tile``
        right-hand sides per pass)."""
        if streams is None:
            streams = min(16, len(self._mats))
        c = _lib.BatchConfig(schedule, streams, threads, grab, rhs_tile, 1 if graph else 0)
        _check(_load().hbdia_batch_set_config(self.handle, ctypes.byref(c)))

    def config(self) -> "_lib.BatchConfig":
        c = _lib.BatchConfig()
        _check(_load().hbdia_batch_get_config(self.handle, ctypes.byref(c)))
        return c

    def autotune(self, stream: Optional[int] = None):
        """Times every configuration on the bound vectors and keeps the
        fastest; returns (ms per run of the best, candidates timed)."""
        ms = ctypes.c_float(0)
        n = ctypes.c_int32(0)
        _check(_load().hbdia_batch_autotune(self.handle, _stream_arg(stream), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def info(self):
        """(count, total 32-row tiles, algorithmic HBM bytes per run)."""
        c, t, b = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int64(0)
        _check(_load().hbdia_batch_info(self.handle, ctypes.byref(c), ctypes.byref(t), ctypes.byref(b)))
        return c.value, t.value, b.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(_load().hbdia_batch_stream(self.handle, ctypes.byref(s)))
        return s.value or 0


def fill_uniform(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    _check(_load().hbdia_fill_uniform(_vp(out), n, lo, hi, seed))
    return out


class Server:
    """Resident matrices and a request queue (hbdia_server_*): SpMV requests
    served with continuous batching (each matrix's pending requests become one
    SpMM whenever the matrix is free), CG requests on a pool of solver threads.  ``options`` overrides
    fields of hbdia_server_default_options (memoryBudget, batching, maxRhs,
    spmvStorage, cgIterStorage, cgWorkers, cgTol, cgUpdateFactor, cgMaxGroup, maxInFlight, ...)."""

    def __init__(self, **options):
        o = _lib.ServerOptions()
        _load().hbdia_server_default_options(ctypes.byref(o))
        for k, v in options.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown server option {k}")
            setattr(o, k, v)
        h = ctypes.c_void_p()
        _check(_load().hbdia_server_create(ctypes.byref(o), ctypes.byref(h)))
        self.handle = h
        self.options = o
        self._live = {}  # ticket -> (x, y): keeps the host arrays alive until collected

    def close(self) -> None:
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            _load().hbdia_server_destroy(h)
            self.handle = None
            self._live.clear()

    def __del__(self):
        self.close()

    def add_matrix(self, matrix: HBDIA) -> int:
        mid = ctypes.c_int32(0)
        _check(_load().hbdia_server_add_matrix(self.handle, matrix.handle, ctypes.byref(mid)))
        return mid.value

    def submit(self, matrix_id: int, kind: int, x: np.ndarray, y: np.ndarray) -> int:
        """x: float64 right-hand side (numCols), y: float64 output (numRows);
        both must stay untouched until wait(ticket) returns."""
        if x.dtype != np.float64 or y.dtype != np.float64 or not x.flags.c_contiguous or not y.flags.c_contiguous:
            raise ValueError("request vectors must be contiguous float64 arrays")
        t = ctypes.c_uint64(0)
        _check(_load().hbdia_server_submit(self.handle, matrix_id, kind, _vp(x), _vp(y), ctypes.byref(t)))
        self._live[t.value] = (x, y)
        return t.value

    def submit_device(self, matrix_id: int, kind: int, x, y) -> int:
        """The same request on CUDA tensors (float64, contiguous), read and
        written in place; keep them untouched until wait(ticket) returns."""
        for t in (x, y):
            if not t.is_cuda or str(t.dtype) != "torch.float64" or not t.is_contiguous():
                raise ValueError("device request vectors must be contiguous float64 CUDA tensors")
        t = ctypes.c_uint64(0)
        _check(_load().hbdia_server_submit_device(self.handle, matrix_id, kind, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(y.data_ptr()), ctypes.byref(t)))
        self._live[t.value] = (x, y)
        return t.value

    def pause(self, paused: bool = True) -> None:
        """Hold (True) or release (False) the queues; released backlogs are
        batched together."""
        _check(_load().hbdia_server_pause(self.handle, 1 if paused else 0))

    def wait(self, ticket: int) -> "_lib.RequestInfo":
        info = _lib.RequestInfo()
        _check(_load().hbdia_server_wait(self.handle, ticket, ctypes.byref(info)))
        self._live.pop(ticket, None)
        return info

    def stats(self) -> "_lib.ServerStats":
        s = _lib.ServerStats()
        _check(_load().hbdia_server_get_stats(self.handle, ctypes.byref(s)))
        return s


def write_storage_report(matrix: HBDIA, folder: str, name: str, nx: int = 0, ny: int = 0, nz: int = 0,
                         noise: float = 0.0, execCOOCPU: bool = False, execCOOGPU: bool = True) -> None:
    """matrix_info.csv and histogram.csv with the columns of the reference's
    benchmark (benchmarking/benchmark.cpp:236-305) for a converted matrix.
    The unified-memory columns of the reference are written as 0 (this
    library keeps the matrix in device memory)."""
    import csv
    import os
    i = matrix.info()
    c = matrix.storageCosts()
    os.makedirs(folder, exist_ok=True)
    lay = matrix.layout() if i.storage == STORE_NATIVE or matrix.info().numSlots == 0 else None
    hist_b = lay["hist_blocks"] if lay is not None else np.zeros(0, np.int32)
    hist_n = lay["hist_nnz"] if lay is not None else np.zeros(0, np.int32)
    header = ["name", "nx", "ny", "nz", "noise", "rows", "cols", "nnz", "num_diagonals",
              "num_blocks", "block_width", "threshold", "max_coo_entries", "coo_fallback_entries",
              "hbdia_data_size", "hbdia_cost_bytes", "coo_cost_bytes", "dia_cost_bytes",
              "sell_cost_bytes", "csr_cost_bytes", "hbdia_vs_coo", "dia_vs_coo", "csr_vs_coo", "sell_vs_coo",
              "execCOOCPU", "execCOOGPU", "unifiedMemory", "unifiedMemory_malloc",
              "unifiedMemory_managedMalloc", "unifiedMemory_NumaAllocOnNode"]
    row = [name, nx, ny, nz, f"{noise:.6f}", i.numRows, i.numCols, i.numNonZeros, i.numberDiagonals,
           i.numBlocks, i.blockWidth, i.threshold, i.maxCooEntries, i.numCoo, i.numSlots,
           c["hbdia"], c["coo"], c["dia"], c["sell"], c["csr"],
           f"{c['hbdia'] / c['coo']:.6f}", f"{c['dia'] / c['coo']:.6f}", f"{c['csr'] / c['coo']:.6f}",
           f"{c['sell'] / c['coo']:.6f}", int(execCOOCPU), int(execCOOGPU), 0, 0, 0, 0]
    with open(os.path.join(folder, "matrix_info.csv"), "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(header)
        w.writerow(row)
    with open(os.path.join(folder, "histogram.csv"), "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["diagonal_count", "blocks_with_diagonals", "nnz_in_blocks"])
        for d in range(len(hist_b)):
            nnzd = int(hist_n[d]) if d < len(hist_n) else 0
            if hist_b[d] > 0 or nnzd > 0:
                w.writerow([d, int(hist_b[d]), nnzd])
