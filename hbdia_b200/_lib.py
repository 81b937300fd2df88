"""ctypes binding of libhbdia_b200.so (the C ABI in include/hbdia_b200.h).

There is no fallback: if the shared library is missing the import fails with
instructions to build it.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhbdia_b200.so")

c_i32, c_i64, c_u64, c_dbl, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double, ctypes.c_void_p
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_vpp = ctypes.POINTER(ctypes.c_void_p)

HBDIA_OK = 0
HBDIA_ERR_INVALID_ARGUMENT = -1
HBDIA_ERR_OUT_OF_RANGE = -2
HBDIA_ERR_RUNTIME = -3
HBDIA_ERR_CUDA = -4
HBDIA_ERR_NO_MEMORY = -5
HBDIA_ERR_NOT_CONVERTED = -6
HBDIA_ERR_UNSUPPORTED = -7
HBDIA_ERR_DEVICE_TIMEOUT = -8

KERNEL_AUTO, KERNEL_ROWWISE, KERNEL_WARP, KERNEL_STAGED, KERNEL_PIPE, KERNEL_QUAD = 0, 1, 2, 3, 4, 5
TUNE_UNROLL, TUNE_SPMM_TILE, TUNE_PREFETCH, TUNE_TAIL, TUNE_STAGES, TUNE_QUAD_GROUP = 1, 2, 3, 4, 5, 6

HBDIA_F64, HBDIA_F32 = 0, 1
BATCH_CONCURRENT, BATCH_QUEUE = 0, 1
REQ_SPMV, REQ_CG = 0, 1
STORE_NATIVE, STORE_F32, STORE_BF16_SCALED, STORE_F32_QUAD, STORE_BF16_QUAD = 0, 1, 2, 3, 4


class MatrixInfo(ctypes.Structure):
    _fields_ = [
        ("dtype", c_i32), ("numRows", c_i32), ("numCols", c_i32), ("hasCOO", c_i32),
        ("numNonZeros", c_i64), ("hasHBDIA", c_i32), ("onDevice", c_i32),
        ("blockWidth", c_i32), ("threshold", c_i32), ("maxCooEntries", c_i64),
        ("numBlocks", c_i32), ("numberDiagonals", c_i32), ("totalOffsets", c_i64),
        ("numSlots", c_i64), ("numCoo", c_i64), ("histogramLength", c_i32), ("storage", c_i32),
        ("deviceBytes", c_i64), ("bytesPerSpmv", c_i64),
    ]


class TuneResult(ctypes.Structure):
    _fields_ = [("kernel", c_i32), ("unroll", c_i32), ("spmmTile", c_i32), ("fromCache", c_i32),
                ("msPerCall", ctypes.c_float)]


class CgOptions(ctypes.Structure):
    _fields_ = [("tol", c_dbl), ("updateFactor", c_dbl), ("maxUpdates", c_i32), ("maxIterations", c_i32),
                ("iterStorage", c_i32), ("checkEvery", c_i32)]


class CgResult(ctypes.Structure):
    _fields_ = [("updates", c_i32), ("iterations", c_i32), ("converged", c_i32),
                ("relResidual", c_dbl), ("seconds", c_dbl)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("schedule", c_i32), ("streams", c_i32), ("threadsPerBlock", c_i32), ("tilesPerGrab", c_i32),
                ("rhsTile", c_i32), ("useGraph", c_i32)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("memoryBudget", c_i64), ("batching", c_i32), ("maxRhs", c_i32), ("spmvStorage", c_i32),
                ("cgIterStorage", c_i32), ("cgWorkers", c_i32), ("cgMaxUpdates", c_i32), ("cgMaxIterations", c_i32),
                ("cgCheckEvery", c_i32), ("cgTol", c_dbl), ("cgUpdateFactor", c_dbl),
                ("maxInFlight", c_i32), ("cgMaxGroup", c_i32)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", c_i32), ("kind", c_i32), ("matrix", c_i32), ("batchRhs", c_i32),
                ("submitted", c_dbl), ("started", c_dbl), ("finished", c_dbl),
                ("cgUpdates", c_i32), ("cgIterations", c_i32), ("cgRelResidual", c_dbl)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", c_i64), ("spmvRequests", c_i64), ("cgRequests", c_i64), ("spmvSteps", c_i64),
                ("spmvLaunches", c_i64), ("deviceBytes", c_i64), ("matrices", c_i32), ("cgGroups", c_i64)]


class StorageCosts(ctypes.Structure):
    _fields_ = [("hbdia", c_i64), ("coo", c_i64), ("dia", c_i64), ("sell", c_i64), ("csr", c_i64)]


class PartialInfo(ctypes.Structure):
    _fields_ = [("isPartial", c_i32), ("hasMetadata", c_i32), ("globalRowStart", c_i32),
                ("numGlobalRows", c_i32), ("numGlobalCols", c_i32), ("rank", c_i32), ("size", c_i32),
                ("numGlobalNonZeros", c_i64), ("numDataRanges", c_i64), ("numProcessRanges", c_i64),
                ("totalBufferSize", c_i64), ("leftBufferSize", c_i64), ("rightBufferSize", c_i64),
                ("windowStart", c_i32), ("windowLength", c_i32)]


class LayoutDesc(ctypes.Structure):
    _fields_ = [("dtype", c_i32), ("storage", c_i32), ("numRows", c_i32), ("numCols", c_i32),
                ("blockWidth", c_i32), ("numBlocks", c_i32), ("totalOffsets", c_i64), ("numCoo", c_i64),
                ("values", c_vp), ("scales", c_vp), ("offsets", c_vp), ("blockStart", c_vp), ("cooRow", c_vp),
                ("cooCol", c_vp), ("cooVal", c_vp), ("cooRowPtr", c_vp)]


class DeviceArrays(ctypes.Structure):
    _fields_ = [("hbdiaData", c_vp), ("flattenedOffsets", c_vp), ("blockStartIndices", c_vp),
                ("blockSizes", c_vp), ("flattenedVectorOffsets", c_vp), ("cpuRowIndices", c_vp),
                ("cpuColIndices", c_vp), ("cpuValues", c_vp), ("cpuRowPtr", c_vp)]


class HBDIACudaError(RuntimeError):
    """A CUDA runtime call inside the library failed."""


class HBDIADeviceTimeout(RuntimeError):
    """A bounded wait inside an SpMV kernel ran out; that result is invalid."""


_EXC = {
    HBDIA_ERR_INVALID_ARGUMENT: ValueError,
    HBDIA_ERR_OUT_OF_RANGE: IndexError,
    HBDIA_ERR_RUNTIME: RuntimeError,
    HBDIA_ERR_CUDA: HBDIACudaError,
    HBDIA_ERR_NO_MEMORY: MemoryError,
    HBDIA_ERR_NOT_CONVERTED: RuntimeError,
    HBDIA_ERR_UNSUPPORTED: NotImplementedError,
    HBDIA_ERR_DEVICE_TIMEOUT: HBDIADeviceTimeout,
}

# (name, restype, argtypes)
_SIGS = [
    ("hbdia_last_error", ctypes.c_char_p, []),
    ("hbdia_version", ctypes.c_char_p, []),
    ("hbdia_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("hbdia_set_device", ctypes.c_int, [c_i32]),
    ("hbdia_get_device", ctypes.c_int, [c_i32p]),
    ("hbdia_matrix_create_empty", ctypes.c_int, [ctypes.c_int, c_vpp]),
    ("hbdia_matrix_create", ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, c_i64, c_i32, c_i32, c_vpp]),
    ("hbdia_matrix_destroy", None, [c_vp]),
    ("hbdia_matrix_stencil27", ctypes.c_int, [c_vp, c_i32, c_i32, c_i32, c_dbl, c_i32]),
    ("hbdia_matrix_load_mtx", ctypes.c_int, [c_vp, ctypes.c_char_p, c_i32, c_i32, c_i32p]),
    ("hbdia_matrix_convert", ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, c_i32, c_i32, c_i32]),
    ("hbdia_matrix_prepare_gpu", ctypes.c_int, [c_vp, c_i32]),
    ("hbdia_matrix_convert_on_device", ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, c_i32]),
    ("hbdia_matrix_remove_duplicates", ctypes.c_int, [c_vp]),
    ("hbdia_matrix_convert_dia", ctypes.c_int, [c_vp, c_i32]),
    ("hbdia_matrix_dia_info", ctypes.c_int, [c_vp, c_i32p, c_i32p, c_i32p]),
    ("hbdia_matrix_export_dia", ctypes.c_int, [c_vp, c_vp, c_vp]),
    ("hbdia_matrix_storage_costs", ctypes.c_int, [c_vp, ctypes.POINTER(StorageCosts)]),
    ("hbdia_matrix_get_info", ctypes.c_int, [c_vp, ctypes.POINTER(MatrixInfo)]),
    ("hbdia_matrix_export_layout", ctypes.c_int, [c_vp] * 10),
    ("hbdia_matrix_export_coo", ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    ("hbdia_matrix_export_nnz_per_row", ctypes.c_int, [c_vp, c_vp]),
    ("hbdia_matrix_stream", ctypes.c_int, [c_vp, c_vpp]),
    ("hbdia_matrix_device_arrays", ctypes.c_int, [c_vp, ctypes.POINTER(DeviceArrays)]),
    ("hbdia_allocation_count", ctypes.c_int, [c_i64p, c_i64p]),
    ("hbdia_matrix_synchronize", ctypes.c_int, [c_vp]),
    ("hbdia_matrix_device_status", ctypes.c_int, [c_vp, c_i32p]),
    ("hbdia_matrix_set_kernel", ctypes.c_int, [c_vp, c_i32]),
    ("hbdia_matrix_selected_kernel", ctypes.c_int, [c_vp, c_vp, c_i32p]),
    ("hbdia_matrix_set_wait_timeout", ctypes.c_int, [c_vp, c_u64]),
    ("hbdia_matrix_set_tuning", ctypes.c_int, [c_vp, c_i32, c_i32]),
    ("hbdia_matrix_autotune", ctypes.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_i32, c_vp, c_i32,
                                             ctypes.POINTER(TuneResult)]),
    ("hbdia_autotune_clear", ctypes.c_int, []),
    ("hbdia_matrix_test_skip_tile", ctypes.c_int, [c_vp, c_i32]),
    ("hbdia_vector_create", ctypes.c_int, [ctypes.c_int, c_vp, c_i64, c_vpp]),
    ("hbdia_vector_destroy", None, [c_vp]),
    ("hbdia_vector_device_ptr", ctypes.c_int, [c_vp, c_vpp]),
    ("hbdia_vector_coo_results_ptr", ctypes.c_int, [c_vp, c_vpp]),
    ("hbdia_vector_size", ctypes.c_int, [c_vp, c_i64p]),
    ("hbdia_vector_upload", ctypes.c_int, [c_vp, c_vp]),
    ("hbdia_vector_download", ctypes.c_int, [c_vp, c_vp]),
    ("hbdia_spmv", ctypes.c_int, [c_vp, c_vp, c_vp, c_i32, c_i32]),
    ("hbdia_spmv_device", ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    ("hbdia_spmm_device", ctypes.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_i32, c_vp]),
    ("hbdia_spmm_device_colmajor", ctypes.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_i32, c_vp]),
    ("hbdia_spmv_host", ctypes.c_int, [c_vp, c_vp, c_vp]),
    ("hbdia_spmv_host_noalloc", ctypes.c_int, [c_vp, c_vp, c_vp]),
    ("hbdia_generate_stencil27", ctypes.c_int,
     [c_i32, c_i32, c_i32, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl, c_u64, c_i64p, c_vp, c_vp, c_vp]),
    ("hbdia_generate_stencil7", ctypes.c_int, [c_i32, c_i32, c_i32, c_dbl, c_dbl, c_i64p, c_vp, c_vp, c_vp]),
    ("hbdia_generate_banded", ctypes.c_int,
     [c_i32, c_vp, c_i32, c_dbl, c_dbl, c_dbl, c_dbl, c_u64, c_i64p, c_vp, c_vp, c_vp]),
    ("hbdia_fill_uniform", ctypes.c_int, [c_vp, c_i64, c_dbl, c_dbl, c_u64]),
    ("hbdia_generate_stencil27_spd", ctypes.c_int,
     [c_i32, c_i32, c_i32, c_dbl, c_dbl, c_u64, c_i64p, c_vp, c_vp, c_vp]),
    ("hbdia_cg_solve", ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.POINTER(CgOptions), c_vp, ctypes.POINTER(CgResult)]),
    ("hbdia_batch_create", ctypes.c_int, [c_vpp, c_i32, c_vpp]),
    ("hbdia_batch_destroy", None, [c_vp]),
    ("hbdia_batch_bind", ctypes.c_int, [c_vp, c_vpp, c_i64p, c_vpp, c_i64p, c_i32p]),
    ("hbdia_batch_run", ctypes.c_int, [c_vp, c_vp]),
    ("hbdia_batch_set_config", ctypes.c_int, [c_vp, ctypes.POINTER(BatchConfig)]),
    ("hbdia_batch_get_config", ctypes.c_int, [c_vp, ctypes.POINTER(BatchConfig)]),
    ("hbdia_batch_autotune", ctypes.c_int, [c_vp, c_vp, ctypes.POINTER(ctypes.c_float), c_i32p]),
    ("hbdia_batch_info", ctypes.c_int, [c_vp, c_i32p, c_i32p, c_i64p]),
    ("hbdia_batch_stream", ctypes.c_int, [c_vp, c_vpp]),
    ("hbdia_server_default_options", None, [ctypes.POINTER(ServerOptions)]),
    ("hbdia_server_create", ctypes.c_int, [ctypes.POINTER(ServerOptions), c_vpp]),
    ("hbdia_server_destroy", None, [c_vp]),
    ("hbdia_server_add_matrix", ctypes.c_int, [c_vp, c_vp, c_i32p]),
    ("hbdia_server_submit", ctypes.c_int, [c_vp, c_i32, c_i32, c_vp, c_vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("hbdia_server_pause", ctypes.c_int, [c_vp, c_i32]),
    ("hbdia_server_wait", ctypes.c_int, [c_vp, ctypes.c_uint64, ctypes.POINTER(RequestInfo)]),
    ("hbdia_server_get_stats", ctypes.c_int, [c_vp, ctypes.POINTER(ServerStats)]),
    ("hbdia_matrix_create_partial", ctypes.c_int, [c_i32, c_vp, c_vp, c_vp, c_i64, c_i32, c_i32, c_i32, c_i64,
                                                   c_i32, c_i32, c_i32, c_vpp]),
    ("hbdia_matrix_partition", ctypes.c_int, [c_vp, c_i32, c_i32, c_vpp]),
    ("hbdia_matrix_partial_info", ctypes.c_int, [c_vp, ctypes.POINTER(PartialInfo)]),
    ("hbdia_matrix_export_ranges", ctypes.c_int, [c_vp, c_vp, c_vp]),
    ("hbdia_halo_create", ctypes.c_int, [c_i32, c_vp, c_vp, c_vp, c_i32, c_i64, c_i64, c_vpp]),
    ("hbdia_halo_copy", ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    ("hbdia_halo_elements", c_i64, [c_vp]),
    ("hbdia_halo_destroy", None, [c_vp]),
    ("hbdia_spmv_list_device", ctypes.c_int, [c_vp, c_vpp, c_vpp, c_i32, c_vp]),
    ("hbdia_spmv_host_many", ctypes.c_int, [c_vp, c_vpp, c_vpp, c_i32]),
    ("hbdia_plan_create", ctypes.c_int, [ctypes.POINTER(LayoutDesc), c_vpp]),
    ("hbdia_plan_spmv", ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    ("hbdia_plan_spmm", ctypes.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_i32, c_vp]),
    ("hbdia_plan_destroy", None, [c_vp]),
    ("hbdia_server_submit_device", ctypes.c_int, [c_vp, c_i32, c_i32, c_vp, c_vp, ctypes.POINTER(ctypes.c_uint64)]),
]

# every C-ABI entry point (the exported-symbol check in the tests uses this list)
EXPORTED = [s[0] for s in _SIGS]

_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -m hbdia_b200.build, or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != HBDIA_OK:
        lib = load()
        msg = lib.hbdia_last_error().decode(errors="replace")
        name = lib.hbdia_status_string(status).decode()
        raise _EXC.get(status, RuntimeError)(f"{name}: {msg}")
