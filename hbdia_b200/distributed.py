"""Row-partitioned SpMV over several GPUs, one process per GPU.

Python mirror of the reference's DataExchange layer (src/DataExchange/*):

* :class:`BasicExtractor` -- row-wise partitioning (BasicExtractor.cpp:16-234);
* :class:`Distributor`    -- BasicDistributor + MPICommunicator: scatterMatrix /
  receiveMatrix, scatterVector / receiveVector, exchangeData, gatherVector,
  verifyDataExchange (BasicDistributor.cpp:17-251, MPICommunicator.cpp:253-543);
* :class:`PartialVector`  -- ``HBDIAVector(localData, matrix, rank, size)``
  (src/Format/HBDIAVector.cpp:39-66).

MPI is replaced by ``torch.distributed``: NCCL between GPUs, gloo between CPU
processes (which carries the same host logic, without a GPU).

Each rank keeps its partial matrix's plan and an x WINDOW in HBM -- the dense
range of global columns its rows read (``HBDIA.window()``) -- so the local
SpMV is the single-GPU fused kernel unchanged.  ``exchangeData`` fills the
window's halo: each rank packs the x ranges every peer asked for into one
send buffer (one halo-copy kernel), the buffers travel by batched NCCL
send/recv over NVLink, and one kernel unpacks what arrived into the window.
Which ranges a peer asks for is agreed once per matrix; the reference
renegotiates counts and tuples on every call (MPICommunicator.cpp:266-350).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch
import torch.distributed as dist

from . import HBDIA, _lib, set_device, spmv_device
from ._lib import check as _check, load as _load

__all__ = ["MatrixData", "Partition", "VectorPartition", "BasicExtractor", "PartialVector", "Distributor",
           "HaloExchange", "ROW_WISE"]

ROW_WISE = 0  # HBDIAExtractor::PartitioningStrategy::ROW_WISE (include/DataExchange/HBDIAExtractor.hpp:36-38)


@dataclass
class MatrixData:
    """include/DataExchange/HBDIAExtractor.hpp:9-16."""
    numGlobalRows: int
    numGlobalCols: int
    numGlobalNonZeros: int
    numLocalRows: int
    numLocalCols: int
    numLocalNonZeros: int


@dataclass
class Partition:
    """include/DataExchange/HBDIAExtractor.hpp:18-24."""
    localRowIndices: np.ndarray
    localColIndices: np.ndarray
    localValues: np.ndarray
    globalRowMapping: np.ndarray


@dataclass
class VectorPartition:
    localValues: np.ndarray = field(default_factory=lambda: np.zeros(0))


def _row_split(n: int, P: int):
    """Rows of each partition: n // P, the last one taking n % P more
    (BasicExtractor.cpp:97-122, 140-175)."""
    rpp = n // P
    starts = [p * rpp for p in range(P)]
    counts = [rpp + (n % P if p == P - 1 else 0) for p in range(P)]
    return starts, counts


class BasicExtractor:
    """Row-wise partitioning of a matrix and a vector (BasicExtractor.cpp)."""

    def __init__(self):
        self._strategy = ROW_WISE
        self._matrixData: List[MatrixData] = []
        self._partitions: List[Partition] = []
        self._handles: List[HBDIA] = []
        self._vectorPartitions: List[VectorPartition] = []

    def setPartitioningStrategy(self, strategy: int) -> None:
        if strategy != ROW_WISE:
            raise ValueError("Unknown partitioning strategy")
        self._strategy = strategy

    def createMatrixPartitions(self, matrix: HBDIA, numProcesses: int) -> bool:
        if numProcesses <= 0:
            raise ValueError(f"Invalid number of processes: {numProcesses}")
        self.clearMatrixPartitions()
        info = matrix.info()
        for p in range(numProcesses):
            part = matrix.partition(numProcesses, p)
            r, c, v = part._coo()
            pi = part.partialInfo()
            nl = part.getNumRows()
            self._handles.append(part)
            self._partitions.append(Partition(r, c, v, np.arange(pi.globalRowStart, pi.globalRowStart + nl,
                                                                 dtype=np.int32)))
            self._matrixData.append(MatrixData(info.numRows, info.numCols, int(info.numNonZeros), nl,
                                               info.numCols, len(v)))
        return True

    def createVectorPartitions(self, globalVector, numProcesses: int) -> bool:
        g = np.asarray(globalVector)
        if numProcesses <= 0:
            raise ValueError(f"Invalid number of processes: {numProcesses}")
        if g.size == 0:
            raise ValueError("Global vector is empty")
        starts, counts = _row_split(len(g), numProcesses)
        self._vectorPartitions = [VectorPartition(g[s:s + c].copy()) for s, c in zip(starts, counts)]
        return True

    def extractPartialMatrixMetadata(self, matrix: HBDIA, numProcesses: int) -> None:
        """The metadata (BasicExtractor.cpp:269-333) is computed when the
        partial matrix is converted; this checks the process count agrees."""
        if matrix.isPartialMatrix() and matrix.partialInfo().size != numProcesses:
            raise ValueError("the matrix was partitioned for a different number of processes")

    def getMatrixData(self) -> List[MatrixData]: return self._matrixData
    def getPartitions(self) -> List[Partition]: return self._partitions
    def getVectorPartitions(self) -> List[VectorPartition]: return self._vectorPartitions

    def clearMatrixPartitions(self) -> None:
        self._matrixData, self._partitions, self._handles = [], [], []

    def clearVectorPartitions(self) -> None:
        self._vectorPartitions = []


_TORCH_DTYPE = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}


class PartialVector:
    """``HBDIAVector(localData, matrix, rank, size)``: this rank's x entries
    and the entries other ranks send, as one dense window of global columns
    in device memory (x_window[c - windowStart] = x[c]).  getLocalSize /
    getTotalSize keep the reference's meaning (local; left + local + right)."""

    def __init__(self, localData, matrix: HBDIA, rank: Optional[int] = None, size: Optional[int] = None,
                 device=None):
        info = matrix.partialInfo()
        if not info.isPartial:
            raise ValueError("PartialVector needs a partial matrix")
        if rank is not None and rank != info.rank or size is not None and size != info.size:
            raise ValueError("rank / size differ from the matrix's")
        self.dtype = matrix.dtype
        data = np.ascontiguousarray(localData, self.dtype)
        nl = matrix.getNumRows()
        if len(data) != nl:
            raise ValueError(f"local data holds {len(data)} entries, the matrix has {nl} rows")
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        self.windowStart, wlen = matrix.window()
        self.window = torch.zeros(wlen, dtype=_TORCH_DTYPE[self.dtype], device=self.device)
        lo = info.globalRowStart - self.windowStart
        self.local = self.window[lo:lo + nl]
        self.local.copy_(torch.from_numpy(data))
        self.globalRowStart = info.globalRowStart
        self.leftSize = int(info.leftBufferSize)
        self.rightSize = int(info.rightBufferSize)

    def getLocalSize(self) -> int: return self.local.numel()
    def getTotalSize(self) -> int: return self.leftSize + self.local.numel() + self.rightSize
    def getDeviceDataPtr(self) -> int: return self.window.data_ptr()
    def getDeviceLocalPtr(self) -> int: return self.local.data_ptr()
    def toHost(self) -> np.ndarray: return self.local.cpu().numpy()

    def globalValue(self, col: int):
        """x[col] as this rank holds it (inside the window)."""
        return self.window[col - self.windowStart].item()


class _HaloPlan:
    """One direction of the exchange (pack or unpack): element segments
    between two buffers, run by the library's halo-copy kernel on CUDA
    tensors.  CPU tensors (gloo ranks) use an index copy instead; that branch
    only carries the host logic between CPU processes -- a CUDA tensor never
    takes it."""

    def __init__(self, src_off, dst_off, length, src_len: int, dst_len: int, elem_bytes: int, device):
        self.device = device
        self.n = int(np.sum(length)) if len(length) else 0
        so = np.ascontiguousarray(src_off, np.int64)
        do = np.ascontiguousarray(dst_off, np.int64)
        ln = np.ascontiguousarray(length, np.int64)
        self._h = ctypes.c_void_p()
        if device.type == "cuda":
            _check(_load().hbdia_halo_create(elem_bytes, so.ctypes.data, do.ctypes.data, ln.ctypes.data, len(ln),
                                             int(src_len), int(dst_len), ctypes.byref(self._h)))
        else:
            if np.any(so + ln > src_len) or np.any(do + ln > dst_len) or np.any(so < 0) or np.any(do < 0):
                raise IndexError("halo segment outside its buffers")
            idx = [np.arange(a, a + k) for a, k in zip(so, ln)]
            jdx = [np.arange(a, a + k) for a, k in zip(do, ln)]
            self._src = torch.from_numpy(np.concatenate(idx) if idx else np.zeros(0, np.int64))
            self._dst = torch.from_numpy(np.concatenate(jdx) if jdx else np.zeros(0, np.int64))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _load().hbdia_halo_destroy(h)
            self._h = None

    def __call__(self, src: torch.Tensor, dst: torch.Tensor) -> None:
        if self.n == 0:
            return
        if self.device.type == "cuda":
            stream = torch.cuda.current_stream(src.device).cuda_stream
            _check(_load().hbdia_halo_copy(self._h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                           ctypes.c_void_p(stream)))
        else:
            dst.index_copy_(0, self._dst, src.index_select(0, self._src))


class HaloExchange:
    """The agreed exchange of one partial matrix's x window.

    Built collectively (every rank of the group, once per matrix): the ranks
    share their processDataRanges, so each knows which of its own x ranges
    every peer needs (MPICommunicator.cpp:266-350 does this per call)."""

    def __init__(self, matrix: HBDIA, group=None, device=None):
        info, _, proc = matrix._ranges()
        self.rank, self.size = int(info.rank), int(info.size)
        if dist.get_world_size(group) != self.size or dist.get_rank(group) != self.rank:
            raise ValueError("the matrix was partitioned for another process group layout")
        self.group = group
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        self.windowStart, self.windowLength = matrix.window()
        gathered: List = [None] * self.size
        dist.all_gather_object(gathered, (proc.tolist(), self.windowStart), group=group)
        me, wlo = self.rank, self.windowStart
        recv = {q: [(s, e) for p, s, e in proc.tolist() if p == q] for q in range(self.size) if q != me}
        send = {q: [(s, e) for p, s, e in gathered[q][0] if p == me] for q in range(self.size) if q != me}
        self.peers = [q for q in range(self.size) if q != me]
        elem = np.dtype(matrix.dtype).itemsize
        self.dtype = _TORCH_DTYPE[np.dtype(matrix.dtype)]

        def table(segs_by_peer, window_is_src):
            so, do, ln, counts = [], [], [], {}
            pos = 0
            for q in self.peers:
                start = pos
                for s, e in segs_by_peer[q]:
                    if window_is_src:
                        so.append(s - wlo); do.append(pos)
                    else:
                        so.append(pos); do.append(s - wlo)
                    ln.append(e - s)
                    pos += e - s
                counts[q] = (start, pos - start)
            return so, do, ln, counts, pos

        so, do, ln, self.sendCounts, self.sendTotal = table(send, True)
        self.pack = _HaloPlan(so, do, ln, self.windowLength, self.sendTotal, elem, self.device)
        so, do, ln, self.recvCounts, self.recvTotal = table(recv, False)
        self.unpack = _HaloPlan(so, do, ln, self.recvTotal, self.windowLength, elem, self.device)
        self.sendBuf = torch.empty(self.sendTotal, dtype=self.dtype, device=self.device)
        self.recvBuf = torch.empty(self.recvTotal, dtype=self.dtype, device=self.device)

    def bytesPerExchange(self) -> int:
        """Bytes this rank sends per exchange (what crosses NVLink from it)."""
        return self.sendTotal * self.sendBuf.element_size()

    def run(self, window: torch.Tensor) -> None:
        """Fill the halo parts of ``window`` from the peers' local x."""
        if window.numel() != self.windowLength or window.device != self.device:
            raise ValueError("window does not match this exchange")
        self.pack(window, self.sendBuf)
        ops = []
        for q in self.peers:
            s0, sn = self.sendCounts[q]
            r0, rn = self.recvCounts[q]
            if sn:
                ops.append(dist.P2POp(dist.isend, self.sendBuf[s0:s0 + sn], q, self.group))
            if rn:
                ops.append(dist.P2POp(dist.irecv, self.recvBuf[r0:r0 + rn], q, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        self.unpack(self.recvBuf, window)


class Distributor:
    """BasicDistributor<T> over MPICommunicator<T>, on torch.distributed.

    ``device``: where partial matrices get their plans and PartialVectors
    their windows -- the rank's GPU (NCCL), or the CPU (gloo ranks, host
    logic only: no SpMV there)."""

    def __init__(self, group=None, rootProcess: int = 0, device=None, blockWidth: int = 32, threshold: int = 1,
                 maxCooEntries: int = 1_000_000_000):
        if not dist.is_initialized():
            raise RuntimeError("Communicator not initialized")
        self.group = group
        self.rootProcess = rootProcess
        self._rank = dist.get_rank(group)
        self._size = dist.get_world_size(group)
        backend = dist.get_backend(group)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        self.device = torch.device(device)
        if self.device.type == "cuda":  # the library's own runtime follows the rank's GPU
            set_device(self.device.index if self.device.index is not None else torch.cuda.current_device())
        # NCCL moves device tensors only; gloo moves host tensors
        self._comm = self.device if backend == "nccl" else torch.device("cpu")
        self.blockWidth, self.threshold, self.maxCooEntries = blockWidth, threshold, maxCooEntries
        self.extractor = BasicExtractor()
        self._exchanges: Dict[int, HaloExchange] = {}

    def getRank(self) -> int: return self._rank
    def getSize(self) -> int: return self._size
    def getRootProcess(self) -> int: return self.rootProcess
    def isRootProcess(self) -> bool: return self._rank == self.rootProcess
    def getExtractor(self) -> BasicExtractor: return self.extractor

    def setPartitioningStrategy(self, strategy: int) -> None:
        self.extractor.setPartitioningStrategy(strategy)

    # ---- point-to-point helpers
    def _send(self, t: torch.Tensor, dst: int) -> None:
        dist.send(t.to(self._comm), dst, group=self.group)

    def _recv(self, shape, dtype, src: int) -> torch.Tensor:
        t = torch.empty(shape, dtype=dtype, device=self._comm)
        dist.recv(t, src, group=self.group)
        return t.cpu()

    def _convert(self, m: HBDIA) -> HBDIA:
        # BasicDistributor.cpp:71-78: convert, analyse ranges, metadata, prepareForGPU
        m.convertToHBDIAFormat(self.blockWidth, self.threshold, self.maxCooEntries,
                               upload=self.device.type == "cuda")
        return m

    # ---- matrix
    def scatterMatrix(self, globalMatrix: HBDIA) -> HBDIA:
        """Root: partition, send every rank its part, keep the root's
        (BasicDistributor.cpp:17-88)."""
        if not self.isRootProcess():
            raise RuntimeError("scatterMatrix should only be called by root process")
        ex = self.extractor
        ex.createMatrixPartitions(globalMatrix, self._size)
        vdt = _TORCH_DTYPE[np.dtype(globalMatrix.dtype)]
        for p in range(self._size):
            if p == self.rootProcess:
                continue
            md, pt = ex.getMatrixData()[p], ex.getPartitions()[p]
            hdr = torch.tensor([md.numGlobalRows, md.numGlobalCols, md.numGlobalNonZeros, md.numLocalRows,
                                md.numLocalCols, md.numLocalNonZeros, int(pt.globalRowMapping[0]),
                                int(np.dtype(globalMatrix.dtype) == np.float32)], dtype=torch.int64)
            self._send(hdr, p)
            if md.numLocalNonZeros:
                self._send(torch.from_numpy(pt.localRowIndices), p)
                self._send(torch.from_numpy(pt.localColIndices), p)
                self._send(torch.from_numpy(pt.localValues).to(vdt), p)
        local = ex._handles[self.rootProcess]
        ex.clearMatrixPartitions()
        return self._convert(local)

    def receiveMatrix(self) -> HBDIA:
        """Other ranks: receive the partition, build and convert the partial
        matrix (BasicDistributor.cpp:90-146)."""
        if self.isRootProcess():
            raise RuntimeError("receiveMatrix should not be called by root process")
        hdr = self._recv((8,), torch.int64, self.rootProcess).tolist()
        nGR, nGC, nGNZ, nLR, nLC, nLNZ, start, f32 = hdr
        dtype = np.float32 if f32 else np.float64
        if nLNZ:
            r = self._recv((nLNZ,), torch.int32, self.rootProcess).numpy()
            c = self._recv((nLNZ,), torch.int32, self.rootProcess).numpy()
            v = self._recv((nLNZ,), _TORCH_DTYPE[np.dtype(dtype)], self.rootProcess).numpy()
        else:
            r = c = np.zeros(0, np.int32)
            v = np.zeros(0, dtype)
        m = HBDIA.partial(r, c, v, nLR, nLC, np.arange(start, start + nLR), True, nGR, nGC, nGNZ,
                          self._rank, self._size, dtype=dtype)
        return self._convert(m)

    # ---- vector
    def scatterVector(self, globalVector) -> np.ndarray:
        if not self.isRootProcess():
            raise RuntimeError("scatterVector should only be called by root process")
        ex = self.extractor
        ex.createVectorPartitions(globalVector, self._size)
        parts = ex.getVectorPartitions()
        for p in range(self._size):
            if p == self.rootProcess:
                continue
            v = parts[p].localValues
            self._send(torch.tensor([len(v), int(v.dtype == np.float32)], dtype=torch.int64), p)
            self._send(torch.from_numpy(np.ascontiguousarray(v)), p)
        out = parts[self.rootProcess].localValues
        ex.clearVectorPartitions()
        return out

    def receiveVector(self) -> np.ndarray:
        if self.isRootProcess():
            raise RuntimeError("receiveVector should not be called by root process")
        n, f32 = self._recv((2,), torch.int64, self.rootProcess).tolist()
        return self._recv((n,), torch.float32 if f32 else torch.float64, self.rootProcess).numpy()

    # ---- exchange and gather
    def _exchange_for(self, matrix: HBDIA) -> HaloExchange:
        key = matrix.handle.value
        ex = self._exchanges.get(key)
        if ex is None:
            ex = HaloExchange(matrix, self.group, self.device)
            self._exchanges[key] = ex
        return ex

    def exchangeData(self, matrix: HBDIA, vector: PartialVector) -> bool:
        """Fill the halo of ``vector``'s window from the other ranks
        (MPICommunicator::exchangeData, MPICommunicator.cpp:253-412).  Every
        rank of the group calls it; the first call per matrix agrees the
        ranges (a collective)."""
        self._exchange_for(matrix).run(vector.window)
        return True

    def verifyDataExchange(self, matrix: HBDIA, vector: PartialVector) -> bool:
        """MPICommunicator::verifyDataExchange (MPICommunicator.cpp:414-488):
        for x[i] = i, every received entry and every local entry must equal
        its global index."""
        meta = matrix.getPartialMatrixMetadata()
        w = vector.window.cpu().numpy()
        ok = True
        for q, ranges in enumerate(meta["processDataRanges"]):
            if q == self._rank:
                continue
            for s, e in ranges:
                got = w[s - vector.windowStart:e - vector.windowStart]
                ok &= bool(np.array_equal(got, np.arange(s, e, dtype=got.dtype)))
        loc = vector.toHost()
        ok &= bool(np.array_equal(loc, np.arange(vector.globalRowStart, vector.globalRowStart + len(loc),
                                                 dtype=loc.dtype)))
        return ok

    def spmv(self, matrix: HBDIA, x: PartialVector, y: torch.Tensor, stream: Optional[int] = None) -> None:
        """This rank's rows of y = A x: exchangeData, then the fused SpMV over
        the window (hbdiaSpMV on a partial matrix).  A rank whose rows hold
        no entries gets y = 0."""
        self.exchangeData(matrix, x)
        if y.numel() != matrix.getNumRows():
            raise ValueError("y must hold the rank's rows")
        if not matrix.getHasHBDIA():
            y.zero_()
            return
        if y.device.type != "cuda":
            raise RuntimeError("the SpMV runs on the GPU: give CUDA tensors")
        spmv_device(matrix, x.window.data_ptr(), y.data_ptr(),
                    stream if stream is not None else torch.cuda.current_stream().cuda_stream)

    def gatherVector(self, localVector) -> Optional[np.ndarray]:
        """Concatenate every rank's rows on the root
        (MPICommunicator::gatherVectorData, MPICommunicator.cpp:490-532)."""
        loc = localVector.local if isinstance(localVector, PartialVector) else localVector
        loc = torch.as_tensor(loc)
        sizes: List = [None] * self._size
        dist.all_gather_object(sizes, int(loc.numel()), group=self.group)
        m = max(sizes)
        buf = torch.zeros(m, dtype=loc.dtype, device=self._comm)
        buf[:loc.numel()] = loc.to(self._comm)
        outs = [torch.empty_like(buf) for _ in range(self._size)]
        dist.all_gather(outs, buf, group=self.group)
        if not self.isRootProcess():
            return None
        return np.concatenate([o[:k].cpu().numpy() for o, k in zip(outs, sizes)])
