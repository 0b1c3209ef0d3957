"""hornet_b200: B200-native Hornet dynamic-graph hot path.

Python binding over the C ABI in include/hornet_b200.h (libhornet_b200.so,
built in-tree by hornet_b200/build.py).  The classes mirror the reference's
C++ names and argument meaning:

* ``HornetInit`` / ``Hornet`` (``HornetGPU``): hornet::HornetInit and
  hornet::gpu::Hornet (hornet/include/Core/Hornet.cuh:56-131);
* ``BatchUpdate``: hornet::gpu::BatchUpdate over a BatchUpdatePtr
  (hornet/include/Core/BatchUpdate/BatchUpdate.cuh:77-272);
* ``BfsTopDown``, ``TriangleCounting2``, ``CC``, ``KTruss``: the
  hornetsnest StaticAlgorithm subclasses (primitives/HornetAlg.cuh:51-150).

Arrays are numpy arrays (host) or CUDA tensors / objects exposing
``data_ptr()`` and ``is_cuda`` (device).  There is no CPU fallback: without
the compiled library every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhornet_b200.so")

HN_OK = 0
HN_ERR_INVALID = 1
HN_ERR_OOM = 2
HN_ERR_CAPACITY = 3
HN_ERR_TIMEOUT = 4
HN_ERR_CUDA = 5
HN_ERR_STATE = 6

HN_MEM_HOST = 0
HN_MEM_DEVICE = 1
HN_CSR_SORTED = 1
HN_DEDUP_BATCH = 1
HN_DEDUP_GRAPH = 2
HN_CC_MIN_ID = 0
HN_CC_REFERENCE = 1
HN_LB_BINARY_SEARCH = 0
HN_LB_VERTEX_BASED = 1

INF = 2147483647


class HornetError(RuntimeError):
    """A C-ABI call returned an HN_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class BfsStats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("visited", ctypes.c_int64), ("edges_scanned", ctypes.c_int64)]


class DeviceView(ctypes.Structure):
    _fields_ = [("nV", ctypes.c_int32), ("pad", ctypes.c_int32), ("nE", ctypes.c_int64),
                ("vtab", ctypes.c_void_p), ("pool", ctypes.c_void_p)]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_INT = ctypes.c_int
_D = ctypes.c_double

# name -> argtypes (all return int unless listed in _RESTYPES)
_SIGNATURES = {
    "hn_last_error_string": [],
    "hn_version": [],
    "hn_kernel_launches": [],
    "hn_profile_enable": [_INT],
    "hn_profile_report": [_P, _I64],
    "hn_graph_create_csr": [_I32, _I64, _P, _P, _U32, _INT, _INT, _P],
    "hn_graph_create_csr64": [_I32, _I64, _P, _P, _U32, _INT, _INT, _P],
    "hn_graph_reset_csr": [_P, _I32, _I64, _P, _P, _U32, _INT],
    "hn_graph_destroy": [_P],
    "hn_graph_set_stream": [_P, _P],
    "hn_graph_nv": [_P, _P],
    "hn_graph_ne": [_P, _P],
    "hn_graph_max_degree": [_P, _P, _P],
    "hn_graph_export_coo": [_P, _INT, _P, _P, _INT],
    "hn_graph_export_csr": [_P, _P, _P, _INT],
    "hn_graph_degrees": [_P, _P, _INT],
    "hn_graph_device_view": [_P, _P],
    "hn_graph_memory": [_P, _P, _P, _P],
    "hn_graph_adjacency_hash": [_P, _P],
    "hn_graph_view_create": [_P, _P, _P],
    "hn_graph_view_refresh": [_P],
    "hn_gather_int32": [_P, _P, _P, _I64, _P],
    "hn_segment_sum_u64": [_P, _P, _P, _I64, _P],
    "hn_read_bandwidth": [_P, _P, _I64, ctypes.c_int32, _P],
    "hn_batch_create": [_P, _I64, _P, _P, _INT, _P],
    "hn_batch_reset": [_P, _I64, _P, _P, _INT],
    "hn_batch_size": [_P, _P],
    "hn_batch_destroy": [_P],
    "hn_insert": [_P, _P, _U32, _P],
    "hn_erase": [_P, _P, _U32, _P],
    "hn_bfs": [_P, _I32, _P, _INT, _P],
    "hn_bfs_multi": [_P, _P, _I32, _P, _INT, _P],
    "hn_bfs_do": [_P, _P, _I32, _P, _INT, _P],
    "hn_bfs_level_trace": [_P, _I32, _P, _P, _P],
    "hn_bfs_validate": [_P, _I32, _P, _INT, _P],
    "hn_cc_validate": [_P, _P, _INT, _P],
    "hn_ktruss_validate": [_P, _I32, _P, _INT, _P],
    "hn_bfs_batch": [_P, _P, _P, _I32, _I32, _P, _INT, _P],
    "hn_tc": [_P, _P, _INT, _P],
    "hn_tc_local": [_P, _P, _I32, _P, _INT],
    "hn_tc_owner": [_P, _P, _INT, _P],
    "hn_update_coalesced": [_P, _I64, _P, _P, _P, _INT, _P, _P],
    "hn_insert_count_triangles": [_P, _P, _P, _P],
    "hn_ktruss_keep": [_P, _I32, _P, _P],
    "hn_graph_create_csr_w": [_I32, _I64, _P, _P, _P, ctypes.c_uint32, _INT, _INT, _P],
    "hn_graph_weighted": [_P, _P],
    "hn_graph_export_coo_w": [_P, _INT, _P, _P, _P, _INT],
    "hn_batch_create_w": [_P, _I64, _P, _P, _P, _INT, _P],
    "hn_batch_reset_w": [_P, _I64, _P, _P, _P, _INT],
    "hn_tune_set": [ctypes.c_char_p, _I64],
    "hn_tune_get": [ctypes.c_char_p, _P],
    "hn_tune_reset": [],
    "hn_tune_name": [_I32],
    "hn_cc": [_P, _INT, _P, _INT, _P],
    "hn_ktruss": [_P, _P, _P, _INT],
    "hn_for_all_edges_count": [_P, _P, _I32, _INT, _INT, _P],
    "hn_for_all_vertices_degree": [_P, _P],
    "hn_gen_rmat_host": [_I32, _I32, _I64, _D, _D, _D, _U64, _P, _P],
    "hn_gen_rmat_device": [_I32, _I32, _I64, _D, _D, _D, _U64, _P, _P, _INT],
    "hn_coo_to_csr_device": [_I32, _I64, _P, _P, _INT, _P, _P, _P],
    "hn_free_device": [_P],
    "hn_cc_csr_noalloc": [_I32, _P, _P, _P, _P, _P],
    "hn_csr_write_bin": [ctypes.c_char_p, _I32, _I32, _P, _P],
    "hn_csr_read_bin": [ctypes.c_char_p, _P, _P, _P, _P],
    "hn_csr_write_mtx": [ctypes.c_char_p, _I32, _I64, _P, _P],
    "hn_graph_write_bin": [_P, ctypes.c_char_p],
    "hn_graph_read_bin": [ctypes.c_char_p, _INT, _P],
}
_RESTYPES = {"hn_last_error_string": ctypes.c_char_p, "hn_kernel_launches": _I64,
             "hn_tune_name": ctypes.c_char_p}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libhornet_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m hornet_b200.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(l, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = l
    return _lib


def _check(rc: int) -> None:
    if rc != HN_OK:
        msg = lib().hn_last_error_string()
        raise HornetError(rc, msg.decode() if msg else "")


def last_error() -> str:
    return lib().hn_last_error_string().decode()


def kernel_launches() -> int:
    return int(lib().hn_kernel_launches())


def profile_enable(on: bool = True) -> None:
    """Bracket every library kernel with CUDA events (clears old records)."""
    _check(lib().hn_profile_enable(1 if on else 0))


def profile_report() -> dict:
    """{kernel: {"launches": n, "ms": total}} since profile_enable."""
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    _check(lib().hn_profile_report(buf, len(buf)))
    return json.loads(buf.value.decode())


# ---------------------------------------------------------------------------
# array plumbing
# ---------------------------------------------------------------------------

def _is_device(a) -> bool:
    return bool(getattr(a, "is_cuda", False))


def _ptr(a, dtype=None):
    """(pointer, mem_kind, keepalive) for a numpy array or CUDA tensor."""
    if a is None:
        return None, HN_MEM_HOST, None
    if _is_device(a):
        return ctypes.c_void_p(a.data_ptr()), HN_MEM_DEVICE, a
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(ctypes.c_void_p), HN_MEM_HOST, arr


def _ptr_u32(a):
    """Like _ptr for 32-bit edge weights: int32 / uint32 / float32 values
    are passed as their raw 32-bit patterns."""
    if _is_device(a):
        assert a.element_size() == 4, "weights must be 32-bit"
        return ctypes.c_void_p(a.data_ptr()), HN_MEM_DEVICE, a
    arr = np.ascontiguousarray(a)
    assert arr.dtype.itemsize == 4, "weights must be 32-bit"
    arr = arr.view(np.uint32)
    return arr.ctypes.data_as(ctypes.c_void_p), HN_MEM_HOST, arr


def _out_ptr(a):
    if _is_device(a):
        return ctypes.c_void_p(a.data_ptr()), HN_MEM_DEVICE
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p), HN_MEM_HOST


# ---------------------------------------------------------------------------
# graph + batches
# ---------------------------------------------------------------------------

class HornetInit:
    """hornet::HornetInit(nV, nE, csr_offsets, csr_edges)
    (hornet/include/Core/HornetInitialize/HornetInit.cuh:70-73).  Borrows
    the CSR until a Hornet is built from it."""

    def __init__(self, nV: int, nE: int, offsets, edges, sorted_adjacency: bool = False):
        self._nV = int(nV)
        self._nE = int(nE)
        self.offsets = offsets
        self.edges = edges
        self.sorted = bool(sorted_adjacency)
        self.weights = None

    def insertEdgeData(self, weights) -> None:
        """HornetInit::insertEdgeData (HornetInit.cuh:79-97) for one 32-bit
        field per edge: int32, uint32 or float32 values (kept as raw bits)."""
        self.weights = weights

    def nV(self) -> int:
        return self._nV

    def nE(self) -> int:
        return self._nE


class Hornet:
    """hornet::gpu::Hornet<int> (hornet/include/Core/Hornet.cuh:56-131)."""

    def __init__(self, init: HornetInit, device: int = 0):
        self._h = ctypes.c_void_p()
        self._device = device
        self._build(init, create=True)

    def _build(self, init: HornetInit, create: bool) -> None:
        off = init.offsets
        if _is_device(off):
            use64 = str(off.dtype).endswith("int64")
        else:
            off = np.asarray(off)
            use64 = off.dtype == np.int64 or init.nE() > 0x7FFFFFFF
            off = np.ascontiguousarray(off, dtype=np.int64 if use64 else np.int32)
        po, mem, keep_o = _ptr(off)
        pa, mem_a, keep_a = _ptr(init.edges, np.int32)
        assert mem == mem_a, "offsets and edges must live in the same memory"
        flags = HN_CSR_SORTED if init.sorted else 0
        if create and init.weights is not None:
            assert not use64, "weighted graphs take int32 offsets"
            pw, mem_w, keep_w = _ptr_u32(init.weights)
            assert mem_w == mem, "weights must live with the CSR"
            _check(lib().hn_graph_create_csr_w(init.nV(), init.nE(), po, pa, pw, flags, mem,
                                               self._device, ctypes.byref(self._h)))
            return
        if create:
            fn = lib().hn_graph_create_csr64 if use64 else lib().hn_graph_create_csr
            _check(fn(init.nV(), init.nE(), po, pa, flags, mem, self._device,
                      ctypes.byref(self._h)))
        else:
            assert not use64, "reset takes int32 offsets"
            _check(lib().hn_graph_reset_csr(self._h, init.nV(), init.nE(), po, pa, flags, mem))

    def reset(self, init: HornetInit) -> None:
        """gpu::Hornet::reset(HornetInit&) (HornetInitialize.i.cuh:190-204)."""
        self._build(init, create=False)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.hn_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    release = __del__

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def nV(self) -> int:
        v = ctypes.c_int32()
        _check(lib().hn_graph_nv(self._h, ctypes.byref(v)))
        return v.value

    def nE(self) -> int:
        v = ctypes.c_int64()
        _check(lib().hn_graph_ne(self._h, ctypes.byref(v)))
        return v.value

    def _maxdeg(self) -> Tuple[int, int]:
        d, i = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().hn_graph_max_degree(self._h, ctypes.byref(d), ctypes.byref(i)))
        return d.value, i.value

    def max_degree(self) -> int:
        return self._maxdeg()[0]

    def max_degree_id(self) -> int:
        return self._maxdeg()[1]

    def getCOO(self, sort: bool = True, src=None, dst=None):
        """getCOO(sort): (src, dst) sorted lexicographically
        (HornetQuery.i.cuh:67-109).  Pass CUDA tensors to keep it on device."""
        n = self.nE()
        if src is None:
            src = np.empty(n, np.int32)
            dst = np.empty(n, np.int32)
        ps, mem = _out_ptr(src)
        pd, _ = _out_ptr(dst)
        _check(lib().hn_graph_export_coo(self._h, int(sort), ps, pd, mem))
        return src, dst

    get_coo = getCOO

    def getCOOWeighted(self, dtype=np.uint32):
        """getCOO(true) with the edge weights of a weighted graph:
        (src, dst, weights); weights viewed as `dtype` (a 32-bit type)."""
        n = self.nE()
        src = np.empty(n, np.int32)
        dst = np.empty(n, np.int32)
        w = np.empty(n, np.uint32)
        _check(lib().hn_graph_export_coo_w(self._h, 1, src.ctypes.data_as(_P),
                                           dst.ctypes.data_as(_P), w.ctypes.data_as(_P),
                                           HN_MEM_HOST))
        return src, dst, w.view(dtype)

    def is_weighted(self) -> bool:
        v = ctypes.c_int32()
        _check(lib().hn_graph_weighted(self._h, ctypes.byref(v)))
        return bool(v.value)

    def getCSR(self):
        """getCSR(true): (offsets[nV+1], edges[nE]) host arrays."""
        off = np.empty(self.nV() + 1, np.int32)
        adj = np.empty(self.nE(), np.int32)
        _check(lib().hn_graph_export_csr(self._h, off.ctypes.data_as(_P),
                                         adj.ctypes.data_as(_P), HN_MEM_HOST))
        return off, adj

    get_csr = getCSR

    def insert_count_triangles(self, batch: "BatchUpdate") -> Tuple[int, int]:
        """insert(batch, True, True) that also returns the triangles it
        created (hn_insert_count_triangles): (edges added, new triangles)."""
        n, t = ctypes.c_int64(), ctypes.c_uint64()
        _check(lib().hn_insert_count_triangles(self._h, batch.handle, ctypes.byref(n),
                                               ctypes.byref(t)))
        return n.value, t.value

    def update_coalesced(self, src, dst, ops) -> Tuple[int, int]:
        """A run of insert/erase batches applied as one (hn_update_coalesced):
        ops[i] != 0 inserts edge i, 0 erases it; the last entry of an edge
        decides.  Host numpy arrays or device tensors (all three alike).
        Returns (inserted, erased)."""
        ins, era = ctypes.c_int64(), ctypes.c_int64()
        if _is_device(src):
            _check(lib().hn_update_coalesced(self._h, int(src.numel()),
                                             ctypes.c_void_p(src.data_ptr()),
                                             ctypes.c_void_p(dst.data_ptr()),
                                             ctypes.c_void_p(ops.data_ptr()), HN_MEM_DEVICE,
                                             ctypes.byref(ins), ctypes.byref(era)))
        else:
            s_ = np.ascontiguousarray(src, np.int32)
            d_ = np.ascontiguousarray(dst, np.int32)
            o_ = np.ascontiguousarray(ops, np.uint8)
            _check(lib().hn_update_coalesced(self._h, len(s_), s_.ctypes.data_as(_P),
                                             d_.ctypes.data_as(_P), o_.ctypes.data_as(_P),
                                             HN_MEM_HOST, ctypes.byref(ins), ctypes.byref(era)))
        return ins.value, era.value

    def degrees(self):
        d = np.empty(self.nV(), np.int32)
        _check(lib().hn_graph_degrees(self._h, d.ctypes.data_as(_P), HN_MEM_HOST))
        return d

    def view(self, stream=None) -> "Hornet":
        """A query view (hn_graph_view_create): the same resident graph on its
        own stream and scratch, for read-only calls that run concurrently
        with those on other views.  Call refresh_view() on it after updating
        this graph; destroy views before the graph."""
        v = Hornet.__new__(Hornet)
        v._h = ctypes.c_void_p()
        v._device = self._device
        v._parent = self
        _check(lib().hn_graph_view_create(self._h, None if stream is None else
                                          ctypes.c_void_p(stream), ctypes.byref(v._h)))
        return v

    def refresh_view(self) -> None:
        _check(lib().hn_graph_view_refresh(self._h))

    def gather(self, dev_ptr: int, idx) -> np.ndarray:
        """src[idx] for a device int32 array at dev_ptr (hn_gather_int32)."""
        ix = np.ascontiguousarray(idx, np.int64)
        out = np.empty(len(ix), np.int32)
        _check(lib().hn_gather_int32(self._h, ctypes.c_void_p(dev_ptr), ix.ctypes.data_as(_P),
                                     len(ix), out.ctypes.data_as(_P)))
        return out

    def save_bin(self, path: str) -> None:
        """getCSR + GraphStd::writeBinary (hn_graph_write_bin): the graph's
        current adjacency in the reference's .bin format."""
        _check(lib().hn_graph_write_bin(self._h, path.encode()))

    @staticmethod
    def load_bin(path: str, device: int = 0) -> "Hornet":
        """GraphStd::readBinary + HornetInit (hn_graph_read_bin): a device
        graph from a .bin file (the fast reload of a saved graph)."""
        h = Hornet.__new__(Hornet)
        h._h = ctypes.c_void_p()
        h._device = device
        _check(lib().hn_graph_read_bin(path.encode(), device, ctypes.byref(h._h)))
        return h

    def adjacency_hash(self) -> int:
        """Order-independent checksum of the edge multiset (computed on the
        device; hn_graph_adjacency_hash)."""
        h = ctypes.c_uint64(0)
        _check(lib().hn_graph_adjacency_hash(self._h, ctypes.byref(h)))
        return int(h.value)

    def device(self) -> DeviceView:
        v = DeviceView()
        _check(lib().hn_graph_device_view(self._h, ctypes.byref(v)))
        return v

    def memory(self) -> Tuple[int, int, int]:
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().hn_graph_memory(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def insert(self, batch: "BatchUpdate", removeBatchDuplicates: bool = False,
               removeGraphDuplicates: bool = False) -> int:
        """gpu::Hornet::insert (hornet/include/Core/HornetOperations/
        HornetInsert.i.cuh:12-27).  Returns the number of edges added."""
        flags = (HN_DEDUP_BATCH if removeBatchDuplicates else 0) | \
                (HN_DEDUP_GRAPH if removeGraphDuplicates else 0)
        applied = ctypes.c_int64()
        _check(lib().hn_insert(self._h, batch.handle, flags, ctypes.byref(applied)))
        return applied.value

    def erase(self, batch: "BatchUpdate", removeBatchDuplicates: bool = False) -> int:
        """gpu::Hornet::erase (HornetInsert.i.cuh:71-89).  Returns the number
        of edges removed."""
        flags = HN_DEDUP_BATCH if removeBatchDuplicates else 0
        applied = ctypes.c_int64()
        _check(lib().hn_erase(self._h, batch.handle, flags, ctypes.byref(applied)))
        return applied.value


HornetGPU = Hornet


class BatchUpdate:
    """gpu::BatchUpdate built from a BatchUpdatePtr<HOST|DEVICE>(n, src, dst)
    (BatchUpdate.cuh:91-99); the batch owns a device copy."""

    def __init__(self, hornet: Hornet, src, dst, weights=None):
        self._hornet = hornet
        self._h = ctypes.c_void_p()
        ps, mem, ks = _ptr(src, np.int32)
        pd, _, kd = _ptr(dst, np.int32)
        n = len(src) if not _is_device(src) else int(src.numel())
        if weights is not None:
            pw, _, kw = _ptr_u32(weights)
            _check(lib().hn_batch_create_w(hornet.handle, n, ps, pd, pw, mem,
                                           ctypes.byref(self._h)))
        else:
            _check(lib().hn_batch_create(hornet.handle, n, ps, pd, mem, ctypes.byref(self._h)))

    def reset(self, src, dst, weights=None) -> None:
        ps, mem, ks = _ptr(src, np.int32)
        pd, _, kd = _ptr(dst, np.int32)
        n = len(src) if not _is_device(src) else int(src.numel())
        if weights is not None:
            pw, _, kw = _ptr_u32(weights)
            _check(lib().hn_batch_reset_w(self._h, n, ps, pd, pw, mem))
        else:
            _check(lib().hn_batch_reset(self._h, n, ps, pd, mem))

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def size(self) -> int:
        n = ctypes.c_int64()
        _check(lib().hn_batch_size(self._h, ctypes.byref(n)))
        return n.value

    nE = size

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.hn_batch_destroy(self._h)
            self._h = ctypes.c_void_p()


# ---------------------------------------------------------------------------
# StaticAlgorithm family (primitives/HornetAlg.cuh:51-150)
# ---------------------------------------------------------------------------

class StaticAlgorithm:
    def __init__(self, hornet: Hornet):
        self.hornet = hornet

    def run(self):
        raise NotImplementedError

    def reset(self):
        raise NotImplementedError

    def release(self):
        pass

    def validate(self) -> bool:
        """Certify the last result on the device (the reference's validate()
        methods are stubs returning true, TopDown.cu:113-128,
        CC.cu:163-203)."""
        raise NotImplementedError


def _violations(fn, *args) -> int:
    v = ctypes.c_int64(-1)
    _check(fn(*args, ctypes.byref(v)))
    return v.value


class BfsTopDown(StaticAlgorithm):
    """hornetsnest BfsTopDown (TopDown.cuh:52-70): set_parameters(src), run().
    validate() certifies the last run's distances on the device
    (hn_bfs_validate: source at 0, no edge skips a level, every reached
    vertex has a parent one level closer); the reference's own validate()
    is a stub returning true (TopDown.cu:113-128)."""

    def __init__(self, hornet: Hornet):
        super().__init__(hornet)
        self.source = 0
        self.distances: Optional[np.ndarray] = None
        self.stats = BfsStats()

    def reset(self):
        self.distances = None

    def set_parameters(self, source: int):
        self.source = int(source)

    def run(self, out=None):
        n = self.hornet.nV()
        if out is None:
            out = np.empty(n, np.int32)
        p, mem = _out_ptr(out)
        _check(lib().hn_bfs(self.hornet.handle, self.source, p, mem, ctypes.byref(self.stats)))
        self.distances = out
        self.distances_source = self.source
        return out

    def validate(self) -> bool:
        if self.distances is None:
            return False
        p, mem = _out_ptr(self.distances)
        return _violations(lib().hn_bfs_validate, self.hornet.handle, self.distances_source, p,
                           mem) == 0

    def run_multi(self, sources, out=None, direction_optimizing: bool = False):
        srcs = np.ascontiguousarray(sources, np.int32)
        n = self.hornet.nV()
        if out is None:
            out = np.empty((len(srcs), n), np.int32)
        p, mem = _out_ptr(out)
        stats = (BfsStats * max(1, len(srcs)))()
        fn = lib().hn_bfs_do if direction_optimizing else lib().hn_bfs_multi
        _check(fn(self.hornet.handle, srcs.ctypes.data_as(_P), len(srcs), p, mem, stats))
        return out, [stats[i] for i in range(len(srcs))]


    def level_trace(self, max_levels: int = 32):
        """Per-level device time (us) and frontier edges of the latest BFS
        source run on this graph (instrumentation, hn_bfs_level_trace)."""
        us = np.zeros(max_levels, np.float64)
        ed = np.zeros(max_levels, np.int64)
        n = ctypes.c_int32(0)
        _check(lib().hn_bfs_level_trace(self.hornet.handle, max_levels, us.ctypes.data_as(_P),
                                        ed.ctypes.data_as(_P), ctypes.byref(n)))
        return us[: n.value], ed[: n.value]

    def run_batch(self, sources, slots=None, nslots=None, out=None):
        """Batched BFS (hn_bfs_batch): up to 64 slots in one traversal.
        Returns (dist[nslots][nV], per-slot stats)."""
        srcs = np.ascontiguousarray(sources, np.int32)
        sl = None if slots is None else np.ascontiguousarray(slots, np.int32)
        if nslots is None:
            nslots = len(srcs) if sl is None else int(sl.max()) + 1
        n = self.hornet.nV()
        if out is None:
            out = np.empty((nslots, n), np.int32)
        p, mem = _out_ptr(out)
        stats = (BfsStats * nslots)()
        _check(lib().hn_bfs_batch(self.hornet.handle, srcs.ctypes.data_as(_P),
                                  None if sl is None else sl.ctypes.data_as(_P),
                                  len(srcs), nslots, p, mem, stats))
        return out, [stats[i] for i in range(nslots)]


class BfsDirectionOptimizing(BfsTopDown):
    """Direction-optimising BFS (hornetsnest BottomUpBFS counterpart): same
    distances as BfsTopDown, fewer edges read on large frontiers."""

    def run(self, out=None):
        n = self.hornet.nV()
        if out is None:
            out = np.empty(n, np.int32)
        p, mem = _out_ptr(out)
        src = np.array([self.source], np.int32)
        _check(lib().hn_bfs_do(self.hornet.handle, src.ctypes.data_as(_P), 1, p, mem,
                               ctypes.byref(self.stats)))
        self.distances = out
        return out

    def getLevels(self) -> int:
        return self.stats.levels


class TriangleCounting2(StaticAlgorithm):
    """hornetsnest TriangleCounting2 (triangle2.cuh:18-37): init(), run(),
    countTriangles(), copyTCToHost()."""

    def __init__(self, hornet: Hornet):
        super().__init__(hornet)
        self._per_vertex = None
        self._total = 0

    def init(self):
        self.reset()

    def reset(self):
        self._per_vertex = None
        self._total = 0

    def run(self, per_vertex: bool = False):
        total = ctypes.c_uint64()
        if per_vertex:
            pv = np.empty(self.hornet.nV(), np.uint64)
            _check(lib().hn_tc(self.hornet.handle, pv.ctypes.data_as(_P), HN_MEM_HOST,
                               ctypes.byref(total)))
            self._per_vertex = pv
        else:
            _check(lib().hn_tc(self.hornet.handle, None, HN_MEM_HOST, ctypes.byref(total)))
        self._total = total.value
        return self._total

    def countTriangles(self) -> int:
        return self._total

    def validate(self) -> bool:
        """The total against two other kernels: the owner counts (each
        triangle credited once) sum to it, and the per-vertex counts (every
        triangle credited to its three vertices) sum to three times it."""
        total = ctypes.c_uint64()
        owner = np.empty(max(1, self.hornet.nV()), np.uint64)
        _check(lib().hn_tc_owner(self.hornet.handle, owner.ctypes.data_as(_P), HN_MEM_HOST,
                                 ctypes.byref(total)))
        pv = self._per_vertex
        if pv is None:
            pv = np.empty(self.hornet.nV(), np.uint64)
            t2 = ctypes.c_uint64()
            _check(lib().hn_tc(self.hornet.handle, pv.ctypes.data_as(_P), HN_MEM_HOST,
                               ctypes.byref(t2)))
        return total.value == self._total and int(pv.sum(dtype=np.uint64)) == 3 * self._total

    def local(self, seeds, out=None):
        """Triangles containing each seed vertex (hn_tc_local).  seeds: host
        int array, or a device int32 tensor (then `out`, a device int64
        tensor, receives the counts)."""
        if _is_device(seeds):
            _check(lib().hn_tc_local(self.hornet.handle, ctypes.c_void_p(seeds.data_ptr()),
                                     int(seeds.numel()), ctypes.c_void_p(out.data_ptr()),
                                     HN_MEM_DEVICE))
            return out
        sd = np.ascontiguousarray(seeds, np.int32)
        res = np.empty(len(sd), np.uint64)
        _check(lib().hn_tc_local(self.hornet.handle, sd.ctypes.data_as(_P), len(sd),
                                 res.ctypes.data_as(_P), HN_MEM_HOST))
        return res

    def copyTCToHost(self):
        if self._per_vertex is None:
            self.run(per_vertex=True)
        return self._per_vertex


class CC(StaticAlgorithm):
    """hornetsnest CC (CC.cuh:53-69).  labels: min vertex id per component;
    reference_colors(): the colours CC::run itself produces."""

    def __init__(self, hornet: Hornet):
        super().__init__(hornet)
        self.labels: Optional[np.ndarray] = None
        self.n_components = 0

    def reset(self):
        self.labels = None

    def run(self, mode: int = HN_CC_MIN_ID, out=None):
        n = self.hornet.nV()
        if out is None:
            out = np.empty(n, np.int32)
        p, mem = _out_ptr(out)
        nc = ctypes.c_int32()
        _check(lib().hn_cc(self.hornet.handle, mode, p, mem, ctypes.byref(nc)))
        self.n_components = nc.value
        if mode == HN_CC_MIN_ID:
            self.labels = out
        return out

    def reference_colors(self):
        return self.run(HN_CC_REFERENCE)

    def validate(self) -> bool:
        """Certify the last minimum-id labels on the device (hn_cc_validate)."""
        if self.labels is None:
            return False
        p, mem = _out_ptr(self.labels)
        return _violations(lib().hn_cc_validate, self.hornet.handle, p, mem) == 0


class KTruss(StaticAlgorithm):
    """hornetsnest KTruss (KTruss.cuh:43-78): run(), getMaxK(); edge_truss
    holds the truss number of every edge in sorted-COO order."""

    def __init__(self, hornet: Hornet):
        super().__init__(hornet)
        self.max_k = 0
        self.edge_truss: Optional[np.ndarray] = None

    def init(self):
        self.reset()

    def reset(self):
        self.max_k = 0
        self.edge_truss = None

    def run(self):
        k = ctypes.c_int32()
        et = np.empty(self.hornet.nE(), np.int32)
        _check(lib().hn_ktruss(self.hornet.handle, ctypes.byref(k), et.ctypes.data_as(_P),
                               HN_MEM_HOST))
        self.max_k = k.value
        self.edge_truss = et
        return self.max_k

    def getMaxK(self) -> int:
        return self.max_k

    def validate(self) -> bool:
        """Certify the last edge truss numbers on the device
        (hn_ktruss_validate: the edges numbered >= t form a t-truss)."""
        if self.edge_truss is None:
            return False
        et = np.ascontiguousarray(self.edge_truss, np.int32)
        return _violations(lib().hn_ktruss_validate, self.hornet.handle, self.max_k,
                           et.ctypes.data_as(_P), HN_MEM_HOST) == 0

    def runForK(self, K: int):
        """KTruss::runForK (KTruss.cu:114-119) + copyOffsetArrayHost: the
        K-truss of the graph (not modified) as CSR offsets (nV + 1) and the
        surviving edges (src, dst) in sorted-COO order."""
        self.run()
        s, d = self.hornet.getCOO(True)
        keep = self.edge_truss >= K
        off = np.zeros(self.hornet.nV() + 1, np.int64)
        np.add.at(off, s[keep].astype(np.int64) + 1, 1)
        self.offsets = np.cumsum(off).astype(np.int32)
        return self.offsets, s[keep], d[keep]

    def copyOffsetArrayHost(self):
        return self.offsets

    def runForKDynamic(self, K: int) -> int:
        """KTruss::runForKDynamic (KTruss.cu:270-295): erase every edge below
        the K-truss from the graph itself (hn_ktruss_keep).  Returns the
        number of directed edges erased; max_k is the graph's max K before."""
        k, n = ctypes.c_int32(), ctypes.c_int64()
        _check(lib().hn_ktruss_keep(self.hornet.handle, int(K), ctypes.byref(k), ctypes.byref(n)))
        self.max_k = k.value
        return n.value


# ---------------------------------------------------------------------------
# operator primitives with built-in operators
# ---------------------------------------------------------------------------

def for_all_edges_count(hornet: Hornet, out, vertices=None, lb: int = HN_LB_BINARY_SEARCH,
                        vw: int = 1) -> None:
    """forAllEdges(hornet, vertices, op=count-dst, lb) into the device int32
    tensor `out` (accumulated)."""
    pv, mem, keep = _ptr(vertices, np.int32)
    n = 0 if vertices is None else (int(vertices.numel()) if _is_device(vertices) else len(vertices))
    if vertices is not None:
        assert mem == HN_MEM_DEVICE, "vertices must be a device array"
    _check(lib().hn_for_all_edges_count(hornet.handle, pv, n, lb, vw, ctypes.c_void_p(out.data_ptr())))


def for_all_vertices_degree(hornet: Hornet, out) -> None:
    _check(lib().hn_for_all_vertices_degree(hornet.handle, ctypes.c_void_p(out.data_ptr())))


# ---------------------------------------------------------------------------
# synthetic inputs
# ---------------------------------------------------------------------------

RMAT_A, RMAT_B, RMAT_C = 0.57, 0.19, 0.19


def gen_rmat_host(scale: int, n_pairs: int, seed: int, n_vertices: Optional[int] = None,
                  a: float = RMAT_A, b: float = RMAT_B, c: float = RMAT_C):
    """R-MAT pairs on the host; identical to gen_rmat_device."""
    n = n_vertices if n_vertices is not None else (1 << scale)
    src = np.empty(n_pairs, np.int32)
    dst = np.empty(n_pairs, np.int32)
    _check(lib().hn_gen_rmat_host(scale, n, n_pairs, a, b, c, seed & (2**64 - 1),
                                  src.ctypes.data_as(_P), dst.ctypes.data_as(_P)))
    return src, dst


def gen_rmat_device(scale: int, n_pairs: int, seed: int, src, dst, n_vertices: Optional[int] = None,
                    a: float = RMAT_A, b: float = RMAT_B, c: float = RMAT_C, device: int = 0):
    n = n_vertices if n_vertices is not None else (1 << scale)
    _check(lib().hn_gen_rmat_device(scale, n, n_pairs, a, b, c, seed & (2**64 - 1),
                                    ctypes.c_void_p(src.data_ptr()),
                                    ctypes.c_void_p(dst.data_ptr()), device))


class DeviceCSR:
    """Undirected CSR built on the device (owns two cudaMalloc buffers)."""

    def __init__(self, nV: int, off_ptr: int, adj_ptr: int, nE: int):
        self.nV, self.nE = nV, nE
        self.off_ptr, self.adj_ptr = off_ptr, adj_ptr

    def __del__(self):
        if _lib is not None:
            for p in (self.off_ptr, self.adj_ptr):
                if p:
                    _lib.hn_free_device(ctypes.c_void_p(p))
            self.off_ptr = self.adj_ptr = 0


def coo_to_csr_device(nV: int, src, dst, device: int = 0) -> DeviceCSR:
    po, pa, ne = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int64()
    _check(lib().hn_coo_to_csr_device(nV, int(src.numel()), ctypes.c_void_p(src.data_ptr()),
                                      ctypes.c_void_p(dst.data_ptr()), device, ctypes.byref(po),
                                      ctypes.byref(pa), ctypes.byref(ne)))
    return DeviceCSR(nV, po.value or 0, pa.value or 0, ne.value)


def write_bin(path: str, off, adj) -> None:
    """GraphStd binary (.bin) from a host CSR (int32 offsets)."""
    off = np.ascontiguousarray(off, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    _check(lib().hn_csr_write_bin(path.encode(), len(off) - 1, len(adj),
                                  off.ctypes.data_as(_P), adj.ctypes.data_as(_P)))


def read_bin(path: str):
    """(off, adj) host CSR from a GraphStd binary (.bin) file."""
    nv, ne = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().hn_csr_read_bin(path.encode(), ctypes.byref(nv), ctypes.byref(ne), None, None))
    off = np.empty(nv.value + 1, np.int32)
    adj = np.empty(max(1, ne.value), np.int32)
    _check(lib().hn_csr_read_bin(path.encode(), ctypes.byref(nv), ctypes.byref(ne),
                                 off.ctypes.data_as(_P), adj.ctypes.data_as(_P)))
    return off, adj[:ne.value]


def write_mtx(path: str, off, adj) -> None:
    """Matrix Market (coordinate pattern general, 1-based) from a host CSR."""
    off = np.ascontiguousarray(off, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    _check(lib().hn_csr_write_mtx(path.encode(), len(off) - 1, len(adj),
                                  off.ctypes.data_as(_P), adj.ctypes.data_as(_P)))


def hornet_from_device_csr(csr: DeviceCSR, device: int = 0) -> Hornet:
    """Build a Hornet straight from a DeviceCSR (sorted, int32 offsets)."""
    h = Hornet.__new__(Hornet)
    h._h = ctypes.c_void_p()
    h._device = device
    _check(lib().hn_graph_create_csr(csr.nV, csr.nE, ctypes.c_void_p(csr.off_ptr),
                                     ctypes.c_void_p(csr.adj_ptr), HN_CSR_SORTED, HN_MEM_DEVICE,
                                     device, ctypes.byref(h._h)))
    return h


def hornet_from_device_arrays(nV: int, nE: int, off, adj, device: int = 0) -> Hornet:
    """Build a Hornet from caller-owned device arrays (torch int32 tensors:
    sorted CSR offsets[nV+1] and edges[nE]); the arrays are copied."""
    h = Hornet.__new__(Hornet)
    h._h = ctypes.c_void_p()
    h._device = device
    _check(lib().hn_graph_create_csr(nV, nE, ctypes.c_void_p(off.data_ptr()),
                                     ctypes.c_void_p(adj.data_ptr()), HN_CSR_SORTED,
                                     HN_MEM_DEVICE, device, ctypes.byref(h._h)))
    return h


def tune_names():
    """Names of the tuning knobs (hn_tune_name)."""
    out, i = [], 0
    while True:
        n = lib().hn_tune_name(i)
        if not n:
            return out
        out.append(n.decode())
        i += 1


def tune_get(name: str) -> int:
    v = ctypes.c_int64()
    _check(lib().hn_tune_get(name.encode(), ctypes.byref(v)))
    return v.value


def tune_set(name: str, value: int) -> None:
    _check(lib().hn_tune_set(name.encode(), int(value)))


def tune_reset() -> None:
    _check(lib().hn_tune_reset())
