"""CPU ORACLE — test infrastructure, not product code.

Python access to the C restatement (oracle/libhn_oracle.so, see
oracle/hn_oracle.h for the reference lines each function follows) and to
the reference's own host code compiled into oracle/_ref/ref_driver
(xlib GraphStd / BFS / WCC, see oracle/ref_driver.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this module,
always as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libhn_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
INF = 2147483647

_P = ctypes.c_void_p
_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=subprocess.DEVNULL)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        l = ctypes.CDLL(LIB)
        I32, I64, U = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint
        l.hno_build_csr_undirected.argtypes = [I32, I64, _P, _P, _P, _P]
        l.hno_build_csr_undirected.restype = I64
        l.hno_orient_by_degree.argtypes = [I32, _P, _P, _P, _P]
        l.hno_orient_by_degree.restype = I64
        for f in (l.hno_insert, l.hno_erase):
            f.argtypes = [I32, _P, _P, I64, _P, _P, U, _P, _P]
            f.restype = I64
        l.hno_bfs.argtypes = [I32, _P, _P, I32, _P]
        l.hno_bfs.restype = I64
        l.hno_tc_oriented.argtypes = [I32, _P, _P, _P]
        l.hno_tc_oriented.restype = ctypes.c_uint64
        l.hno_cc_min_label.argtypes = [I32, _P, _P, _P]
        l.hno_cc_min_label.restype = I32
        l.hno_cc_reference_colors.argtypes = [I32, _P, _P, _P]
        l.hno_cc_reference_colors.restype = None
        l.hno_ktruss.argtypes = [I32, _P, _P, _P]
        l.hno_ktruss.restype = I32
        l.hno_tc_oriented_sample.argtypes = [I32, _P, _P, I32, I32, _P]
        l.hno_tc_oriented_sample.restype = ctypes.c_uint64
        l.hno_ktruss_peel.argtypes = [I32, _P, _P, _P]
        l.hno_ktruss_peel.restype = I32
        l.hno_gen_rmat.argtypes = [I32, I32, I64, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_uint64, _P, _P, I32]
        l.hno_gen_rmat.restype = ctypes.c_int
        l.hno_adjacency_hash.argtypes = [I32, _P, _P]
        l.hno_adjacency_hash.restype = ctypes.c_uint64
        _lib = l
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P)


class Csr:
    """CSR with int64 offsets (oracle side)."""

    def __init__(self, off: np.ndarray, adj: np.ndarray):
        self.off = np.ascontiguousarray(off, np.int64)
        self.adj = np.ascontiguousarray(adj, np.int32)

    @property
    def nV(self) -> int:
        return len(self.off) - 1

    @property
    def nE(self) -> int:
        return int(self.off[-1])

    def off32(self) -> np.ndarray:
        return self.off.astype(np.int32)

    def coo(self) -> Tuple[np.ndarray, np.ndarray]:
        src = np.repeat(np.arange(self.nV, dtype=np.int32), np.diff(self.off))
        return src, self.adj.copy()


def gen_rmat(scale: int, np_pairs: int, seed: int, n_vertices: Optional[int] = None,
             a: float = 0.57, b: float = 0.19, c: float = 0.19,
             threads: Optional[int] = None) -> Tuple[np.ndarray, np.ndarray]:
    """The repository's R-MAT input pairs (restated generator, bit-identical
    to the library's hn_gen_rmat_host)."""
    n = (1 << scale) if n_vertices is None else int(n_vertices)
    src = np.empty(np_pairs, np.int32)
    dst = np.empty(np_pairs, np.int32)
    t = threads or min(32, os.cpu_count() or 1)
    rc = lib().hno_gen_rmat(scale, n, np_pairs, a, b, c, seed & (2**64 - 1), _p(src), _p(dst), t)
    if rc != 0:
        raise ValueError("bad R-MAT parameters")
    return src, dst


def adjacency_hash(g: "Csr") -> int:
    """Order-independent checksum of the graph's edge multiset."""
    return int(lib().hno_adjacency_hash(g.nV, _p(g.off), _p(g.adj)))


def build_csr_undirected(nV: int, src, dst) -> Csr:
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    off = np.empty(nV + 1, np.int64)
    adj = np.empty(2 * len(src) + 1, np.int32)
    m = lib().hno_build_csr_undirected(nV, len(src), _p(src), _p(dst), _p(off), _p(adj))
    return Csr(off, adj[:m].copy())


def orient_by_degree(g: Csr) -> Csr:
    off = np.empty(g.nV + 1, np.int64)
    adj = np.empty(g.nE + 1, np.int32)
    m = lib().hno_orient_by_degree(g.nV, _p(g.off), _p(g.adj), _p(off), _p(adj))
    return Csr(off, adj[:m].copy())


def insert(g: Csr, bsrc, bdst, flags: int) -> Tuple[Csr, int]:
    bsrc = np.ascontiguousarray(bsrc, np.int32)
    bdst = np.ascontiguousarray(bdst, np.int32)
    off = np.empty(g.nV + 1, np.int64)
    adj = np.empty(g.nE + len(bsrc) + 1, np.int32)
    n = lib().hno_insert(g.nV, _p(g.off), _p(g.adj), len(bsrc), _p(bsrc), _p(bdst), flags,
                         _p(off), _p(adj))
    if n < 0:
        raise ValueError("batch id out of range")
    return Csr(off, adj[:off[-1]].copy()), int(n)


def erase(g: Csr, bsrc, bdst, flags: int) -> Tuple[Csr, int]:
    bsrc = np.ascontiguousarray(bsrc, np.int32)
    bdst = np.ascontiguousarray(bdst, np.int32)
    off = np.empty(g.nV + 1, np.int64)
    adj = np.empty(g.nE + 1, np.int32)
    n = lib().hno_erase(g.nV, _p(g.off), _p(g.adj), len(bsrc), _p(bsrc), _p(bdst), flags,
                        _p(off), _p(adj))
    if n < 0:
        raise ValueError("batch id out of range")
    return Csr(off, adj[:off[-1]].copy()), int(n)


def bfs(g: Csr, src: int) -> Tuple[np.ndarray, int]:
    dist = np.empty(g.nV, np.int32)
    scanned = lib().hno_bfs(g.nV, _p(g.off), _p(g.adj), src, _p(dist))
    return dist, int(scanned)


def tc(g: Csr, per_vertex: bool = False):
    """Triangles of an undirected graph via the degree orientation."""
    o = orient_by_degree(g)
    pv = np.empty(g.nV, np.uint64) if per_vertex else None
    t = lib().hno_tc_oriented(o.nV, _p(o.off), _p(o.adj), _p(pv) if pv is not None else None)
    return (int(t), pv) if per_vertex else int(t)


def time_tc_sample(g: Csr, stride: int, first: int = 0) -> Tuple[float, int]:
    """Seconds of the restated hostCountTriangles over a uniform sample of
    the degree-oriented graph's edges (every stride-th in CSR order), and
    the number of sampled edges.  The orientation is not timed."""
    import time
    o = orient_by_degree(g)
    e = ctypes.c_int64()
    t0 = time.perf_counter()
    lib().hno_tc_oriented_sample(o.nV, _p(o.off), _p(o.adj), first, stride, ctypes.byref(e))
    return time.perf_counter() - t0, int(e.value)


def cc_min_label(g: Csr) -> Tuple[np.ndarray, int]:
    lab = np.empty(g.nV, np.int32)
    n = lib().hno_cc_min_label(g.nV, _p(g.off), _p(g.adj), _p(lab))
    return lab, int(n)


def cc_reference_colors(g: Csr) -> np.ndarray:
    col = np.empty(g.nV, np.int32)
    lib().hno_cc_reference_colors(g.nV, _p(g.off), _p(g.adj), _p(col))
    return col


def ktruss(g: Csr) -> Tuple[int, np.ndarray]:
    et = np.empty(max(1, g.nE), np.int32)
    k = lib().hno_ktruss(g.nV, _p(g.off), _p(g.adj), _p(et))
    return int(k), et[:g.nE].copy()


def ktruss_peel(g: Csr) -> Tuple[int, np.ndarray]:
    """Truss numbers by support peeling (independent of ktruss(); same
    results, fast enough for benchmark-scale graphs)."""
    et = np.empty(max(1, g.nE), np.int32)
    k = lib().hno_ktruss_peel(g.nV, _p(g.off), _p(g.adj), _p(et))
    return int(k), et[:g.nE].copy()


def canon_labels_fast(lab: np.ndarray) -> np.ndarray:
    """canon_labels, vectorised: every vertex gets the smallest vertex id
    carrying its label."""
    lab = np.asarray(lab)
    uniq, first, inv = np.unique(lab, return_index=True, return_inverse=True)
    return first.astype(np.int32)[inv]


# ---------------------------------------------------------------------------
# reference host code (oracle/_ref/ref_driver)
# ---------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_DRIVER)


def write_csr(path: str, g: Csr) -> None:
    with open(path, "wb") as f:
        np.array([g.nV, g.nE], np.int64).tofile(f)
        g.off.astype(np.int32).tofile(f)
        g.adj.astype(np.int32).tofile(f)


def read_csr(path: str) -> Csr:
    b = open(path, "rb").read()
    nV, nE = np.frombuffer(b[:16], np.int64)
    a = np.frombuffer(b[16:], np.int32)
    return Csr(a[: nV + 1].astype(np.int64), a[nV + 1: nV + 1 + nE].copy())


def ref_bfs(g: Csr, sources) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        cp, op = os.path.join(d, "g.csr"), os.path.join(d, "o.bin")
        write_csr(cp, g)
        subprocess.run([REF_DRIVER, "bfs", cp, op] + [str(int(s)) for s in sources], check=True,
                       stdout=subprocess.DEVNULL)
        return np.fromfile(op, np.int32).reshape(len(sources), g.nV)


def ref_wcc(g: Csr) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        cp, op = os.path.join(d, "g.csr"), os.path.join(d, "o.bin")
        write_csr(cp, g)
        subprocess.run([REF_DRIVER, "wcc", cp, op], check=True, stdout=subprocess.DEVNULL)
        return np.fromfile(op, np.int32)


def ref_time_wcc(g: Csr) -> Tuple[float, int]:
    """Seconds spent in graph::WCC::run (reference host code) and the
    component count."""
    with tempfile.TemporaryDirectory() as d:
        cp, op = os.path.join(d, "g.csr"), os.path.join(d, "o.bin")
        write_csr(cp, g)
        out = subprocess.run([REF_DRIVER, "wcc", cp, op], check=True, capture_output=True,
                             text=True).stdout.split()
        return float(out[0]), int(out[1])


def time_update(g: Csr, bsrc, bdst) -> Tuple[float, float, int, int]:
    """Seconds of the restated insert (both dedup flags) and of the erase
    (removeBatchDuplicates) of one batch on g, and the edges each applied."""
    import time
    t0 = time.perf_counter()
    g2, a = insert(g, bsrc, bdst, 3)
    t1 = time.perf_counter()
    _, r = erase(g2, bsrc, bdst, 1)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, a, r


def ref_time_bfs(g: Csr, sources) -> Tuple[float, int]:
    """Seconds spent in graph::BFS::run over `sources` and edges visited."""
    with tempfile.TemporaryDirectory() as d:
        cp = os.path.join(d, "g.csr")
        write_csr(cp, g)
        out = subprocess.run([REF_DRIVER, "time_bfs", cp] + [str(int(s)) for s in sources],
                             check=True, capture_output=True, text=True).stdout.split()
        return float(out[0]), int(out[1])


def ref_time_bfs_parallel(g: Csr, sources, procs: int) -> Tuple[float, int, int]:
    """graph::BFS::run over `sources` split across `procs` concurrent
    ref_driver processes (the reference BFS is single-threaded; the host's
    cores run independent sources).  Returns (seconds of the slowest
    process's BFS phase, edges visited in total, processes used)."""
    procs = max(1, min(procs, len(sources)))
    parts = [list(sources[i::procs]) for i in range(procs)]
    with tempfile.TemporaryDirectory() as d:
        cp = os.path.join(d, "g.csr")
        write_csr(cp, g)
        ps = [subprocess.Popen([REF_DRIVER, "time_bfs", cp] + [str(int(x)) for x in part],
                               stdout=subprocess.PIPE, text=True) for part in parts]
        secs, edges = [], 0
        for p_ in ps:
            out, _ = p_.communicate()
            if p_.returncode != 0:
                raise RuntimeError("ref_driver failed")
            a = out.split()
            secs.append(float(a[0]))
            edges += int(a[1])
        return max(secs), edges, procs


def ref_read_mtx(path: str, undirected: bool = True, by_degree: bool = False) -> Csr:
    with tempfile.TemporaryDirectory() as d:
        op = os.path.join(d, "o.csr")
        subprocess.run([REF_DRIVER, "read_mtx", path, "undirected" if undirected else "directed",
                        "1" if by_degree else "0", op], check=True, stdout=subprocess.DEVNULL)
        return read_csr(op)


def write_mtx(path: str, nV: int, src, dst) -> None:
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{nV} {nV} {len(src)}\n")
        for u, v in zip(src, dst):
            f.write(f"{int(u) + 1} {int(v) + 1}\n")


def canon_labels(lab: np.ndarray) -> np.ndarray:
    """Relabel any component labelling to the minimum vertex id per label."""
    lab = np.asarray(lab)
    n = len(lab)
    first = {}
    out = np.empty(n, np.int32)
    for v in range(n):
        first.setdefault(int(lab[v]), v)
        out[v] = first[int(lab[v])]
    return out
