"""GPU: hn_cc_csr_noalloc — connected components for callers that cannot
allocate device memory (a host framework that owns all device memory, a
fixed up-front memory budget, or a loop that cannot afford cudaMalloc's
implicit synchronisation).  Called through the C ABI on a caller-owned
device CSR, twice in a row (the shared static scratch keeps the previous
call's contents), and compared with the allocating entry point hn_cc and
with the CPU oracle on the same graph; at its vertex limit (4,194,304, the
benchmark's scale-22 graph) with the reference's graph::WCC labels pinned in
tests/golden/fullsize.json.  Labels are integers, so every comparison is
exact.  Edge cases: no vertices, isolated vertices, every degree at most 2
(no vertex left for the second linking pass), a call on a non-default
stream, and malformed CSRs (ids out of range, offsets that decrease or do
not start at 0) reported without following them.

Collected last on purpose: it must pass alone in a fresh process and after
every other test."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from tests import helpers as T

pytestmark = pytest.mark.gpu

LIMIT = 1 << 22


def _noalloc(nV, off_t, adj_t, out_t, stream=None):
    nc = ctypes.c_int32(-1)
    rc = H.lib().hn_cc_csr_noalloc(nV, ctypes.c_void_p(off_t.data_ptr()),
                                   ctypes.c_void_p(adj_t.data_ptr()),
                                   ctypes.c_void_p(out_t.data_ptr()), ctypes.byref(nc),
                                   None if stream is None else ctypes.c_void_p(stream))
    return rc, nc.value


def _run_twice_and_compare(g, stream=None):
    import torch
    ref, ref_n = O.cc_min_label(g)
    off_t = torch.from_numpy(g.off32()).cuda()
    adj_t = torch.from_numpy(g.adj if g.nE else np.zeros(1, np.int32)).cuda()
    for call in range(2):
        out_t = torch.full((max(1, g.nV),), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()   # inputs ready before a call on another stream
        rc, n = _noalloc(g.nV, off_t, adj_t, out_t, stream)
        assert rc == H.HN_OK, H.last_error()
        if stream is not None:
            torch.cuda.synchronize()
        np.testing.assert_array_equal(out_t.cpu().numpy()[: g.nV], ref, err_msg=f"call {call}")
        assert n == ref_n
    return ref


@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 41), (14, 4, 42)])
def test_noalloc_cc_matches_hn_cc_and_oracle_twice(scale, ef, seed):
    g = T.rmat_graph(scale, ef, seed=seed)
    ref = _run_twice_and_compare(g)
    h = H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))
    np.testing.assert_array_equal(H.CC(h).run(), ref)


def test_noalloc_cc_small_shapes():
    # isolated vertices around a triangle and an edge
    g = O.build_csr_undirected(5, np.array([1, 2, 1], np.int32), np.array([2, 3, 3], np.int32))
    _run_twice_and_compare(g)
    # a path: every degree <= 2, so the giant-component pass lists nothing
    n = 5000
    s = np.arange(n - 1, dtype=np.int32)
    _run_twice_and_compare(O.build_csr_undirected(n, s, s + 1))
    # a forest of paths and isolated vertices
    rng = np.random.default_rng(8)
    s = rng.integers(0, 3000, 1500).astype(np.int32)
    _run_twice_and_compare(O.build_csr_undirected(3000, s, (s + 1) % 3000))


def test_noalloc_cc_no_vertices():
    import torch
    off_t = torch.zeros(1, dtype=torch.int32, device="cuda")
    out_t = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc, n = _noalloc(0, off_t, off_t, out_t)
    assert rc == H.HN_OK and n == 0


def test_noalloc_cc_on_a_stream():
    import torch
    g = T.rmat_graph(11, 8, seed=5)
    s = torch.cuda.Stream()
    _run_twice_and_compare(g, stream=s.cuda_stream)


def test_noalloc_cc_at_its_limit_pinned_to_reference():
    """4,194,304 vertices (the benchmark's scale-22 graph, built on the
    device): the labels equal the reference's graph::WCC labels relabelled
    to minimum ids (SHA-256 in tests/golden/fullsize.json), twice."""
    import torch
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fullsize.json")))
    cc = gold["rmat22"]["cc"]
    n = LIMIT
    src = torch.empty(16 * n, dtype=torch.int32, device="cuda")
    dst = torch.empty_like(src)
    H.gen_rmat_device(22, 16 * n, 1, src, dst)
    csr = H.coo_to_csr_device(n, src, dst)
    del src, dst
    for call in range(2):
        out_t = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        nc = ctypes.c_int32(-1)
        rc = H.lib().hn_cc_csr_noalloc(n, ctypes.c_void_p(csr.off_ptr),
                                       ctypes.c_void_p(csr.adj_ptr),
                                       ctypes.c_void_p(out_t.data_ptr()), ctypes.byref(nc), None)
        assert rc == H.HN_OK, H.last_error()
        lab = out_t.cpu().numpy().astype("<i4")
        assert hashlib.sha256(lab.tobytes()).hexdigest() == cc["sha256_min_id"], call
        assert nc.value == cc["components"]


def test_noalloc_cc_rejects_oversize_and_malformed_csr():
    import torch
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(LIMIT + 1, dummy, dummy, dummy)
    assert rc == H.HN_ERR_CAPACITY
    assert "4194304" in H.last_error()
    out_t = torch.full((3,), -7, dtype=torch.int32, device="cuda")
    cases = [
        ([0, 1, 2, 2], [1, 5]),        # a neighbour id out of range
        ([0, 2, 1, 2], [1, 0]),        # offsets decrease
        ([1, 2, 3, 3], [1, 0, 0]),     # offsets do not start at 0
        ([0, 1, 2, 2], [1, -1]),       # a negative id
    ]
    for off, adj in cases:
        off_t = torch.tensor(off, dtype=torch.int32, device="cuda")
        adj_t = torch.tensor(adj, dtype=torch.int32, device="cuda")
        rc, _ = _noalloc(3, off_t, adj_t, out_t)
        assert rc == H.HN_ERR_INVALID, (off, adj)
    # a valid call right after the rejected ones (the counters are cleared)
    g = O.build_csr_undirected(3, np.array([0], np.int32), np.array([2], np.int32))
    _run_twice_and_compare(g)
