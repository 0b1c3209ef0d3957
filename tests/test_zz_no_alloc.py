"""GPU: hn_cc_csr_noalloc — connected components for callers that cannot
allocate device memory (a host framework that owns all device memory, a
fixed up-front memory budget, or a loop that cannot afford cudaMalloc's
implicit synchronisation).  Called through the C ABI on a caller-owned
device CSR, twice in a row (the shared static scratch keeps the previous
call's contents), and compared with the allocating entry point hn_cc on
the same graph.  Labels are integers, so the comparison is exact.

Collected last on purpose: it must pass alone in a fresh process and after
every other test."""
import ctypes

import numpy as np
import pytest

import hornet_b200 as H
from tests import helpers as T

pytestmark = pytest.mark.gpu


def _noalloc(nV, off_t, adj_t, out_t):
    nc = ctypes.c_int32(-1)
    rc = H.lib().hn_cc_csr_noalloc(nV, ctypes.c_void_p(off_t.data_ptr()),
                                   ctypes.c_void_p(adj_t.data_ptr()),
                                   ctypes.c_void_p(out_t.data_ptr()), ctypes.byref(nc), None)
    return rc, nc.value


@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 41), (14, 4, 42)])
def test_noalloc_cc_matches_hn_cc_twice(scale, ef, seed):
    import torch
    g = T.rmat_graph(scale, ef, seed=seed)
    h = H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))
    cc = H.CC(h)
    ref = cc.run()
    ref_n = cc.n_components
    off_t = torch.from_numpy(g.off32()).cuda()
    adj_t = torch.from_numpy(g.adj).cuda()
    for call in range(2):
        out_t = torch.full((g.nV,), -7, dtype=torch.int32, device="cuda")
        rc, n = _noalloc(g.nV, off_t, adj_t, out_t)
        assert rc == H.HN_OK, H.last_error()
        np.testing.assert_array_equal(out_t.cpu().numpy(), ref, err_msg=f"call {call}")
        assert n == ref_n


def test_noalloc_cc_rejects_oversize_and_bad_ids():
    import torch
    big = (1 << 22) + 1
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(big, dummy, dummy, dummy)
    assert rc == H.HN_ERR_CAPACITY
    assert "4194304" in H.last_error()
    # a neighbour id out of range is reported, not followed
    off_t = torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda")
    adj_t = torch.tensor([1, 5], dtype=torch.int32, device="cuda")
    out_t = torch.empty(2, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(2, off_t, adj_t, out_t)
    assert rc == H.HN_ERR_INVALID
