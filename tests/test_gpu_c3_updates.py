"""GPU: the dynamic-update configuration at its own size.

R-MAT scale 24 (16,777,216 vertices, edge factor 16, seed 1) resident on the
device.  Batches of 1K, 10K, 100K, 1M and 10M directed edges, each drawn
two ways: uniformly at random, and from the R-MAT distribution with about
5 % in-batch duplicates (copies of other pairs of the same batch).  Each
batch holds both directions of its pairs, so the graph stays undirected.
Every batch is inserted (removeBatchDuplicates, removeGraphDuplicates, with
the incremental triangle count) and then erased (removeBatchDuplicates):
the insert/erase semantics of hornet/include/Core/HornetOperations/
HornetInsert.i.cuh:12-27,71-89 as the reference's HornetInsertTest.cu and
HornetDeleteTest.cu check them.

After every batch the device graph's adjacency checksum (hn_graph_adjacency_
hash) equals the CPU model's, and the applied/removed counts agree.  After
each 10M batch the sorted lists of 2,000 touched vertices are compared
exactly.  After each insert, the incrementally counted new triangles equal
the change of the full recount (TriangleCounting2).

The CPU model (tests.helpers.UpdateModel, checked against the oracle's
restated update model by tests/test_update_model_cpu.py) holds the initial
graph as sorted 64-bit (src, dst) keys plus the sets of keys added and
removed since, so it needs no copy of the graph per batch.
"""
import ctypes

import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from tests.helpers import UpdateModel

pytestmark = pytest.mark.gpu

SCALE = 24
SIZES = [1_000, 10_000, 100_000, 1_000_000, 10_000_000]


def make_batch(rng, kind: str, b: int, nV: int, seed: int):
    """b directed entries: b/2 pairs (no self loops) and their mirrors; the
    R-MAT kind replaces ~5 % of its pairs by copies of other pairs."""
    half = b // 2
    if kind == "uniform":
        u = rng.integers(0, nV, half).astype(np.int32)
        v = rng.integers(0, nV, half).astype(np.int32)
    else:
        u, v = O.gen_rmat(SCALE, half, seed)
        ndup = half // 20
        to = rng.choice(half, ndup, replace=False)
        frm = rng.integers(0, half, ndup)
        u[to], v[to] = u[frm], v[frm]
    keep = u != v
    u, v = u[keep], v[keep]
    return np.concatenate([u, v]), np.concatenate([v, u])


def test_c3_batches_at_scale_24():
    import torch
    n = 1 << SCALE
    src = torch.empty(16 * n, dtype=torch.int32, device="cuda")
    dst = torch.empty_like(src)
    H.gen_rmat_device(SCALE, 16 * n, 1, src, dst)
    csr = H.coo_to_csr_device(n, src, dst)
    del src, dst
    h = H.hornet_from_device_csr(csr)
    nV, nE = h.nV(), h.nE()
    off = torch.empty(nV + 1, dtype=torch.int32, device="cuda")
    adj = torch.empty(nE, dtype=torch.int32, device="cuda")
    H._check(H.lib().hn_graph_export_csr(h.handle, ctypes.c_void_p(off.data_ptr()),
                                         ctypes.c_void_p(adj.data_ptr()), H.HN_MEM_DEVICE))
    g = O.Csr(off.cpu().numpy().astype(np.int64), adj.cpu().numpy())
    del off, adj, csr
    h0 = O.adjacency_hash(g)
    assert h.adjacency_hash() == h0
    base = (np.repeat(np.arange(nV, dtype=np.int64), np.diff(g.off)) << 32) | \
        g.adj.astype(np.int64)
    del g
    model = UpdateModel(base, h0)
    tc = H.TriangleCounting2(h)
    tri = tc.run()
    rng = np.random.default_rng(2024)
    for kind in ("uniform", "rmat"):
        for i, b in enumerate(SIZES):
            bs, bd = make_batch(rng, kind, b, nV, seed=77 + i)
            keys = (bs.astype(np.int64) << 32) | bd.astype(np.int64)
            batch = H.BatchUpdate(h, torch.from_numpy(bs).cuda(), torch.from_numpy(bd).cuda())
            applied, new_tri = h.insert_count_triangles(batch)
            assert applied == model.insert(keys), (kind, b)
            assert h.adjacency_hash() == model.hash, (kind, b, "insert")
            tri_after = tc.run()
            assert tri_after - tri == new_tri, (kind, b)
            if b == SIZES[-1]:
                touched = np.unique(bs)
                sample = rng.choice(touched, 2000, replace=False)
                offd = torch.empty(nV + 1, dtype=torch.int32, device="cuda")
                adjd = torch.empty(h.nE(), dtype=torch.int32, device="cuda")
                H._check(H.lib().hn_graph_export_csr(
                    h.handle, ctypes.c_void_p(offd.data_ptr()), ctypes.c_void_p(adjd.data_ptr()),
                    H.HN_MEM_DEVICE))
                oh = offd.cpu().numpy()
                for u in sample:
                    got = adjd[int(oh[u]):int(oh[u + 1])].cpu().numpy()
                    np.testing.assert_array_equal(got, model.neighbours(int(u)))
                del offd, adjd
            removed = h.erase(batch, True)
            assert removed == model.erase(keys), (kind, b)
            assert h.adjacency_hash() == model.hash, (kind, b, "erase")
            tri = tc.run()
    assert h.nE() == len(model.base) - len(model.removed) + len(model.added)
