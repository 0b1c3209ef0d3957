"""GPU: weighted graphs (one 32-bit value per edge, the reference's
HornetInit::insertEdgeData / weighted BatchUpdate) against the weighted
oracle: construction from an unsorted multigraph CSR, inserts under every
dedup flag combination with batch weights, erases, an unweighted batch on
a weighted graph (weight 0), and float weights kept bit-exact."""
import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from oracle.weighted import WGraph

pytestmark = pytest.mark.gpu


def _unsorted_multigraph(rng, nV=300, m=3000):
    s = rng.integers(0, nV, m).astype(np.int32)
    d = rng.integers(0, nV, m).astype(np.int32)
    order = np.argsort(s, kind="stable")   # grouped by source, neighbours unsorted
    s, d = s[order], d[order]
    off = np.zeros(nV + 1, np.int64)
    np.add.at(off, s + 1, 1)
    return np.cumsum(off).astype(np.int32), d, rng.integers(0, 1 << 32, m, dtype=np.uint64).astype(np.uint32)


def _check(h, wg):
    s, d, w = h.getCOOWeighted()
    rs, rd, rw = wg.coo()
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(d, rd)
    np.testing.assert_array_equal(w, rw)


def test_weighted_construct_insert_erase_sequence():
    rng = np.random.default_rng(3)
    off, adj, w = _unsorted_multigraph(rng)
    init = H.HornetInit(len(off) - 1, len(adj), off, adj)
    init.insertEdgeData(w)
    h = H.Hornet(init)
    assert h.is_weighted()
    wg = WGraph.from_csr(off, adj, w)
    _check(h, wg)
    nV = len(off) - 1
    for it, flags in enumerate([0, 1, 2, 3, 3, 0]):
        es, ed, _ = wg.coo()
        pick = rng.integers(0, len(es), 100)
        bs = np.concatenate([rng.integers(0, nV, 400), es[pick], es[pick[:20]]]).astype(np.int32)
        bd = np.concatenate([rng.integers(0, nV, 400), ed[pick], ed[pick[:20]]]).astype(np.int32)
        bw = rng.integers(0, 1 << 32, len(bs), dtype=np.uint64).astype(np.uint32)
        n = h.insert(H.BatchUpdate(h, bs, bd, bw), removeBatchDuplicates=bool(flags & 1),
                     removeGraphDuplicates=bool(flags & 2))
        assert n == wg.insert(bs, bd, bw, flags)
        _check(h, wg)
        es, ed, _ = wg.coo()
        pick = rng.integers(0, len(es), 150)
        n = h.erase(H.BatchUpdate(h, es[pick], ed[pick]), removeBatchDuplicates=bool(it & 1))
        assert n == wg.erase(es[pick], ed[pick], it & 1)
        _check(h, wg)


def test_unweighted_batch_and_float_weights():
    rng = np.random.default_rng(5)
    g = O.build_csr_undirected(500, rng.integers(0, 500, 2000), rng.integers(0, 500, 2000))
    wf = rng.standard_normal(g.nE).astype(np.float32)
    init = H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True)
    init.insertEdgeData(wf)
    h = H.Hornet(init)
    s, d, w = h.getCOOWeighted(np.float32)
    np.testing.assert_array_equal(w.view(np.uint32), wf.view(np.uint32))
    wg = WGraph.from_csr(g.off, g.adj, wf.view(np.uint32))
    bs = rng.integers(0, 500, 300).astype(np.int32)
    bd = rng.integers(0, 500, 300).astype(np.int32)
    h.insert(H.BatchUpdate(h, bs, bd), True, True)          # no weights: 0
    wg.insert(bs, bd, None, 3)
    _check(h, wg)
    # device-resident weighted batch
    import torch
    ds = torch.from_numpy(bs).cuda()
    dd = torch.from_numpy((bd + 1) % 500).cuda()
    dw = torch.arange(300, dtype=torch.int32, device="cuda")
    h.insert(H.BatchUpdate(h, ds, dd, dw), False, False)
    wg.insert(bs, (bd + 1) % 500, np.arange(300, dtype=np.uint32), 0)
    _check(h, wg)
    # BFS ignores weights
    bfs = H.BfsTopDown(h)
    bfs.set_parameters(0)
    ref = O.Csr(*_csr_of(wg))
    np.testing.assert_array_equal(bfs.run(), O.bfs(ref, 0)[0])


def _csr_of(wg):
    s, d, _ = wg.coo()
    off = np.zeros(wg.nV + 1, np.int64)
    np.add.at(off, s.astype(np.int64) + 1, 1)
    return np.cumsum(off), d


def test_export_weights_of_unweighted_graph_rejected():
    g = O.build_csr_undirected(10, np.arange(9), np.arange(1, 10))
    h = H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))
    assert not h.is_weighted()
    with pytest.raises(H.HornetError):
        h.getCOOWeighted()
