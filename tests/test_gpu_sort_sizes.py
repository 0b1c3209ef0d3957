"""GPU: batch sizes around the update sort's tiles and pass counts.

The batch sort (hn_sort.cu) takes 8 key bits a pass over 2*key_bits bits
(1 pass for 5 vertices, 3 for 3,000, 5 for 2^20), in tiles of 4,096 keys
(2,048 with weights), with a look-back across tiles.  Inserts and erases
of batches of 1..20,001 entries, with in-batch duplicates spread across
tile boundaries, equal the oracle's multiset model; on a weighted graph the
weights of duplicate batch entries keep their batch order across tiles (the
sort is stable), as the weighted oracle requires."""
import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from oracle.weighted import WGraph
from tests import helpers as T

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 2047, 2048, 2049, 4095, 4096, 4097, 8193, 20001]


def _same(h, g):
    s, d = h.getCOO()
    rs, rd = g.coo()
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(d, rd)


@pytest.mark.parametrize("nV", [5, 3000, 1 << 20])
def test_update_batch_sizes_around_sort_tiles(nV):
    rng = np.random.default_rng(nV)
    g = T.er_graph(nV, 4, seed=7) if nV > 5 else \
        O.build_csr_undirected(5, np.array([0, 1], np.int32), np.array([1, 2], np.int32))
    h = H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))
    for i, n in enumerate(SIZES):
        s = rng.integers(0, nV, n).astype(np.int32)
        d = rng.integers(0, nV, n).astype(np.int32)
        if n > 8:   # duplicates far apart in the batch (other tiles)
            k = n // 8
            s[-k:], d[-k:] = s[:k], d[:k]
        flags = (True, True) if i % 2 else (False, False)
        a = h.insert(H.BatchUpdate(h, s, d), *flags)
        g, na = O.insert(g, s, d, 3 if flags[0] else 0)
        assert a == na, n
        _same(h, g)
        es, ed = g.coo()
        pick = rng.integers(0, len(es), n)
        dedup = bool(i % 2)
        r = h.erase(H.BatchUpdate(h, es[pick], ed[pick]), dedup)
        g, nr = O.erase(g, es[pick], ed[pick], 1 if dedup else 0)
        assert r == nr, n
        _same(h, g)


def test_weighted_duplicates_across_sort_tiles():
    rng = np.random.default_rng(12)
    nV = 4000
    g = T.er_graph(nV, 3, seed=1)
    w0 = rng.integers(0, 1 << 32, g.nE, dtype=np.uint64).astype(np.uint32)
    init = H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True)
    init.insertEdgeData(w0)
    h = H.Hornet(init)
    wg = WGraph.from_csr(g.off32(), g.adj, w0)
    for n in [2047, 2049, 4097, 6145]:
        s = rng.integers(0, nV, n).astype(np.int32)
        d = rng.integers(0, nV, n).astype(np.int32)
        k = n // 4   # the first quarter again at the end: equal keys two tiles apart
        s[-k:], d[-k:] = s[:k], d[:k]
        w = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        for flags in (0, 1):
            assert h.insert(H.BatchUpdate(h, s, d, w), removeBatchDuplicates=bool(flags & 1),
                            removeGraphDuplicates=False) == wg.insert(s, d, w, flags)
            hs, hd, hw = h.getCOOWeighted()
            rs, rd, rw = wg.coo()
            np.testing.assert_array_equal(hs, rs)
            np.testing.assert_array_equal(hd, rd)
            np.testing.assert_array_equal(hw, rw)
