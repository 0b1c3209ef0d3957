"""CPU: the update model that the scale-24 GPU test (test_gpu_c3_updates)
compares the device against agrees with the oracle's restated update model
(hno_insert / hno_erase, BatchUpdate.i.cuh:485-524) and with the oracle's
adjacency checksum, batch after batch, on a small graph."""
import numpy as np

from oracle import oracle as O
from tests import helpers as T


def test_update_model_matches_oracle():
    g = T.rmat_graph(10, 8, seed=12)
    base = (np.repeat(np.arange(g.nV, dtype=np.int64), np.diff(g.off)) << 32) | \
        g.adj.astype(np.int64)
    m = T.UpdateModel(base, O.adjacency_hash(g))
    rng = np.random.default_rng(3)
    for step in range(12):
        b = int(rng.integers(1, 3000))
        if step % 3 == 2:   # pairs taken from the graph itself: real deletions
            s, d = g.coo()
            idx = rng.integers(0, len(s), b)
            bs, bd = s[idx], d[idx]
        else:
            bs = rng.integers(0, g.nV, b).astype(np.int32)
            bd = rng.integers(0, g.nV, b).astype(np.int32)
        keys = (bs.astype(np.int64) << 32) | bd.astype(np.int64)
        if step % 2 == 0:
            g, n = O.insert(g, bs, bd, 3)   # removeBatchDuplicates | removeGraphDuplicates
            assert m.insert(keys) == n
        else:
            g, n = O.erase(g, bs, bd, 1)    # removeBatchDuplicates
            assert m.erase(keys) == n
        assert m.hash == O.adjacency_hash(g)
        for u in rng.integers(0, g.nV, 20):
            np.testing.assert_array_equal(m.neighbours(int(u)), g.adj[g.off[u]:g.off[u + 1]])
