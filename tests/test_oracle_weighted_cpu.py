"""CPU: the weighted update model (oracle/weighted.py) agrees, on the
(src, dst) keys, with the C oracle's multiset insert/erase (itself checked
against the reference's insert/delete test identities), for every flag
combination, on multigraphs with repeated edges."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.weighted import WGraph


def _multigraph(rng, nV=60, m=400):
    s = rng.integers(0, nV, m).astype(np.int32)
    d = rng.integers(0, nV, m).astype(np.int32)
    order = np.lexsort((d, s))
    s, d = s[order], d[order]
    off = np.zeros(nV + 1, np.int64)
    np.add.at(off, s + 1, 1)
    return O.Csr(np.cumsum(off), d), rng.integers(0, 1 << 31, m).astype(np.uint32)


@pytest.mark.parametrize("flags", [0, 1, 2, 3])
def test_weighted_insert_keys_match_c_oracle(flags):
    rng = np.random.default_rng(flags + 10)
    g, w = _multigraph(rng)
    wg = WGraph.from_csr(g.off, g.adj, w)
    es, ed = g.coo()
    pick = rng.integers(0, len(es), 60)
    bs = np.concatenate([rng.integers(0, g.nV, 200), es[pick], es[pick[:10]]]).astype(np.int32)
    bd = np.concatenate([rng.integers(0, g.nV, 200), ed[pick], ed[pick[:10]]]).astype(np.int32)
    bw = rng.integers(0, 1 << 31, len(bs)).astype(np.uint32)
    ref, n_ref = O.insert(g, bs, bd, flags)
    n = wg.insert(bs, bd, bw, flags)
    assert n == n_ref
    s, d, _ = wg.coo()
    rs, rd = ref.coo()
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(d, rd)


@pytest.mark.parametrize("flags", [0, 1])
def test_weighted_erase_keys_match_c_oracle(flags):
    rng = np.random.default_rng(flags + 20)
    g, w = _multigraph(rng)
    wg = WGraph.from_csr(g.off, g.adj, w)
    es, ed = g.coo()
    pick = rng.integers(0, len(es), 150)
    bs, bd = es[pick].astype(np.int32), ed[pick].astype(np.int32)
    ref, n_ref = O.erase(g, bs, bd, flags)
    assert wg.erase(bs, bd, flags) == n_ref
    s, d, _ = wg.coo()
    rs, rd = ref.coo()
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(d, rd)


def test_weights_follow_insertion_order():
    wg = WGraph.from_csr(np.array([0, 2, 2]), np.array([1, 1]), np.array([7, 8], np.uint32))
    wg.insert(np.array([0, 0]), np.array([1, 0]), np.array([9, 5], np.uint32), 0)
    s, d, w = wg.coo()
    assert list(zip(s, d, w)) == [(0, 0, 5), (0, 1, 7), (0, 1, 8), (0, 1, 9)]
    wg.erase(np.array([0]), np.array([1]), 1)
    assert list(zip(*wg.coo())) == [(0, 0, 5), (0, 1, 8), (0, 1, 9)]
