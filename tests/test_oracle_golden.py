"""CPU: pin the oracle against the reference's own outputs.

tests/golden/*.npz were produced by the reference's host code (xlib GraphStd
reader, graph::BFS, graph::WCC) on the reference's example graphs and on a
small R-MAT graph (tests/golden/make_golden.py).  When oracle/_ref was built
in this container the same comparisons also run live on fresh inputs."""
import itertools
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as T

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["G", "G_cc2", "rome99", "rmat8"]


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    return z, O.Csr(z["off"], z["adj"])


def sorted_lists(g: O.Csr) -> O.Csr:
    adj = g.adj.copy()
    for v in range(g.nV):
        adj[g.off[v]:g.off[v + 1]].sort()
    return O.Csr(g.off, adj)


@pytest.mark.parametrize("name", FIXTURES)
def test_bfs_matches_reference(name):
    z, g = load(name)
    for i, s in enumerate(z["bfs_src"]):
        dist, _ = O.bfs(g, int(s))
        np.testing.assert_array_equal(dist, z["bfs"][i])


@pytest.mark.parametrize("name", FIXTURES)
def test_cc_matches_reference_wcc(name):
    z, g = load(name)
    lab, n = O.cc_min_label(g)
    np.testing.assert_array_equal(lab, O.canon_labels(z["wcc"]))
    assert n == len(np.unique(z["wcc"]))


@pytest.mark.parametrize("name", FIXTURES)
def test_orientation_matches_reference(name):
    z, g = load(name)
    o = O.orient_by_degree(sorted_lists(g))
    ref = sorted_lists(O.Csr(z["ooff"], z["oadj"]))
    np.testing.assert_array_equal(o.off, ref.off)
    np.testing.assert_array_equal(o.adj, ref.adj)


def test_csr_builder_matches_reference_graphstd():
    """GraphStd mirrors every pair, sorts and dedups, but keeps ONE copy of
    each self loop (GraphStd.cpp:175-190 skips only the mirror).  The
    configurations drop self loops, which is the only difference."""
    z, gref = load("rmat8")
    p = np.load(os.path.join(GOLD, "rmat8_pairs.npz"))
    g = O.build_csr_undirected(256, p["src"], p["dst"])
    s, d = gref.coo()
    keep = s != d
    np.testing.assert_array_equal(g.coo()[0], s[keep])
    np.testing.assert_array_equal(g.coo()[1], d[keep])


def test_known_answers_example_graph():
    """example/G.mtx: 9 vertices, 12 pairs -> 11 undirected edges, one
    component, BFS levels from vertex 0 and 2 triangles (0-2-3, 2-3-8)."""
    z, g = load("G")
    assert g.nV == 9 and g.nE == 22
    np.testing.assert_array_equal(O.bfs(g, 0)[0], [0, 2, 1, 1, 1, 2, 2, 2, 2])
    assert O.tc(g) == 2
    assert O.cc_min_label(g)[1] == 1


def brute_triangles(g: O.Csr) -> int:
    adj = [set(g.adj[g.off[v]:g.off[v + 1]].tolist()) for v in range(g.nV)]
    return sum(1 for a, b, c in itertools.combinations(range(g.nV), 3)
               if b in adj[a] and c in adj[a] and c in adj[b])


def brute_truss(g: O.Csr):
    """k-truss by definition: largest k whose k-truss (support >= k-2 inside
    it) contains the edge."""
    edges = {(int(u), int(v)) for u, v in zip(*g.coo()) if u < v}
    truss = {e: 2 for e in edges}
    k = 3
    cur = set(edges)
    while True:
        changed = True
        while changed:
            adj = {}
            for u, v in cur:
                adj.setdefault(u, set()).add(v)
                adj.setdefault(v, set()).add(u)
            bad = {(u, v) for u, v in cur if len(adj[u] & adj[v]) < k - 2}
            changed = bool(bad)
            cur -= bad
        if not cur:
            return k - 1, truss
        for e in cur:
            truss[e] = k
        k += 1


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_tc_and_ktruss_against_brute_force(seed):
    g = T.er_graph(40, 9, seed)
    assert O.tc(g) == brute_triangles(g)
    k, et = O.ktruss(g)
    bk, bt = brute_truss(g)
    assert k == bk
    s, d = g.coo()
    for e, (u, v) in enumerate(zip(s, d)):
        assert et[e] == bt[(min(u, v), max(u, v))]


def test_update_model_roundtrip_and_multiset():
    g = T.rmat_graph(8, 8, seed=3)
    rng = np.random.default_rng(0)
    bs = rng.integers(0, g.nV, 300).astype(np.int32)
    bd = rng.integers(0, g.nV, 300).astype(np.int32)
    g1, n = O.insert(g, bs, bd, 0)           # plain multiset union
    assert n == 300 and g1.nE == g.nE + 300
    g2, r = O.erase(g1, bs, bd, 0)           # multiset difference undoes it
    assert r == 300
    np.testing.assert_array_equal(g2.adj, g.adj)
    np.testing.assert_array_equal(g2.off, g.off)
    # graph de-duplication drops only the FIRST copy of an existing edge
    s, d = g.coo()
    g3, n3 = O.insert(g, [s[0], s[0]], [d[0], d[0]], 2)
    assert n3 == 1
    g4, n4 = O.insert(g, [s[0], s[0]], [d[0], d[0]], 3)
    assert n4 == 0 and g4.nE == g.nE
    # erase removes min(batch, graph) copies
    g5, r5 = O.erase(g3, [s[0]] * 3, [d[0]] * 3, 0)
    assert r5 == 2
    g6, r6 = O.erase(g3, [s[0]] * 3, [d[0]] * 3, 1)
    assert r6 == 1
    with pytest.raises(ValueError):
        O.insert(g, [g.nV], [0], 0)


def test_reference_colors_definition():
    z, g = load("G_cc2")
    col = O.cc_reference_colors(g)
    lab, _ = O.cc_min_label(g)
    deg = np.diff(g.off)
    giant = lab[int(np.argmax(deg))]
    for v in range(g.nV):
        if lab[v] == giant:
            assert col[v] == 0
        else:
            assert col[v] == max(u for u in range(g.nV) if lab[u] == lab[v]) + 1


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_live_reference_bfs_wcc_on_rmat():
    g = T.rmat_graph(11, 8, seed=21)
    srcs = [0, 5, 1000, 2047]
    ref = O.ref_bfs(g, srcs)
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(O.bfs(g, s)[0], ref[i])
    np.testing.assert_array_equal(O.cc_min_label(g)[0], O.canon_labels(O.ref_wcc(g)))
