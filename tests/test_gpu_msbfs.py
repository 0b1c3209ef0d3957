"""GPU parity of the batched BFS (hn_bfs_batch): up to 64 BFS slots in one
traversal.  Every slot's distances are compared bit-exactly with the
oracle's single-source BFS (the restatement of
hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu), and the per-slot
statistics with the oracle's counts."""
import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from tests import helpers as T

pytestmark = pytest.mark.gpu


def build(g: O.Csr) -> H.Hornet:
    return H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))


def oracle_slots(g, sources, slots, nslots):
    """Per slot: the minimum over its sources of the single-source BFS
    distance (the multi-source BFS distance), with visited/scanned/levels."""
    dist = np.full((nslots, g.nV), O.INF, np.int64)
    for s, b in zip(sources, slots):
        d, _ = O.bfs(g, int(s))
        dist[b] = np.minimum(dist[b], d)
    stats = []
    for b in range(nslots):
        reached = dist[b] != O.INF
        deg = np.diff(g.off)
        lv = int(dist[b][reached].max()) + 1 if reached.any() else 0
        stats.append((int(reached.sum()), int(deg[reached].sum()), lv))
    return dist.astype(np.int32), stats


def check(out, st, ref, ref_stats):
    np.testing.assert_array_equal(out, ref)
    for b, (vis, scanned, lv) in enumerate(ref_stats):
        assert st[b].visited == vis, b
        assert st[b].edges_scanned == scanned, b
        assert st[b].levels == lv, b


@pytest.mark.parametrize("name,k", [("rmat10", 64), ("er2000", 17), ("rmat12_nonpow2", 64)])
def test_batch_one_source_per_slot(name, k):
    g = {"rmat10": lambda: T.rmat_graph(10, 16, seed=3),
         "er2000": lambda: T.er_graph(2000, 8, seed=5),
         "rmat12_nonpow2": lambda: T.rmat_graph(12, 8, seed=7, n_vertices=3000)}[name]()
    h = build(g)
    rng = np.random.default_rng(11)
    srcs = np.concatenate([[0], rng.integers(0, g.nV, k - 1)]).astype(np.int32)
    out, st = H.BfsTopDown(h).run_batch(srcs)
    ref, ref_stats = oracle_slots(g, srcs, range(k), k)
    check(out, st, ref, ref_stats)
    # the same as k single-source runs through hn_bfs_multi
    multi, mst = H.BfsTopDown(h).run_multi(srcs)
    np.testing.assert_array_equal(out, multi)
    for b in range(k):
        assert st[b].levels == mst[b].levels


def test_batch_duplicate_sources_and_sparse_slots():
    g = T.rmat_graph(11, 8, seed=9)
    h = build(g)
    # the same vertex in several slots, two sources in one slot, slots 3..7 empty
    srcs = np.array([5, 5, 17, 900, 5, 5], np.int32)
    slots = np.array([0, 1, 1, 2, 8, 8], np.int32)
    out, st = H.BfsTopDown(h).run_batch(srcs, slots=slots, nslots=9)
    ref, ref_stats = oracle_slots(g, srcs, slots, 9)
    check(out, st, ref, ref_stats)
    assert (out[3:8] == O.INF).all()


def test_batch_disjoint_union_many_graphs():
    """4096-graph pattern, scaled down: 96 small graphs in one union, one
    source per graph, 8 slots; every graph's distances equal its own BFS."""
    graphs = [T.rmat_graph(6, 4, seed=100 + i) if i % 3 else T.er_graph(50, 3, seed=i)
              for i in range(96)]
    u, base = T.disjoint_union(graphs)
    h = build(u)
    rng = np.random.default_rng(3)
    srcs = np.array([base[i] + rng.integers(0, graphs[i].nV) for i in range(96)], np.int32)
    slots = np.arange(96, dtype=np.int32) % 8
    out, st = H.BfsTopDown(h).run_batch(srcs, slots=slots, nslots=8)
    for i, gi in enumerate(graphs):
        d, _ = O.bfs(gi, int(srcs[i] - base[i]))
        np.testing.assert_array_equal(out[slots[i], base[i]:base[i] + gi.nV], d)
    ref, ref_stats = oracle_slots(u, srcs, slots, 8)
    check(out, st, ref, ref_stats)


def test_batch_after_updates_and_isolated():
    g = T.rmat_graph(10, 8, seed=21)
    h = build(g)
    bfs = H.BfsTopDown(h)
    srcs = np.arange(0, 640, 10, dtype=np.int32)
    out0, _ = bfs.run_batch(srcs)
    np.testing.assert_array_equal(out0, oracle_slots(g, srcs, range(64), 64)[0])
    s, d = T.uniform_new_edges(g, 3000, seed=2)
    h.insert(H.BatchUpdate(h, s, d), removeBatchDuplicates=True, removeGraphDuplicates=True)
    g2, _ = O.insert(g, s, d, 3)
    out1, st1 = bfs.run_batch(srcs)
    ref, ref_stats = oracle_slots(g2, srcs, range(64), 64)
    check(out1, st1, ref, ref_stats)


def test_batch_device_output_and_errors():
    import torch
    g = T.er_graph(500, 4, seed=1)
    h = build(g)
    srcs = np.array([1, 2, 3], np.int32)
    dev = torch.empty((3, g.nV), dtype=torch.int32, device="cuda")
    H.BfsTopDown(h).run_batch(srcs, out=dev)
    np.testing.assert_array_equal(dev.cpu().numpy(), oracle_slots(g, srcs, range(3), 3)[0])
    with pytest.raises(H.HornetError):
        H.BfsTopDown(h).run_batch(np.arange(65, dtype=np.int32) % g.nV, nslots=65)
    with pytest.raises(H.HornetError):
        H.BfsTopDown(h).run_batch(srcs, slots=np.array([0, 1, 4], np.int32), nslots=4 - 1)
    with pytest.raises(H.HornetError):
        H.BfsTopDown(h).run_batch(np.array([g.nV], np.int32))


@pytest.mark.parametrize("block,ctas,bu", [(128, 2, 1), (512, 8, 0), (256, 6, 1), (256, 4, 0)])
def test_batch_block_size_knobs(block, ctas, bu):
    """Every batched-BFS launch shape the autotuner may pick gives the same
    distances (the CUDA graph is rebuilt when a knob changes)."""
    g = T.rmat_graph(11, 16, seed=13)
    h = build(g)
    srcs = np.arange(0, 2048, 64, dtype=np.int32)
    ref, ref_stats = oracle_slots(g, srcs, range(len(srcs)), len(srcs))
    try:
        H.tune_set("msbfs.block", block)
        H.tune_set("msbfs.ctas_per_sm", ctas)
        H.tune_set("msbfs.bottom_up", bu)
        out, st = H.BfsTopDown(h).run_batch(srcs)
        check(out, st, ref, ref_stats)
    finally:
        H.tune_reset()


@pytest.mark.parametrize("alpha,beta", [(1, 1 << 20), (1 << 20, 1), (14, 24)])
def test_batch_bottom_up_switching(alpha, beta):
    """Bottom-up levels from the first level on (alpha 1), never (huge
    alpha), and the default switch: distances and statistics unchanged."""
    g = T.rmat_graph(12, 16, seed=23)
    h = build(g)
    srcs = np.arange(0, 4096, 97, dtype=np.int32)
    ref, ref_stats = oracle_slots(g, srcs, range(len(srcs)), len(srcs))
    try:
        H.tune_set("msbfs.bottom_up", 1)
        H.tune_set("bfs.do_alpha", alpha)
        H.tune_set("bfs.do_beta", beta)
        out, st = H.BfsTopDown(h).run_batch(srcs)
        check(out, st, ref, ref_stats)
    finally:
        H.tune_reset()
