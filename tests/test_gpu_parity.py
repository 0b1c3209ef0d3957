"""GPU parity: the sm_100a library through the C ABI against the CPU oracle
(and the reference's own host BFS/WCC where oracle/_ref was built).
Every comparison is bit-exact (integer results)."""
import ctypes

import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from tests import helpers as T

pytestmark = pytest.mark.gpu

DEDUP_BOTH = dict(removeBatchDuplicates=True, removeGraphDuplicates=True)


def build(g: O.Csr, sorted_adj=True) -> H.Hornet:
    return H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=sorted_adj))


def assert_same_graph(h: H.Hornet, g: O.Csr):
    assert h.nE() == g.nE
    s, d = h.getCOO(True)
    gs, gd = g.coo()
    np.testing.assert_array_equal(s, gs)
    np.testing.assert_array_equal(d, gd)


GRAPHS = {
    "rmat10": lambda: T.rmat_graph(10, 16, seed=3),
    "er2000": lambda: T.er_graph(2000, 8, seed=5),
    "rmat12_nonpow2": lambda: T.rmat_graph(12, 8, seed=7, n_vertices=3000),
}


@pytest.mark.parametrize("name", list(GRAPHS))
def test_construct_export(name):
    g = GRAPHS[name]()
    h = build(g)
    assert h.nV() == g.nV
    assert_same_graph(h, g)
    off, adj = h.getCSR()
    np.testing.assert_array_equal(off, g.off32())
    np.testing.assert_array_equal(adj, g.adj)
    deg = np.diff(g.off)
    np.testing.assert_array_equal(h.degrees(), deg)
    assert h.max_degree() == deg.max()
    assert h.max_degree_id() == int(np.argmax(deg))  # lowest id on ties


def test_construct_unsorted_input_is_sorted():
    g = T.rmat_graph(9, 8, seed=11)
    rng = np.random.default_rng(0)
    adj = g.adj.copy()
    for v in range(g.nV):
        a, b = g.off[v], g.off[v + 1]
        rng.shuffle(adj[a:b])
    h = H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), adj, sorted_adjacency=False))
    assert_same_graph(h, g)


def test_construct_unsorted_large_multigraph():
    """A larger unsorted CSR (2^17 vertices: five 8-bit sort passes over
    34-bit keys), with empty lists first, in the middle and last, a hub, and
    repeated neighbours: the lists come out sorted, multiplicities kept."""
    rng = np.random.default_rng(4)
    nV = 1 << 17
    s, d = H.gen_rmat_host(16, 400_000, 3)
    s = s.astype(np.int64) + 5          # vertices 0..4 empty
    d = d.astype(np.int32) + 5
    keep = (s < nV - 7) & (s != 40000)  # the last 7 and vertex 40000 empty
    s, d = s[keep], d[keep]
    dup = rng.choice(len(s), 20000)
    s = np.concatenate([s, s[dup]])
    d = np.concatenate([d, d[dup]])
    order = np.argsort(s, kind="stable")   # grouped by source, neighbours unsorted
    s, d = s[order], d[order]
    off = np.zeros(nV + 1, np.int64)
    np.add.at(off, s + 1, 1)
    off = np.cumsum(off)
    for v in rng.choice(nV, 50, replace=False):   # shuffle some lists more
        a, b = off[v], off[v + 1]
        rng.shuffle(d[a:b])
    h = H.Hornet(H.HornetInit(nV, len(d), off.astype(np.int32), d, sorted_adjacency=False))
    hs, hd = h.getCOO(True)
    ref = np.lexsort((d, s))
    np.testing.assert_array_equal(hs, s[ref])
    np.testing.assert_array_equal(hd, d[ref])


def test_construct_with_isolated_and_empty():
    # vertices 0, 5, 9 isolated
    s = np.array([1, 2, 3, 6, 7], np.int32)
    d = np.array([2, 3, 4, 7, 8], np.int32)
    g = O.build_csr_undirected(10, s, d)
    h = build(g)
    assert_same_graph(h, g)
    e = O.Csr(np.zeros(5, np.int64), np.zeros(0, np.int32))
    h0 = build(e)
    assert h0.nE() == 0 and h0.nV() == 4
    assert h0.max_degree() == 0 and h0.max_degree_id() == 0


def test_invalid_ids_rejected_graph_unchanged():
    g = T.rmat_graph(8, 8, seed=2)
    h = build(g)
    b = H.BatchUpdate(h, np.array([0, g.nV], np.int32), np.array([1, 1], np.int32))
    with pytest.raises(H.HornetError) as ei:
        h.insert(b)
    assert ei.value.code == H.HN_ERR_INVALID
    assert_same_graph(h, g)
    with pytest.raises(H.HornetError):
        H.Hornet(H.HornetInit(3, 1, np.array([0, 1, 1, 1], np.int32), np.array([7], np.int32)))


@pytest.mark.parametrize("flags", [(False, False), (True, False), (False, True), (True, True)])
def test_insert_multiset_semantics(flags):
    """Batch with in-batch duplicates and edges already present, all four
    removeBatchDuplicates/removeGraphDuplicates combinations."""
    g = T.rmat_graph(9, 8, seed=4)
    rng = np.random.default_rng(1)
    es, ed = g.coo()
    pick = rng.choice(len(es), 300, replace=False)
    bs = np.concatenate([rng.integers(0, g.nV, 700).astype(np.int32), es[pick]])
    bd = np.concatenate([rng.integers(0, g.nV, 700).astype(np.int32), ed[pick]])
    dup = rng.choice(len(bs), 150)
    bs = np.concatenate([bs, bs[dup]])
    bd = np.concatenate([bd, bd[dup]])
    h = build(g)
    b = H.BatchUpdate(h, bs, bd)
    applied = h.insert(b, removeBatchDuplicates=flags[0], removeGraphDuplicates=flags[1])
    f = (O_FLAG_BATCH if flags[0] else 0) | (O_FLAG_GRAPH if flags[1] else 0)
    ref, n = O.insert(g, bs, bd, f)
    assert applied == n
    assert_same_graph(h, ref)


O_FLAG_BATCH, O_FLAG_GRAPH = 1, 2


@pytest.mark.parametrize("dedup", [False, True])
def test_erase_multiset_semantics(dedup):
    g0 = T.rmat_graph(9, 8, seed=6)
    rng = np.random.default_rng(2)
    # make a multigraph first: insert some existing edges again
    es, ed = g0.coo()
    pick = rng.choice(len(es), 400, replace=False)
    h = build(g0)
    h.insert(H.BatchUpdate(h, es[pick], ed[pick]))
    g, _ = O.insert(g0, es[pick], ed[pick], 0)
    assert_same_graph(h, g)
    # erase: existing (some duplicated in the batch) + absent edges
    pick2 = rng.choice(len(es), 500, replace=False)
    bs = np.concatenate([es[pick2], es[pick2[:100]], rng.integers(0, g.nV, 200).astype(np.int32)])
    bd = np.concatenate([ed[pick2], ed[pick2[:100]], rng.integers(0, g.nV, 200).astype(np.int32)])
    removed = h.erase(H.BatchUpdate(h, bs, bd), removeBatchDuplicates=dedup)
    ref, n = O.erase(g, bs, bd, O_FLAG_BATCH if dedup else 0)
    assert removed == n
    assert_same_graph(h, ref)


def test_update_sequence_alternating():
    """Alternately insert and delete batches of several sizes, sorted
    adjacency re-checked after every batch."""
    g = T.rmat_graph(11, 16, seed=8)
    h = build(g)
    rng = np.random.default_rng(3)
    for it, k in enumerate([10, 1000, 5000, 1, 20000, 300]):
        bs = rng.integers(0, g.nV, k).astype(np.int32)
        bd = rng.integers(0, g.nV, k).astype(np.int32)
        b = H.BatchUpdate(h, bs, bd)
        a = h.insert(b, **DEDUP_BOTH)
        g, n = O.insert(g, bs, bd, 3)
        assert a == n
        assert_same_graph(h, g)
        es, ed = g.coo()
        sel = rng.choice(len(es), min(k, len(es)), replace=False)
        b.reset(es[sel], ed[sel])
        r = h.erase(b, removeBatchDuplicates=True)
        g, n = O.erase(g, es[sel], ed[sel], 1)
        assert r == n
        assert_same_graph(h, g)
    pool, used, free_blocks = h.memory()
    assert used <= pool


def test_erase_everything_then_reinsert():
    g = T.rmat_graph(8, 8, seed=9)
    h = build(g)
    s, d = g.coo()
    assert h.erase(H.BatchUpdate(h, s, d)) == g.nE
    assert h.nE() == 0
    assert (h.degrees() == 0).all()
    assert h.insert(H.BatchUpdate(h, s, d)) == g.nE
    assert_same_graph(h, g)


@pytest.mark.parametrize("name", ["rmat10", "er2000"])
def test_bfs(name):
    g = GRAPHS[name]()
    h = build(g)
    bfs = H.BfsTopDown(h)
    rng = np.random.default_rng(4)
    srcs = [0] + list(rng.integers(0, g.nV, 4))
    for s in srcs:
        bfs.set_parameters(int(s))
        dist = bfs.run()
        ref, scanned = O.bfs(g, int(s))
        np.testing.assert_array_equal(dist, ref)
        assert bfs.stats.edges_scanned == scanned
        assert bfs.stats.visited == int((ref != O.INF).sum())
    if O.ref_available():
        out, _ = bfs.run_multi(srcs)
        np.testing.assert_array_equal(out, O.ref_bfs(g, srcs))


@pytest.mark.parametrize("name", ["rmat10", "er2000", "rmat12_nonpow2"])
def test_bfs_direction_optimizing(name):
    """Direction-optimising BFS (bottom-up levels on large frontiers) gives
    exactly the top-down distances and counts the same scanned edges."""
    g = GRAPHS[name]()
    h = build(g)
    rng = np.random.default_rng(6)
    srcs = [0] + [int(x) for x in rng.integers(0, g.nV, 5)]
    td, td_stats = H.BfsTopDown(h).run_multi(srcs)
    do, do_stats = H.BfsTopDown(h).run_multi(srcs, direction_optimizing=True)
    np.testing.assert_array_equal(do, td)
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(do[i], O.bfs(g, s)[0])
        assert do_stats[i].edges_scanned == td_stats[i].edges_scanned
        assert do_stats[i].visited == td_stats[i].visited
        assert do_stats[i].levels == td_stats[i].levels


def _shape_graph(kind):
    """Graphs that reach every branch of the level kernels: a star whose hub
    spans many 256- and 1024-edge chunks, a long path (one vertex per
    level), many vertices of degree 1-2 (windows of more than 32 vertices
    per chunk) and hubs joined by paths."""
    rng = np.random.default_rng(17)
    if kind == "star":
        n = 20001
        s = np.zeros(n - 1, np.int32)
        d = np.arange(1, n, dtype=np.int32)
    elif kind == "path":
        n = 3000
        s = np.arange(n - 1, dtype=np.int32)
        d = s + 1
    elif kind == "sparse":
        n = 50000
        s = rng.integers(0, n, n // 2).astype(np.int32)
        d = rng.integers(0, n, n // 2).astype(np.int32)
        s = np.concatenate([s, np.arange(n - 1, dtype=np.int32)])
        d = np.concatenate([d, np.arange(1, n, dtype=np.int32)])
    else:   # "hubs": four stars of 6000 leaves whose hubs are joined by a path
        n = 4 * 6001 + 100
        ss, dd = [], []
        for h in range(4):
            hub = h * 6001
            ss.append(np.full(6000, hub, np.int32))
            dd.append(np.arange(hub + 1, hub + 6001, dtype=np.int32))
        chain = np.array([0, 24004, 6001, 24010, 12002, 24020, 18003], np.int32)
        ss.append(chain[:-1])
        dd.append(chain[1:])
        s, d = np.concatenate(ss), np.concatenate(dd)
    return O.build_csr_undirected(n, s, d)


@pytest.mark.parametrize("kernel", [1, 0])
@pytest.mark.parametrize("kind", ["star", "path", "sparse", "hubs"])
def test_bfs_graph_shapes_both_kernels(kind, kernel):
    """Both level kernels (warp chunks and CTA chunks), top-down and
    direction-optimising, equal the oracle on graphs that stress the chunk
    table: hubs spanning many chunks, one vertex per level, and windows of
    many low-degree vertices."""
    g = _shape_graph(kind)
    h = build(g)
    srcs = [0, g.nV - 1, g.nV // 2]
    try:
        H.tune_set("bfs.kernel", kernel)
        td, st = H.BfsTopDown(h).run_multi(srcs)
        do, _ = H.BfsTopDown(h).run_multi(srcs, direction_optimizing=True)
    finally:
        H.tune_reset()
    for i, s in enumerate(srcs):
        ref, scanned = O.bfs(g, s)
        np.testing.assert_array_equal(td[i], ref)
        np.testing.assert_array_equal(do[i], ref)
        assert st[i].edges_scanned == scanned


def test_bfs_isolated_source():
    s = np.array([1, 2], np.int32)
    d = np.array([2, 3], np.int32)
    g = O.build_csr_undirected(5, s, d)
    h = build(g)
    bfs = H.BfsTopDown(h)
    bfs.set_parameters(0)
    dist = bfs.run()
    assert dist[0] == 0 and (dist[1:] == O.INF).all()


@pytest.mark.parametrize("name", list(GRAPHS))
def test_tc(name):
    g = GRAPHS[name]()
    h = build(g)
    tc = H.TriangleCounting2(h)
    tc.init()
    total = tc.run(per_vertex=True)
    ref, pv = O.tc(g, per_vertex=True)
    assert total == ref
    np.testing.assert_array_equal(tc.copyTCToHost(), pv)


@pytest.mark.parametrize("name", list(GRAPHS))
def test_cc(name):
    g = GRAPHS[name]()
    h = build(g)
    cc = H.CC(h)
    lab = cc.run()
    ref, ncomp = O.cc_min_label(g)
    np.testing.assert_array_equal(lab, ref)
    assert cc.n_components == ncomp
    np.testing.assert_array_equal(cc.reference_colors(), O.cc_reference_colors(g))
    if O.ref_available():
        np.testing.assert_array_equal(lab, O.canon_labels(O.ref_wcc(g)))


@pytest.mark.parametrize("scale,ef,seed", [(7, 8, 1), (8, 16, 2), (9, 8, 3)])
def test_ktruss(scale, ef, seed):
    g = T.rmat_graph(scale, ef, seed=seed)
    h = build(g)
    kt = H.KTruss(h)
    kt.init()
    k = kt.run()
    rk, ret = O.ktruss(g)
    assert k == rk
    np.testing.assert_array_equal(kt.edge_truss, ret)


def test_ktruss_no_triangles_and_empty():
    # a path has no triangles: max_K = 2, every edge truss 2
    s = np.arange(0, 9, dtype=np.int32)
    g = O.build_csr_undirected(10, s, s + 1)
    h = build(g)
    kt = H.KTruss(h)
    assert kt.run() == 2
    assert (kt.edge_truss == 2).all()
    e = O.Csr(np.zeros(4, np.int64), np.zeros(0, np.int32))
    assert H.KTruss(build(e)).run() == 2


def test_generators_match_host():
    import torch
    s_h, d_h = H.gen_rmat_host(12, 50000, 42, n_vertices=3000)
    s = torch.empty(50000, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    H.gen_rmat_device(12, 50000, 42, s, d, n_vertices=3000)
    np.testing.assert_array_equal(s.cpu().numpy(), s_h)
    np.testing.assert_array_equal(d.cpu().numpy(), d_h)
    csr = H.coo_to_csr_device(3000, s, d)
    h = H.hornet_from_device_csr(csr)
    ref = O.build_csr_undirected(3000, s_h, d_h)
    assert_same_graph(h, ref)


@pytest.mark.parametrize("lb,vw", [(H.HN_LB_BINARY_SEARCH, 1), (H.HN_LB_VERTEX_BASED, 1),
                                   (H.HN_LB_VERTEX_BASED, 4), (H.HN_LB_VERTEX_BASED, 32)])
def test_for_all_edges(lb, vw):
    import torch
    g = T.rmat_graph(10, 16, seed=12)
    h = build(g)
    out = torch.zeros(g.nV, dtype=torch.int32, device="cuda")
    H.for_all_edges_count(h, out, lb=lb, vw=vw)
    ref = np.bincount(g.adj, minlength=g.nV)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    # a frontier subset with repeats and isolated vertices
    rng = np.random.default_rng(5)
    verts = rng.integers(0, g.nV, 500).astype(np.int32)
    out.zero_()
    H.for_all_edges_count(h, out, vertices=torch.from_numpy(verts).cuda(), lb=lb, vw=vw)
    ref = np.zeros(g.nV, np.int64)
    for v in verts:
        np.add.at(ref, g.adj[g.off[v]:g.off[v + 1]], 1)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    deg = torch.zeros(g.nV, dtype=torch.int32, device="cuda")
    H.for_all_vertices_degree(h, deg)
    np.testing.assert_array_equal(deg.cpu().numpy(), np.diff(g.off))


def test_config_plain_small_end_to_end():
    """The CPU-runnable workload: R-MAT scale 14, ef 16, seed 1; insert 10,000
    uniform new undirected edges, delete 5,000 existing ones; BFS from 0,
    TC and CC checked against the oracle (and the reference's host BFS/WCC)."""
    g = T.rmat_graph(14, 16, seed=1)
    h = build(g)
    ins_s, ins_d = T.uniform_new_edges(g, 10000, seed=101)
    a = h.insert(H.BatchUpdate(h, ins_s, ins_d), **DEDUP_BOTH)
    g, n = O.insert(g, ins_s, ins_d, 3)
    assert a == n == 20000
    del_s, del_d = T.sample_existing_edges(g, 5000, seed=102)
    r = h.erase(H.BatchUpdate(h, del_s, del_d), removeBatchDuplicates=True)
    g, n = O.erase(g, del_s, del_d, 1)
    assert r == n == 10000
    assert_same_graph(h, g)
    bfs = H.BfsTopDown(h)
    bfs.set_parameters(0)
    np.testing.assert_array_equal(bfs.run(), O.bfs(g, 0)[0])
    assert H.TriangleCounting2(h).run() == O.tc(g)
    np.testing.assert_array_equal(H.CC(h).run(), O.cc_min_label(g)[0])
    if O.ref_available():
        np.testing.assert_array_equal(bfs.distances, O.ref_bfs(g, [0])[0])


@pytest.mark.parametrize("name", list(GRAPHS))
def test_tc_local(name):
    """Triangles containing each seed == TriangleCounting2's per-vertex
    counts (oracle) at those seeds; repeated seeds, isolated seeds, hubs."""
    g = GRAPHS[name]()
    h = build(g)
    _, pv = O.tc(g, per_vertex=True)
    deg = np.diff(g.off)
    rng = np.random.default_rng(8)
    seeds = np.concatenate([rng.integers(0, g.nV, 1000), [int(np.argmax(deg))] * 3,
                            np.nonzero(deg == 0)[0][:5]]).astype(np.int32)
    tc = H.TriangleCounting2(h)
    np.testing.assert_array_equal(tc.local(seeds), pv[seeds])
    import torch
    sd = torch.from_numpy(seeds).cuda()
    out = torch.empty(len(seeds), dtype=torch.int64, device="cuda")
    tc.local(sd, out)
    np.testing.assert_array_equal(out.cpu().numpy().astype(np.uint64), pv[seeds])
    with pytest.raises(H.HornetError):
        tc.local(np.array([g.nV], np.int32))


@pytest.mark.parametrize("knobs", [
    {"tc.warp_cap": 32, "tc.chunk": 1, "tc.warp_ctas_per_sm": 1},
    {"tc.warp_cap": 64, "tc.chunk": 256, "tc.warp_ctas_per_sm": 16},
    {"tc.narrow_min": 1024, "tc.warp_cap": 128},
    # rmat10's oriented degrees reach 44: all three listed-vertex paths
    {"tc.warp_cap": 32, "tc.mid_cap": 36, "tc.cta_table_cap": 40},
    {"tc.warp_cap": 32, "tc.mid_cap": 32, "tc.cta_table_cap": 32, "tc.narrow_min": 8},
    {"tc.warp_work": 1024, "tc.item_work": 1024, "tc.warp_cap": 64},
    {"tc.flip": 0, "tc.warp_work": 1024, "tc.item_work": 1024},
    {"tc.thread_du": 64, "tc.thread_dc": 1024},
    {"tc.thread_du": 0},
    {"tc.thread_du": 4, "tc.thread_dc": 3},
    {"tc.warp_work": 1024, "tc.item_work": 1500, "tc.mid_cap": 36, "tc.warp_cap": 32},
    {"bfs.kernel": 0, "bfs.ctas_per_sm": 1, "bfs.do_alpha": 1, "bfs.do_beta": 1},
    {"bfs.kernel": 0, "bfs.ctas_per_sm": 3, "bfs.dynamic_chunks": 1},
    {"bfs.kernel": 0, "bfs.warp_strided": 1},
    {"bfs.kernel": 0, "bfs.host_levels": 1, "bfs.warp_strided": 1},
    {"bfs.kernel": 0, "bfs.warp_strided": 1, "bfs.dynamic_chunks": 1, "bfs.ctas_per_sm": 8},
    {"bfs.kernel": 0, "bfs.ctas_per_sm": 8, "bfs.do_alpha": 1 << 20, "bfs.do_beta": 1 << 20},
    {"bfs.warp_ctas_per_sm": 1, "bfs.do_alpha": 1, "bfs.do_beta": 1},
    {"bfs.warp_ctas_per_sm": 8, "bfs.host_levels": 1},
    {"bfs.warp_ctas_per_sm": 2, "bfs.do_alpha": 1 << 20, "bfs.do_beta": 1 << 20},
])
def test_tuning_knobs_keep_results(knobs):
    """The knob extremes the autotuner can set change only the speed: TC
    totals and per-vertex counts, TD and DO BFS distances stay exact."""
    g = GRAPHS["rmat10"]()
    h = build(g)
    ref_tc, ref_pv = O.tc(g, per_vertex=True)
    srcs = [0, 5, 77]
    try:
        for k, v in knobs.items():
            H.tune_set(k, v)
        tc = H.TriangleCounting2(h)
        tc.init()
        assert tc.run(per_vertex=True) == ref_tc
        np.testing.assert_array_equal(tc.copyTCToHost(), ref_pv)
        td, _ = H.BfsTopDown(h).run_multi(srcs)
        do, _ = H.BfsTopDown(h).run_multi(srcs, direction_optimizing=True)
        for i, s in enumerate(srcs):
            np.testing.assert_array_equal(td[i], O.bfs(g, s)[0])
            np.testing.assert_array_equal(do[i], td[i])
    finally:
        H.tune_reset()


@pytest.mark.parametrize("name", ["rmat10", "er2000"])
def test_insert_count_triangles(name):
    """Triangles created by each insert == the oracle's T(after) - T(before),
    over a sequence of batches (some edges already present, some repeated
    inside a batch, triangles with 1, 2 and 3 new edges)."""
    g = GRAPHS[name]()
    h = build(g)
    rng = np.random.default_rng(12)
    for it in range(4):
        s, d = T.uniform_new_edges(g, 400, seed=100 + it)
        es, ed = g.coo()
        pick = rng.integers(0, len(es), 50)
        # a closed triangle of brand-new edges among three random vertices
        tri = rng.choice(g.nV, 3, replace=False).astype(np.int32)
        ts = np.array([tri[0], tri[1], tri[2], tri[1], tri[2], tri[0]], np.int32)
        td = np.array([tri[1], tri[2], tri[0], tri[0], tri[1], tri[2]], np.int32)
        bs = np.concatenate([s, es[pick], ts, s[:20]]).astype(np.int32)
        bd = np.concatenate([d, ed[pick], td, d[:20]]).astype(np.int32)
        before = O.tc(g)
        g, n_ref = O.insert(g, bs, bd, 3)
        n, new = h.insert_count_triangles(H.BatchUpdate(h, bs, bd))
        assert n == n_ref
        assert new == O.tc(g) - before
    assert_same_graph(h, g)


@pytest.mark.parametrize("K", [3, 4, 6])
def test_ktruss_keep_runForKDynamic(K):
    """runForKDynamic(K): the graph keeps exactly the edges whose truss
    number (oracle) is at least K; the rest leave through the erase path."""
    g = T.rmat_graph(10, 16, seed=8)
    h = build(g)
    rk, ret = O.ktruss(g)
    kt = H.KTruss(h)
    removed = kt.runForKDynamic(K)
    assert kt.getMaxK() == rk
    s, d = g.coo()
    keep = ret >= K
    assert removed == int((~keep).sum())
    hs, hd = h.getCOO(True)
    np.testing.assert_array_equal(hs, s[keep])
    np.testing.assert_array_equal(hd, d[keep])
    # the kept graph is its own K-truss: running again removes nothing
    assert kt.runForKDynamic(K) == 0
    # runForK on a fresh copy: same surviving edges, graph unchanged
    h2 = build(g)
    kt2 = H.KTruss(h2)
    off, ks, kd = kt2.runForK(K)
    np.testing.assert_array_equal(ks, s[keep])
    np.testing.assert_array_equal(kd, d[keep])
    assert off[-1] == int(keep.sum()) and h2.nE() == g.nE


@pytest.mark.parametrize("flip", [1, 0])
@pytest.mark.parametrize("name", ["rmat10", "er2000"])
def test_tc_owner_counts(name, flip):
    """Owner counts: each triangle credited once, to its lowest vertex in the
    degree orientation (oracle: |N+(u) ∩ N+(v)| summed over v in N+(u)),
    whichever endpoint of an oriented edge counts it (tc.flip)."""
    H.tune_set("tc.flip", flip)
    try:
        _check_owner_counts(name)
    finally:
        H.tune_reset()


def _check_owner_counts(name):
    g = GRAPHS[name]()
    h = build(g)
    o = O.orient_by_degree(g)
    ref = np.zeros(g.nV, np.uint64)
    for u in range(g.nV):
        nu = set(o.adj[o.off[u]:o.off[u + 1]].tolist())
        for v in nu:
            ref[u] += len(nu & set(o.adj[o.off[v]:o.off[v + 1]].tolist()))
    out = np.empty(g.nV, np.uint64)
    total = ctypes.c_uint64()
    rc = H.lib().hn_tc_owner(h.handle, out.ctypes.data_as(ctypes.c_void_p), H.HN_MEM_HOST,
                             ctypes.byref(total))
    assert rc == H.HN_OK
    np.testing.assert_array_equal(out, ref)
    assert total.value == int(ref.sum()) == O.tc(g)


def test_graph_batch_triangles_per_graph():
    import torch
    from hornet_b200.batching import GraphBatch
    graphs = [T.rmat_graph(7, 8, seed=200 + i) if i % 2 else T.er_graph(90, 6, seed=i)
              for i in range(24)]
    u, base = T.disjoint_union(graphs)
    h = build(u)
    gb = GraphBatch(h, base, [gi.nV for gi in graphs])
    pv = torch.empty(u.nV, dtype=torch.int64, device="cuda")
    tri, total = gb.triangles(pv)
    np.testing.assert_array_equal(tri.cpu().numpy(), [O.tc(gi) for gi in graphs])
    assert total == O.tc(u)


def test_bfs_multi_many_sources_host_and_device():
    """More sources than the library's 64-entry staging ring, host output
    (copies overlapped with the next BFS) and device output: every row and
    every per-source statistic equals the oracle's."""
    import torch
    g = GRAPHS["rmat12_nonpow2"]()
    h = build(g)
    rng = np.random.default_rng(17)
    srcs = rng.integers(0, g.nV, 150).astype(np.int32)
    host = torch.empty((150, g.nV), dtype=torch.int32, pin_memory=True).numpy()
    out, st = H.BfsTopDown(h).run_multi(srcs, out=host)
    dev = torch.empty((150, g.nV), dtype=torch.int32, device="cuda")
    _, st_do = H.BfsTopDown(h).run_multi(srcs, out=dev, direction_optimizing=True)
    for i, s in enumerate(srcs):
        ref, scanned = O.bfs(g, int(s))
        np.testing.assert_array_equal(out[i], ref)
        assert st[i].edges_scanned == scanned and st_do[i].edges_scanned == scanned
        assert st[i].visited == int((ref != O.INF).sum()) == st_do[i].visited
    np.testing.assert_array_equal(dev.cpu().numpy(), out)


def test_pool_grows_in_place_under_many_inserts():
    """A small graph receiving several million edges: the edge pool grows
    (mapped in place where the device supports it) several times, and the
    graph stays exactly the oracle's; weighted graphs grow their weights
    alongside."""
    g = T.er_graph(5000, 4, seed=3)
    h = build(g)
    wg_init = H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True)
    wg_init.insertEdgeData(np.arange(g.nE, dtype=np.uint32))
    hw = H.Hornet(wg_init)
    rng = np.random.default_rng(0)
    ref = g
    for it in range(3):
        bs = rng.integers(0, g.nV, 1_500_000).astype(np.int32)
        bd = rng.integers(0, g.nV, 1_500_000).astype(np.int32)
        n = h.insert(H.BatchUpdate(h, bs, bd))          # no dedup: every edge added
        ref, n_ref = O.insert(ref, bs, bd, 0)
        assert n == n_ref == len(bs)
        hw.insert(H.BatchUpdate(hw, bs, bd, np.full(len(bs), (1 << 30) + it, np.uint32)))
    assert_same_graph(h, ref)
    s, d, w = hw.getCOOWeighted()
    np.testing.assert_array_equal(d, ref.coo()[1])
    # weights of the original edges survive the moves; inserted ones carry
    # their batch's weight
    np.testing.assert_array_equal(np.sort(w[w < (1 << 30)]), np.arange(g.nE, dtype=np.uint32))
    assert set(np.unique(w[w >= (1 << 30)]).tolist()) == {1 << 30, (1 << 30) + 1, (1 << 30) + 2}


def test_validate_certifies_results_and_catches_errors():
    """validate() (device certificates; the reference's are stubs returning
    true) accepts the computed BFS, CC, TC and k-truss results and rejects
    results with one error planted on the host."""
    g = GRAPHS["rmat10"]()
    h = build(g)
    bfs = H.BfsTopDown(h)
    bfs.set_parameters(3)
    dist = bfs.run()
    assert bfs.validate()
    reached = np.nonzero((dist != O.INF) & (dist > 1))[0]
    wrong = dist.copy()
    wrong[reached[0]] += 1                       # a vertex one level too far
    bfs.distances = wrong
    assert not bfs.validate()
    wrong = dist.copy()
    wrong[reached[1]] = O.INF                    # a reached vertex dropped
    bfs.distances = wrong
    assert not bfs.validate()
    cc = H.CC(h)
    lab = cc.run()
    assert cc.validate()
    comps = np.unique(lab)
    if len(comps) >= 2:
        merged = lab.copy()
        merged[merged == comps[1]] = comps[0]    # two components under one label
        cc.labels = merged
        assert not cc.validate()
    tc = H.TriangleCounting2(h)
    tc.run()
    assert tc.validate()
    tc._total += 1
    assert not tc.validate()
    kt = H.KTruss(build(T.rmat_graph(8, 16, seed=2)))
    kt.run()
    assert kt.validate()
    et = kt.edge_truss.copy()
    top = np.nonzero(et == kt.max_k)[0]
    kt.edge_truss = et.copy()
    kt.edge_truss[top[0]] = 2                    # one direction of an edge changed
    assert not kt.validate()


def test_device_graph_save_and_reload(tmp_path):
    """A device graph saved after updates (hn_graph_write_bin, the
    reference's GraphStd .bin format) reloads into an identical graph
    (hn_graph_read_bin), and the file is byte-identical to the host writer's
    output for the exported CSR (pinned to the reference's example/G.bin by
    the CPU format tests)."""
    g = T.rmat_graph(10, 8, seed=21)
    h = build(g)
    rng = np.random.default_rng(2)
    bs = rng.integers(0, g.nV, 3000).astype(np.int32)
    bd = rng.integers(0, g.nV, 3000).astype(np.int32)
    h.insert(H.BatchUpdate(h, bs, bd), True, True)
    p = str(tmp_path / "g.bin")
    h.save_bin(p)
    h2 = H.Hornet.load_bin(p)
    assert h2.nV() == h.nV() and h2.nE() == h.nE()
    s1, d1 = h.getCOO(True)
    s2, d2 = h2.getCOO(True)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(d1, d2)
    assert h2.adjacency_hash() == h.adjacency_hash()
    off, adj = h.getCSR()
    q = str(tmp_path / "host.bin")
    H.write_bin(q, off.astype(np.int32), adj)
    assert open(p, "rb").read() == open(q, "rb").read()
    # the reloaded graph is a full dynamic graph: it takes further updates
    assert h2.erase(H.BatchUpdate(h2, bs, bd), True) == h.erase(H.BatchUpdate(h, bs, bd), True)
    assert h2.adjacency_hash() == h.adjacency_hash()


@pytest.mark.parametrize("device_rounds", [1, 0])
def test_ktruss_round_drivers(device_rounds):
    """The peel rounds driven on the device (a CUDA graph's WHILE node) and
    from the host give the oracle's truss numbers."""
    g = T.rmat_graph(9, 8, seed=3)
    h = build(g)
    kmax, et = O.ktruss(g)
    try:
        H.tune_set("ktruss.device_rounds", device_rounds)
        kt = H.KTruss(h)
        assert kt.run() == kmax
        np.testing.assert_array_equal(kt.edge_truss, et)
    finally:
        H.tune_reset()


@pytest.mark.parametrize("in_place", [1, 0])
def test_in_place_updates_on_long_suffixes(in_place):
    """Updates of vertices whose block class does not change rewrite their
    list inside the block from the first entry that moves (update.in_place
    1), or move it to a new block (0); both equal the oracle's multiset
    model.  64 lists of 1,500 entries (block class 2048) beside an R-MAT
    graph get batch entries below most of their values, so the moved parts
    (up to ~1,500 entries) span scatter tiles and take the whole-vertex
    path; a multigraph stage and an erase with batch duplicates exercise
    the rank rule for equal entries in place; a last insert pushes some of
    the lists past 2,048 entries (a class change, a new block)."""
    rng = np.random.default_rng(21)
    g = T.rmat_graph(14, 8, seed=3)
    heads = np.arange(8000, 8064, dtype=np.int32)
    hs = np.repeat(heads, 1500)
    hd = np.concatenate([rng.choice(np.arange(1000, g.nV), 1500, replace=False)
                         for _ in heads]).astype(np.int32)
    g, _ = O.insert(g, hs, hd, 3)
    try:
        H.tune_set("update.in_place", in_place)
        h = build(g)
        # 1: small ids into the long lists (moved parts ~1,500) + random edges
        s = np.concatenate([np.repeat(heads, 3), rng.integers(0, g.nV, 3000).astype(np.int32)])
        d = np.concatenate([rng.integers(0, 500, 3 * len(heads)).astype(np.int32),
                            rng.integers(0, g.nV, 3000).astype(np.int32)])
        assert h.insert(H.BatchUpdate(h, s, d), True, True) == O.insert(g, s, d, 3)[1]
        g, _ = O.insert(g, s, d, 3)
        assert_same_graph(h, g)
        # 2: a multigraph: existing entries of the long lists inserted again
        es, ed = g.coo()
        mine = np.nonzero((es >= 8000) & (es < 8064))[0]
        pick = rng.choice(mine, 2000, replace=False)
        h.insert(H.BatchUpdate(h, es[pick], ed[pick]), False, False)
        g, _ = O.insert(g, es[pick], ed[pick], 0)
        assert_same_graph(h, g)
        # 3: erase with batch duplicates: some of the doubled entries lose one
        # copy, some both
        s = np.concatenate([es[pick[:800]], es[pick[:300]], es[rng.choice(mine, 500)]])
        d = np.concatenate([ed[pick[:800]], ed[pick[:300]], ed[rng.choice(mine, 500)]])
        assert h.erase(H.BatchUpdate(h, s, d), False) == O.erase(g, s, d, 0)[1]
        g, _ = O.erase(g, s, d, 0)
        assert_same_graph(h, g)
        # 4: erase low entries (moved parts start near the front) with dedup
        es, ed = g.coo()
        low = np.nonzero((es >= 8000) & (es < 8064) & (ed < 3000))[0]
        s, d = es[low], ed[low]
        h.erase(H.BatchUpdate(h, s, d), True)
        g, _ = O.erase(g, s, d, 1)
        assert_same_graph(h, g)
        # 5: some lists past 2,048 entries (class change) beside in-place ones
        s = np.repeat(heads[:8], 1000)
        d = rng.integers(0, g.nV, len(s)).astype(np.int32)
        h.insert(H.BatchUpdate(h, s, d), True, True)
        g, _ = O.insert(g, s, d, 3)
        assert_same_graph(h, g)
    finally:
        H.tune_reset()


@pytest.mark.parametrize("in_place", [1, 0])
def test_in_place_hub_updates(in_place):
    """A hub (20,000 leaves, then a run of 5,000 copies of one neighbour that
    spans chunk boundaries) updated with at most 256 batch entries at a
    time keeps its block and is rewritten chunk by chunk in place (the slots
    a neighbouring chunk may overwrite first come from the boundary
    snapshot), or moved to a new block (update.in_place 0); both equal the
    oracle's multiset model.  Batches: entries spread over every chunk,
    entries only at the front (the later chunks move as blocks), erasing
    three copies of the long run (the first-copy rule across chunks), and
    random erases."""
    rng = np.random.default_rng(33)
    n_star = 20001
    star = O.build_csr_undirected(n_star, np.zeros(n_star - 1, np.int32),
                                  np.arange(1, n_star, dtype=np.int32))
    g, _ = T.disjoint_union([star, T.rmat_graph(11, 8, seed=2)])
    g, _ = O.insert(g, np.zeros(5000, np.int32), np.full(5000, 12345, np.int32), 0)
    try:
        H.tune_set("update.in_place", in_place)
        h = build(g)
        assert_same_graph(h, g)
        holes = rng.choice(np.arange(1, n_star, dtype=np.int32), 150, replace=False)
        steps = [
            ("erase", holes, True),                                    # spread over the chunks
            ("insert", np.concatenate([holes, rng.integers(n_star, g.nV, 50).astype(np.int32)]),
             (True, True)),                                            # spread again
            ("insert", rng.integers(1, 40, 10).astype(np.int32), (False, False)),   # front only
            ("erase", np.full(3, 12345, np.int32), False),             # the long run
            ("insert", np.full(7, 12345, np.int32), (False, False)),
            ("erase", np.array([12345] * 5 + [3, 3], np.int32), False),
        ]
        for kind, d, flags in steps:
            src = np.zeros(len(d), np.int32)
            if kind == "insert":
                h.insert(H.BatchUpdate(h, src, d), *flags)
                g, _ = O.insert(g, src, d, (1 if flags[0] else 0) | (2 if flags[1] else 0))
            else:
                h.erase(H.BatchUpdate(h, src, d), flags)
                g, _ = O.erase(g, src, d, 1 if flags else 0)
            assert_same_graph(h, g)
    finally:
        H.tune_reset()


@pytest.mark.parametrize("big_min", [2048, 4, 1 << 30])
def test_updates_on_long_lists(big_min):
    """Insert and erase batches that reach long adjacency lists (a star with
    20,000 leaves beside an R-MAT graph) equal the oracle's multiset model,
    with the long lists moved by the chunked hub scatter (update.big_min:
    the default 2048, 4 = nearly every list) or by the tiles alone (2^30).
    Batches hit chunks with and without batch entries inside, and a
    multigraph stage makes the erase rank rule apply inside hub chunks."""
    n_star = 20001
    star = O.build_csr_undirected(n_star, np.zeros(n_star - 1, np.int32),
                                  np.arange(1, n_star, dtype=np.int32))
    g, base = T.disjoint_union([star, T.rmat_graph(12, 16, seed=7)])
    rng = np.random.default_rng(11)
    try:
        H.tune_set("update.big_min", big_min)
        h = build(g)
        for step in range(8):
            if step % 2 == 0:
                # edges from the hub (or, every other time, from the first
                # R-MAT vertex) to leaves in one id range, so most chunks of
                # the hub's list see no batch entry, plus random edges
                hub = 0 if step % 4 == 0 else n_star
                lo = int(rng.integers(1, n_star - 600))
                leaves = rng.integers(lo, lo + 500, 300).astype(np.int32)
                s = np.concatenate([np.full(300, hub, np.int32),
                                    rng.integers(0, g.nV, 2000).astype(np.int32)])
                d = np.concatenate([leaves, rng.integers(0, g.nV, 2000).astype(np.int32)])
                flags = (True, True) if step != 4 else (False, False)   # step 4: multigraph
                h.insert(H.BatchUpdate(h, s, d), *flags)
                g, _ = O.insert(g, s, d, 3 if flags[0] else 0)
            else:
                es, ed = g.coo()
                hub_edges = np.nonzero(es == 0)[0]
                pick = np.concatenate([rng.choice(hub_edges, 400, replace=False),
                                       rng.integers(0, len(es), 1500)])
                s, d = es[pick], ed[pick]
                if step == 5:   # duplicates in the batch: several copies of an edge go
                    s = np.concatenate([s, s[:50]])
                    d = np.concatenate([d, d[:50]])
                dedup = step != 5
                h.erase(H.BatchUpdate(h, s, d), dedup)
                g, _ = O.erase(g, s, d, 1 if dedup else 0)
            assert_same_graph(h, g)
    finally:
        H.tune_reset()
