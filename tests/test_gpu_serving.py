"""GPU: coalesced update batches and the serving loop against the oracle.

* hn_update_coalesced on a mixed run of insert/erase batches equals the
  oracle applying the batches one by one (insert with both dedup flags,
  erase with batch dedup), including edges inserted and erased several
  times inside the run.
* The batched serving loop and the plain per-request loop give identical
  per-request results, and both equal the oracle replaying the stream in
  arrival order (BFS distances at the targets and vertices reached; local
  triangle counts from TriangleCounting2's per-vertex counts)."""
import numpy as np
import pytest

import hornet_b200 as H
from hornet_b200 import serving as S
from oracle import oracle as O
from tests import helpers as T

pytestmark = pytest.mark.gpu


def build(g):
    return H.Hornet(H.HornetInit(g.nV, g.nE, g.off32(), g.adj, sorted_adjacency=True))


def assert_same_graph(h, g):
    assert h.nE() == g.nE
    s, d = h.getCOO(True)
    gs, gd = g.coo()
    np.testing.assert_array_equal(s, gs)
    np.testing.assert_array_equal(d, gd)


def sym(s, d):
    return np.concatenate([s, d]).astype(np.int32), np.concatenate([d, s]).astype(np.int32)


def test_update_coalesced_equals_sequential():
    g = T.rmat_graph(10, 8, seed=31)
    h = build(g)
    rng = np.random.default_rng(1)
    es, ed = g.coo()
    batches = []
    hot_s = rng.integers(0, g.nV, 50).astype(np.int32)
    hot_d = rng.integers(0, g.nV, 50).astype(np.int32)
    for b in range(12):
        if b % 2 == 0:
            s = np.concatenate([rng.integers(0, g.nV, 300), hot_s]).astype(np.int32)
            d = np.concatenate([rng.integers(0, g.nV, 300), hot_d]).astype(np.int32)
            keep = s != d
            batches.append(("insert",) + sym(s[keep], d[keep]))
        else:
            pick = rng.integers(0, len(es), 200)
            s = np.concatenate([es[pick], hot_s]).astype(np.int32)
            d = np.concatenate([ed[pick], hot_d]).astype(np.int32)
            batches.append(("erase",) + sym(s, d))
    ref = g
    for kind, s, d in batches:
        ref, _ = O.insert(ref, s, d, 3) if kind == "insert" else O.erase(ref, s, d, 1)
    src = np.concatenate([s for _, s, _ in batches])
    dst = np.concatenate([d for _, _, d in batches])
    ops = np.concatenate([np.full(len(s), k == "insert", np.uint8) for k, s, _ in batches])
    ins, era = h.update_coalesced(src, dst, ops)
    assert_same_graph(h, ref)
    assert g.nE + ins - era == ref.nE
    # device arrays, and an out-of-range id is rejected with the graph unchanged
    import torch
    before = h.getCOO(True)
    bad = torch.tensor([0, g.nV], dtype=torch.int32, device="cuda")
    with pytest.raises(H.HornetError):
        h.update_coalesced(bad, bad, torch.ones(2, dtype=torch.uint8, device="cuda"))
    after = h.getCOO(True)
    np.testing.assert_array_equal(before[1], after[1])


def oracle_replay(g, reqs):
    out = {}
    for r in sorted(reqs, key=lambda r: (r.arrival, r.rid)):
        if r.kind == "insert":
            g, _ = O.insert(g, r.src, r.dst, 3)
            out[r.rid] = None
        elif r.kind == "erase":
            g, _ = O.erase(g, r.src, r.dst, 1)
            out[r.rid] = None
        elif r.kind == "bfs":
            d, _ = O.bfs(g, r.source)
            out[r.rid] = (d[r.targets].astype(np.int32), int((d != O.INF).sum()))
        else:
            _, pv = O.tc(g, per_vertex=True)
            out[r.rid] = pv[r.seeds].astype(np.uint64)
    return out, g


@pytest.mark.parametrize("rate", [0.0, 2000.0])
def test_serving_batched_equals_plain_equals_oracle(rate):
    g = T.rmat_graph(11, 8, seed=17)
    es, ed = g.coo()

    def erase_pool(rng, k):
        pick = rng.integers(0, len(es), k)
        return es[pick].astype(np.int32), ed[pick].astype(np.int32)

    reqs = S.make_requests(160, rate, g.nV, np.diff(g.off), erase_pool, seed=5,
                           median_edges=300, sigma=1.0, clip=(20, 3000), n_seeds=64)
    ref, g_end = oracle_replay(g, reqs)
    reports = {}
    for batched, single, msmin in ((False, "td", 4), (False, "do", 4), (True, "do", 2)):
        h = build(g)
        srv = S.Server(h, batched=batched, max_slots=16, reserve_bytes=0, single_bfs=single,
                       msbfs_min=msmin)
        rep = srv.run(reqs)
        assert S.same_results(rep.results, ref), f"batched={batched} single={single}"
        assert_same_graph(h, g_end)
        reports[batched] = rep
    assert reports[True].calls < reports[False].calls
    assert reports[True].latency_ms["all"]["n"] == len(reqs)


def test_serving_splits_updates_to_fit_memory():
    g = T.er_graph(3000, 6, seed=2)
    es, ed = g.coo()

    def erase_pool(rng, k):
        pick = rng.integers(0, len(es), k)
        return es[pick].astype(np.int32), ed[pick].astype(np.int32)

    reqs = S.make_requests(80, 0.0, g.nV, np.diff(g.off), erase_pool, seed=9,
                           mix=(0.9, 0.05, 0.05), median_edges=200, sigma=0.5,
                           clip=(50, 1000), n_seeds=32)
    ref, g_end = oracle_replay(g, reqs)
    h = build(g)
    # pretend only ~1000 update entries fit at a time
    srv = S.Server(h, batched=True, reserve_bytes=0,
                   free_bytes_fn=lambda: 1000 * S.Server.UPDATE_BYTES_PER_EDGE)
    rep = srv.run(reqs)
    assert rep.split_for_memory > 0
    assert S.same_results(rep.results, ref)
    assert_same_graph(h, g_end)


def test_query_views_run_concurrently_and_reject_updates():
    """Query views of one resident graph answer BFS and local-TC calls from
    several host threads at once with the graph's own results, reject
    updates (HN_ERR_STATE), and see an update of the graph after
    refresh_view()."""
    from concurrent.futures import ThreadPoolExecutor
    g = T.rmat_graph(12, 8, seed=3)
    h = build(g)
    views = [h.view() for _ in range(3)]
    srcs = [0, 5, 17, 99, 1234, 777, 2048, 4000]

    def one(i):
        v = views[i % 3]
        d = H.BfsTopDown(v).run_multi([srcs[i]], direction_optimizing=bool(i & 1))[0][0]
        return d, H.TriangleCounting2(v).local(np.array([srcs[i]], np.int32))

    def per_view(j):
        # a handle serves one host thread at a time: thread j owns view j
        return {i: one(i) for i in range(j, len(srcs), 3)}

    with ThreadPoolExecutor(3) as ex:
        done = {}
        for part in ex.map(per_view, range(3)):
            done.update(part)
    outs = [done[i] for i in range(len(srcs))]
    _, pv = O.tc(g, per_vertex=True)
    for s, (d, t) in zip(srcs, outs):
        np.testing.assert_array_equal(d, O.bfs(g, s)[0])
        assert int(t[0]) == int(pv[s])
    bs = np.array([1, 2], np.int32)
    bd = np.array([2, 1], np.int32)
    with pytest.raises(H.HornetError) as e:
        views[0].insert(H.BatchUpdate(views[0], bs, bd), True, True)
    assert e.value.code == H.HN_ERR_STATE
    s2, d2 = T.uniform_new_edges(g, 500, seed=8)
    h.insert(H.BatchUpdate(h, s2, d2), True, True)
    g2, _ = O.insert(g, s2, d2, 3)
    for v in views:
        v.refresh_view()
        assert v.nE() == g2.nE
    d, _ = H.BfsTopDown(views[1]).run_multi([5])
    np.testing.assert_array_equal(d[0], O.bfs(g2, 5)[0])
