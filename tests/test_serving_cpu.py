"""CPU: the serving loop's host logic — grouping keeps arrival-order
semantics (no group crosses an update/query boundary, BFS groups hold at
most max_slots sources), request streams are deterministic, and result
comparison."""
from collections import deque

import numpy as np

from hornet_b200 import serving as S


def _stream(kinds):
    return [S.Request(i, k, 0.0) for i, k in enumerate(kinds)]


def _groups(kinds, batched, max_slots=64):
    pend = deque(_stream(kinds))
    out = []
    while pend:
        out.append([r.kind for r in S.take_group(pend, batched, max_slots)])
    return out


def test_groups_respect_update_query_boundaries():
    kinds = ["insert", "erase", "insert", "bfs", "tc_local", "bfs", "erase", "bfs"]
    assert _groups(kinds, True) == [["insert", "erase", "insert"], ["bfs", "tc_local", "bfs"],
                                    ["erase"], ["bfs"]]
    assert _groups(kinds, False) == [[k] for k in kinds]


def test_bfs_groups_capped_at_slots():
    kinds = ["bfs"] * 5 + ["tc_local"] + ["bfs"] * 2
    g = _groups(kinds, True, max_slots=3)
    assert g == [["bfs"] * 3, ["bfs", "bfs", "tc_local", "bfs"], ["bfs"]]
    for grp in g:
        assert sum(k == "bfs" for k in grp) <= 3


def test_requests_deterministic_and_mixed():
    deg = np.ones(1000, np.int32)

    def erase_pool(rng, k):
        return rng.integers(0, 1000, k).astype(np.int32), rng.integers(0, 1000, k).astype(np.int32)

    a = S.make_requests(400, 1000.0, 1000, deg, erase_pool, seed=3)
    b = S.make_requests(400, 1000.0, 1000, deg, erase_pool, seed=3)
    assert [(r.kind, r.arrival, r.n_edges) for r in a] == [(r.kind, r.arrival, r.n_edges) for r in b]
    kinds = [r.kind for r in a]
    frac_upd = sum(k in S.UPDATE_KINDS for k in kinds) / len(kinds)
    assert 0.5 < frac_upd < 0.7
    assert all(np.all(np.diff([r.arrival for r in a]) >= 0) for _ in [0])
    for r in a:
        if r.kind in S.UPDATE_KINDS:
            assert 100 <= r.n_edges // 2 <= 2_000_000 or r.kind == "insert"
            # both directions of every pair
            h = len(r.src) // 2
            np.testing.assert_array_equal(r.src[:h], r.dst[h:])


def test_same_results():
    a = {0: None, 1: (np.array([1, 2], np.int32), 5), 2: np.array([3], np.uint64)}
    b = {0: None, 1: (np.array([1, 2], np.int32), 5), 2: np.array([3], np.uint64)}
    assert S.same_results(a, b)
    b[1] = (np.array([1, 3], np.int32), 5)
    assert not S.same_results(a, b)


def test_query_units_stop_at_updates_and_return_the_rest():
    kinds = ["bfs", "tc_local", "bfs", "bfs", "tc_local", "insert", "bfs"]
    pend = deque(_stream(kinds))
    units = S.query_units(pend, 2, msbfs_min=4, max_slots=16)
    # two free views: the TC unit (both TC queries) and the first lone BFS
    assert [(k, [r.rid for r in g]) for k, g in units] == [("tc_local", [1, 4]), ("bfs", [0])]
    # the other BFS queries wait at the front, in arrival order, before the update
    assert [r.rid for r in pend] == [2, 3, 5, 6]
    # enough BFS queries share one batched unit, capped at max_slots
    pend = deque(_stream(["bfs"] * 7 + ["erase"]))
    units = S.query_units(pend, 4, msbfs_min=3, max_slots=5)
    assert [len(g) for _, g in units] == [5, 1, 1]
    assert [r.kind for r in pend] == ["erase"]
