"""GPU: the benchmark's full-size graph (R-MAT scale 22, ef 16, generated on
the device: 4,194,304 vertices, 128,302,074 directed edges).

Pinned to the reference (tests/golden/fullsize.json, made on the CPU by
tests/golden/make_fullsize.py): the graph's edge count and adjacency
checksum; BFS distances from 8 of the benchmark's sources equal the
reference's graph::BFS (xlib/src/Graph/BFS.cpp) byte for byte; CC labels
equal graph::WCC (xlib/src/Graph/WCC.cpp) relabelled to minimum ids; the
triangle total equals the restated hostCountTriangles
(hornetsnest/test/TriangleTest2.cu:22-69); k-truss edge truss numbers equal
the CPU truss decomposition (scale 18 and, when pinned, scale 22).

Also checked through size-independent properties:

* BFS: a BFS certificate on every source (source at 0; along every edge
  distances differ by at most one; every reached vertex other than the
  source has a neighbour one level closer), and direction-optimising BFS
  and every slot of a batched BFS equal top-down BFS exactly;
* CC: labels constant along edges, at most the vertex id, fixed points, and
  the component of a BFS source labelled with its minimum vertex id;
* TC: independent kernels agree — the warp/CTA counting split at two bin
  thresholds, per-vertex counts summing to three times the total, and the
  local-count kernel on a half-million-vertex sample;
* updates: a 1M-edge insert then the erase of the same batch restores the
  exported CSR exactly, and after the insert every list is strictly sorted.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import hornet_b200 as H

pytestmark = pytest.mark.gpu

SCALE = 22
GOLD_PATH = os.path.join(os.path.dirname(__file__), "golden", "fullsize.json")
GOLD = json.load(open(GOLD_PATH)) if os.path.exists(GOLD_PATH) else {}


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, "<i4").tobytes()).hexdigest()


def _device_rmat(scale, ef=16, seed=1):
    import torch
    n = 1 << scale
    src = torch.empty(ef * n, dtype=torch.int32, device="cuda")
    dst = torch.empty_like(src)
    H.gen_rmat_device(scale, ef * n, seed, src, dst)
    csr = H.coo_to_csr_device(n, src, dst)
    del src, dst
    return H.hornet_from_device_csr(csr), csr


@pytest.fixture(scope="module")
def big():
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
    deg = off[1:] - off[:-1]
    srcv = torch.repeat_interleave(torch.arange(nV, device="cuda", dtype=torch.int32), deg)
    yield h, off, adj, srcv
    H.tune_reset()


def test_c2_pinned_to_reference(big):
    """Graph, BFS (top-down and direction-optimising), CC and TC at scale 22
    equal the reference's host code / the restated TC on the same graph."""
    g = GOLD["rmat22"]
    h, off, adj, srcv = big
    assert (h.nV(), h.nE()) == (g["nV"], g["nE"])
    assert h.adjacency_hash() == int(g["adjacency_hash"])
    srcs = np.array(g["bfs"]["sources"], np.int32)
    bfs = H.BfsTopDown(h)
    for do in (False, True):
        dist, st = bfs.run_multi(srcs, direction_optimizing=do)
        for j in range(len(srcs)):
            assert _sha(dist[j]) == g["bfs"]["sha256"][j], (do, j)
            assert st[j].visited == g["bfs"]["reached"][j]
            assert st[j].levels == g["bfs"]["levels"][j]
    cc = H.CC(h)
    lab = cc.run()
    assert cc.n_components == g["cc"]["components"]
    assert _sha(lab) == g["cc"]["sha256_min_id"]
    assert H.TriangleCounting2(h).run() == g["tc"]["triangles"]


def _check_ktruss(h, entry):
    kt = H.KTruss(h)
    kmax = kt.run()
    et = kt.edge_truss
    assert kmax == entry["max_k"]
    ks, cnt = np.unique(et, return_counts=True)
    assert {str(int(k)): int(c) for k, c in zip(ks, cnt)} == entry["edges_per_truss"]
    assert _sha(et) == entry["edge_truss_sha256"]


@pytest.mark.skipif("ktruss" not in GOLD.get("rmat22", {}), reason="scale-22 truss not pinned")
def test_ktruss_scale22_pinned(big):
    h, off, adj, srcv = big
    _check_ktruss(h, GOLD["rmat22"]["ktruss"])


def test_ktruss_scale18_pinned():
    h, csr = _device_rmat(18)
    assert h.nE() == GOLD["ktruss18"]["nE"]
    _check_ktruss(h, GOLD["ktruss18"])


def _bfs_certificate(dist, srcv, adj, s):
    import torch
    INF = 2147483647
    assert int(dist[s]) == 0
    du, dv = dist[srcv].long(), dist[adj].long()
    reached_u = du != INF
    # along every edge from a reached vertex: neighbour reached, |du - dv| <= 1
    assert bool((dv[reached_u] != INF).all())
    assert int((du[reached_u] - dv[reached_u]).abs().max()) <= 1
    # every reached vertex but the source has a neighbour one level closer
    best = torch.full_like(dist, INF, dtype=torch.int64)
    best.scatter_reduce_(0, adj.long(), du, reduce="amin")
    reached = (dist != INF)
    reached[s] = False
    assert bool((best[reached] == dist[reached].long() - 1).all())


def test_bfs_certificate_do_and_batch_equal(big):
    import torch
    h, off, adj, srcv = big
    nV = h.nV()
    deg = (off[1:] - off[:-1]).cpu().numpy()
    rng = np.random.default_rng(99)
    srcs = rng.choice(np.nonzero(deg > 0)[0], 8, replace=False).astype(np.int32)
    bfs = H.BfsTopDown(h)
    td = torch.empty((8, nV), dtype=torch.int32, device="cuda")
    for j, s in enumerate(srcs):
        bfs.set_parameters(int(s))
        bfs.run(out=td[j])
        _bfs_certificate(td[j], srcv, adj, int(s))
    do = torch.empty_like(td)
    bfs.run_multi(srcs, out=do, direction_optimizing=True)
    assert torch.equal(do, td)
    ms = torch.empty_like(td)
    bfs.run_batch(srcs, out=ms)
    assert torch.equal(ms, td)


def test_cc_properties(big):
    import torch
    h, off, adj, srcv = big
    nV = h.nV()
    lab = torch.empty(nV, dtype=torch.int32, device="cuda")
    H.CC(h).run(out=lab)
    ids = torch.arange(nV, device="cuda", dtype=torch.int32)
    assert torch.equal(lab[srcv], lab[adj])
    assert bool((lab <= ids).all())
    assert torch.equal(lab[lab.long()], lab)
    # the component of a BFS source: all reached, labelled with their min id
    s = int(torch.argmax((off[1:] - off[:-1])).item())
    dist = torch.empty(nV, dtype=torch.int32, device="cuda")
    bfs = H.BfsTopDown(h)
    bfs.set_parameters(s)
    bfs.run(out=dist)
    reached = dist != 2147483647
    mn = int(ids[reached].min())
    assert bool((lab[reached] == mn).all())
    assert bool((lab[~reached] != mn).all())


def test_tc_three_ways(big):
    import torch
    h, off, adj, srcv = big
    nV = h.nV()
    tc = H.TriangleCounting2(h)
    totals = []
    for cap in (512, 64):
        H.tune_set("tc.warp_cap", cap)
        totals.append(tc.run())
    H.tune_reset()
    assert totals[0] == totals[1]
    pv_total = tc.run(per_vertex=True)
    assert pv_total == totals[0]
    pv = tc.copyTCToHost()
    assert int(pv.sum()) == 3 * totals[0]
    # local counts (a separate kernel) on a seeded half-million-vertex sample
    seeds_h = np.random.default_rng(4).choice(nV, 500_000, replace=False).astype(np.int32)
    seeds = torch.from_numpy(seeds_h).cuda()
    loc = torch.empty(len(seeds_h), dtype=torch.int64, device="cuda")
    tc.local(seeds, loc)
    np.testing.assert_array_equal(loc.cpu().numpy().astype(np.uint64), pv[seeds_h])


def test_update_round_trip(big):
    import torch
    h, off, adj, srcv = big
    nV = h.nV()
    rng = np.random.default_rng(5)
    b = 1_000_000
    bs = torch.from_numpy(rng.integers(0, nV, b).astype(np.int32)).cuda()
    bd = torch.from_numpy(rng.integers(0, nV, b).astype(np.int32)).cuda()
    # keep the pairs absent from the graph, once each: then insert + erase
    # of the batch is an exact round trip
    gkeys = (srcv.long() << 32) | adj.long()
    bkeys = torch.unique((bs.long() << 32) | bd.long())
    pos = torch.searchsorted(gkeys, bkeys).clamp(max=gkeys.numel() - 1)
    bkeys = bkeys[gkeys[pos] != bkeys]
    bs, bd = (bkeys >> 32).int(), (bkeys & 0xFFFFFFFF).int()
    batch = H.BatchUpdate(h, bs, bd)
    added = h.insert(batch, True, True)
    assert added == bkeys.numel()
    assert h.nE() == adj.numel() + added
    off2 = torch.empty(nV + 1, dtype=torch.int32, device="cuda")
    adj2 = torch.empty(h.nE(), dtype=torch.int32, device="cuda")
    H._check(H.lib().hn_graph_export_csr(h.handle, ctypes.c_void_p(off2.data_ptr()),
                                         ctypes.c_void_p(adj2.data_ptr()), H.HN_MEM_DEVICE))
    deg2 = off2[1:] - off2[:-1]
    src2 = torch.repeat_interleave(torch.arange(nV, device="cuda", dtype=torch.int32), deg2)
    same_seg = src2[1:] == src2[:-1]
    assert bool((adj2[1:][same_seg] > adj2[:-1][same_seg]).all())
    removed = h.erase(batch, True)
    assert removed == added
    off3 = torch.empty_like(off)
    adj3 = torch.empty_like(adj)
    H._check(H.lib().hn_graph_export_csr(h.handle, ctypes.c_void_p(off3.data_ptr()),
                                         ctypes.c_void_p(adj3.data_ptr()), H.HN_MEM_DEVICE))
    assert torch.equal(off3, off)
    assert torch.equal(adj3, adj)
