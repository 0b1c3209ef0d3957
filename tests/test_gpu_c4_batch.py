"""GPU: the many-small-graphs configuration at its own size, every graph
checked against the oracle.

4,096 graphs (vertex counts log-uniform in [1024, 65536]; half Erdos-Renyi
with mean degree 8, half R-MAT with edge factor 16) generated on the device
into one disjoint union; 8 seeded sources per graph traversed by one batched
BFS, and per-graph triangles from the owner counts (GraphBatch).  On the CPU,
a pool of spawned worker processes regenerates each graph from its seed
(the oracle's restated generator), builds its CSR (GraphStd's COOtoCSR,
restated) and computes its 8 BFS (BFS.cpp:54-76) and its triangle count
(TriangleTest2.cu:22-69).  Every graph's CSR, every (graph, source)
distance array and every triangle count must match; arrays are compared by
SHA-256.
"""
import ctypes
import hashlib
import multiprocessing as mp
import os

import numpy as np
import pytest

import hornet_b200 as H
from hornet_b200.batching import GraphBatch, synthetic_specs, synthetic_union

pytestmark = pytest.mark.gpu

N_GRAPHS = 4096
SLOTS = 8


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, "<i4").tobytes()).hexdigest()


def _oracle_graph(job):
    """(spec, local sources) -> SHA-256 of the CSR and of each BFS, and the
    triangle count of one graph (runs in a worker process)."""
    from oracle import oracle as O
    (sc, npairs, pseed, n, a, b, c), srcs = job
    s, d = O.gen_rmat(sc, npairs, pseed, n_vertices=n, a=a, b=b, c=c, threads=1)
    g = O.build_csr_undirected(n, s, d)
    csr = hashlib.sha256(g.off.astype("<i4").tobytes() + g.adj.astype("<i4").tobytes()).hexdigest()
    bfs = [_sha(O.bfs(g, int(x))[0]) for x in srcs]
    return csr, bfs, O.tc(g)


def test_c4_every_graph_matches_oracle():
    import torch
    sizes0, bases0, kinds0, specs = synthetic_specs(N_GRAPHS, seed=4096)
    h, csr, sizes, bases, kinds = synthetic_union(N_GRAPHS, seed=4096)
    assert (sizes == sizes0).all() and (bases == bases0).all()
    nV, nE = h.nV(), h.nE()
    deg = h.degrees()
    rng = np.random.default_rng(77)
    local = np.zeros((N_GRAPHS, SLOTS), np.int64)
    for i in range(N_GRAPHS):
        cand = np.nonzero(deg[bases[i]:bases[i] + sizes[i]] > 0)[0]
        local[i] = rng.choice(cand, size=SLOTS, replace=len(cand) < SLOTS)
    # CPU side first, in spawned workers (no fork after CUDA is in use)
    ctx = mp.get_context("spawn")
    procs = max(1, min(32, os.cpu_count() or 1))
    with ctx.Pool(procs) as pool:
        pending = pool.map_async(_oracle_graph, list(zip(specs, local.tolist())), chunksize=16)
        gb = GraphBatch(h, bases, sizes)
        out = torch.empty((SLOTS, nV), dtype=torch.int32, device="cuda")
        gb.bfs(local, out)
        pv = torch.empty(nV, dtype=torch.int64, device="cuda")
        tri, _ = gb.triangles(pv)
        tri = tri.cpu().numpy()
        dist = out.cpu().numpy()
        off = torch.empty(nV + 1, dtype=torch.int32, device="cuda")
        adj = torch.empty(nE, dtype=torch.int32, device="cuda")
        H._check(H.lib().hn_graph_export_csr(h.handle, ctypes.c_void_p(off.data_ptr()),
                                             ctypes.c_void_p(adj.data_ptr()), H.HN_MEM_DEVICE))
        off, adj = off.cpu().numpy(), adj.cpu().numpy()
        ref = pending.get(timeout=1800)
    bad = []
    for i, (csr_sha, bfs_sha, t) in enumerate(ref):
        b, n = int(bases[i]), int(sizes[i])
        o = off[b:b + n + 1] - off[b]
        a = adj[off[b]:off[b + n]] - b
        if hashlib.sha256(o.astype("<i4").tobytes() + a.astype("<i4").tobytes()).hexdigest() \
                != csr_sha:
            bad.append((i, "csr"))
        for j in range(SLOTS):
            if _sha(dist[j, b:b + n]) != bfs_sha[j]:
                bad.append((i, "bfs", j))
        if int(tri[i]) != t:
            bad.append((i, "tc", int(tri[i]), t))
    assert not bad, bad[:20]
