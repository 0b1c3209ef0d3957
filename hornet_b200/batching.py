"""Many graphs, one launch: a batch of independent graphs of uneven size held
as one Hornet (their disjoint union, vertex ids shifted by each graph's
base), traversed together by the batched BFS and counted together by
triangle counting.

The reference runs one StaticAlgorithm per graph and per source
(hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:88-106,
hornetsnest/src/Static/TriangleCounting/triangle2.cu:158-171); a batch gives
the same per-graph results:

* BFS: source j of every graph goes to slot j, so one hn_bfs_batch call
  with `sources_per_graph` slots computes every (graph, source) pair; the
  graphs are disjoint, so a slot's distances inside graph i are graph i's
  own BFS from its source j.
* Triangles: the union's owner counts (hn_tc_owner: each triangle credited
  once, to its lowest vertex in the degree orientation) summed over each
  graph's vertex range; every triangle lies inside one graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import HN_MEM_DEVICE, Hornet, _check, _P, lib


def synthetic_specs(n_graphs: int, seed: int = 4096):
    """The many-small-graphs workload: n_graphs graphs with vertex counts
    log-uniform in [1024, 65536]; half Erdos-Renyi with mean degree 8
    (4n uniform pairs), half R-MAT with edge factor 16 (a=.57 b=.19 c=.19,
    16n pairs drawn at scale ceil(log2 n), endpoints >= n redrawn).  Returns
    (sizes, bases, kinds, specs); graph i's pairs are
    gen_rmat(scale, pairs, pair_seed, n_vertices=n, a, b, c) with
    (scale, pairs, pair_seed, n, a, b, c) = specs[i]; kinds[i] is 0 for ER."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1024), np.log(65536), n_graphs)).astype(np.int64)
    kinds = rng.permutation(np.repeat([0, 1], [n_graphs // 2, n_graphs - n_graphs // 2]))
    pairs = np.where(kinds == 0, 4 * sizes, 16 * sizes)
    bases = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    specs = []
    for i in range(n_graphs):
        n = int(sizes[i])
        abc = (0.25, 0.25, 0.25) if kinds[i] == 0 else (0.57, 0.19, 0.19)
        specs.append((int(np.ceil(np.log2(n))), int(pairs[i]), seed * 1_000_003 + i, n) + abc)
    return sizes, bases, kinds, specs


def synthetic_union(n_graphs: int, seed: int = 4096, device: int = 0):
    """The graphs of synthetic_specs generated on the device into one
    disjoint union.  Returns (hornet, device csr, sizes, bases, kinds)."""
    import torch
    from . import coo_to_csr_device, gen_rmat_device, hornet_from_device_csr
    sizes, bases, kinds, specs = synthetic_specs(n_graphs, seed)
    poff = np.concatenate([[0], np.cumsum([sp[1] for sp in specs])]).astype(np.int64)
    src = torch.empty(int(poff[-1]), dtype=torch.int32, device=f"cuda:{device}")
    dst = torch.empty_like(src)
    for i, (sc, npairs, pseed, n, a, b, c) in enumerate(specs):
        s, d = src[poff[i]:poff[i + 1]], dst[poff[i]:poff[i + 1]]
        gen_rmat_device(sc, npairs, pseed, s, d, n_vertices=n, a=a, b=b, c=c, device=device)
        s += int(bases[i])
        d += int(bases[i])
    csr = coo_to_csr_device(int(sizes.sum()), src, dst, device=device)
    del src, dst
    h = hornet_from_device_csr(csr, device=device)
    return h, csr, sizes, bases, kinds


class GraphBatch:
    """A batch of graphs as one Hornet.  `bases[i]` is the first vertex id of
    graph i in the union; `sizes[i]` its vertex count."""

    def __init__(self, hornet: Hornet, bases, sizes):
        self.hornet = hornet
        self.bases = np.ascontiguousarray(bases, np.int64)
        self.sizes = np.ascontiguousarray(sizes, np.int64)
        assert len(self.bases) == len(self.sizes)
        assert int(self.bases[-1] + self.sizes[-1]) == hornet.nV()

    @property
    def n_graphs(self) -> int:
        return len(self.sizes)

    def bfs(self, local_sources, out):
        """local_sources: int[n_graphs][k] vertex ids local to each graph
        (k <= 64).  out: device int32 tensor [k][nV] (the union's ids);
        graph i's distances from its source j are out[j, bases[i]:bases[i]+sizes[i]].
        Returns the per-slot statistics."""
        from . import BfsStats
        ls = np.ascontiguousarray(local_sources, np.int64)
        k = ls.shape[1]
        if (ls < 0).any() or (ls >= self.sizes[:, None]).any():
            raise ValueError("source outside its graph")
        srcs = (ls + self.bases[:, None]).astype(np.int32).ravel()
        slots = np.tile(np.arange(k, dtype=np.int32), self.n_graphs)
        stats = (BfsStats * k)()
        _check(lib().hn_bfs_batch(self.hornet.handle, srcs.ctypes.data_as(_P),
                                  slots.ctypes.data_as(_P), len(srcs), k,
                                  ctypes.c_void_p(out.data_ptr()), HN_MEM_DEVICE, stats))
        return [stats[i] for i in range(k)]

    def triangles(self, per_vertex):
        """Per-graph triangle counts (device int64 tensor [n_graphs]);
        per_vertex is a device int64 scratch tensor [nV] that receives the
        owner counts (each triangle credited once, to a vertex of its own
        graph)."""
        import torch
        total = ctypes.c_uint64()
        _check(lib().hn_tc_owner(self.hornet.handle, ctypes.c_void_p(per_vertex.data_ptr()),
                                 HN_MEM_DEVICE, ctypes.byref(total)))
        off = np.ascontiguousarray(np.concatenate([self.bases, self.bases[-1:] + self.sizes[-1:]]),
                                   np.int64)
        out = torch.empty(self.n_graphs, dtype=torch.int64, device=per_vertex.device)
        _check(lib().hn_segment_sum_u64(self.hornet.handle,
                                        ctypes.c_void_p(per_vertex.data_ptr()),
                                        off.ctypes.data_as(ctypes.c_void_p), self.n_graphs,
                                        ctypes.c_void_p(out.data_ptr())))
        return out, total.value
