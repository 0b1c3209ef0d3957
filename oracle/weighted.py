"""Oracle (test infrastructure only): the update model with one 32-bit
weight per edge, in plain Python for small graphs.

Restates what the weighted insert test of the reference checks
(hornet/test/HornetInsertTestWeighted.cu: the graph after an insert equals
the initial COO with the batch appended, compared as a multimap of
(src, dst) -> weights) together with the insert/erase key rules of the
unweighted model (hornet/include/Core/BatchUpdate/BatchUpdateKernels.cuh:
27-58, 263-300; BatchUpdate.i.cuh:485-524), which the C oracle
(`hn_oracle.c`) restates for keys only:

* insert: the batch is ordered stably by (src, dst); an entry is kept when
  (it is the first of its run or batch duplicates are allowed) and not
  (graph duplicates are removed and it is the first of its run and the
  edge is already in the graph); kept entries join their source's list
  after the stored copies of an equal neighbour, in batch order, carrying
  their weights;
* erase: per edge, min(copies in the batch after batch dedup, copies in the
  graph) copies leave, the first ones in stored order.

Lists stay ordered by neighbour, equal neighbours in insertion order — the
order the library keeps, so the exported (src, dst, weight) triples are
compared exactly.
"""
from typing import Dict, List, Tuple

import numpy as np

DEDUP_BATCH = 1
DEDUP_GRAPH = 2


class WGraph:
    def __init__(self, nV: int):
        self.nV = nV
        self.adj: List[List[Tuple[int, int]]] = [[] for _ in range(nV)]

    @classmethod
    def from_csr(cls, off, adj, w) -> "WGraph":
        g = cls(len(off) - 1)
        for u in range(g.nV):
            lst = [(int(adj[i]), int(w[i])) for i in range(off[u], off[u + 1])]
            # stable by neighbour: equal neighbours keep their input order
            g.adj[u] = sorted(lst, key=lambda t: t[0])
        return g

    def coo(self):
        s, d, w = [], [], []
        for u in range(self.nV):
            for v, x in self.adj[u]:
                s.append(u)
                d.append(v)
                w.append(x)
        return (np.array(s, np.int32), np.array(d, np.int32), np.array(w, np.uint32))

    @property
    def nE(self) -> int:
        return sum(len(a) for a in self.adj)

    def insert(self, bs, bd, bw, flags: int) -> int:
        order = sorted(range(len(bs)), key=lambda i: (int(bs[i]), int(bd[i])))
        add: Dict[int, List[Tuple[int, int]]] = {}
        prev = None
        for i in order:
            key = (int(bs[i]), int(bd[i]))
            first = key != prev
            prev = key
            present = any(v == key[1] for v, _ in self.adj[key[0]])
            keep = (first or not (flags & DEDUP_BATCH)) and \
                not ((flags & DEDUP_GRAPH) and first and present)
            if keep:
                add.setdefault(key[0], []).append((key[1], int(bw[i]) if bw is not None else 0))
        n = 0
        for u, lst in add.items():
            merged = self.adj[u] + lst   # stored copies first, then the batch
            self.adj[u] = sorted(merged, key=lambda t: t[0])
            n += len(lst)
        return n

    def erase(self, bs, bd, flags: int) -> int:
        cnt: Dict[Tuple[int, int], int] = {}
        for i in range(len(bs)):
            key = (int(bs[i]), int(bd[i]))
            cnt[key] = 1 if (flags & DEDUP_BATCH) else cnt.get(key, 0) + 1
        n = 0
        for (u, v), c in cnt.items():
            out = []
            for t in self.adj[u]:
                if t[0] == v and c > 0:
                    c -= 1
                    n += 1
                else:
                    out.append(t)
            self.adj[u] = out
        return n
