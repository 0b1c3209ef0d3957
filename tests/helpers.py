"""Shared input synthesis for the tests (seeded, deterministic)."""
import numpy as np

import hornet_b200 as H
from oracle import oracle as O


def rmat_graph(scale: int, ef: int = 16, seed: int = 1, n_vertices=None) -> O.Csr:
    """Undirected R-MAT graph (a=.57 b=.19 c=.19), self loops and duplicates
    removed, sorted adjacency — built by the oracle from the library's
    host generator."""
    n = n_vertices if n_vertices is not None else (1 << scale)
    s, d = H.gen_rmat_host(scale, ef * n, seed, n_vertices=n)
    return O.build_csr_undirected(n, s, d)


def er_graph(n: int, mean_deg: float, seed: int) -> O.Csr:
    rng = np.random.default_rng(seed)
    m = int(n * mean_deg / 2)
    s = rng.integers(0, n, m, dtype=np.int32)
    d = rng.integers(0, n, m, dtype=np.int32)
    return O.build_csr_undirected(n, s, d)


def uniform_new_edges(g: O.Csr, k: int, seed: int):
    """k undirected edges (both directions) absent from g and from each other,
    no self loops."""
    rng = np.random.default_rng(seed)
    have = set((g.coo()[0].astype(np.int64) << 32 | g.coo()[1].astype(np.int64)).tolist())
    out = set()
    while len(out) < k:
        u, v = (int(x) for x in rng.integers(0, g.nV, 2))
        if u == v:
            continue
        key = (min(u, v) << 32) | max(u, v)
        if key in out or ((u << 32) | v) in have:
            continue
        out.add(key)
    a = np.array(sorted(out), np.int64)
    u, v = (a >> 32).astype(np.int32), (a & 0xFFFFFFFF).astype(np.int32)
    return np.concatenate([u, v]), np.concatenate([v, u])


def sample_existing_edges(g: O.Csr, k: int, seed: int):
    """k existing undirected edges (both directions), uniform."""
    rng = np.random.default_rng(seed)
    s, d = g.coo()
    mask = s < d
    s, d = s[mask], d[mask]
    idx = rng.choice(len(s), size=min(k, len(s)), replace=False)
    return np.concatenate([s[idx], d[idx]]), np.concatenate([d[idx], s[idx]])


def disjoint_union(graphs):
    """One CSR holding `graphs` side by side (vertex ids shifted by the
    running vertex count).  Returns (union, first vertex id of each graph)."""
    offs, adjs, base = [np.zeros(1, np.int64)], [], []
    nv = 0
    ne = 0
    for g in graphs:
        base.append(nv)
        offs.append(g.off[1:] + ne)
        adjs.append(g.adj + nv)
        nv += g.nV
        ne += g.nE
    return O.Csr(np.concatenate(offs), np.concatenate(adjs).astype(np.int32)), np.array(base)


def mix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    x = x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def hsum(keys: np.ndarray) -> int:
    if len(keys) == 0:
        return 0
    return int(mix64(keys.astype(np.uint64)).sum(dtype=np.uint64))


class UpdateModel:
    """A simple directed graph under insert(removeBatchDuplicates,
    removeGraphDuplicates) and erase(removeBatchDuplicates) batches, as
    (initial sorted (src << 32 | dst) keys - removed) | added, with the
    order-independent adjacency checksum kept up to date."""

    def __init__(self, base: np.ndarray, h0: int):
        self.base = base
        self.added = np.zeros(0, np.int64)
        self.removed = np.zeros(0, np.int64)
        self.hash = h0

    @staticmethod
    def _isin_sorted(a: np.ndarray, q: np.ndarray) -> np.ndarray:
        if len(a) == 0:
            return np.zeros(len(q), bool)
        p = np.searchsorted(a, q)
        p[p == len(a)] = 0
        return a[p] == q

    def present(self, q: np.ndarray) -> np.ndarray:
        return (self._isin_sorted(self.base, q) & ~self._isin_sorted(self.removed, q)) | \
            self._isin_sorted(self.added, q)

    def insert(self, keys: np.ndarray) -> int:
        uq = np.unique(keys)
        new = uq[~self.present(uq)]
        in_base = self._isin_sorted(self.base, new)
        self.removed = np.setdiff1d(self.removed, new[in_base], assume_unique=True)
        self.added = np.union1d(self.added, new[~in_base])
        self.hash = (self.hash + hsum(new)) % (1 << 64)
        return len(new)

    def erase(self, keys: np.ndarray) -> int:
        uq = np.unique(keys)
        gone = uq[self.present(uq)]
        in_added = self._isin_sorted(self.added, gone)
        self.added = np.setdiff1d(self.added, gone[in_added], assume_unique=True)
        self.removed = np.union1d(self.removed, gone[~in_added])
        self.hash = (self.hash - hsum(gone)) % (1 << 64)
        return len(gone)

    def neighbours(self, u: int) -> np.ndarray:
        lo, hi = np.searchsorted(self.base, [u << 32, (u + 1) << 32])
        b = self.base[lo:hi]
        b = b[~self._isin_sorted(self.removed, b)]
        lo, hi = np.searchsorted(self.added, [u << 32, (u + 1) << 32])
        return np.sort(np.concatenate([b, self.added[lo:hi]]) & 0xFFFFFFFF).astype(np.int32)
