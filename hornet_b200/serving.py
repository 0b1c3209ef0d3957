"""Serving: one resident graph answering a timed stream of requests.

Requests are update batches (insert or erase), single-source BFS queries
(distances to a few target vertices plus the number of vertices reached) and
local triangle-count queries (triangles containing each vertex of a seed
set).  The graph stays on the device for the whole run.  Two loops serve the
same stream:

* the plain per-request loop: one library call per request, in arrival
  order (hn_insert / hn_erase, hn_bfs — or hn_bfs_do with single_bfs="do" —,
  hn_tc_local);
* the batched loop, which keeps arrival-order semantics — a query sees
  exactly the updates that arrived before it — while
  - coalescing a run of consecutive update batches into one
    hn_update_coalesced call (the last operation on an edge decides it, which
    on a simple graph is what applying the batches in order gives),
  - answering a run of consecutive queries together: up to `max_slots` BFS
    sources in one hn_bfs_batch traversal (one slot per request, so every
    request gets its own single-source distances) when the run holds at
    least `msbfs_min` of them, otherwise one direction-optimising traversal
    per BFS (hn_bfs_do: the same distances, fewer edges read); all local-TC
    seed sets in one hn_tc_local call,
  - admitting a coalesced update only while its working memory fits in
    the free device memory (less a reserve); a run that does not fit is split.

Latency of a request = completion time of the call that answered it minus its
arrival time, both on the host clock; the run reports p50/p99 per request
kind and overall, and the throughput (requests / time of the last
completion).
"""
from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import (HN_DEDUP_BATCH, HN_DEDUP_GRAPH, HN_MEM_DEVICE, HN_MEM_HOST, BfsStats, Hornet,
               _check, _P, lib)

UPDATE_KINDS = ("insert", "erase")
QUERY_KINDS = ("bfs", "tc_local")


@dataclass
class Request:
    rid: int
    kind: str                              # "insert" | "erase" | "bfs" | "tc_local"
    arrival: float                         # seconds after the start of the run
    src: Optional[np.ndarray] = None       # updates: int32 edge endpoints
    dst: Optional[np.ndarray] = None
    source: int = 0                        # bfs
    targets: Optional[np.ndarray] = None   # bfs: int32 vertices reported
    seeds: Optional[np.ndarray] = None     # tc_local: int32 seed set

    @property
    def n_edges(self) -> int:
        return 0 if self.src is None else len(self.src)


@dataclass
class ServeReport:
    mode: str
    n_requests: int
    makespan_s: float
    throughput_rps: float
    latency_ms: Dict[str, Dict[str, float]]
    calls: int
    groups: Dict[str, int]
    split_for_memory: int
    results: Dict[int, object] = field(repr=False, default_factory=dict)

    def summary(self) -> dict:
        return {"mode": self.mode, "requests": self.n_requests,
                "makespan_s": round(self.makespan_s, 4),
                "throughput_rps": round(self.throughput_rps, 1), "latency_ms": self.latency_ms,
                "library_calls": self.calls, "groups": self.groups,
                "updates_split_for_memory": self.split_for_memory,
                "service_ms": getattr(self, "service_ms", None),
                "single_bfs": getattr(self, "single_bfs", None)}


def _pct(a, q):
    return float(np.percentile(a, q)) if len(a) else float("nan")


class Server:
    """Serves a request stream on `hornet` (kept resident).  `batched`
    selects the batched loop; otherwise the plain per-request loop."""

    # device bytes per coalesced update entry: keys and sort buffers,
    # scan values, net sets, the update pipeline's own per-edge buffers
    UPDATE_BYTES_PER_EDGE = 96

    def __init__(self, hornet: Hornet, batched: bool = True, max_slots: int = 64,
                 max_update_edges: int = 1 << 24, reserve_bytes: int = 2 << 30,
                 free_bytes_fn=None, single_bfs: str = "", msbfs_min: int = 4):
        import torch
        self.h = hornet
        self.batched = batched
        # traversal for a BFS answered alone: "td" (BfsTopDown) or "do"
        # (direction-optimising, same distances); groups of at least
        # msbfs_min BFS queries go to one batched traversal
        self.single_bfs = single_bfs or ("do" if batched else "td")
        self.msbfs_min = max(2, int(msbfs_min))
        self.max_slots = max(1, min(64, int(max_slots)))
        self.max_update_edges = int(max_update_edges)
        self.reserve = int(reserve_bytes)
        self.dev = hornet._device
        self.nV = hornet.nV()
        self._free = free_bytes_fn or (lambda: torch.cuda.mem_get_info(self.dev)[0])
        slots = self.max_slots if batched else 1
        self.dist = torch.empty((slots, self.nV), dtype=torch.int32, device=f"cuda:{self.dev}")
        self.dist_flat = self.dist.view(-1)
        self.calls = 0
        self.split_for_memory = 0
        self.groups = {"update": 0, "bfs": 0, "tc_local": 0}
        self.service_s = {"update": 0.0, "bfs": 0.0, "tc_local": 0.0}

    # ---- library calls ---------------------------------------------------
    def _update_plain(self, r: Request):
        s = np.ascontiguousarray(r.src, np.int32)
        d = np.ascontiguousarray(r.dst, np.int32)
        b = ctypes.c_void_p()
        _check(lib().hn_batch_create(self.h.handle, len(s), s.ctypes.data_as(_P),
                                     d.ctypes.data_as(_P), HN_MEM_HOST, ctypes.byref(b)))
        try:
            n = ctypes.c_int64()
            if r.kind == "insert":
                _check(lib().hn_insert(self.h.handle, b, HN_DEDUP_BATCH | HN_DEDUP_GRAPH,
                                       ctypes.byref(n)))
            else:
                _check(lib().hn_erase(self.h.handle, b, HN_DEDUP_BATCH, ctypes.byref(n)))
        finally:
            lib().hn_batch_destroy(b)
        self.calls += 1
        return None

    def _update_group(self, group: List[Request]):
        """Coalesced updates, split where the working set would not fit."""
        start = 0
        while start < len(group):
            budget = max(0, self._free() - self.reserve) // self.UPDATE_BYTES_PER_EDGE
            budget = min(budget, self.max_update_edges)
            end, total = start, 0
            while end < len(group) and (end == start or total + group[end].n_edges <= budget):
                total += group[end].n_edges
                end += 1
            if end < len(group):
                self.split_for_memory += 1
            part = group[start:end]
            src = np.concatenate([r.src for r in part]).astype(np.int32, copy=False)
            dst = np.concatenate([r.dst for r in part]).astype(np.int32, copy=False)
            ops = np.concatenate([np.full(r.n_edges, 1 if r.kind == "insert" else 0, np.uint8)
                                  for r in part])
            self.h.update_coalesced(src, dst, ops)
            self.calls += 1
            self.groups["update"] += 1
            start = end

    def _bfs_group(self, group: List[Request], results):
        import torch
        k = len(group)
        srcs = np.array([r.source for r in group], np.int32)
        stats = (BfsStats * k)()
        if k >= self.msbfs_min:
            _check(lib().hn_bfs_batch(self.h.handle, srcs.ctypes.data_as(_P), None, k, k,
                                      ctypes.c_void_p(self.dist.data_ptr()), HN_MEM_DEVICE,
                                      stats))
            self.calls += 1
        else:
            for j in range(k):
                row = ctypes.c_void_p(self.dist.data_ptr() + 4 * j * self.nV)
                if self.single_bfs == "do":
                    one = srcs[j:j + 1]
                    _check(lib().hn_bfs_do(self.h.handle, one.ctypes.data_as(_P), 1, row,
                                           HN_MEM_DEVICE, ctypes.byref(stats[j])))
                else:
                    _check(lib().hn_bfs(self.h.handle, int(srcs[j]), row, HN_MEM_DEVICE,
                                        ctypes.byref(stats[j])))
                self.calls += 1
        self.groups["bfs"] += 1
        idx = np.concatenate([j * self.nV + np.asarray(r.targets, np.int64)
                              for j, r in enumerate(group)])
        got = torch.take(self.dist_flat, torch.from_numpy(idx).to(self.dist.device)).cpu().numpy()
        at = 0
        for j, r in enumerate(group):
            n = len(r.targets)
            results[r.rid] = (got[at:at + n].copy(), int(stats[j].visited))
            at += n

    def _tc_group(self, group: List[Request], results):
        seeds = np.concatenate([np.asarray(r.seeds, np.int32) for r in group])
        out = np.empty(len(seeds), np.uint64)
        _check(lib().hn_tc_local(self.h.handle, seeds.ctypes.data_as(_P), len(seeds),
                                 out.ctypes.data_as(_P), HN_MEM_HOST))
        self.calls += 1
        self.groups["tc_local"] += 1
        at = 0
        for r in group:
            results[r.rid] = out[at:at + len(r.seeds)].copy()
            at += len(r.seeds)

    # ---- loop --------------------------------------------------------------
    def _take(self, pending: deque) -> List[Request]:
        return take_group(pending, self.batched, self.max_slots)

    def _execute(self, group: List[Request], results):
        t0 = time.perf_counter()
        self._execute_group(group, results)
        kind = "update" if group[0].kind in UPDATE_KINDS else \
            ("bfs" if group[0].kind == "bfs" else "tc_local")
        self.service_s[kind] += time.perf_counter() - t0

    def _execute_group(self, group: List[Request], results):
        if group[0].kind in UPDATE_KINDS:
            if self.batched:
                self._update_group(group)
            else:
                self._update_plain(group[0])
                self.groups["update"] += 1
            for r in group:
                results[r.rid] = None
            return
        bfs = [r for r in group if r.kind == "bfs"]
        tcs = [r for r in group if r.kind == "tc_local"]
        if bfs:
            self._bfs_group(bfs, results)
        if tcs:
            self._tc_group(tcs, results)

    def run(self, requests: List[Request]) -> ServeReport:
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        n = len(reqs)
        lat = np.zeros(n)
        kinds = [r.kind for r in reqs]
        pos = {r.rid: i for i, r in enumerate(reqs)}
        results: Dict[int, object] = {}
        pending: deque = deque()
        i = 0
        done = 0
        t0 = time.perf_counter()
        last = 0.0
        while done < n:
            now = time.perf_counter() - t0
            while i < n and reqs[i].arrival <= now:
                pending.append(reqs[i])
                i += 1
            if not pending:
                wait = reqs[i].arrival - (time.perf_counter() - t0)
                if wait > 2e-3:
                    time.sleep(wait - 1e-3)
                continue
            group = self._take(pending)
            self._execute(group, results)
            last = time.perf_counter() - t0
            for r in group:
                lat[pos[r.rid]] = last - r.arrival
            done += len(group)
        lat_ms = {}
        for kind in ("insert", "erase", "bfs", "tc_local", "all"):
            sel = lat if kind == "all" else lat[[k == kind for k in kinds]]
            if len(sel):
                lat_ms[kind] = {"n": int(len(sel)), "p50": round(_pct(sel, 50) * 1e3, 3),
                                "p99": round(_pct(sel, 99) * 1e3, 3),
                                "mean": round(float(sel.mean()) * 1e3, 3)}
        rep = ServeReport("batched" if self.batched else "per_request", n, last,
                          n / last if last > 0 else float("inf"), lat_ms, self.calls,
                          dict(self.groups), self.split_for_memory, results)
        rep.service_ms = {k: round(v * 1e3, 2) for k, v in self.service_s.items()}
        rep.single_bfs = self.single_bfs
        return rep


def take_group(pending: deque, batched: bool, max_slots: int) -> List[Request]:
    """The next group to execute, popped from the front of `pending`:
    a run of consecutive updates, or a run of consecutive queries holding at
    most `max_slots` BFS queries (one request when not batched).  Groups
    never cross an update/query boundary, so every query sees exactly the
    updates that arrived before it."""
    if not batched:
        return [pending.popleft()]
    group = [pending.popleft()]
    if group[0].kind in UPDATE_KINDS:
        while pending and pending[0].kind in UPDATE_KINDS:
            group.append(pending.popleft())
    else:
        nbfs = int(group[0].kind == "bfs")
        while pending and pending[0].kind in QUERY_KINDS:
            if pending[0].kind == "bfs":
                if nbfs == max_slots:
                    break
                nbfs += 1
            group.append(pending.popleft())
    return group


def same_results(a: Dict[int, object], b: Dict[int, object]) -> bool:
    """Per-request results of two runs are identical."""
    if a.keys() != b.keys():
        return False
    for k, x in a.items():
        y = b[k]
        if x is None or y is None:
            if x is not y:
                return False
        elif isinstance(x, tuple):
            if x[1] != y[1] or not np.array_equal(x[0], y[0]):
                return False
        elif not np.array_equal(x, y):
            return False
    return True


def make_requests(n: int, rate: float, nV: int, deg: np.ndarray, erase_pool, seed: int,
                  mix=(0.6, 0.3, 0.1), median_edges: int = 10_000, sigma: float = 1.5,
                  clip=(100, 2_000_000), n_targets: int = 16, n_seeds: int = 1000,
                  insert_pairs=None) -> List[Request]:
    """A seeded request stream: Poisson arrivals at `rate` per second
    (rate <= 0: everything arrives at time 0); `mix` = fractions of update
    batches (half insert, half erase), BFS queries and local-TC queries;
    update sizes LogNormal(median, sigma) clipped, as undirected pairs
    stored in both directions.  erase_pool(rng, k) -> (src, dst) samples k
    existing edges; insert_pairs(rng, k) -> (src, dst) draws k new pairs
    (uniform when None)."""
    rng = np.random.default_rng(seed)
    if rate > 0:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    else:
        arrivals = np.zeros(n)
    u = rng.random(n)
    nonzero = np.nonzero(deg > 0)[0]
    out = []
    for i in range(n):
        a = float(arrivals[i])
        if u[i] < mix[0]:
            k = int(np.clip(rng.lognormal(np.log(median_edges), sigma), clip[0], clip[1]))
            if rng.random() < 0.5:
                if insert_pairs is None:
                    s = rng.integers(0, nV, k).astype(np.int32)
                    d = rng.integers(0, nV, k).astype(np.int32)
                else:
                    s, d = insert_pairs(rng, k)
                keep = s != d
                s, d = s[keep], d[keep]
                out.append(Request(i, "insert", a, np.concatenate([s, d]),
                                   np.concatenate([d, s])))
            else:
                s, d = erase_pool(rng, k)
                out.append(Request(i, "erase", a, np.concatenate([s, d]),
                                   np.concatenate([d, s])))
        elif u[i] < mix[0] + mix[1]:
            out.append(Request(i, "bfs", a, source=int(rng.choice(nonzero)),
                               targets=rng.integers(0, nV, n_targets).astype(np.int32)))
        else:
            out.append(Request(i, "tc_local", a,
                               seeds=rng.integers(0, nV, n_seeds).astype(np.int32)))
    return out
