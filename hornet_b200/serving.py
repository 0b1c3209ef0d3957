"""Serving: one resident graph answering a timed stream of requests.

Requests are update batches (insert or erase), single-source BFS queries
(distances to a few target vertices plus the number of vertices reached) and
local triangle-count queries (triangles containing each vertex of a seed
set).  The graph stays on the device for the whole run.  Two loops serve the
same stream, and a query always sees exactly the updates that arrived
before it (arrival-order semantics, as the reference's one-call-per-request
use gives):

* the plain per-request loop: one library call per request, in arrival
  order, on one stream (hn_insert / hn_erase, hn_bfs -- or hn_bfs_do with
  single_bfs="do" --, hn_tc_local);
* the continuous-batching loop:
  - queries run on query views (hn_graph_view_create: the same resident
    graph, each view with its own stream and scratch), one per worker
    thread, so queries overlap on the device.  A query that arrives while
    others are on the GPU is admitted as soon as a view is free, whatever
    the state of the ones already running;
  - the queries of one epoch (between two updates) are grouped when they
    can share work: at least `msbfs_min` waiting BFS queries go to one
    batched traversal (hn_bfs_batch, one slot per request), waiting
    local-TC queries to one hn_tc_local call; a BFS that waits alone runs
    direction-optimising (hn_bfs_do: same distances, fewer edges read);
  - an update is a fence: it starts when the queries of the previous epoch
    have finished, and a run of consecutive waiting updates is coalesced
    into one hn_update_coalesced call (the last operation on an edge decides
    it, which on a simple graph is what applying the batches in order
    gives), split where its working memory would not fit in the free device
    memory (less a reserve); the views then take the graph's new shape
    (hn_graph_view_refresh).

Latency of a request = completion time of the call that answered it minus
its arrival time, on the host clock; the run reports p50/p99/p999 per
request kind and overall, and the throughput (requests / time of the last
completion).
"""
from __future__ import annotations

import ctypes
import threading
import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
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


class _View:
    """A query view with its own distance rows (device int32 [slots][nV])."""

    def __init__(self, hornet: Hornet, slots: int):
        import torch
        self.g = hornet if slots == 0 else hornet.view()
        self.rows = max(1, slots)
        self.dist = torch.empty((self.rows, hornet.nV()), dtype=torch.int32,
                                device=f"cuda:{hornet._device}")


class Server:
    """Serves a request stream on `hornet` (kept resident).  `batched`
    selects the continuous-batching loop (query views on `workers` threads);
    otherwise the plain per-request loop."""

    # device bytes per coalesced update entry: keys and sort buffers,
    # scan values, net sets, the update pipeline's own per-edge buffers
    UPDATE_BYTES_PER_EDGE = 96

    def __init__(self, hornet: Hornet, batched: bool = True, max_slots: int = 16,
                 max_update_edges: int = 1 << 24, reserve_bytes: int = 2 << 30,
                 free_bytes_fn=None, single_bfs: str = "", msbfs_min: int = 16,
                 workers: int = 4):
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
        self._free_fn = free_bytes_fn or (lambda: torch.cuda.mem_get_info(self.dev)[0])
        self._free_at, self._free_val = -1.0, 0
        self.workers = max(1, int(workers)) if batched else 1
        # the plain loop queries the graph itself; the batched loop one view
        # per worker
        self.views = [_View(hornet, self.max_slots if batched else 0)
                      for _ in range(self.workers)]
        self.calls = 0
        self.split_for_memory = 0
        self.groups = {"update": 0, "bfs": 0, "tc_local": 0}
        self.service_s = {"update": 0.0, "bfs": 0.0, "tc_local": 0.0}
        self.max_inflight = 0
        self.update_call_s: List[float] = []     # device-synchronous update call times
        self.update_parts_s = {"free_query": 0.0, "concat": 0.0, "call": 0.0, "refresh": 0.0}
        self._lock = threading.Lock()

    def _free(self) -> int:
        """Free device bytes, queried at most every 0.25 s (the query takes
        about a millisecond; the free memory moves only with pool growth)."""
        now = time.perf_counter()
        if now - self._free_at > 0.25:
            self._free_val = self._free_fn()
            self._free_at = now
        return self._free_val

    def close(self):
        """Release the views (before the graph)."""
        self.views = []

    # ---- library calls ---------------------------------------------------
    def _update_plain(self, r: Request):
        s = np.ascontiguousarray(r.src, np.int32)
        d = np.ascontiguousarray(r.dst, np.int32)
        b = ctypes.c_void_p()
        _check(lib().hn_batch_create(self.h.handle, len(s), s.ctypes.data_as(_P),
                                     d.ctypes.data_as(_P), HN_MEM_HOST, ctypes.byref(b)))
        try:
            n = ctypes.c_int64()
            tc = time.perf_counter()
            if r.kind == "insert":
                _check(lib().hn_insert(self.h.handle, b, HN_DEDUP_BATCH | HN_DEDUP_GRAPH,
                                       ctypes.byref(n)))
            else:
                _check(lib().hn_erase(self.h.handle, b, HN_DEDUP_BATCH, ctypes.byref(n)))
            self.update_call_s.append(time.perf_counter() - tc)
        finally:
            lib().hn_batch_destroy(b)
        self.calls += 1

    def _update_group(self, group: List[Request]):
        """Coalesced updates, split where the working set would not fit."""
        start = 0
        while start < len(group):
            tq = time.perf_counter()
            free_b = self._free()
            self.update_parts_s["free_query"] += time.perf_counter() - tq
            budget = max(0, free_b - self.reserve) // self.UPDATE_BYTES_PER_EDGE
            budget = min(budget, self.max_update_edges)
            end, total = start, 0
            while end < len(group) and (end == start or total + group[end].n_edges <= budget):
                total += group[end].n_edges
                end += 1
            if end < len(group):
                self.split_for_memory += 1
            part = group[start:end]
            tq = time.perf_counter()
            src = np.concatenate([r.src for r in part]).astype(np.int32, copy=False)
            dst = np.concatenate([r.dst for r in part]).astype(np.int32, copy=False)
            ops = np.concatenate([np.full(r.n_edges, 1 if r.kind == "insert" else 0, np.uint8)
                                  for r in part])
            tc = time.perf_counter()
            self.update_parts_s["concat"] += tc - tq
            self.h.update_coalesced(src, dst, ops)
            self.update_call_s.append(time.perf_counter() - tc)
            self.update_parts_s["call"] += time.perf_counter() - tc
            self.calls += 1
            self.groups["update"] += 1
            start = end

    def _bfs_unit(self, v: _View, group: List[Request], results):
        k = len(group)
        srcs = np.array([r.source for r in group], np.int32)
        stats = (BfsStats * k)()
        g = v.g.handle
        base = v.dist.data_ptr()
        if k >= self.msbfs_min:
            _check(lib().hn_bfs_batch(g, srcs.ctypes.data_as(_P), None, k, k,
                                      ctypes.c_void_p(base), HN_MEM_DEVICE, stats))
            calls = 1
        else:
            for j in range(k):
                row = ctypes.c_void_p(base + 4 * j * self.nV)
                if self.single_bfs == "do":
                    one = srcs[j:j + 1]
                    _check(lib().hn_bfs_do(g, one.ctypes.data_as(_P), 1, row, HN_MEM_DEVICE,
                                           ctypes.byref(stats[j])))
                else:
                    _check(lib().hn_bfs(g, int(srcs[j]), row, HN_MEM_DEVICE,
                                        ctypes.byref(stats[j])))
            calls = k
        idx = np.concatenate([j * self.nV + np.asarray(r.targets, np.int64)
                              for j, r in enumerate(group)])
        got = v.g.gather(base, idx)
        at = 0
        for j, r in enumerate(group):
            n = len(r.targets)
            results[r.rid] = (got[at:at + n].copy(), int(stats[j].visited))
            at += n
        return calls

    def _tc_unit(self, v: _View, group: List[Request], results):
        seeds = np.concatenate([np.asarray(r.seeds, np.int32) for r in group])
        out = np.empty(len(seeds), np.uint64)
        _check(lib().hn_tc_local(v.g.handle, seeds.ctypes.data_as(_P), len(seeds),
                                 out.ctypes.data_as(_P), HN_MEM_HOST))
        at = 0
        for r in group:
            results[r.rid] = out[at:at + len(r.seeds)].copy()
            at += len(r.seeds)
        return 1

    def _run_unit(self, v: _View, kind: str, group: List[Request], results, t0):
        """One query unit on view v (a worker thread); returns the unit's
        completion time (seconds since t0)."""
        ts = time.perf_counter()
        calls = self._bfs_unit(v, group, results) if kind == "bfs" else \
            self._tc_unit(v, group, results)
        te = time.perf_counter()
        with self._lock:
            self.calls += calls
            self.groups[kind] += 1
            self.service_s[kind] += te - ts
        return te - t0

    # ---- loops ---------------------------------------------------------------
    def run(self, requests: List[Request]) -> ServeReport:
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        n = len(reqs)
        lat = np.zeros(n)
        kinds = [r.kind for r in reqs]
        pos = {r.rid: i for i, r in enumerate(reqs)}
        results: Dict[int, object] = {}
        t0 = time.perf_counter()
        if self.batched:
            last = self._run_batched(reqs, lat, pos, results, t0)
        else:
            last = self._run_plain(reqs, lat, pos, results, t0)
        lat_ms = {}
        for kind in ("insert", "erase", "bfs", "tc_local", "all"):
            sel = lat if kind == "all" else lat[[k == kind for k in kinds]]
            if len(sel):
                lat_ms[kind] = {"n": int(len(sel)), "p50": round(_pct(sel, 50) * 1e3, 3),
                                "p99": round(_pct(sel, 99) * 1e3, 3),
                                "p999": round(_pct(sel, 99.9) * 1e3, 3),
                                "mean": round(float(sel.mean()) * 1e3, 3)}
        rep = ServeReport("batched" if self.batched else "per_request", n, last,
                          n / last if last > 0 else float("inf"), lat_ms, self.calls,
                          dict(self.groups), self.split_for_memory, results)
        rep.service_ms = {k: round(v * 1e3, 2) for k, v in self.service_s.items()}
        rep.single_bfs = self.single_bfs
        rep.workers = self.workers
        rep.max_inflight = self.max_inflight
        u = np.array(self.update_call_s)
        rep.update_parts_ms = {k: round(v * 1e3, 2) for k, v in self.update_parts_s.items()}
        rep.update_calls_ms = {"n": int(len(u)), "p50": round(_pct(u, 50) * 1e3, 3),
                               "p99": round(_pct(u, 99) * 1e3, 3),
                               "max": round(float(u.max()) * 1e3 if len(u) else 0.0, 3),
                               "sum": round(float(u.sum()) * 1e3, 2)}
        return rep

    def _run_plain(self, reqs, lat, pos, results, t0) -> float:
        n = len(reqs)
        v = self.views[0]
        i = done = 0
        last = 0.0
        while done < n:
            now = time.perf_counter() - t0
            if reqs[i].arrival > now:
                wait_s = reqs[i].arrival - now
                if wait_s > 2e-3:
                    time.sleep(wait_s - 1e-3)
                continue
            r = reqs[i]
            ts = time.perf_counter()
            if r.kind in UPDATE_KINDS:
                self._update_plain(r)
                self.groups["update"] += 1
                results[r.rid] = None
                kind = "update"
            else:
                kind = r.kind
                self.calls += self._bfs_unit(v, [r], results) if kind == "bfs" else \
                    self._tc_unit(v, [r], results)
                self.groups[kind] += 1
            te = time.perf_counter()
            self.service_s[kind] += te - ts
            last = te - t0
            lat[pos[r.rid]] = last - r.arrival
            i += 1
            done += 1
        return last

    def _run_batched(self, reqs, lat, pos, results, t0) -> float:
        n = len(reqs)
        pending: deque = deque()
        free = list(self.views)
        inflight = {}                      # future -> (view, requests)
        i = done = 0
        last = 0.0
        with ThreadPoolExecutor(max_workers=self.workers) as ex:

            def harvest(futs):
                nonlocal done, last
                for f in futs:
                    v, grp = inflight.pop(f)
                    t = f.result()
                    free.append(v)
                    last = max(last, t)
                    for r in grp:
                        lat[pos[r.rid]] = t - r.arrival
                    done += len(grp)

            while done < n:
                now = time.perf_counter() - t0
                while i < n and reqs[i].arrival <= now:
                    pending.append(reqs[i])
                    i += 1
                ready = [f for f in inflight if f.done()]
                if ready:
                    harvest(ready)
                    continue
                if pending and pending[0].kind in UPDATE_KINDS:
                    if inflight:                       # fence: the epoch's queries first
                        harvest(wait(list(inflight), return_when=FIRST_COMPLETED)[0])
                        continue
                    group = [pending.popleft()]
                    while pending and pending[0].kind in UPDATE_KINDS:
                        group.append(pending.popleft())
                    ts = time.perf_counter()
                    self._update_group(group)
                    tr = time.perf_counter()
                    for v in self.views:
                        v.g.refresh_view()
                    te = time.perf_counter()
                    self.update_parts_s["refresh"] += te - tr
                    self.service_s["update"] += te - ts
                    last = max(last, te - t0)
                    for r in group:
                        results[r.rid] = None
                        lat[pos[r.rid]] = te - t0 - r.arrival
                    done += len(group)
                    continue
                if pending and free:
                    for kind, grp in query_units(pending, len(free), self.msbfs_min,
                                                 self.max_slots):
                        v = free.pop()
                        f = ex.submit(self._run_unit, v, kind, grp, results, t0)
                        inflight[f] = (v, grp)
                    self.max_inflight = max(self.max_inflight, len(inflight))
                    continue
                # nothing to start: wait for a completion or the next arrival
                timeout = None
                if i < n:
                    timeout = max(0.0, reqs[i].arrival - (time.perf_counter() - t0))
                if inflight:
                    harvest(wait(list(inflight), timeout=timeout,
                                 return_when=FIRST_COMPLETED)[0])
                elif timeout is not None and timeout > 2e-3:
                    time.sleep(timeout - 1e-3)
        return last


def query_units(pending: deque, nfree: int, msbfs_min: int, max_slots: int):
    """Query units for up to nfree free views, popped from the front of
    `pending` up to the first update (so a unit never crosses an update):
    the waiting local-TC queries as one unit; the waiting BFS queries as one
    batched unit when there are at least msbfs_min of them (at most
    max_slots per unit), else one unit each.  Requests that get no view now
    go back to the front of `pending`, in arrival order."""
    qs = []
    while pending and pending[0].kind in QUERY_KINDS:
        qs.append(pending.popleft())
    units = []
    bfs = [r for r in qs if r.kind == "bfs"]
    tcs = [r for r in qs if r.kind == "tc_local"]
    if tcs:
        units.append(("tc_local", tcs))
    while bfs:
        if len(bfs) >= msbfs_min:
            units.append(("bfs", bfs[:max_slots]))
            bfs = bfs[max_slots:]
        else:
            units.append(("bfs", [bfs.pop(0)]))
    keep = units[:nfree]
    back = sorted([r for _, g in units[nfree:] for r in g], key=lambda r: (r.arrival, r.rid))
    for r in reversed(back):
        pending.appendleft(r)
    return keep


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
