"""Autotuner for the library's tuning knobs (hn_tune_set / hn_tune_get).

The knobs are load-balancing bin thresholds and launch shapes:

* tc.warp_cap — the oriented-degree boundary between the warp-per-vertex and
  the CTA-per-vertex triangle kernels; tc.chunk — vertices per work grab;
  tc.warp_ctas_per_sm — grid of the warp kernel;
* msbfs.block — block size of the batched BFS (128/256/512 threads, the
  same 2048-edge chunks); msbfs.ctas_per_sm — its grid;
* bfs.kernel — the warp-chunk (1) or CTA-chunk (0) BFS level kernel;
  bfs.warp_ctas_per_sm / bfs.ctas_per_sm — their grids; bfs.dynamic_chunks —
  frontier chunks taken from a counter instead of round-robin (CTA kernel);
  bfs.do_alpha / do_beta — the direction-optimising switch thresholds.

`tune` runs coordinate descent over a knob space: every candidate value of a
knob is timed (median of `reps` runs, after one warm-up run that also
rebuilds any CUDA graph the knob is baked into) with the other knobs at
their best values so far, and every candidate's result must equal the
result at the defaults — a knob only ever changes speed.  Results are kept
in a JSON file keyed by device name and a workload signature (workload
kind, log2 of the vertex count, average degree, log2 of the maximum degree),
so a later run on the same kind of input and device loads them with
`apply_saved`.
"""
from __future__ import annotations

import json
import math
import os
import time
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import tune_get, tune_names, tune_reset, tune_set

SPACES: Dict[str, Dict[str, List[int]]] = {
    "bfs": {"bfs.kernel": [1, 0], "bfs.warp_ctas_per_sm": [2, 3, 4, 6, 8],
            "bfs.ctas_per_sm": [4, 6, 8, 9, 12, 16], "bfs.dynamic_chunks": [0, 1],
            "bfs.warp_strided": [0, 1]},
    "bfs_do": {"bfs.do_alpha": [4, 8, 14, 24, 48], "bfs.do_beta": [8, 24, 64, 256]},
    "msbfs": {"msbfs.block": [128, 256, 512], "msbfs.ctas_per_sm": [2, 4, 6, 8],
              "msbfs.bottom_up": [0, 1]},
    "tc": {"tc.warp_cap": [64, 128, 256, 512], "tc.chunk": [4, 16, 64],
           "tc.warp_ctas_per_sm": [4, 8, 12, 16], "tc.narrow_min": [0, 8, 32, 128],
           "tc.mid_cap": [1024, 2048, 4096], "tc.warp_work": [16384, 65536, 262144],
           "tc.item_work": [65536, 262144, 1048576], "tc.flip": [0, 1],
           "tc.thread_du": [0, 8, 16, 32], "tc.thread_dc": [16, 32, 128]},
}

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")


def signature(workload: str, nV: int, nE: int, max_degree: int) -> str:
    avg = nE / max(1, nV)
    return (f"{workload}|lognV={round(math.log2(max(2, nV)))}|avgdeg={round(avg)}"
            f"|logmaxdeg={round(math.log2(max(2, max_degree)))}")


def current() -> Dict[str, int]:
    return {n: tune_get(n) for n in tune_names()}


def _time(run: Callable[[], object], reps: int) -> Tuple[float, object]:
    out = run()   # warm-up: graph rebuilds, caches
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = run()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), out


def tune(run: Callable[[], object], same: Callable[[object, object], bool],
         space: Dict[str, List[int]], reps: int = 3) -> Tuple[Dict[str, int], List[dict]]:
    """Coordinate descent over `space`.  run() executes the workload once
    (and synchronises); same(a, b) compares two results.  Returns the best
    knob values and the trial log; the best values are left set."""
    base_t, base_out = _time(run, reps)
    best = {k: tune_get(k) for k in space}
    best_t = base_t
    log = [{"knobs": dict(best), "s": base_t, "default": True}]
    for knob, values in space.items():
        start = best[knob]
        for v in values:
            if v == start:
                continue
            tune_set(knob, v)
            t, out = _time(run, reps)
            ok = same(out, base_out)
            log.append({"knobs": {**best, knob: v}, "s": t, "same_result": ok})
            if not ok:
                raise RuntimeError(f"knob {knob}={v} changed the result")
            if t < best_t:
                best_t, best[knob] = t, v
        tune_set(knob, best[knob])
    return best, log


def load(path: str = DEFAULT_PATH) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save(device_name: str, sig: str, knobs: Dict[str, int], speedup: float,
         path: str = DEFAULT_PATH) -> None:
    db = load(path)
    db.setdefault(device_name, {})[sig] = {"knobs": knobs, "speedup_vs_default": round(speedup, 3)}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply_saved(device_name: str, sig: str, path: str = DEFAULT_PATH) -> Optional[Dict[str, int]]:
    """Set the knobs saved for (device, signature); None when there are none."""
    rec = load(path).get(device_name, {}).get(sig)
    if not rec:
        return None
    for k, v in rec["knobs"].items():
        tune_set(k, v)
    return dict(rec["knobs"])


def reset() -> None:
    tune_reset()
