"""Benchmark of the Hornet dynamic-graph hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload static|update] [--scale S]

static (default): undirected R-MAT (a=.57 b=.19 c=.19), scale 22, edge
    factor 16, int32 ids, sorted adjacency; BFS TopDown from 64 seeded random
    non-isolated sources.  One step = one BFS from the next source.
    Headline metric: BFS GTEPS (directed edges scanned per second).
    Also measured on the same graph: TriangleCounting2 (TC edges/s), CC
    (edges/s) and a 1M-edge insert + erase batch (update edges/s).
update: R-MAT scale 24; batches of 1K..10M uniform edges alternately
    inserted and erased.  One step = one batch.  Metric: update edges/s.

The graph is synthetic (seeded) and resident in HBM before timing; graph
data (>= 0.6 GB) exceeds the 126 MB L2, so no L2 flush is needed between
steps.  Device time is measured with CUDA events on the stream the library
launches on, max over ranks.  With N > 1 every rank runs an independent
replica (the path has no exchange step).

--impl reference times the reference's own CPU implementation on the host
(graph::BFS from xlib, compiled into oracle/_ref/ref_driver), rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def hbm_peak():
    try:
        p = json.load(open(PEAKS_FILE))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class Dist:
    """Rank aggregation for the replica benchmark: device time is the MAX
    over ranks, work is the SUM (works with nccl on cuda tensors and with
    gloo on cpu tensors)."""

    def __init__(self, world: int, device: str = "cpu"):
        self.world = world
        self.device = device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def _reduce(self, x, op):
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.MAX) if self.world > 1 else x

    def sum(self, x):
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.SUM) if self.world > 1 else x


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"hn_clocks_{os.getpid()}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        # a short timed region may end before nvidia-smi's first sample:
        # wait (at most a second) for one line
        for _ in range(50):
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                try:
                    rows.append(f)
                except Exception:
                    pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def load_traffic(name):
    """Per-launch DRAM bytes of kernel `name` from a committed ncu summary
    (profiles/*.md line 'traffic_bytes_per_launch <kernel> <workload> <bytes>')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(d, fn)):
            p = line.strip().strip("`").split()
            if len(p) == 4 and p[0] == "traffic_bytes_per_launch" and p[1] == name:
                return p[2], float(p[3])
    return None


# ---------------------------------------------------------------------------
# graph construction
# ---------------------------------------------------------------------------

def make_graph_device(H, scale, ef, seed, device):
    import torch
    n = 1 << scale
    np_pairs = ef * n
    src = torch.empty(np_pairs, dtype=torch.int32, device=f"cuda:{device}")
    dst = torch.empty_like(src)
    H.gen_rmat_device(scale, np_pairs, seed, src, dst, device=device)
    csr = H.coo_to_csr_device(n, src, dst, device=device)
    del src, dst
    return H.hornet_from_device_csr(csr, device=device), csr


def static_config(scale, nV, nE, world):
    """The static-analytics workload's config, identical in both arms."""
    return {"workload": f"static analytics: R-MAT scale {scale}, edge factor 16, "
                        f"a=.57 b=.19 c=.19, BFS TopDown from 64 seeded non-isolated sources",
            "nV": nV, "nE": nE, "sources": 64,
            "parallelism": f"replicas x{world}",
            "l2": "graph data > 126 MB L2; no flush"}


def pick_sources(deg, k, seed):
    rng = np.random.default_rng(seed)
    cand = np.nonzero(deg > 0)[0]
    return rng.choice(cand, size=k, replace=False).astype(np.int32)


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch
    import torch.distributed as dist
    import hornet_b200 as H

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = local
    peak, peak_kind = hbm_peak()
    stream = torch.cuda.Stream(device=dev)

    d = Dist(world, f"cuda:{dev}")
    barrier, max_over_ranks, sum_over_ranks = d.barrier, d.max, d.sum

    if args.workload == "serve":
        result = bench_serve(args, H, dev, rank, world)
        if rank == 0:
            print(json.dumps(result))
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload == "batch":
        result = bench_batch(args, H, dev, stream, rank, world, peak, peak_kind, barrier,
                             max_over_ranks, sum_over_ranks)
        if rank == 0:
            print(json.dumps(result))
        if world > 1:
            dist.destroy_process_group()
        return
    scale = args.scale or (22 if args.workload == "static" else 24)
    h, csr = make_graph_device(H, scale, 16, 1, dev)
    H.lib().hn_graph_set_stream(h.handle, __import__("ctypes").c_void_p(stream.cuda_stream))
    nV, nE = h.nV(), h.nE()
    deg = h.degrees()
    result = {}
    if args.workload == "static":
        result = bench_static(args, H, h, deg, nV, nE, stream, dev, rank, world, peak, peak_kind,
                              barrier, max_over_ranks, sum_over_ranks, scale)
    else:
        result = bench_update(args, H, h, deg, nV, nE, stream, dev, rank, world, peak, peak_kind,
                              barrier, max_over_ranks, sum_over_ranks, scale)
    if rank == 0:
        print(json.dumps(result))
    del h, csr
    if world > 1:
        dist.destroy_process_group()


def event_time(stream, fn):
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3


def measure_l2_gbs(H, h, dev, mib=48, reps=20):
    """L2 read bandwidth on this GPU, measured now: a `mib` MiB device buffer
    (resident in the 126 MB L2 after a first pass) read `reps` times with
    16-byte loads by the library's probe (hn_read_bandwidth, CUDA events)."""
    import ctypes
    import torch
    buf = torch.ones(mib * (1 << 20) // 4, dtype=torch.int32, device=dev)
    gbs = ctypes.c_double(0)
    H._check(H.lib().hn_read_bandwidth(h.handle, ctypes.c_void_p(buf.data_ptr()),
                                       buf.numel() * 4, reps, ctypes.byref(gbs)))
    del buf
    return gbs.value


def roofline_entry(H, prefixes, algo_bytes_fn, peak, peak_kind, report, workload,
                   bound="hbm"):
    """Roofline of a path from the event-profiled pass: achieved = the
    path's algorithmic bytes / the summed device time of its kernels
    (`prefixes`), per launch of the dominant kernel; the dominant kernel and
    its share of the path time are named.  `bound` names the memory level
    whose bandwidth `peak` is."""
    if isinstance(prefixes, str):
        prefixes = [prefixes]
    cand = {k: v for k, v in report.items() if any(k.startswith(p) for p in prefixes)}
    if not cand:
        return None
    name, rec = max(cand.items(), key=lambda kv: kv[1]["ms"])
    path_s = sum(v["ms"] for v in cand.values()) / 1e3
    launches = rec["launches"]
    algo_total = algo_bytes_fn()
    achieved = algo_total / path_s / 1e9
    tr = load_traffic(name)
    return {"kernel": name, "bound": bound, "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": tr[1] if tr else None,
            "algorithmic_bytes_per_launch": round(algo_total / launches),
            "avg_launch_us": round(rec["ms"] * 1e3 / launches, 2), "launches": launches,
            "path_kernels": sorted(cand), "path_us": round(path_s * 1e6, 2),
            "share_of_path": round(rec["ms"] / 1e3 / path_s, 3) if path_s else None,
            "peak_kind": peak_kind, "workload": workload}


def tuning_setup(args, space, nV, nE, max_degree, run, same):
    """Knobs for this workload: tuned now (--autotune, then saved) or loaded
    from a saved entry for this device and workload signature (defaults
    when there is none)."""
    import torch
    from hornet_b200 import autotune as A
    devname = torch.cuda.get_device_name()
    sig = A.signature(space, nV, nE, max_degree)
    path = args.tuned_path or A.DEFAULT_PATH
    if args.autotune:
        best, log = A.tune(run, same, A.SPACES[space], reps=3)
        base, top = log[0]["s"], min(x["s"] for x in log)
        A.save(devname, sig, best, base / top, path=path)
        return {"signature": sig, "knobs": best, "tuned_now": True, "trials": len(log),
                "speedup_vs_default": round(base / top, 3)}
    return {"signature": sig, "knobs": A.apply_saved(devname, sig, path), "tuned_now": False}


def bench_static(args, H, h, deg, nV, nE, stream, dev, rank, world, peak, peak_kind, barrier,
                 max_over_ranks, sum_over_ranks, scale):
    import torch
    K, W = args.steps, args.warmup
    sources = pick_sources(deg, 64, seed=2022 + rank)
    out = torch.empty(nV, dtype=torch.int32, device=f"cuda:{dev}")
    bfs = H.BfsTopDown(h)
    tune8 = torch.empty((8, nV), dtype=torch.int32, device=f"cuda:{dev}")

    def bfs8():
        for j in range(8):
            bfs.set_parameters(int(sources[j]))
            bfs.run(out=tune8[j])
        return tune8.clone()

    tuning = {"bfs": tuning_setup(args, "bfs", nV, nE, h.max_degree(), bfs8, torch.equal)}

    # steps run back to back through the multi-source call (groups of up to
    # 16 sources, distances into a device buffer): one BFS per step, no host
    # synchronisation between steps
    G = 16
    dev_out = torch.empty((G, nV), dtype=torch.int32, device=f"cuda:{dev}")

    def run_steps(i0, n):
        e = v = 0
        for g0 in range(i0, i0 + n, G):
            grp = [int(sources[i % len(sources)]) for i in range(g0, min(i0 + n, g0 + G))]
            _, st = bfs.run_multi(grp, out=dev_out[:len(grp)])
            e += sum(x.edges_scanned for x in st)
            v += sum(x.visited for x in st)
        return e, v

    run_steps(0, W)
    # ---- timed region (device) ----
    clocks = ClockSampler(dev)
    clocks.start()
    launches0 = H.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    scanned = [0]
    visited = [0]

    def timed():
        # NVTX range "hn_bfs" lets a profiler select exactly these launches
        torch.cuda.nvtx.range_push("hn_bfs")
        e, v = run_steps(W, K)
        scanned[0] += e
        visited[0] += v
        torch.cuda.nvtx.range_pop()

    t = event_time(stream, timed)
    barrier()
    launches = H.kernel_launches() - launches0
    clk = clocks.stop()
    t_max = max_over_ranks(t)
    total_edges = sum_over_ranks(scanned[0])
    value = total_edges / t_max / 1e9

    # ---- e2e: public API (BfsTopDown multi-source run), every step's
    # distances copied into pinned host memory, wall clock; calls of up to
    # 16 sources, so the library overlaps each copy with the next BFS ----
    G = min(K, 16)
    host_out = torch.empty((G, nV), dtype=torch.int32, pin_memory=True).numpy()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    e2e_edges = 0
    for i0 in range(0, K, G):
        grp = [int(sources[(W + i) % len(sources)]) for i in range(i0, min(K, i0 + G))]
        _, st = bfs.run_multi(grp, out=host_out[:len(grp)])
        e2e_edges += sum(x.edges_scanned for x in st)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_value = sum_over_ranks(e2e_edges) / t_e2e / 1e9

    # ---- profiled pass for the kernel roofline ----
    H.profile_enable(True)
    prof_edges, prof_vis = run_steps(W, min(K, 16))
    rep = H.profile_report()
    H.profile_enable(False)
    roof = roofline_entry(H, ["k_bfs_level<false>", "k_bfs_wlevel<false>"], lambda: 8 * prof_edges + 20 * prof_vis, peak,
                          peak_kind, rep, f"R-MAT scale {scale} BFS, {min(K, 16)} sources")

    also = {}
    if not args.no_extras and rank == 0:
        also = static_extras(args, H, h, nV, nE, stream, dev, peak, peak_kind, scale, tuning)
        # direction-optimising BFS on the same sources (same distances)
        dev_out = torch.empty((1, nV), dtype=torch.int32, device=f"cuda:{dev}")

        def bfs8_do():
            for j in range(8):
                bfs.run_multi([int(sources[j])], out=tune8[j:j + 1], direction_optimizing=True)
            return tune8.clone()

        tuning["bfs_do"] = tuning_setup(args, "bfs_do", nV, nE, h.max_degree(), bfs8_do,
                                        torch.equal)
        for i in range(W):
            bfs.run_multi([int(sources[i % len(sources)])], out=dev_out, direction_optimizing=True)
        do_edges = [0]

        def timed_do():
            for i in range(K):
                _, st = bfs.run_multi([int(sources[(W + i) % len(sources)])], out=dev_out,
                                      direction_optimizing=True)
                do_edges[0] += st[0].edges_scanned

        t_do = event_time(stream, timed_do)
        if not args.no_c3c5:
            also["c3_updates"] = c3_summary(H, dev, peak, peak_kind)
            also["c5_serve"] = c5_summary(args, H, dev, rank, world)
        also["bfs_direction_optimizing"] = {
            "metric": "BFS GTEPS", "value": round(do_edges[0] / t_do / 1e9, 4), "unit": "GTEPS",
            "ms_per_step": round(t_do * 1e3 / K, 4),
            "note": "same sources and distances as the top-down headline; bottom-up levels "
                    "read fewer edges, GTEPS counts the same edges (sum of degrees reached)"}

    cpu = cpu_baseline_bfs(h, sources, args) if (rank == 0 and world == 1 and not args.no_cpu) else None
    return {
        "metric": "BFS GTEPS", "value": round(value, 4), "unit": "GTEPS", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": round(t_max * 1e3 / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic R-MAT (seeded), no dataset",
        "config": static_config(scale, nV, nE, world),
        "graph500_gteps": round(value / 2, 4),
        "e2e": {"value": round(e2e_value, 4), "unit": "GTEPS", "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 4 * nV + 8},
        "roofline": roof,
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
        "clocks": clk,
        "tuning": tuning,
        "also": also,
    }


def static_extras(args, H, h, nV, nE, stream, dev, peak, peak_kind, scale, tuning):
    import torch
    also = {}
    # triangle counting (orientation + intersection per run)
    tc = H.TriangleCounting2(h)
    tuning["tc"] = tuning_setup(args, "tc", nV, nE, h.max_degree(), tc.run,
                                lambda a, b: a == b)
    for _ in range(2):
        tc.run()
    reps = 3
    clk = ClockSampler(dev)
    clk.start()
    tc_reps = [event_time(stream, tc.run) for _ in range(reps)]
    tc_clocks = clk.stop()
    t = statistics.median(tc_reps)
    H.profile_enable(True)
    tc.run()
    rep = H.profile_report()
    H.profile_enable(False)
    m_plus = nE // 2
    # TC model bytes need sum over oriented edges of d+(u)+d+(v): computed
    # from the exported oriented degrees on the host
    off, adj = h.getCSR()
    d = np.diff(off).astype(np.int64)
    src = np.repeat(np.arange(nV, dtype=np.int64), d)
    keep = (d[src] < d[adj]) | ((d[src] == d[adj]) & (src < adj))
    dplus = np.bincount(src[keep], minlength=nV).astype(np.int64)
    tc_bytes = 8 * m_plus + 4 * int((dplus[src[keep]] + dplus[adj[keep]]).sum())
    # the model counts both lists of every oriented edge; nearly all of it
    # is served by L2 (the oriented graph, 0.29 GB, is read from DRAM about
    # once), so the path is measured against L2 bandwidth, not HBM
    l2_gbs = measure_l2_gbs(H, h, dev)
    troof = roofline_entry(H, ["k_orient", "k_cand", "k_tc_", "k_degrees"], lambda: tc_bytes,
                           round(l2_gbs, 1),
                           "measured now: L2 read bandwidth of a 48 MiB buffer resident in L2 "
                           "(16-byte loads, 20 passes, CUDA events; hn_read_bandwidth)", rep,
                           f"R-MAT scale {scale} TC", bound="l2")
    also["tc"] = {"metric": "TC edges/s", "value": round(m_plus / t, 1), "unit": "edges/s",
                  "triangles": int(tc.countTriangles()), "ms": round(t * 1e3, 3),
                  "roofline": troof, "kernels_ms": {k: round(v["ms"], 3) for k, v in rep.items()},
                  "rep_ms": [round(x * 1e3, 2) for x in tc_reps], "clocks": tc_clocks}
    cpu = not args.no_cpu
    if cpu:
        from oracle import oracle as O
        g_host = O.Csr(off.astype(np.int64), adj)
        sec, e = O.time_tc_sample(g_host, stride=16, first=7)
        also["tc"]["cpu_baseline"] = {
            "value": round(e / sec, 1), "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"restated hostCountTriangles (hornetsnest/test/TriangleTest2.cu:22-69) "
                      f"over every 16th edge of the degree-oriented graph: {e} oriented "
                      f"edges in {sec:.1f} s"}
    # connected components
    cc = H.CC(h)
    lab = torch.empty(nV, dtype=torch.int32, device=f"cuda:{dev}")
    cc.run(out=lab)
    t = event_time(stream, lambda: [cc.run(out=lab) for _ in range(reps)]) / reps
    H.profile_enable(True)
    cc.run(out=lab)
    rep = H.profile_report()
    H.profile_enable(False)
    croof = roofline_entry(H, ["k_cc_"], lambda: 4 * nE + 8 * (nV + 1) + 8 * nV, peak,
                           peak_kind, rep, f"R-MAT scale {scale} CC")
    also["cc"] = {"metric": "CC edges/s", "value": round(nE / t, 1), "unit": "edges/s",
                  "components": cc.n_components, "ms": round(t * 1e3, 3), "roofline": croof}
    if cpu and O.ref_available():
        sec, ncomp = O.ref_time_wcc(g_host)
        also["cc"]["cpu_baseline"] = {
            "value": round(nE / sec, 1), "unit": "edges/s", "cores": 1, "kind": "reference",
            "sample": f"graph::WCC (xlib/src/Graph/WCC.cpp) on the whole graph, {sec:.2f} s, "
                      f"{ncomp} components"}
    # k-truss decomposition (all K, incremental peel): one untimed run (its
    # CUDA graph and buffers), then the median of three runs timed with CUDA
    # events on the graph's stream
    if not args.no_ktruss:
        kt = H.KTruss(h)
        kmax = kt.run()
        reps_k = [event_time(stream, kt.run) for _ in range(3)]
        tk = statistics.median(reps_k)
        also["ktruss"] = {"metric": "k-truss edges/s", "value": round(nE / tk, 1),
                          "unit": "edges/s", "max_k": int(kmax), "ms": round(tk * 1e3, 3),
                          "rep_ms": [round(x * 1e3, 1) for x in reps_k],
                          "note": "all K from 3 to max_k; median of 3 event-timed runs after "
                                  "one untimed run"}
        if cpu:
            s16, d16 = O.gen_rmat(16, 16 << 16, 1)
            g16 = O.build_csr_undirected(1 << 16, s16, d16)
            t0 = time.perf_counter()
            k16, _ = O.ktruss_peel(g16)
            sec = time.perf_counter() - t0
            also["ktruss"]["cpu_baseline"] = {
                "value": round(g16.nE / sec, 1), "unit": "edges/s", "cores": 1, "kind": "port",
                "sample": f"support-peeling truss decomposition (the oracle's; the restated "
                          f"KTruss.cu:90-174 loop needs minutes at scale 14) on the R-MAT scale-16 "
                          f"graph of the same generator: {g16.nE} edges, max K {k16}, "
                          f"{sec:.1f} s"}
    # one 1M-edge uniform insert + erase on the same graph
    rng = np.random.default_rng(77)
    b = 1_000_000
    bs = torch.from_numpy(rng.integers(0, nV, b).astype(np.int32)).cuda(dev)
    bd = torch.from_numpy(rng.integers(0, nV, b).astype(np.int32)).cuda(dev)
    batch = H.BatchUpdate(h, bs, bd)
    ti = event_time(stream, lambda: h.insert(batch, True, True))
    te = event_time(stream, lambda: h.erase(batch, True))
    also["update_1M"] = {"metric": "update edges/s", "insert": round(b / ti, 1),
                         "erase": round(b / te, 1), "unit": "edges/s",
                         "note": "one 1M uniform batch on the scale-22 graph; see --workload update"}
    if cpu:
        sbi, sbe, _, _ = O.time_update(g_host, bs.cpu().numpy(), bd.cpu().numpy())
        also["update_1M"]["cpu_baseline"] = {
            "value": round(2 * b / (sbi + sbe), 1), "unit": "edges/s", "cores": 1,
            "kind": "port", "insert": round(b / sbi, 1), "erase": round(b / sbe, 1),
            "sample": "restated multiset update model (BatchUpdate.i.cuh:485-524; the "
                      "reference has no CPU dynamic graph): the same 1M batch inserted then "
                      f"erased on the same graph, {sbi:.2f} s + {sbe:.2f} s"}
    return also


def c3_batch(H, rng, kind, b, nV, scale, seed):
    """b directed entries of the dynamic-update configuration: b/2 pairs (no
    self loops) with their mirrors, uniform or R-MAT-distributed; the R-MAT
    kind replaces ~5 % of its pairs by copies of other pairs of the batch."""
    half = b // 2
    if kind == "uniform":
        u = rng.integers(0, nV, half).astype(np.int32)
        v = rng.integers(0, nV, half).astype(np.int32)
    else:
        u, v = H.gen_rmat_host(scale, half, seed)
        ndup = half // 20
        to = rng.choice(half, ndup, replace=False)
        frm = rng.integers(0, half, ndup)
        u[to], v[to] = u[frm], v[frm]
    keep = u != v
    u, v = u[keep], v[keep]
    return np.concatenate([u, v]), np.concatenate([v, u])


def c3_summary(H, dev, peak, peak_kind, scale=24):
    """The dynamic-update configuration, compact: R-MAT scale 24 resident;
    batches of 1K..10M directed edges, uniform and R-MAT-distributed with ~5 %
    in-batch duplicates, each inserted (both dedup flags) then erased
    (batch dedup); device time per call from CUDA events on the graph's
    stream."""
    import ctypes
    import torch
    t0 = time.perf_counter()
    stream = torch.cuda.Stream(device=dev)
    h, csr = make_graph_device(H, scale, 16, 1, dev)
    H.lib().hn_graph_set_stream(h.handle, ctypes.c_void_p(stream.cuda_stream))
    nV, nE = h.nV(), h.nE()
    deg0 = np.asarray(h.degrees(), np.int64)
    rng = np.random.default_rng(2024)
    rows, tot_e, tot_t = [], 0, 0.0
    for kind in ("uniform", "rmat"):
        for i, b in enumerate([1_000, 10_000, 100_000, 1_000_000, 10_000_000]):
            bs_h, bd_h = c3_batch(H, rng, kind, b, nV, scale, 77 + i)
            batch = H.BatchUpdate(h, torch.from_numpy(bs_h).cuda(dev),
                                  torch.from_numpy(bd_h).cuda(dev))
            n = len(bs_h)
            ins = [0]
            ti = event_time(stream, lambda: ins.__setitem__(0, h.insert(batch, True, True)))
            te = event_time(stream, lambda: h.erase(batch, True))
            keys = np.unique((bs_h.astype(np.int64) << 32) | bd_h.astype(np.int64))
            uu = np.unique(keys >> 32)
            # model bytes (insert): 8 b + 4 applied + 4 sum of the touched
            # sources' degrees
            ib = 8 * n + 4 * ins[0] + 4 * int(deg0[uu].sum())
            rows.append({"kind": kind, "batch": n, "insert_edges_per_s": round(n / ti, 1),
                         "erase_edges_per_s": round(n / te, 1),
                         "insert_ms": round(ti * 1e3, 4), "erase_ms": round(te * 1e3, 4),
                         "applied": int(ins[0]), "insert_frac": round(ib / ti / 1e9 / peak, 4)})
            tot_e += 2 * n
            tot_t += ti + te
    del h, csr
    return {"metric": "update edges/s", "value": round(tot_e / tot_t, 1), "unit": "edges/s",
            "config": f"R-MAT scale {scale} ef 16 (nV {nV}, nE {nE}); batches 1K..10M, uniform "
                      "and R-MAT with ~5% in-batch duplicates, each inserted then erased",
            "per_batch": rows, "peak_kind": peak_kind,
            "wall_s": round(time.perf_counter() - t0, 1)}


def c5_summary(args, H, dev, rank, world):
    """The serving configuration, compact: scale 25 resident, the seeded
    request mix at saturation (all requests at time 0), the plain
    per-request loops and the continuous-batching loop."""
    import copy
    a = copy.copy(args)
    a.rates = "0,0"   # two seeded streams; throughputs averaged, latencies the worse
    a.requests = args.c5_requests
    a.scale = 0
    t0 = time.perf_counter()
    r = bench_serve(a, H, dev, rank, world)
    rows = r["per_rate"]
    out = {"metric": "served requests/s", "unit": "requests/s",
           "config": r["config"]["workload"], "requests_per_stream": a.requests,
           "streams": len(rows), "results_identical": r["results_identical"]}
    for m in ("per_request", "per_request_do", "batched"):
        out[m] = {"throughput_rps": round(statistics.mean(
                      row[m]["throughput_rps"] for row in rows), 1),
                  "per_stream_rps": [row[m]["throughput_rps"] for row in rows]}
        for q in ("p50", "p99", "p999"):
            out[m][q + "_ms"] = max(row[m]["latency_ms"]["all"][q] for row in rows)
    out["value"] = out["batched"]["throughput_rps"]
    out["throughput_x_vs_per_request"] = round(
        out["batched"]["throughput_rps"] / out["per_request"]["throughput_rps"], 2)
    out["throughput_x_vs_per_request_do"] = round(
        out["batched"]["throughput_rps"] / out["per_request_do"]["throughput_rps"], 2)
    out["wall_s"] = round(time.perf_counter() - t0, 1)
    return out


def cpu_baseline_bfs(h, sources, args):
    """Reference graph::BFS (xlib/src/Graph/BFS.cpp) on the host, 1 thread,
    on a bounded sample of the same sources."""
    from oracle import oracle as O
    off, adj = h.getCSR()
    g = O.Csr(off.astype(np.int64), adj)
    sample = [int(s) for s in sources[: args.cpu_sources]]
    if O.ref_available():
        sec, edges = O.ref_time_bfs(g, sample)
        kind = "reference"
    else:
        t0 = time.perf_counter()
        edges = 0
        for s in sample:
            edges += O.bfs(g, s)[1]
        sec = time.perf_counter() - t0
        kind = "port"
    return {"value": round(edges / sec / 1e9, 5), "unit": "GTEPS", "cores": 1, "kind": kind,
            "sample": f"graph::BFS from {len(sample)} of the 64 sources on the same graph, "
                      f"{sec:.2f} s"}


# ---------------------------------------------------------------------------
# update workload
# ---------------------------------------------------------------------------

def bench_update(args, H, h, deg, nV, nE, stream, dev, rank, world, peak, peak_kind, barrier,
                 max_over_ranks, sum_over_ranks, scale):
    import torch
    K, W = args.steps, args.warmup
    sizes = [int(x) for x in args.batch_sizes.split(",")]
    rng = np.random.default_rng(5 + rank)
    batches = []
    deg0 = np.asarray(deg, np.int64)
    model = []   # algorithmic bytes of (insert, erase) per batch
    for b in sizes:
        bs_h = rng.integers(0, nV, b).astype(np.int32)
        bd_h = rng.integers(0, nV, b).astype(np.int32)
        bs = torch.from_numpy(bs_h).cuda(dev)
        bd = torch.from_numpy(bd_h).cuda(dev)
        batches.append((H.BatchUpdate(h, bs, bd), b, bs, bd))
        # insert: 8b + 4*applied + 4*sum deg_old(u) over distinct sources;
        # the erase that follows sees deg_old + the inserted edges
        keys = np.unique((bs_h.astype(np.int64) << 32) | bd_h.astype(np.int64))
        u = (keys >> 32).astype(np.int64)
        uu, cnt = np.unique(u, return_counts=True)
        model.append((8 * b + 4 * len(keys) + 4 * int(deg0[uu].sum()),
                      8 * b + 4 * len(keys) + 4 * int((deg0[uu] + cnt).sum())))
    applied = [0]

    def step(i):
        bt, b, _, _ = batches[(i // 2) % len(batches)]
        if i % 2 == 0:
            applied[0] += h.insert(bt, True, True)
        else:
            applied[0] += h.erase(bt, True)
        return b

    for i in range(W + (W % 2)):
        step(i)
    start = W + (W % 2)
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = H.kernel_launches()
    barrier()
    edges = [0]

    def timed():
        torch.cuda.nvtx.range_push("hn_update")
        for i in range(K):
            edges[0] += step(start + i)
        torch.cuda.nvtx.range_pop()

    t = event_time(stream, timed)
    launches = H.kernel_launches() - l0
    clk = clocks.stop()
    t_max = max_over_ranks(t)
    value = sum_over_ranks(edges[0]) / t_max
    # path roofline: model bytes of the timed steps over their device time
    # (graph de-duplication makes insert then erase of a batch a round trip,
    # so every step sees the initial degrees, plus the batch for erases)
    model_bytes = sum(model[((start + i) // 2) % len(model)][(start + i) % 2] for i in range(K))
    achieved = model_bytes / t / 1e9
    per_size = []
    for j, b in enumerate(sizes):
        ti = event_time(stream, lambda: step(2 * j))
        te = event_time(stream, lambda: step(2 * j + 1))
        # stage breakdown (kernels, CUB calls, the host round trip) of one
        # more insert and erase of the same batch
        stages = {}
        for which in (0, 1):
            H.profile_enable(True)
            step(2 * j + which)
            r = H.profile_report()
            H.profile_enable(False)
            stages["insert" if which == 0 else "erase"] = {
                k: round(v["ms"], 4) for k, v in sorted(r.items(), key=lambda kv: -kv[1]["ms"])}
        # insert + incremental triangle count (then the erase restores)
        bt_j = batches[j][0]
        newtri = [0]

        def ins_tc():
            newtri[0] = h.insert_count_triangles(bt_j)[1]

        tt = event_time(stream, ins_tc)
        step(2 * j + 1)
        per_size.append({"batch": b, "insert_edges_per_s": round(b / ti, 1),
                         "erase_edges_per_s": round(b / te, 1),
                         "insert_ms": round(ti * 1e3, 4), "erase_ms": round(te * 1e3, 4),
                         "insert_with_new_triangles_ms": round(tt * 1e3, 4),
                         "new_triangles": int(newtri[0]),
                         "insert_frac": round(model[j][0] / ti / 1e9 / peak, 4),
                         "erase_frac": round(model[j][1] / te / 1e9 / peak, 4),
                         "stages_ms": stages})
    roof = {"kernel": "update path (sort, mark, scan, plan, assign, scatter, commit)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None,
            "algorithmic_bytes_per_launch": round(model_bytes / K),
            "peak_kind": peak_kind, "per_batch_size": per_size,
            "note": "device time of whole insert/erase calls (includes the one host "
                    "synchronisation per batch)"}
    # e2e: pinned host batch arrays copied in every step
    host = [(bs.cpu().pin_memory().numpy(), bd.cpu().pin_memory().numpy(), b)
            for (_, b, bs, bd) in batches]
    # the batch's device buffers sized once for the largest batch, outside
    # the timed region (a growing batch would reallocate inside it)
    big = max(range(len(host)), key=lambda j: host[j][2])
    bt = H.BatchUpdate(h, host[big][0], host[big][1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_edges = 0
    hb = 0
    for i in range(K):
        s, d, b = host[((start + i) // 2) % len(host)]
        bt.reset(s, d)
        hb += 8 * b
        if (start + i) % 2 == 0:
            h.insert(bt, True, True)
        else:
            h.erase(bt, True)
        e_edges += b
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    H.profile_enable(True)
    step(start)
    step(start + 1)
    rep = H.profile_report()
    H.profile_enable(False)
    return {
        "metric": "update edges/s", "value": round(value, 1), "unit": "edges/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": round(t_max * 1e3 / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic R-MAT (seeded) + uniform batches",
        "config": {"workload": f"dynamic batch updates: R-MAT scale {scale}, ef 16; uniform "
                               f"batches {args.batch_sizes} alternately inserted/erased",
                   "nV": nV, "nE": nE, "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(sum_over_ranks(e_edges) / t_e2e, 1), "unit": "edges/s",
                "h2d_bytes_per_step": hb // K, "d2h_bytes_per_step": 8},
        "roofline": roof, "kernels_ms": {k: round(v["ms"], 4) for k, v in rep.items()},
        "cpu_baseline": None, "gpu_launches": int(launches), "clocks": clk,
    }


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# batch workload: many small graphs of uneven size
# ---------------------------------------------------------------------------

def bench_batch(args, H, dev, stream, rank, world, peak, peak_kind, barrier, max_over_ranks,
                sum_over_ranks):
    """Batched form (one hn_bfs_batch over all graphs x 8 sources + one TC
    over the union) against the plain per-request loop (one BfsTopDown::run
    per graph and source, one TriangleCounting2 run per graph, each on the
    graph's own Hornet) on a seeded sample of the same graphs."""
    import ctypes
    import torch
    from hornet_b200.batching import GraphBatch, synthetic_union
    K, W = max(1, min(args.steps, 8)), max(3, min(args.warmup, 3))
    t0 = time.perf_counter()
    h, csr, sizes, bases, kinds = synthetic_union(args.graphs, seed=4096 + rank, device=dev)
    H.lib().hn_graph_set_stream(h.handle, ctypes.c_void_p(stream.cuda_stream))
    build_s = time.perf_counter() - t0
    nV, nE = h.nV(), h.nE()
    gb = GraphBatch(h, bases, sizes)
    deg = h.degrees()
    rng = np.random.default_rng(77 + rank)
    S = 8
    local = np.zeros((len(sizes), S), np.int64)
    for i in range(len(sizes)):
        cand = np.nonzero(deg[bases[i]:bases[i] + sizes[i]] > 0)[0]
        local[i] = rng.choice(cand, size=S, replace=len(cand) < S)
    out = torch.empty((S, nV), dtype=torch.int32, device=f"cuda:{dev}")
    pv = torch.empty(nV, dtype=torch.int64, device=f"cuda:{dev}")

    def bfs_all():
        gb.bfs(local, out)
        return out.clone()

    tuning = {"msbfs": tuning_setup(args, "msbfs", nV, nE, h.max_degree(), bfs_all, torch.equal),
              "tc": tuning_setup(args, "tc", nV, nE, h.max_degree(),
                                 lambda: gb.triangles(pv)[0].clone(), torch.equal)}

    def step():
        st = gb.bfs(local, out)
        tri, _ = gb.triangles(pv)
        return st, tri

    for _ in range(W):
        st, tri = step()
    barrier()
    t = event_time(stream, lambda: [step() for _ in range(K)]) / K
    t = max_over_ranks(t)
    torch.cuda.nvtx.range_push("hn_msbfs")
    tb = event_time(stream, lambda: gb.bfs(local, out))
    torch.cuda.nvtx.range_pop()
    edges = sum(x.edges_scanned for x in st)
    tri_host = tri.cpu().numpy()

    # per-request loop on a seeded sample of the same graphs
    off_d = torch.empty(nV + 1, dtype=torch.int32, device=f"cuda:{dev}")
    adj_d = torch.empty(nE, dtype=torch.int32, device=f"cuda:{dev}")
    H._check(H.lib().hn_graph_export_csr(h.handle, ctypes.c_void_p(off_d.data_ptr()),
                                         ctypes.c_void_p(adj_d.data_ptr()), H.HN_MEM_DEVICE))
    off_h = off_d.cpu().numpy().astype(np.int64)
    sample = np.sort(np.random.default_rng(5).choice(len(sizes), args.sample_graphs,
                                                     replace=False))
    per = []
    for i in sample:
        b, n = int(bases[i]), int(sizes[i])
        o = (off_d[b:b + n + 1] - int(off_h[b])).contiguous()
        a = (adj_d[int(off_h[b]):int(off_h[b + n])] - b).contiguous()
        hi = H.hornet_from_device_arrays(n, int(off_h[b + n] - off_h[b]), o, a, device=dev)
        H.lib().hn_graph_set_stream(hi.handle, ctypes.c_void_p(stream.cuda_stream))
        per.append((i, hi, torch.empty(n, dtype=torch.int32, device=f"cuda:{dev}"),
                    H.BfsTopDown(hi), H.TriangleCounting2(hi)))
    del o, a

    def per_request():
        res = []
        for i, hi, d_i, bfs, tc in per:
            for j in range(S):
                bfs.set_parameters(int(local[i, j]))
                bfs.run(out=d_i)
            res.append(tc.run())
        return res

    # the plain loop runs with the default knobs (those tuned for the union
    # are not meant for graphs of a few thousand vertices)
    H.tune_reset()
    per_request()
    tp = event_time(stream, per_request)
    # the two forms agree on the sample (distances and triangle counts)
    agree = True
    for i, hi, d_i, bfs, tc in per[:16]:
        b, n = int(bases[i]), int(sizes[i])
        for j in range(S):
            bfs.set_parameters(int(local[i, j]))
            bfs.run(out=d_i)
            agree &= bool(torch.equal(d_i, out[j, b:b + n]))
        agree &= tc.run() == int(tri_host[i])
    agree = bool(max_over_ranks(0.0 if agree else 1.0) == 0.0)
    ng = len(sizes)
    value = sum_over_ranks(ng / t)
    per_rate = len(sample) / tp
    res = {"metric": "C4 graphs/s", "value": round(value, 1), "unit": "graphs/s",
           "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": round(t * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic ER + R-MAT (seeded), no dataset",
           "config": {"workload": f"batch: {ng} graphs, n ~ LogUniform[1024, 65536], half ER "
                                  "mean degree 8, half R-MAT ef 16; 8 BFS sources per graph "
                                  "+ triangle count per graph",
                      "nV_total": nV, "nE_total": nE, "bfs_per_step": ng * S,
                      "parallelism": f"replicas x{world}", "l2": "union > 126 MB L2; no flush"},
           "batched": {"bfs_ms": round(tb * 1e3, 3), "bfs_gteps": round(edges / tb / 1e9, 3),
                       "bfs_edges_scanned": int(edges), "slots": S},
           "per_request_loop": {"graphs_per_s": round(per_rate, 2),
                                "sample_graphs": int(len(sample)),
                                "ms_per_graph": round(tp / len(sample) * 1e3, 3)},
           "speedup_vs_per_request": round((ng / t) / per_rate, 2),
           "results_identical_on_sample": agree, "build_s": round(build_s, 2),
           "tuning": tuning}
    del per
    return res


# ---------------------------------------------------------------------------
# serve workload: a request stream on a resident scale-25 graph
# ---------------------------------------------------------------------------

def bench_serve(args, H, dev, rank, world):
    """The batched serving loop against the plain per-request loop on the
    same seeded request stream (Poisson arrivals at each rate; rate 0 = all
    requests at time 0, the saturation throughput).  60 % update batches
    (LogNormal median 10K pairs, sigma 1.5, clipped to [100, 2M], half
    insert / half erase, both directions stored), 30 % BFS queries (distances
    to 16 targets + vertices reached), 10 % local triangle counts of 1K-vertex
    seed sets.  Each run starts from a fresh copy of the same graph; the two
    loops' per-request results are compared."""
    import ctypes
    import gc
    import torch
    from hornet_b200 import serving as S
    scale = args.scale or 25
    t0 = time.perf_counter()
    h0, csr = make_graph_device(H, scale, 16, 1, dev)
    nV, nE = h0.nV(), h0.nE()
    deg = h0.degrees()
    off_d = torch.empty(nV + 1, dtype=torch.int32, device=f"cuda:{dev}")
    adj_d = torch.empty(nE, dtype=torch.int32, device=f"cuda:{dev}")
    H._check(H.lib().hn_graph_export_csr(h0.handle, ctypes.c_void_p(off_d.data_ptr()),
                                         ctypes.c_void_p(adj_d.data_ptr()), H.HN_MEM_DEVICE))
    del h0
    gc.collect()
    off64 = off_d.long()

    def erase_pool(rng, k):
        idx = torch.from_numpy(rng.integers(0, nE, k)).to(off64.device)
        u = torch.searchsorted(off64, idx, right=True) - 1
        return u.int().cpu().numpy(), adj_d[idx].cpu().numpy()

    def insert_pairs(rng, k):
        return H.gen_rmat_host(scale, k, int(rng.integers(1, 2**62)))

    build_s = time.perf_counter() - t0
    rates = [float(x) for x in args.rates.split(",")]
    table = []
    identical = True
    for ri, rate in enumerate(rates):
        reqs = S.make_requests(args.requests, rate, nV, deg, erase_pool, seed=1000 + ri,
                               insert_pairs=insert_pairs)
        warm = [r for r in S.make_requests(80, 0.0, nV, deg, erase_pool, seed=7,
                                           insert_pairs=insert_pairs)
                if r.kind in S.QUERY_KINDS]
        row = {"rate_rps": rate if rate > 0 else "saturation"}
        res = {}
        for mode in args.serve_modes.split(","):
            h = H.hornet_from_device_arrays(nV, nE, off_d, adj_d, device=dev)
            srv = S.Server(h, batched=mode == "batched",
                           single_bfs="do" if mode != "per_request" else "td",
                           msbfs_min=args.msbfs_min, workers=args.serve_workers)
            srv.run(warm)                       # CUDA graphs built, read-only
            srv.calls, srv.split_for_memory, srv.max_inflight = 0, 0, 0
            srv.groups = {k: 0 for k in srv.groups}
            srv.service_s = {k: 0.0 for k in srv.service_s}
            rep = srv.run(reqs)
            res[mode] = rep.results
            row[mode] = rep.summary()
            row[mode]["workers"] = rep.workers
            row[mode]["max_queries_in_flight"] = rep.max_inflight
            row[mode]["update_calls_ms"] = rep.update_calls_ms
            row[mode]["update_parts_ms"] = rep.update_parts_ms
            srv.close()
            del srv, h
            gc.collect()
        modes = list(res)
        same = all(S.same_results(res[modes[0]], res[m]) for m in modes[1:])
        identical &= same
        row["results_identical"] = same
        bt = row["batched"]
        if "per_request" in row:
            row["throughput_x"] = round(bt["throughput_rps"] / row["per_request"]["throughput_rps"], 2)
        if "per_request_do" in row:
            row["throughput_x_vs_per_request_do"] = round(
                bt["throughput_rps"] / row["per_request_do"]["throughput_rps"], 2)
        row["p99_ms"] = {m: row[m]["latency_ms"]["all"]["p99"] for m in modes}
        row["p999_ms"] = {m: row[m]["latency_ms"]["all"]["p999"] for m in modes}
        table.append(row)
    sat = [r for r in table if r["rate_rps"] == "saturation"]
    head = sat[0] if sat else table[-1]
    return {"metric": "served requests/s", "value": head["batched"]["throughput_rps"],
            "unit": "requests/s", "n_gpus": world, "steps": args.requests, "warmup": 1,
            "ms_per_step": round(1e3 / head["batched"]["throughput_rps"], 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic R-MAT (seeded) + seeded request stream, no dataset",
            "config": {"workload": f"serve: R-MAT scale {scale} ef 16 resident; 60% updates "
                                   "(LogNormal median 10K, sigma 1.5, [100, 2M]; half insert, "
                                   "half erase), 30% BFS (16 targets), 10% local TC (1K seeds)",
                       "nV": nV, "nE": nE, "requests_per_rate": args.requests,
                       "parallelism": f"replicas x{world}", "l2": "graph > 126 MB L2; no flush"},
            "per_rate": table, "results_identical": identical,
            "saturation_throughput_x": head.get("throughput_x"), "build_s": round(build_s, 2)}


def run_reference(args):
    """The reference's own CPU BFS (graph::BFS, xlib/src/Graph/BFS.cpp,
    compiled from the reference sources into oracle/_ref/ref_driver) on the
    same graph and sources.  The graph comes from the oracle's restatement
    of the input generator, so this arm loads nothing of hornet_b200."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    scale = args.scale or 22
    n = 1 << scale
    s, d = O.gen_rmat(scale, 16 * n, 1)
    g = O.build_csr_undirected(n, s, d)
    del s, d
    deg = np.diff(g.off)
    sources = pick_sources(deg, 64, seed=2022)
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_driver (reference graph::BFS) was not built"}))
        return
    K, W = args.steps, args.warmup
    O.ref_time_bfs(g, [int(x) for x in sources[:W]])
    per_step = 1
    # the reference BFS is single-threaded: the host's cores run the steps'
    # sources concurrently, one process per core (bounded)
    cores = min(os.cpu_count() or 1, 32)
    sec, edges, used = O.ref_time_bfs_parallel(
        g, [int(sources[i % 64]) for i in range(W, W + K * per_step)], cores)
    value = edges / sec / 1e9
    print(json.dumps({
        "impl": "reference", "metric": "BFS GTEPS", "value": round(value, 5), "unit": "GTEPS",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": round(sec * 1e3 / K, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic R-MAT (seeded), no dataset",
        "config": static_config(scale, g.nV, g.nE, world),
        "cpu_baseline": {"value": round(value, 5), "unit": "GTEPS", "cores": used,
                         "kind": "reference",
                         "sample": f"graph::BFS (xlib/src/Graph/BFS.cpp), {per_step} source per "
                                   f"step, {K} steps over {used} concurrent processes; time = "
                                   f"the slowest process's BFS phase"},
        "e2e": {"value": round(value, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="static", choices=["static", "update", "batch", "serve"])
    ap.add_argument("--rates", default="250,500,1000,2000,0")
    ap.add_argument("--requests", type=int, default=1000)
    ap.add_argument("--msbfs-min", type=int, default=16,
                    help="serve: smallest run of BFS queries answered by one batched traversal")
    ap.add_argument("--serve-modes", default="per_request,per_request_do,batched",
                    help="serve: the loops to run, in this order")
    ap.add_argument("--serve-workers", type=int, default=4,
                    help="serve: query views (worker threads) of the batched loop")
    ap.add_argument("--graphs", type=int, default=4096)
    ap.add_argument("--sample-graphs", type=int, default=128)
    ap.add_argument("--scale", type=int, default=0)
    ap.add_argument("--batch-sizes", default="1000,10000,100000,1000000,10000000")
    ap.add_argument("--cpu-sources", type=int, default=8)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ktruss", action="store_true")
    ap.add_argument("--no-c3c5", action="store_true",
                    help="static: skip the compact dynamic-update and serving summaries")
    ap.add_argument("--c5-requests", type=int, default=600)
    ap.add_argument("--autotune", action="store_true",
                    help="tune the knobs of each workload first and save them")
    ap.add_argument("--knob", action="append", default=[],
                    help="name=value tuning knob set before the run (repeatable)")
    ap.add_argument("--tuned-path", default="",
                    help="knob file to load / save (default: the package's tuned.json)")
    args = ap.parse_args()
    if args.knob and args.impl != "reference":
        import hornet_b200 as H
        for kv in args.knob:
            k, v = kv.split("=")
            H.tune_set(k, int(v))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
