"""TEST INFRASTRUCTURE — times the reference's own GPU programs on this GPU.

    python oracle/run_ref_gpu.py [out.json] [--scale 22] [--only bfs,tc,cc]
    python oracle/run_ref_gpu.py [out.json] --only update [--scale 24]

The programs are the reference's hornetsnest test drivers (BFSTest.cu,
TriangleTest2.cu, CCTest.cu) with their algorithm sources, built as
compute_70 PTX by `make -C oracle ref_gpu` (oracle/_ref/ref_gpu_*); the
driver JIT-compiles the PTX for the GPU at hand.  Each is run once per
input, under a time limit, on the benchmark's graph (R-MAT scale 22, edge
factor 16, seed 1, from the oracle's restatement of the input generator),
written in the reference's GraphStd .bin format:

  * BFS (TopDown.cu) from the first 8 of the benchmark's 64 sources, on the
    symmetric graph; GTEPS = edges scanned (counted by graph::BFS on the
    CPU) / the program's own Timer<DEVICE> time of BfsTopDown::run;
  * TriangleCounting2 (triangle2.cu, work factor 1) on the degree-oriented
    graph (GraphStd's DIRECTED_BY_DEGREE orientation, which the .bin reader
    does not apply itself): its printed triangle total and its time.  Its
    vertex 0 (the largest hub, which keeps no out-edge) swaps ids with the
    first vertex of out-degree 1: the reference's HornetInit sizes the first
    block array of its smallest bin by the first such vertex's degree and
    asserts on degree 0 (ceil_log2(0): hornet/include/Core/MemoryManager/
    BlockArray/BlockArray.i.cuh:150-153, HornetInitialize.i.cuh:126-129).
    A relabelled acyclic orientation counts every triangle once all the
    same, so the total is the graph's;
  * CC (CC.cu) on the symmetric graph: its time;
  * update (`--only update`, scale 24 by default): gpu::Hornet::insert and
    erase through this repository's driver oracle/ref_gpu_update.cu, on the
    dynamic-update configuration's graph (R-MAT scale 24, edge factor 16,
    seed 1, built with the library's device generator, which the CPU tests
    pin bit-identical to the oracle's) and its ten batches (uniform and
    R-MAT, 1K..10M directed entries, as bench.py's c3_batch makes them),
    each inserted (both de-duplications) then erased (batch
    de-duplication) in order on one graph.  The same sequence then runs
    through this library, and the edge count after every call is compared:
    equal counts after all twenty calls are a full-size check of the
    update semantics against the reference's own GPU code.

The .bin files are written by this repository's writer, which the CPU tests
pin byte-identical to the reference's own writeBinary output.  Results
(times as the programs print them, plus the full program output) go to a
JSON file.
"""
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this directory comes first on the path; the package
# imports need the repository root instead
sys.path[:] = [ROOT] + [x for x in sys.path if os.path.abspath(x or ".") != HERE]

from oracle import oracle as O  # noqa: E402

BIN = {k: os.path.join(HERE, "_ref", f"ref_gpu_{k}")
       for k in ("bfs", "triangle2", "cc", "update")}
C3_BATCHES = [1_000, 10_000, 100_000, 1_000_000, 10_000_000]
ANSI = re.compile(r"\x1b\[[0-9;]*m")


def timer_ms(out: str, label: str):
    """The reference Timer's printout '<label>  <value>ms' -> value."""
    m = re.search(re.escape(label) + r"\s+([0-9.]+)\s*ms", ANSI.sub("", out))
    return float(m.group(1)) if m else None


def run(cmd, limit):
    t0 = time.perf_counter()
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=limit)
        return {"rc": p.returncode, "wall_s": round(time.perf_counter() - t0, 2),
                "out": ANSI.sub("", p.stdout)[-3000:], "err": p.stderr[-2000:]}
    except subprocess.TimeoutExpired:
        return {"rc": None, "timeout_s": limit, "wall_s": round(time.perf_counter() - t0, 2)}


def relabel_first_vertex(g: "O.Csr") -> "O.Csr":
    """g with vertex 0 and the first vertex of out-degree 1 swapping ids
    (lists re-sorted)."""
    deg = np.diff(g.off)
    x = int(np.nonzero(deg == 1)[0][0])
    perm = np.arange(g.nV, dtype=np.int64)
    perm[0], perm[x] = x, 0
    src = perm[np.repeat(np.arange(g.nV, dtype=np.int64), deg)]
    keys = np.sort((src << 32) | perm[g.adj.astype(np.int64)])
    off = np.zeros(g.nV + 1, np.int64)
    np.add.at(off, (keys >> 32) + 1, 1)
    return O.Csr(np.cumsum(off), (keys & 0xFFFFFFFF).astype(np.int32))


def json_lines(text):
    out = []
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("{"):
            try:
                out.append(json.loads(line))
            except ValueError:
                pass
    return out


def run_update(scale, out_path):
    """The reference's GPU insert / erase and this library's on the same
    graph and batch sequence; edge counts compared after every call."""
    import ctypes
    import types
    import torch
    import hornet_b200 as H
    import bench
    h0, csr = bench.make_graph_device(H, scale, 16, 1, 0)
    nV_full = h0.nV()
    off_full, adj_full = h0.getCSR()
    del h0, csr
    # The reference's HornetInit cannot start a block array with an isolated
    # vertex: it sizes the array as 1 << ceil_log2(degree), and ceil_log2(0)
    # asserts (hornet/include/Core/HornetInitialize/HornetInitialize.i.cuh:
    # 126-129 -> xlib/include/Host/impl/Numeric.i.hpp:432), which the
    # scale-24 graph's isolated vertices reach.  Both arms therefore run on
    # the graph without its isolated vertices, ids compacted in order (lists
    # stay sorted, the edges are the same); the batches are drawn on the
    # compacted ids (R-MAT pairs with an isolated endpoint are dropped).
    deg = np.diff(np.asarray(off_full, np.int64))
    keep_v = deg > 0
    newid = np.cumsum(keep_v) - 1
    off = np.concatenate([[0], np.cumsum(deg[keep_v])]).astype(np.int64)
    adj = newid[np.asarray(adj_full)].astype(np.int32)
    del off_full, adj_full
    nV = int(keep_v.sum())
    rng = np.random.default_rng(2024)
    gen = types.SimpleNamespace(gen_rmat_host=O.gen_rmat)
    batches = []
    for kind in ("uniform", "rmat"):
        for i, b in enumerate(C3_BATCHES):
            if kind == "uniform":
                bs, bd = bench.c3_batch(gen, rng, kind, b, nV, scale, 77 + i)
            else:
                bs, bd = bench.c3_batch(gen, rng, kind, b, nV_full, scale, 77 + i)
                ok = keep_v[bs] & keep_v[bd]
                bs, bd = newid[bs[ok]].astype(np.int32), newid[bd[ok]].astype(np.int32)
            batches.append((kind, bs, bd))
    h = H.Hornet(H.HornetInit(nV, len(adj), off, adj, sorted_adjacency=True))
    nE0 = h.nE()
    res = {"graph": {"scale": scale, "nV_with_isolated": nV_full, "nV": nV, "nE": nE0,
                     "note": "isolated vertices removed (ids compacted) for the reference's "
                             "HornetInit"}}
    with tempfile.TemporaryDirectory() as tmp:
        gb = os.path.join(tmp, "g.bin")
        H.write_bin(gb, off.astype(np.int32), adj)
        files = []
        for j, (kind, bs, bd) in enumerate(batches):
            f = os.path.join(tmp, f"b{j}.bin")
            with open(f, "wb") as fh:
                fh.write(np.int64(len(bs)).tobytes())
                fh.write(bs.astype("<i4").tobytes())
                fh.write(bd.astype("<i4").tobytes())
            files.append(f)
        r = run([BIN["update"], gb] + files, 1800)
        lines = json_lines(r.get("out", ""))
        res["reference_run"] = {k: v for k, v in r.items() if k != "out"}
        res["reference_out"] = r.get("out", "")[-3000:]
    ref_rows = [x for x in lines if "batch" in x]
    # this library, same sequence, timed the same way (CUDA events around
    # each call, the graph's own stream)
    stream = torch.cuda.Stream()
    H.lib().hn_graph_set_stream(h.handle, ctypes.c_void_p(stream.cuda_stream))
    ours, ours_ms = [], []
    for kind, bs, bd in batches:
        b = H.BatchUpdate(h, torch.from_numpy(bs).cuda(), torch.from_numpy(bd).cuda())
        torch.cuda.synchronize()
        ti = bench.event_time(stream, lambda: h.insert(b, True, True))
        ne_i = h.nE()
        te = bench.event_time(stream, lambda: h.erase(b, True))
        ours.append((ne_i, h.nE()))
        ours_ms.append((round(ti * 1e3, 4), round(te * 1e3, 4)))
    rows = []
    for j, (kind, bs, bd) in enumerate(batches):
        row = {"kind": kind, "batch": len(bs), "ours_nE": list(ours[j]),
               "ours_insert_ms": ours_ms[j][0], "ours_erase_ms": ours_ms[j][1]}
        if j < len(ref_rows):
            x = ref_rows[j]
            row.update({"ref_insert_ms": x["insert_ms"], "ref_erase_ms": x["erase_ms"],
                        "ref_nE": [x["nE_after_insert"], x["nE_after_erase"]]})
            row["nE_equal"] = row["ref_nE"] == row["ours_nE"]
        rows.append(row)
    res["update"] = rows
    res["all_nE_equal"] = len(ref_rows) == len(batches) and all(r.get("nE_equal") for r in rows)
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({"rows": len(ref_rows), "all_nE_equal": res["all_nE_equal"],
                      "ref_ms": [(r.get("ref_insert_ms"), r.get("ref_erase_ms")) for r in rows]}))


def main():
    out_path = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else \
        "ref_gpu.json"
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else \
        ["bfs", "tc", "cc"]
    scale = 24 if only == ["update"] else 22
    if "--scale" in sys.argv:
        scale = int(sys.argv[sys.argv.index("--scale") + 1])
    need = {"bfs": "bfs", "tc": "triangle2", "cc": "cc", "update": "update"}
    for k in only:
        if not os.path.exists(BIN[need[k]]):
            raise SystemExit(f"{BIN[need[k]]} missing: make -C oracle ref_gpu")
    if only == ["update"]:
        run_update(scale, out_path)
        return
    import hornet_b200 as H   # only its .bin writer (pinned to the reference's bytes)
    s, d = O.gen_rmat(scale, 16 << scale, 1)
    g = O.build_csr_undirected(1 << scale, s, d)
    del s, d
    og = relabel_first_vertex(O.orient_by_degree(g))
    rng = np.random.default_rng(2022)
    cand = np.nonzero(np.diff(g.off) > 0)[0]
    sources = [int(x) for x in rng.choice(cand, size=64, replace=False)[:8]]
    res = {"graph": {"scale": scale, "nV": g.nV, "nE": g.nE, "oriented_nE": og.nE},
           "sources": sources}
    with tempfile.TemporaryDirectory() as tmp:
        gb = os.path.join(tmp, "g.bin")
        ob = os.path.join(tmp, "g_oriented.bin")
        H.write_bin(gb, g.off32(), g.adj)
        H.write_bin(ob, og.off32(), og.adj)
        bfs = []
        for src in (sources if "bfs" in only else []):
            r = run([BIN["bfs"], gb, str(src)], 600)
            r["source"] = src
            r["ms"] = timer_ms(r.get("out", ""), "TopDown")
            _, edges = O.ref_time_bfs(g, [src])
            r["edges_scanned"] = edges
            if r["ms"]:
                r["gteps"] = round(edges / (r["ms"] * 1e-3) / 1e9, 4)
            bfs.append(r)
            if r["rc"] is None:
                break   # a program that ran out of time is not run again
        res["bfs"] = bfs
        if "tc" in only:
            r = run([BIN["triangle2"], ob], 900)
            m = re.search(r"Device triangles:\s*([0-9]+)", r.get("out", ""))
            r["triangles"] = int(m.group(1)) if m else None
            r["ms"] = timer_ms(r.get("out", ""), "Computation time:")
            res["tc"] = r
        if "cc" in only:
            r = run([BIN["cc"], gb], 600)
            r["ms"] = timer_ms(r.get("out", ""), "CC")
            res["cc"] = r
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    ok = [b["gteps"] for b in res["bfs"] if b.get("gteps")]
    print(json.dumps({"bfs_gteps": ok,
                      "tc_triangles": res.get("tc", {}).get("triangles"),
                      "tc_ms": res.get("tc", {}).get("ms"), "cc_ms": res.get("cc", {}).get("ms")}))


if __name__ == "__main__":
    main()
