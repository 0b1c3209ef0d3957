"""TEST INFRASTRUCTURE — times the reference's own GPU programs on this GPU.

    python oracle/run_ref_gpu.py [out.json] [--scale 22]

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
  * CC (CC.cu) on the symmetric graph: its time.

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

BIN = {k: os.path.join(HERE, "_ref", f"ref_gpu_{k}") for k in ("bfs", "triangle2", "cc")}
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


def main():
    out_path = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else \
        "ref_gpu.json"
    scale = 22
    if "--scale" in sys.argv:
        scale = int(sys.argv[sys.argv.index("--scale") + 1])
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else \
        ["bfs", "tc", "cc"]
    for k, b in BIN.items():
        if not os.path.exists(b):
            raise SystemExit(f"{b} missing: make -C oracle ref_gpu")
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
