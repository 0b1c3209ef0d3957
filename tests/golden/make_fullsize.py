"""Full-size pins for the benchmark graphs -> tests/golden/fullsize.json.

    python tests/golden/make_fullsize.py [part ...]     (parts: c2, ktruss18, ktruss22)

The graphs are the repository's seeded R-MAT inputs (a=.57 b=.19 c=.19, edge
factor 16, seed 1, symmetrised, self loops and duplicates removed), generated
on the CPU by the oracle's restatement of the input generator.  The pinned
results come from the reference's own host code where it has some, else
from the C oracle:

  c2        scale 22: nV, nE, the adjacency checksum; BFS distances from the
            first 8 of the 64 seeded sources by graph::BFS
            (xlib/src/Graph/BFS.cpp, oracle/_ref/ref_driver); CC labels by
            graph::WCC (xlib/src/Graph/WCC.cpp) relabelled to the minimum
            vertex id; the triangle total by the restated hostCountTriangles
            (hornetsnest/test/TriangleTest2.cu:22-69) on the degree
            orientation (xlib/src/Graph/GraphStd.cpp:247-268).
  ktruss18  scale 18: edge truss numbers by both CPU k-truss computations
            (the restated KTruss.cu:90-174 loop is too slow here, so the
            support-peeling oracle, which the CPU tests check against it).
  ktruss22  scale 22: the same by support peeling (about an hour).

Arrays are pinned by SHA-256 of their little-endian bytes plus summary
counts, so the fixture stays small.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "fullsize.json")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rmat(scale: int, ef: int = 16, seed: int = 1) -> O.Csr:
    s, d = O.gen_rmat(scale, ef << scale, seed)
    return O.build_csr_undirected(1 << scale, s, d)


def sources(g: O.Csr, k: int = 64, seed: int = 2022) -> np.ndarray:
    """The benchmark's sources: k seeded distinct non-isolated vertices."""
    rng = np.random.default_rng(seed)
    cand = np.nonzero(np.diff(g.off) > 0)[0]
    return rng.choice(cand, size=k, replace=False).astype(np.int32)


def load() -> dict:
    return json.load(open(OUT)) if os.path.exists(OUT) else {}


def save(db: dict) -> None:
    tmp = OUT + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, OUT)


def ktruss_entry(g: O.Csr, scale: int) -> dict:
    t0 = time.time()
    kmax, et = O.ktruss_peel(g)
    ks, cnt = np.unique(et, return_counts=True)
    return {"scale": scale, "nE": g.nE, "max_k": kmax,
            "edges_per_truss": {str(int(k)): int(c) for k, c in zip(ks, cnt)},
            "edge_truss_sha256": sha(et.astype("<i4")), "by": "hno_ktruss_peel",
            "cpu_s": round(time.time() - t0, 1)}


def part_c2(db: dict) -> None:
    assert O.ref_available(), "build oracle/_ref first: make -C oracle ref"
    g = rmat(22)
    e = {"scale": 22, "edge_factor": 16, "seed": 1, "nV": g.nV, "nE": g.nE,
         "adjacency_hash": str(O.adjacency_hash(g))}
    src = sources(g)[:8]
    dist = O.ref_bfs(g, src)
    e["bfs"] = {"sources": [int(x) for x in src],
                "sha256": [sha(d.astype("<i4")) for d in dist],
                "reached": [int((d != O.INF).sum()) for d in dist],
                "levels": [int(d[d != O.INF].max()) + 1 for d in dist],
                "by": "graph::BFS (oracle/_ref)"}
    lab = O.canon_labels_fast(O.ref_wcc(g))
    e["cc"] = {"components": int(len(np.unique(lab))), "sha256_min_id": sha(lab.astype("<i4")),
               "by": "graph::WCC (oracle/_ref), relabelled to min id"}
    e["tc"] = {"triangles": O.tc(g), "by": "hno_tc_oriented (TriangleTest2.cu:22-69)"}
    db["rmat22"] = {**db.get("rmat22", {}), **e}


def main(parts) -> None:
    db = load()
    for p in parts:
        t0 = time.time()
        if p == "c2":
            part_c2(db)
        elif p == "ktruss18":
            db["ktruss18"] = ktruss_entry(rmat(18), 18)
        elif p == "ktruss22":
            db.setdefault("rmat22", {})["ktruss"] = ktruss_entry(rmat(22), 22)
        else:
            raise SystemExit(f"unknown part {p}")
        save(db)
        print(f"{p}: {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c2", "ktruss18"])
