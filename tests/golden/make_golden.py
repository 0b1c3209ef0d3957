"""Regenerate the golden fixtures in tests/golden/ from the REFERENCE's own
host code (oracle/_ref/ref_driver: xlib GraphStd reader, graph::BFS,
graph::WCC) and the reference's example graphs.

    python tests/golden/make_golden.py [/path/to/hornet/source]

The source path defaults to the environment variable HORNET_REFERENCE.

Run in a container that has the reference sources; the fixtures are
committed so the tests never need them.  Each fixture holds:
  off, adj          undirected CSR as GraphStd builds it (mirror, drop self
                    loops, sort, dedup: xlib/src/Graph/GraphStd.cpp:174-206)
  ooff, oadj        the DIRECTED_BY_DEGREE | SORT orientation used by
                    TriangleCounting2 (GraphStd.cpp:247-310)
  bfs_src, bfs      graph::BFS::run distances from a few sources
  wcc               graph::WCC::run colours
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HORNET_REFERENCE", "")


def fixture(name: str, path: str, nsrc: int = 4) -> None:
    g = O.ref_read_mtx(path, undirected=True)
    og = O.ref_read_mtx(path, undirected=True, by_degree=True)
    srcs = sorted(set([0] + list(np.linspace(0, g.nV - 1, nsrc).astype(int))))
    bfs = O.ref_bfs(g, srcs)
    wcc = O.ref_wcc(g)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), off=g.off, adj=g.adj, ooff=og.off,
                        oadj=og.adj, bfs_src=np.array(srcs, np.int32), bfs=bfs, wcc=wcc)
    print(f"{name}: nV={g.nV} nE={g.nE} oriented={og.nE}")


def fixture_bin(name: str, path: str) -> None:
    """The reference's own GraphStd binary file: its SHA-256 and the CSR it
    holds (header: 6 bytes, nV, nE, 16 more bytes; then off[nV+1], adj[nE])."""
    import hashlib
    raw = open(path, "rb").read()
    nV = int.from_bytes(raw[6:10], "little")
    nE = int.from_bytes(raw[10:14], "little")
    body = np.frombuffer(raw[30:], np.int32)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), off=body[: nV + 1].copy(),
                        adj=body[nV + 1: nV + 1 + nE].copy(),
                        sha256=np.frombuffer(hashlib.sha256(raw).digest(), np.uint8),
                        size=np.int64(len(raw)))
    print(f"{name}: nV={nV} nE={nE} bytes={len(raw)}")


def main() -> None:
    assert REF, "give the reference source path (argument or HORNET_REFERENCE)"
    assert O.ref_available(), "build oracle/_ref first: make -C oracle ref"
    ex = os.path.join(REF, "example")
    fixture_bin("G_bin", os.path.join(ex, "G.bin"))
    fixture("G", os.path.join(ex, "G.mtx"))
    fixture("G_cc2", os.path.join(ex, "G_cc2.mtx"))
    fixture("rome99", os.path.join(ex, "rome99.gr"))
    # a small R-MAT graph from this repository's generator, written as a
    # Matrix Market file and read back by the reference's GraphStd
    import hornet_b200 as H
    import tempfile
    s, d = H.gen_rmat_host(8, 8 * 256, 7)
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "rmat8.mtx")
        O.write_mtx(p, 256, s, d)
        fixture("rmat8", p)
    np.savez_compressed(os.path.join(HERE, "rmat8_pairs.npz"), src=s, dst=d)


if __name__ == "__main__":
    main()
