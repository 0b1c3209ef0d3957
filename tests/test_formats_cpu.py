"""CPU: GraphStd binary (.bin) and Matrix Market formats, pinned against the
reference: byte-identical to the reference's own example/G.bin (its SHA-256
and CSR are the fixture tests/golden/G_bin.npz, made by
tests/golden/make_golden.py), and read back by the reference's GraphStd
reader (oracle/_ref) when it was built."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

import hornet_b200 as H
from oracle import oracle as O
from tests import helpers as T

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_bin_roundtrip():
    g = T.rmat_graph(9, 8, seed=3)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.bin")
        H.write_bin(p, g.off32(), g.adj)
        off, adj = H.read_bin(p)
    np.testing.assert_array_equal(off, g.off32())
    np.testing.assert_array_equal(adj, g.adj)


def test_bin_matches_reference_example_bytes():
    """example/G.mtx read as DIRECTED by GraphStd and written with
    writeBinary is example/G.bin; the same CSR written here gives the same
    bytes (same length and SHA-256), and reads back as the same CSR."""
    z = np.load(os.path.join(GOLD, "G_bin.npz"))
    off, adj = z["off"], z["adj"]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "G.bin")
        H.write_bin(p, off, adj)
        raw = open(p, "rb").read()
        assert len(raw) == int(z["size"])
        assert hashlib.sha256(raw).digest() == z["sha256"].tobytes()
        o2, a2 = H.read_bin(p)
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(a2, adj)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_reader_reads_our_files():
    g = T.rmat_graph(8, 8, seed=5)
    with tempfile.TemporaryDirectory() as d:
        pb = os.path.join(d, "g.bin")
        H.write_bin(pb, g.off32(), g.adj)
        r = O.ref_read_mtx(pb, undirected=False)
        np.testing.assert_array_equal(r.off, g.off)
        np.testing.assert_array_equal(r.adj, g.adj)
        pm = os.path.join(d, "g.mtx")
        H.write_mtx(pm, g.off32(), g.adj)
        r = O.ref_read_mtx(pm, undirected=True)   # mirror + dedup is a no-op here
        np.testing.assert_array_equal(r.off, g.off)
        np.testing.assert_array_equal(r.adj, g.adj)
