"""CPU: the C-ABI library loads, exports every entry point include/*.h
declares, and its host-only logic (the R-MAT generator, error reporting)
behaves; no device compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

import hornet_b200 as H
from tests.conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(hn_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = H.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), f"{n} declared but not exported"
        assert n in H._SIGNATURES, f"{n} has no Python binding"


def test_library_is_built_for_sm100a():
    so = H.LIB_PATH
    assert os.path.getsize(so) > 100_000
    # the fatbin names its target architecture
    data = open(so, "rb").read()
    assert b"sm_100a" in data


def test_version_and_error_string():
    assert H.lib().hn_version() >= 10000
    assert isinstance(H.last_error(), str)


def test_rmat_host_generator_deterministic_and_in_range():
    s1, d1 = H.gen_rmat_host(12, 20000, 5)
    s2, d2 = H.gen_rmat_host(12, 20000, 5)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(d1, d2)
    assert s1.min() >= 0 and s1.max() < 4096 and d1.max() < 4096
    s3, _ = H.gen_rmat_host(12, 20000, 6)
    assert (s3 != s1).any()
    # a = .57 skews ids toward 0: the top half of the id range is rarer
    assert (s1 < 2048).mean() > 0.7
    # non-power-of-two vertex count: all endpoints below n
    s4, d4 = H.gen_rmat_host(12, 20000, 5, n_vertices=3000)
    assert s4.max() < 3000 and d4.max() < 3000
    # pair i depends only on (seed, i): a prefix is reproducible
    s5, d5 = H.gen_rmat_host(12, 1000, 5)
    np.testing.assert_array_equal(s5, s1[:1000])


def test_rmat_multithreaded_equals_single():
    s1, d1 = H.gen_rmat_host(14, 200000, 9)   # multi-threaded path
    s2 = np.empty_like(s1)
    d2 = np.empty_like(d1)
    for lo in range(0, 200000, 50000):         # single-threaded chunks
        a, b = H.gen_rmat_host(14, lo + 50000, 9)
        s2[lo:lo + 50000] = a[lo:]
        d2[lo:lo + 50000] = b[lo:]
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(d1, d2)


def test_invalid_arguments_are_status_codes():
    lib = H.lib()
    src = np.zeros(4, np.int32)
    rc = lib.hn_gen_rmat_host(0, 1, 4, 0.57, 0.19, 0.19, 1, src.ctypes.data_as(ctypes.c_void_p),
                              src.ctypes.data_as(ctypes.c_void_p))
    assert rc == H.HN_ERR_INVALID
    assert "scale" in H.last_error()
    out = ctypes.c_void_p()
    rc = lib.hn_graph_create_csr(-1, 0, None, None, 0, 0, 0, ctypes.byref(out))
    assert rc == H.HN_ERR_INVALID
    rc = lib.hn_insert(None, None, 0, None)
    assert rc == H.HN_ERR_INVALID


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_reports_cuda_error_without_exiting():
    off = np.array([0, 1, 2], np.int32)
    adj = np.array([1, 0], np.int32)
    with pytest.raises(H.HornetError) as ei:
        H.Hornet(H.HornetInit(2, 2, off, adj))
    assert ei.value.code in (H.HN_ERR_CUDA, H.HN_ERR_OOM)


def test_oracle_generator_equals_library_generator_for_update_batches():
    """The reference GPU update run (oracle/run_ref_gpu.py) draws the
    dynamic-update configuration's R-MAT batches with the oracle's
    generator; they equal the benchmark's, drawn with the library's."""
    import types
    import bench
    from oracle import oracle as O
    for kind, b, seed in (("uniform", 10000, 77), ("rmat", 10000, 78), ("rmat", 4001, 80)):
        r1 = np.random.default_rng(2024)
        r2 = np.random.default_rng(2024)
        a = bench.c3_batch(H, r1, kind, b, 1 << 20, 20, seed)
        o = bench.c3_batch(types.SimpleNamespace(gen_rmat_host=O.gen_rmat), r2, kind, b,
                           1 << 20, 20, seed)
        np.testing.assert_array_equal(a[0], o[0])
        np.testing.assert_array_equal(a[1], o[1])
