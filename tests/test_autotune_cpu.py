"""CPU: the autotuner's search and persistence over the library's knob
registry (hn_tune_*), with a fake workload whose speed depends on the
knobs; knob ranges are enforced by the library."""
import time

import pytest

import hornet_b200 as H
from hornet_b200 import autotune as A


@pytest.fixture(autouse=True)
def _defaults():
    H.tune_reset()
    yield
    H.tune_reset()


def test_registry_defaults_and_ranges():
    names = H.tune_names()
    assert {"tc.warp_cap", "msbfs.block", "bfs.ctas_per_sm"} <= set(names)
    assert H.tune_get("tc.warp_cap") == 512 and H.tune_get("msbfs.block") == 256
    for bad in [("msbfs.block", 384), ("tc.warp_cap", 1024), ("bfs.ctas_per_sm", 0)]:
        with pytest.raises(H.HornetError):
            H.tune_set(*bad)
    with pytest.raises(H.HornetError):
        H.tune_set("no.such.knob", 1)


def test_coordinate_descent_picks_fastest_and_keeps_it_set():
    def run():
        cap, chunk = H.tune_get("tc.warp_cap"), H.tune_get("tc.chunk")
        time.sleep(0.001 * (abs(cap - 128) / 64 + abs(chunk - 64) / 16))
        return 42

    best, log = A.tune(run, lambda a, b: a == b,
                       {"tc.warp_cap": [64, 128, 256, 512], "tc.chunk": [4, 16, 64]}, reps=1)
    assert best == {"tc.warp_cap": 128, "tc.chunk": 64}
    assert H.tune_get("tc.warp_cap") == 128 and H.tune_get("tc.chunk") == 64
    assert log[0]["default"] and len(log) == 1 + 3 + 2


def test_a_knob_that_changes_results_is_rejected():
    with pytest.raises(RuntimeError):
        A.tune(lambda: H.tune_get("tc.chunk"), lambda a, b: a == b, {"tc.chunk": [4]}, reps=1)


def test_save_and_apply(tmp_path):
    p = str(tmp_path / "tuned.json")
    sig = A.signature("tc", 1 << 22, 128_000_000, 200_000)
    assert A.apply_saved("B200", sig, p) is None
    A.save("B200", sig, {"tc.warp_cap": 256, "tc.chunk": 4}, 1.2, p)
    assert A.apply_saved("B200", sig, p) == {"tc.warp_cap": 256, "tc.chunk": 4}
    assert H.tune_get("tc.warp_cap") == 256
    assert A.apply_saved("other", sig, p) is None


def test_search_spaces_and_saved_knobs_are_registered():
    """Every value the autotuner may try, and every knob saved in the
    shipped tuned file, is accepted by the library's registry."""
    import json
    names = set(H.tune_names())
    for space in A.SPACES.values():
        for knob, values in space.items():
            assert knob in names, knob
            for v in values:
                H.tune_set(knob, v)
                assert H.tune_get(knob) == v
    with open(A.DEFAULT_PATH) as f:
        db = json.load(f)
    for dev in db.values():
        for rec in dev.values():
            for knob, v in rec["knobs"].items():
                H.tune_set(knob, v)
                assert H.tune_get(knob) == v


def test_knobs_start_at_their_defaults():
    """In a fresh process every knob already holds its default before any
    hn_tune_reset (the values are not a second hand-kept list)."""
    import subprocess
    import sys
    code = ("import hornet_b200 as H\n"
            "before = {n: H.tune_get(n) for n in H.tune_names()}\n"
            "H.tune_reset()\n"
            "after = {n: H.tune_get(n) for n in H.tune_names()}\n"
            "assert before == after, (before, after)\n")
    root = __import__("os").path.dirname(__import__("os").path.dirname(__file__))
    subprocess.run([sys.executable, "-c", code], check=True, cwd=root)
