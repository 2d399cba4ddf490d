"""CPU checks of the C ABI: the library loads and exports every entry point
that include/*.h declares (no compute calls: there may be no GPU here)."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "graptor_b200", "libgg.so")


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"GG_API\s+[\w\s\*]+?\b(gg_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared()
    for must in ["gg_ctx_create", "gg_graph_upload", "gg_edgemap", "gg_vertexmap",
                 "gg_bfs_level", "gg_cc", "gg_pagerank", "gg_frontier_create", "gg_prop_create"]:
        assert must in names


def test_library_exports_all_declared():
    if not os.path.exists(LIB):
        from graptor_b200 import build
        build.build()
    L = C.CDLL(LIB)
    missing = [n for n in sorted(declared()) if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert declared() <= exported
    # nothing but the C ABI leaks out of the shared object
    assert all(n.startswith("gg_") for n in exported), sorted(n for n in exported if not n.startswith("gg_"))


def test_status_strings_and_sizes():
    from graptor_b200 import gg
    L = gg.lib()
    assert L.gg_status_string(gg.GG_ERR_TIMEOUT) == b"GG_ERR_TIMEOUT"
    assert L.gg_dtype_size(gg.BF16) == 2 and L.gg_dtype_size(gg.F64) == 8
    assert L.gg_dtype_size(gg.FP8E4M3) == 1


def test_null_arguments_rejected_without_gpu():
    from graptor_b200 import gg
    L = gg.lib()
    assert L.gg_ctx_create(0, None) == gg.GG_ERR_ARG
    assert L.gg_edgemap(None, None, None, None, None) == gg.GG_ERR_ARG
    assert L.gg_graph_destroy(None) == gg.GG_ERR_ARG


def test_ctx_create_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from graptor_b200 import gg
    h = C.c_void_p()
    assert gg.lib().gg_ctx_create(0, C.byref(h)) == gg.GG_ERR_NOT_FOUND


def test_tuning_knobs_roundtrip():
    from graptor_b200 import gg
    old = gg.tuning_get("pull_k")
    try:
        gg.tuning_set("pull_k", 12)
        assert gg.tuning_get("pull_k") == 12
    finally:
        gg.tuning_set("pull_k", old)
    with pytest.raises(gg.GGError):
        gg.tuning_set("no_such_knob", 1)
    with pytest.raises(gg.GGError):
        gg.tuning_set("pull_k", 0)
    small = gg.tuning_get("bin_small_max")
    with pytest.raises(gg.GGError):  # small bin above the medium bin
        gg.tuning_set("bin_small_max", gg.tuning_get("bin_medium_max") + 1)
    assert gg.tuning_get("bin_small_max") == small  # a rejected set changes nothing


def test_traversal_mode_knobs():
    """Defaults and ranges of the knobs that pick how a BFS run is driven:
    graph-driven levels, the hand-over to the device-driven kernel (after
    how many levels, on how many CTAs) and the small-frontier cluster."""
    from graptor_b200 import gg
    names = ("graph", "graph_handoff", "handoff_ctas", "small_frontier")
    old = {k: gg.tuning_get(k) for k in names}
    assert old == {"graph": 1, "graph_handoff": 32, "handoff_ctas": 148, "small_frontier": 1}
    try:
        for k, v in (("graph_handoff", 0), ("graph_handoff", 1000), ("handoff_ctas", 0), ("handoff_ctas", 37),
                     ("small_frontier", 0)):
            gg.tuning_set(k, v)
            assert gg.tuning_get(k) == v
        for k, v in (("graph", 2), ("small_frontier", 2), ("graph_handoff", -1), ("handoff_ctas", 1 << 20)):
            with pytest.raises(gg.GGError):
                gg.tuning_set(k, v)
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)


def test_pull_knobs():
    """Defaults and ranges of the dense pull's knobs: the per-vertex record
    mode (0-4), the KiB of frontier bitmap a CTA stages in shared memory
    (0, 4, 8, 16 or 32) and the skipped level loads after a pull."""
    from graptor_b200 import gg
    names = ("pull_first", "pull_stage", "pull_fresh", "pull_split", "graph_pdl", "graph_unroll", "pull_ctas",
             "push_ctas", "pr_blocks_per_sm")
    old = {k: gg.tuning_get(k) for k in names}
    try:
        for k, v in (("pull_first", 3), ("pull_first", 4), ("pull_stage", 4), ("pull_stage", 32),
                     ("pull_stage", 0), ("pull_fresh", 0), ("pull_fresh", 1), ("graph_pdl", 1),
                     ("graph_unroll", 4), ("graph_unroll", 1), ("pull_ctas", 4), ("push_ctas", 5),
                     ("pr_blocks_per_sm", 8)):
            gg.tuning_set(k, v)
            assert gg.tuning_get(k) == v
        for k, v in (("pull_first", 5), ("pull_stage", 12), ("pull_stage", 64), ("pull_fresh", 2),
                     ("graph_pdl", 2), ("graph_unroll", 0), ("graph_unroll", 5), ("pull_ctas", 3),
                     ("push_ctas", 9)):
            before = gg.tuning_get(k)
            with pytest.raises(gg.GGError):
                gg.tuning_set(k, v)
            assert gg.tuning_get(k) == before
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)


def test_autotune_apply_orders_the_bin_pair():
    from graptor_b200 import autotune, gg
    old = {k: gg.tuning_get(k) for k in ("bin_small_max", "bin_medium_max", "pull_k")}
    try:
        # both directions: the new small bin above the old medium one, and back
        autotune.apply({"bin_small_max": 4096, "bin_medium_max": 8192, "pull_k": 4})
        assert (gg.tuning_get("bin_small_max"), gg.tuning_get("bin_medium_max")) == (4096, 8192)
        autotune.apply({"bin_medium_max": 64, "bin_small_max": 16})
        assert (gg.tuning_get("bin_small_max"), gg.tuning_get("bin_medium_max")) == (16, 64)
        assert gg.tuning_get("pull_k") == 4
    finally:
        autotune.apply(old)


def test_tuning_accepts_long_timeouts():
    from graptor_b200 import gg
    old = gg.tuning_get("barrier_timeout_ns")
    gg.tuning_set("barrier_timeout_ns", 10_000_000_000)
    assert gg.tuning_get("barrier_timeout_ns") == 10_000_000_000
    gg.tuning_set("barrier_timeout_ns", old)
