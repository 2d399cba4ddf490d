"""Autotune the library's knobs for a graph family and keep the result.

The search itself is native (gg_autotune: coordinate descent over the
degree-bin thresholds, per-lane scan depths, chunk sizes, CTAs per SM, the
heavy-row cut and the device-driven switch, with every candidate's BFS levels
and CC labels checked against the first run's).  This module runs it on a
generated graph, stores the chosen values as JSON and applies stored values.

    python -m graptor_b200.autotune --rmat 22 --out tuning_rmat22.json
    python -m graptor_b200.autotune --grid 2048 --out tuning_grid.json
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import gg


def apply(knobs: dict) -> None:
    """Set stored knob values (graphs built afterwards pick up heavy_*)."""
    k = dict(knobs)
    if "bin_small_max" in k or "bin_medium_max" in k:
        # bin_small_max <= bin_medium_max must hold after every single set
        lo = int(k.pop("bin_small_max", gg.tuning_get("bin_small_max")))
        hi = int(k.pop("bin_medium_max", gg.tuning_get("bin_medium_max")))
        gg.tuning_set("bin_medium_max", max(hi, gg.tuning_get("bin_small_max")))
        gg.tuning_set("bin_small_max", lo)
        gg.tuning_set("bin_medium_max", hi)
    for name, v in k.items():
        gg.tuning_set(name, int(v))


def load(path: str) -> dict:
    with open(path) as f:
        d = json.load(f)
    apply(d["knobs"])
    return d


def tune_graph(g: gg.Graph, analytics: int, nroots: int = 4, seed: int = 1, passes: int = 2, reps: int = 2):
    off, _ = g.download()
    nz = np.flatnonzero(np.diff(off))
    roots = np.random.default_rng(seed).choice(nz, size=min(nroots, len(nz)), replace=False) if len(nz) else []
    return gg.autotune(g, analytics, roots if analytics & gg.TUNE_BFS else (), passes=passes, reps=reps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rmat", type=int, help="R-MAT scale (edge factor 16, symmetrised)")
    ap.add_argument("--grid", type=int, help="grid side")
    ap.add_argument("--analytics", default="bfs,cc", help="comma list of bfs, cc, pr")
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    mask = sum({"bfs": gg.TUNE_BFS, "cc": gg.TUNE_CC, "pr": gg.TUNE_PR}[x] for x in a.analytics.split(","))
    ctx = gg.Context(0)
    if a.rmat:
        g, what = ctx.rmat(a.rmat, 16 << a.rmat, 1), f"rmat{a.rmat}"
    elif a.grid:
        g, what = ctx.grid(a.grid, a.grid, 1, del_bp=100), f"grid{a.grid}"
    else:
        ap.error("--rmat or --grid")
    res = tune_graph(g, mask, passes=a.passes, reps=a.reps)
    res["graph"] = what
    res["analytics"] = a.analytics
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
