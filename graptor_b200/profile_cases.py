"""Single workloads of the library, for profilers and per-iteration breakdowns.

Each case builds its graph on the device, runs a few warm-up repetitions and
then the measured ones, and prints one JSON line with device times (CUDA
events inside the library) and, where the run has iterations, the per-iteration
variant / frontier / kernel-time table of the last repetition.  The commands in
profiles/*.md run these cases under ncu.

    python -m graptor_b200.profile_cases bfs   --scale 24 --roots 4
    python -m graptor_b200.profile_cases pr    --scale 24 --format bf16 --iters 5
    python -m graptor_b200.profile_cases cc    --graph grid --side 2896
    python -m graptor_b200.profile_cases msbfs --scale 22
    python -m graptor_b200.profile_cases ppr   --scale 22 --iters 5
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import gg

FORMATS = {"f32": gg.F32, "bf16": gg.BF16, "f16": gg.F16, "fp8": gg.FP8E4M3, "cfp": gg.CFP_6_10,
           "bf16t": gg.BF16_TRUNC, "f64": gg.F64}


def roots_of(g: gg.Graph, k: int, seed: int = 12345):
    off, _ = g.download()
    nz = np.flatnonzero(np.diff(off))
    return [int(r) for r in np.random.default_rng(seed).choice(nz, size=k, replace=False)]


def iter_table(st: gg.RunStats):
    t = min(st.iterations, gg.MAX_ITERS)
    return [[i, st.variant[i], int(st.nactv[i]), int(st.nacte[i]), round(st.iter_ms[i], 4)] for i in range(t)]


def make_graph(ctx: gg.Context, a) -> gg.Graph:
    if a.graph == "grid":
        return ctx.grid(a.side, a.side, 77, del_bp=100)
    if a.graph == "er":
        return ctx.er(1 << a.scale, 32.0, 1, dangling_bp=100, symmetric=False)
    return ctx.rmat(a.scale, 16 << a.scale, 1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["bfs", "pr", "cc", "msbfs", "ppr"])
    ap.add_argument("--graph", default="rmat", choices=["rmat", "grid", "er"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--side", type=int, default=2048)
    ap.add_argument("--roots", type=int, default=4)
    ap.add_argument("--format", default="f32", choices=sorted(FORMATS))
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seeds", type=int, default=128)
    ap.add_argument("--persistent", type=int, default=None, help="tuning knob: device-driven analytics mask")
    ap.add_argument("--threshold", default="default", choices=["default", "learned"])
    ap.add_argument("--graph-mode", type=int, default=None, help="tuning knob: graph-driven BFS levels (0/1)")
    a = ap.parse_args()
    if a.persistent is not None:
        gg.tuning_set("persistent", a.persistent)
    if a.graph_mode is not None:
        gg.tuning_set("graph", a.graph_mode)
    ctx = gg.Context(0)
    g = make_graph(ctx, a)
    out = {"case": a.case, "graph": a.graph, "n": g.n, "m": g.m, "persistent": gg.tuning_get("persistent")}
    opts = gg.default_opts(gg.THRESH_LEARNED if a.threshold == "learned" else gg.THRESH_DEFAULT, collect=True)
    if a.threshold == "learned":
        from .selector_train import load_selector
        sel = load_selector(ctx)
        gg.attach_selector(g, sel)
    if a.case == "bfs":
        rs = roots_of(g, a.roots)
        for r in rs[: a.warmup]:
            g.bfs_level(r, host=False)
        tot, ker, last, worst = [], [], None, None
        for _ in range(a.reps):
            for r in rs:
                st = gg.RunStats()
                g.bfs_level(r, host=False, opts=opts, stats=st)
                tot.append(st.total_ms)
                ker.append(sum(st.iter_ms[i] for i in range(min(st.iterations, gg.MAX_ITERS))))
                last = st
                if worst is None or st.total_ms > worst[1]:
                    worst = (r, st.total_ms, iter_table(st))
        out.update(ms_per_bfs=round(float(np.mean(tot)), 4), kernel_ms_per_bfs=round(float(np.mean(ker)), 4),
                   ms_per_bfs_median=round(float(np.median(tot)), 4),
                   per_root_ms=[round(x, 3) for x in tot[: len(rs)]], iterations=iter_table(last),
                   worst_root=worst[0], worst_ms=round(worst[1], 3), worst_iterations=worst[2])
    elif a.case == "cc":
        for _ in range(a.warmup):
            g.cc(host=False)
        ts = []
        for _ in range(a.reps):
            st = gg.RunStats()
            g.cc(host=False, opts=gg.default_opts(gg.THRESH_FRAC, 5, collect=True), stats=st)
            ts.append(st.total_ms)
        out.update(ms=round(float(np.median(ts)), 4), iterations=iter_table(st))
    elif a.case == "pr":
        fmt = FORMATS[a.format]
        for _ in range(a.warmup):
            g.pagerank(maxiter=2, tol=-1.0, contrib=fmt, host=False)
        ts = []
        for _ in range(a.reps):
            st = gg.RunStats()
            g.pagerank(maxiter=a.iters, tol=-1.0, contrib=fmt, accum_f64=fmt in (gg.F32, gg.F64), host=False,
                       stats=st)
            ts.append(st.total_ms / max(st.iterations, 1))
        out.update(format=a.format, ms_per_iter=round(float(np.median(ts)), 4))
    elif a.case == "msbfs":
        rs = roots_of(g, 64)
        for _ in range(a.warmup):
            gg.msbfs(g, rs, host=False)
        ts = []
        for _ in range(a.reps):
            st = gg.RunStats()
            gg.msbfs(g, rs, host=False, stats=st)
            ts.append(st.total_ms)
        out.update(ms=round(float(np.median(ts)), 4), edges_reached=int(st.edges_reached),
                   iterations=[[i, st.variant[i], round(st.iter_ms[i], 4)] for i in range(st.iterations)])
    else:
        rs = roots_of(g, min(a.seeds, gg.PPR_MAX_SEEDS))
        for _ in range(a.warmup):
            gg.ppr(g, rs, iters=1, host=False)
        ts = []
        for _ in range(a.reps):
            st = gg.RunStats()
            gg.ppr(g, rs, iters=a.iters, host=False, stats=st)
            ts.append(st.total_ms / max(a.iters, 1))
        out.update(seeds=len(rs), ms_per_iter=round(float(np.median(ts)), 4))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
