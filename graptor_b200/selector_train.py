"""Train the traversal-variant selector on timings the library measures itself.

Training set (seeded): R-MAT scales 18-22 with the first quadrant probability
a drawn from [0.45, 0.65] (d = 0.05, b = c), Erdos-Renyi graphs with average
degree 4-64, and 2-D grids of 2^20-2^22 vertices with 1% of the edges
deleted.  For every graph, gg_selector_collect runs BFS (from a seeded
non-isolated root) and CC device-driven, forcing each of the four traversal
variants at sampled iterations, and records the iteration's features and the
measured log2 time of every variant.  The network is then trained by the
library's GPU kernels (gg_selector_train) on the records of four fifths of
the graphs (every fifth graph is held out: its records are only scored, so
the held-out figures are on graphs the network never saw) and the
parameters are written to graptor_b200/data/selector.npz, which
load_selector() attaches to graphs.  The collected records are kept in
graptor_b200/data/selector_records.npz with the index of the graph each
record comes from.

    python -m graptor_b200.selector_train [--graphs 200] [--out path]
    python -m graptor_b200.selector_train --dataset-in graptor_b200/data/selector_records.npz
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import gg

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "selector.npz")


def graph_family(i: int, rng: np.random.Generator):
    """The i-th training graph: (kind, kwargs, label)."""
    k = i % 3
    if k == 0:
        scale = int(rng.integers(18, 23))
        a = float(rng.uniform(0.45, 0.65))
        b = (1.0 - a - 0.05) / 2
        return "rmat", dict(scale=scale, nedges=16 << scale, seed=1000 + i, a=a, b=b, c=b), f"rmat{scale}_a{a:.2f}"
    if k == 1:
        scale = int(rng.integers(18, 22))
        deg = float(np.exp(rng.uniform(np.log(4), np.log(64))))
        return "er", dict(n=1 << scale, avgdeg=deg, seed=2000 + i), f"er{scale}_d{deg:.0f}"
    side = int(2 ** rng.uniform(10, 11))
    return "grid", dict(rows=side, cols=side, seed=3000 + i, del_bp=100), f"grid{side}"


def make_graph(ctx: gg.Context, kind: str, kw: dict) -> gg.Graph:
    if kind == "rmat":
        return ctx.rmat(kw["scale"], kw["nedges"], kw["seed"], a=kw["a"], b=kw["b"], c=kw["c"])
    if kind == "er":
        return ctx.er(kw["n"], kw["avgdeg"], kw["seed"])
    return ctx.grid(kw["rows"], kw["cols"], kw["seed"], del_bp=kw["del_bp"])


def collect(ctx: gg.Context, n_graphs: int, seed: int = 7, samples: int = 6, log=print):
    rng = np.random.default_rng(seed)
    Xs, Ys, Gs, meta = [], [], [], []
    t0 = time.time()
    for i in range(n_graphs):
        kind, kw, label = graph_family(i, rng)
        g = make_graph(ctx, kind, kw)
        off, _ = g.download()
        deg = np.diff(off)
        nz = np.flatnonzero(deg)
        root = int(rng.choice(nz)) if len(nz) else 0
        for analytic in (0, 1):
            X, Y = gg.selector_collect(g, analytic, root=root, max_samples=samples)
            Xs.append(X)
            Ys.append(Y)
            Gs.append(np.full(len(X), i, dtype=np.int64))
            meta += [(label, analytic)] * len(X)
        g.close()
        if log and (i + 1) % 20 == 0:
            log(f"collected {i + 1}/{n_graphs} graphs, {sum(len(x) for x in Xs)} records, {time.time() - t0:.0f} s")
    return np.concatenate(Xs), np.concatenate(Ys), np.concatenate(Gs), meta


def clean(X, Y):
    """Mask of usable (record, variant) timings and sanitised arrays: a NaN
    timing (the forced run ended before the sampled iteration) is masked out;
    a negative unreached count reads as 0, as on the device."""
    X = np.nan_to_num(np.asarray(X, dtype=np.float32), nan=0.0)
    Y = np.asarray(Y, dtype=np.float32)
    M = np.isfinite(Y).astype(np.float32)
    return X, np.nan_to_num(Y, nan=0.0), M


def split(graph: np.ndarray):
    """(training, held-out) record indices: the records of every fifth
    training graph are held out, so that no held-out record shares a graph
    (or a run) with a training record."""
    graph = np.asarray(graph)
    idx = np.arange(len(graph))
    hold = graph % 5 == 0
    return idx[~hold], idx[hold]


def train(ctx: gg.Context, X, Y, epochs: int = 3000, lr: float = 3e-3, seed: int = 0):
    sel = gg.Selector(ctx)
    X, Y, M = clean(X, Y)
    loss = sel.train(X, Y, M, epochs=epochs, lr=lr)
    return sel, loss


def quality(sel: gg.Selector, X, Y):
    """Argmin agreement with the measured best variant, and the relative time
    lost against it, over records whose four timings are all valid."""
    X, Y, M = clean(X, Y)
    ok = M.all(1)
    pred = sel.forward(X[ok]).argmin(1)
    t = 2.0 ** Y[ok]
    chosen = t[np.arange(len(t)), pred]
    return float((pred == t.argmin(1)).mean()), float(chosen.sum() / t.min(1).sum() - 1.0)


def save_selector(sel: gg.Selector, path: str = WEIGHTS, info: dict | None = None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=sel.params, info=json.dumps(info or {}))


def load_selector(ctx: gg.Context, path: str = WEIGHTS) -> gg.Selector | None:
    if not os.path.exists(path):
        return None
    z = np.load(path)
    sel = gg.Selector(ctx)
    sel.params = z["params"]
    return sel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--graphs", type=int, default=200)
    ap.add_argument("--samples", type=int, default=6)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--dataset-out", default=None, help="also save the collected records (.npz)")
    ap.add_argument("--dataset-in", default=None, help="train on saved records instead of collecting")
    args = ap.parse_args()
    ctx = gg.Context(0)
    t0 = time.time()
    if args.dataset_in:
        d = np.load(args.dataset_in)
        X, Y, G = d["X"], d["Y"], d["graph"]
    else:
        X, Y, G, _ = collect(ctx, args.graphs, samples=args.samples)
    t1 = time.time()
    # every fifth graph is held out (never trained on) to report generalisation
    tr, te = split(G)
    sel, loss = train(ctx, X[tr], Y[tr], epochs=args.epochs, lr=args.lr)
    hold = quality(sel, X[te], Y[te])
    t2 = time.time()
    agree, regret = quality(sel, X[tr], Y[tr])
    info = dict(records=int(len(X)), graphs=int(len(np.unique(G))), heldout_graphs=int(len(np.unique(G[te]))),
                train_mse=loss, argmin_agreement=agree,
                regret_vs_best=regret, heldout_argmin_agreement=hold[0], heldout_regret_vs_best=hold[1],
                collect_s=round(t1 - t0, 1), train_s=round(t2 - t1, 1), epochs=args.epochs, lr=args.lr)
    save_selector(sel, args.out, info)
    if args.dataset_out:
        np.savez(args.dataset_out, X=X, Y=Y, graph=G)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
