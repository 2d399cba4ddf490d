"""What the trained selector gains over the density threshold, on measured
per-variant iteration timings it was not trained on.

The records (graptor_b200/data/selector_records.npz) hold, per sampled
iteration of BFS / CC on the training graph families, the features and the
measured time of all four traversal variants, and the graph each comes from;
the records of every fifth graph are held out of training, so the held-out
records come from graphs the network never saw.  The shipped network (graptor_b200/data/selector.npz, trained on
the GPU by gg_selector_train) is evaluated here with the float64 oracle on
bfloat16-rounded weights, applying the same rule as the device: the
threshold's choice (push_sparse iff |F| + outdeg(F) <= m/20, else pull_dense)
stands unless the network predicts another variant 2^0.2 times faster (2^0.5
for CC steps, whose records carry no unreached count: feature 2 is 0)."""
import os

import numpy as np
import pytest

from oracle import mlp_oracle as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "graptor_b200", "data")
MARGIN, MARGIN_CC = 0.2, 0.5


def heldout():
    from graptor_b200.selector_train import clean, split
    d = np.load(os.path.join(DATA, "selector_records.npz"))
    X, Y, Mk = clean(d["X"], d["Y"])
    _, te = split(d["graph"])
    ok = Mk[te].all(1)
    return X[te][ok], Y[te][ok]


def choices(params, X):
    out, _ = M.forward(M.bf16_round(params), X)
    thr = np.where(X[:, 8] <= 0.05, 0, 2)  # feature 8 = (|F| + outdeg F) / m
    best = out.argmin(1)
    r = np.arange(len(X))
    margin = np.where(X[:, 2] == 0, MARGIN_CC, MARGIN)
    return np.where(out[r, best] < out[r, thr] - margin, best, thr), thr


def test_records_are_usable():
    X, Y = heldout()
    assert len(X) > 100
    assert np.isfinite(X).all() and np.isfinite(Y).all()


def regret(t, choice):
    """Mean over records of the chosen variant's time over the best one's:
    every sampled decision counts once, whatever its absolute duration (a CC
    record's time runs to the end of the run and dwarfs a BFS iteration)."""
    r = np.arange(len(t))
    return float(np.mean(t[r, choice] / t.min(1)))


def test_trained_selector_beats_threshold_on_heldout_records():
    z = np.load(os.path.join(DATA, "selector.npz"))
    X, Y = heldout()
    learned, thr = choices(z["params"].astype(np.float64), X)
    t = 2.0 ** Y.astype(np.float64)  # microseconds
    r = np.arange(len(X))
    # the gain, stated: mean time over the oracle-best variant, and totals
    print(f"held-out records {len(X)}: threshold {regret(t, thr):.3f} x best, learned {regret(t, learned):.3f} x best; "
          f"totals threshold {t[r, thr].sum():.0f} us, learned {t[r, learned].sum():.0f} us, "
          f"best {t.min(1).sum():.0f} us")
    assert regret(t, learned) < regret(t, thr)
    assert regret(t, learned) <= 1.10  # within 10% of the oracle-best choice


def test_untrained_network_does_not_beat_threshold_by_luck():
    # a control: random networks under the same margin rule are no better
    X, Y = heldout()
    t = 2.0 ** Y.astype(np.float64)
    z = np.load(os.path.join(DATA, "selector.npz"))
    trained, thr = choices(z["params"].astype(np.float64), X)
    rnd = [regret(t, choices(M.init_params(seed), X)[0]) for seed in range(5)]
    assert regret(t, trained) < min(rnd)


def test_heldout_records_come_from_unseen_graphs():
    from graptor_b200.selector_train import split
    d = np.load(os.path.join(DATA, "selector_records.npz"))
    tr, te = split(d["graph"])
    assert len(te) > 100 and len(tr) > 4 * len(te) // 2
    assert not set(d["graph"][tr]) & set(d["graph"][te])
