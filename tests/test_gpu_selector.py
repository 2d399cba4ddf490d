"""The selector network's GPU kernels against the float64 CPU oracle, its
training, and that a learned (any) choice never changes the exact results."""
import numpy as np
import pytest

from graptor_b200 import gg
from oracle import mlp_oracle as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(n=300, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.random((n, 10)).astype(np.float32)
    # a smooth target: which variant is "fast" depends on two features
    Y = np.stack([3 + 4 * X[:, 0], 4 + 2 * X[:, 1], 6 - 5 * X[:, 8], 5 + X[:, 3]], 1).astype(np.float32)
    Mk = (rng.random((n, 4)) > 0.1).astype(np.float32)
    return X, Y, Mk


def test_gradient_matches_float64_oracle(ctx):
    sel = gg.Selector(ctx)
    rng = np.random.default_rng(3)
    p = (M.init_params(5) + rng.normal(0, 0.05, M.N_PARAMS)).astype(np.float32)
    sel.params = p
    X, Y, Mk = _data(200, 1)
    loss, g = sel.loss_grad(X, Y, Mk)
    lo, go = M.loss_and_grad(p.astype(np.float64), X, Y, Mk)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    assert np.allclose(g, go, rtol=2e-3, atol=2e-5 * np.abs(go).max())


def test_inference_uses_bf16_weights(ctx):
    sel = gg.Selector(ctx)
    p = M.init_params(7)
    sel.params = p
    X, _, _ = _data(64, 2)
    out = sel.forward(X)
    ref, _ = M.forward(M.bf16_round(p), X)
    assert np.allclose(out, ref, rtol=1e-4, atol=1e-4)


def test_training_reduces_loss(ctx):
    sel = gg.Selector(ctx)
    X, Y, Mk = _data(400, 4)
    l0, _ = sel.loss_grad(X, Y, Mk)
    l1 = sel.train(X, Y, Mk, epochs=400, lr=3e-3)
    assert l1 < 0.1 * l0, (l0, l1)
    # the trained network ranks the variants like the target on most samples
    pred = sel.forward(X).argmin(1)
    assert (pred == Y.argmin(1)).mean() > 0.8


def test_learned_choice_never_changes_results(ctx):
    og = O.rmat(14, 16 << 14, seed=21)
    g = ctx.upload(og.off, og.adj)
    opts = gg.default_opts(gg.THRESH_LEARNED)
    ref_l, ref_c = O.bfs_level(og, 0), O.cc(og)
    for seed in range(3):  # arbitrary networks pick arbitrary variants
        sel = gg.Selector(ctx)
        sel.params = M.init_params(100 + seed) * 3
        gg.attach_selector(g, sel)
        st = gg.RunStats()
        assert np.array_equal(g.bfs_level(0, opts=opts, stats=st), ref_l)
        assert np.array_equal(g.cc(opts=opts), ref_c)
        assert O.check_parents(og, 0, g.bfs_parent(0, opts=opts), ref_l) == 0
    gg.attach_selector(g, None)
    assert np.array_equal(g.bfs_level(0, opts=opts), ref_l)  # threshold fallback


def test_graph_keeps_its_copy_of_the_weights(ctx):
    """A graph attached to a selector that is then destroyed still runs its
    learned choices (graph-driven, device-driven and host-driven) on its own
    copy of the weights, with the same results."""
    import gc
    og = O.rmat(14, 16 << 14, seed=22)
    g = ctx.upload(og.off, og.adj)
    sel = gg.Selector(ctx)
    sel.params = M.init_params(7) * 3
    gg.attach_selector(g, sel)
    sel.close()
    del sel
    gc.collect()
    opts = gg.default_opts(gg.THRESH_LEARNED)
    ref_l = O.bfs_level(og, 3)
    old = {k: gg.tuning_get(k) for k in ("graph", "persistent")}
    try:
        for graph_mode, persistent in ((1, 4), (0, 5), (0, 4)):
            gg.tuning_set("graph", graph_mode)
            gg.tuning_set("persistent", persistent)
            assert np.array_equal(g.bfs_level(3, opts=opts), ref_l), (graph_mode, persistent)
        assert np.array_equal(g.cc(opts=opts), O.cc(og))
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)
        gg.attach_selector(g, None)
        g.close()


@pytest.mark.parametrize("variant", [gg.VAR_PUSH_SPARSE, gg.VAR_PUSH_MERGE, gg.VAR_PULL_DENSE, gg.VAR_PUSH_DENSE])
def test_device_driven_every_variant(ctx, variant):
    og = O.grid(40, 50, seed=6, del_bp=200)
    g = ctx.upload(og.off, og.adj)
    old = gg.tuning_get("persistent")
    gg.tuning_set("persistent", 7)
    try:
        o = gg.default_opts(variant=variant)
        assert np.array_equal(g.bfs_level(3, opts=o), O.bfs_level(og, 3))
        assert np.array_equal(g.cc(opts=o), O.cc(og))
    finally:
        gg.tuning_set("persistent", old)


def test_collect_records(ctx):
    g = ctx.rmat(13, 16 << 13, seed=2)
    X, Y = gg.selector_collect(g, 0, root=0, max_samples=4)
    assert 1 <= len(X) <= 4
    assert np.all(np.isfinite(Y)) and np.all(Y > -3) and np.all(Y < 25)
    assert np.all(X >= 0) and np.all(X <= 4.5)
    X2, Y2 = gg.selector_collect(g, 1, max_samples=3)
    assert len(X2) >= 1
