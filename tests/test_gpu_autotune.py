"""The native autotuner on a small graph: it only keeps values that lower the
measured objective, leaves them set, and results stay exact under them."""
import numpy as np
import pytest

from graptor_b200 import autotune, gg
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KNOBS = ["bin_small_max", "bin_medium_max", "pull_k", "push_k", "large_chunk", "blocks_per_sm",
         "heavy_deg", "heavy_chunk", "persistent", "pr_stream", "pr_blocks_per_sm", "pull_split"]


@pytest.fixture
def saved_knobs():
    old = {k: gg.tuning_get(k) for k in KNOBS}
    yield old
    autotune.apply(old)


def test_autotune_keeps_results_exact(ctx, saved_knobs):
    g = O.rmat(12, 1 << 16, 77)
    G = ctx.upload(g.off, g.adj, True)
    res = autotune.tune_graph(G, gg.TUNE_BFS | gg.TUNE_CC | gg.TUNE_PR, nroots=2, passes=1, reps=1)
    assert res["best_ms"] <= res["initial_ms"]
    assert res["evaluations"] > 10
    for k, v in res["knobs"].items():
        assert gg.tuning_get(k) == v
    root = int(np.flatnonzero(np.diff(g.off))[0])
    assert np.array_equal(G.bfs_level(root), O.bfs_level(g, root))
    assert np.array_equal(G.cc(), O.cc(g))
    G.close()


def test_retune_rebuilds_heavy_rows(ctx, saved_knobs):
    g = O.rmat(11, 1 << 15, 5)
    G = ctx.upload(g.off, g.adj, True)
    x0 = G.pagerank(maxiter=10)
    gg.tuning_set("heavy_deg", 32)
    gg.tuning_set("heavy_chunk", 64)
    gg.graph_retune(G)
    x1 = G.pagerank(maxiter=10)
    ref, _, _ = O.pagerank(g, maxiter=10)
    assert np.abs(x1 - ref).sum() < 1e-6 and np.abs(x0 - ref).sum() < 1e-6
    G.close()
