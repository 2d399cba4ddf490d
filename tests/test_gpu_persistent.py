"""Device-driven (one cooperative launch) traversals against the host-driven
loop and the oracle, and the bounded grid barrier's timeout path."""
import numpy as np
import pytest

from graptor_b200 import gg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def persistent_knob():
    old = gg.tuning_get("persistent")
    yield
    gg.tuning_set("persistent", old)


ALL = 7  # persistent bitmask: BFS levels | BFS parents | CC


@pytest.mark.parametrize("gen", ["rmat", "grid", "er_directed"])
def test_persistent_equals_host_loop(ctx, persistent_knob, gen):
    if gen == "rmat":
        og, sym = O.rmat(14, 16 << 14, seed=61), True
    elif gen == "grid":
        og, sym = O.grid(70, 90, seed=4, del_bp=200), True
    else:
        og, sym = O.er(8192, 6.0, seed=9, dangling_bp=100, symmetric=False), False
    g = ctx.upload(og.off, og.adj, symmetric=sym)
    roots = [0, 5, int(np.argmax(og.outdeg()))]
    res = {}
    for p in (0, 1):
        gg.tuning_set("persistent", ALL * p)
        res[p] = ([g.bfs_level(r) for r in roots], [g.bfs_parent(r) for r in roots],
                  g.cc() if sym else None)
    for i, r in enumerate(roots):
        ref = O.bfs_level(og, r)
        assert np.array_equal(res[0][0][i], ref)
        assert np.array_equal(res[1][0][i], ref)
        assert O.check_parents(og, r, res[1][1][i], ref) == 0
    if sym:
        assert np.array_equal(res[1][2], O.cc(og))
        assert np.array_equal(res[0][2], res[1][2])


def test_persistent_stats_and_thresholds(ctx, persistent_knob):
    gg.tuning_set("persistent", ALL)
    og = O.rmat(13, 16 << 13, seed=3)
    g = ctx.upload(og.off, og.adj)
    ref = O.bfs_level(og, 0)
    for th, k in [(gg.THRESH_DEFAULT, 0), (gg.THRESH_ALWAYS_SPARSE, 0), (gg.THRESH_ALWAYS_DENSE, 0),
                  (gg.THRESH_FRAC, 20)]:
        st = gg.RunStats()
        assert np.array_equal(g.bfs_level(0, opts=gg.default_opts(th, k, collect=True), stats=st), ref)
        # one iteration per non-empty frontier: levels 0 .. depth
        assert st.iterations == int(ref[ref <= og.n].max()) + 1
        assert st.vertices_reached == int((ref <= og.n).sum())
        assert st.edges_reached == O.reached_edges(og, ref)
        kinds = {st.variant[i] for i in range(st.iterations)}
        if th == gg.THRESH_ALWAYS_SPARSE:
            assert kinds == {gg.VAR_PUSH_SPARSE}
        if th == gg.THRESH_ALWAYS_DENSE:
            assert kinds == {gg.VAR_PULL_DENSE}


def test_grid_barrier_timeout_is_reported_and_recoverable(ctx, persistent_knob):
    """A barrier wait that runs out (limit 1 ns) ends the launch with
    GG_ERR_TIMEOUT; no trap, no hang, and the context keeps working."""
    gg.tuning_set("persistent", ALL)
    og = O.rmat(15, 16 << 15, seed=8)
    g = ctx.upload(og.off, og.adj)
    old = gg.tuning_get("barrier_timeout_ns")
    gg.tuning_set("barrier_timeout_ns", 1)
    try:
        with pytest.raises(gg.GGError) as e:
            g.bfs_level(0)
        assert e.value.status == gg.GG_ERR_TIMEOUT
    finally:
        gg.tuning_set("barrier_timeout_ns", old)
    assert np.array_equal(g.bfs_level(0), O.bfs_level(og, 0))
    assert np.array_equal(g.cc(), O.cc(og))
