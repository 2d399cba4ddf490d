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


@pytest.fixture
def fusion_knobs():
    old = {k: gg.tuning_get(k) for k in ("persistent", "fusion", "fusion_queue", "cc_hook")}
    yield
    for k, v in old.items():
        gg.tuning_set(k, v)


@pytest.mark.parametrize("gen", ["rmat", "grid", "union"])
@pytest.mark.parametrize("queue", [0, 32])  # 32 entries: most appends spill into the next frontier
def test_fused_cc_exact(ctx, fusion_knobs, gen, queue):
    if gen == "rmat":
        og = O.rmat(14, 16 << 14, seed=62)
    elif gen == "grid":
        og = O.grid(90, 110, seed=5, del_bp=300)
    else:
        from oracle import batch_oracle as B
        og, _ = B.union([O.grid(20 + i, 30, seed=i, del_bp=500) for i in range(6)] +
                        [O.rmat(9, 4000, seed=i) for i in range(6)])
    g = ctx.upload(og.off, og.adj)
    ref = O.cc(og)
    gg.tuning_set("persistent", 4)
    gg.tuning_set("cc_hook", 0)  # label propagation throughout
    gg.tuning_set("fusion_queue", queue)
    st = {}
    for f in (0, 4):
        gg.tuning_set("fusion", f)
        s = gg.RunStats()
        assert np.array_equal(g.cc(stats=s), ref), (gen, queue, f)
        st[f] = s
    if gen == "grid" and queue == 0:
        # labels cross the grid inside one fused step instead of one hop per level
        assert st[4].iterations < st[0].iterations, (st[4].iterations, st[0].iterations)
    g.close()


def _shuffled_rows(og, seed):
    """The same graph with every adjacency row in a random order (a valid
    symmetric CSR that a caller may upload)."""
    rng = np.random.default_rng(seed)
    adj = og.adj.copy()
    for v in range(og.n):
        b, e = int(og.off[v]), int(og.off[v + 1])
        if e - b > 1:
            adj[b:e] = rng.permutation(adj[b:e])
    return adj


@pytest.mark.parametrize("gen", ["rmat", "grid", "grid_shuffled", "union", "edgeless"])
def test_cc_hooking_exact(ctx, fusion_knobs, gen):
    from oracle import batch_oracle as B
    adj = None
    if gen == "rmat":
        og = O.rmat(14, 16 << 14, seed=63)
    elif gen == "grid":
        og = O.grid(120, 130, seed=6, del_bp=400)
    elif gen == "grid_shuffled":
        # unsorted rows: hooking must not stop a row at its first larger id
        og = O.grid(120, 130, seed=8, del_bp=400)
        adj = _shuffled_rows(og, 9)
        assert not all(np.all(np.diff(adj[og.off[v]:og.off[v + 1]].astype(np.int64)) > 0)
                       for v in range(og.n))
    elif gen == "union":
        og, _ = B.union([O.grid(20 + i, 30, seed=i, del_bp=500) for i in range(8)] +
                        [O.rmat(10, 12 << 10, seed=i) for i in range(8)] + [O.from_edges(9, [])])
    else:
        og = O.from_edges(50, [(1, 2), (3, 4)])
    g = ctx.upload(og.off, og.adj if adj is None else adj)
    ref = O.cc(og)
    gg.tuning_set("persistent", 4)
    st = {}
    for h in (0, 1, 2):
        gg.tuning_set("cc_hook", h)
        s = gg.RunStats()
        assert np.array_equal(g.cc(stats=s), ref), (gen, h)
        st[h] = s
    used = {h: [st[h].variant[i] for i in range(min(st[h].iterations, gg.MAX_ITERS))] for h in (1, 2)}
    if gen == "rmat":
        # vertex 0 reaches most of an R-MAT graph in one step: no road test
        # pass; with cc_hook 2 the rest of the run is hooking all the same
        assert gg.VAR_HOOK not in used[1]
        assert used[2][-1] == gg.VAR_HOOK and st[2].iterations == 2, used[2]
    else:
        # road-like: the run ends with the hooking step
        for h in (1, 2):
            assert used[h][-1] == gg.VAR_HOOK and st[h].iterations == 2, (h, used[h])
    g.close()


@pytest.mark.parametrize("gen", ["rmat", "er", "union", "two_hubs"])
def test_cc_hooking_after_first_step_exact(ctx, fusion_knobs, gen):
    """CC with cc_hook 2 on graphs that fail the road-network test: after
    the first step, the vertices label 0 has not reached hook all their edges
    (vertex 0's component is done): the oracle's labels, also for components
    that label 0 never reaches and for vertex 0 in a small component."""
    from oracle import batch_oracle as B
    if gen == "rmat":
        og = O.rmat(16, 16 << 16, seed=64)
    elif gen == "er":
        og = O.er(40000, 3.0, seed=65)
    elif gen == "union":
        og, _ = B.union([O.rmat(11, 16 << 11, seed=i) for i in range(6)] + [O.grid(30, 40, seed=3, del_bp=200)])
    else:
        # vertex 0 isolated-ish: a small component holding 0, two large ones elsewhere
        e = [(0, 1), (1, 2)] + [(3, 3 + i) for i in range(1, 500)] + [(600, 600 + i) for i in range(1, 400)] + \
            [(4 + i, 5 + i) for i in range(0, 450, 3)]
        og = O.from_edges(1200, e)
    g = ctx.upload(og.off, og.adj)
    gg.tuning_set("persistent", 4)
    gg.tuning_set("cc_hook", 2)
    assert np.array_equal(g.cc(), O.cc(og)), gen
    g.close()


@pytest.mark.parametrize("gen", ["rmat", "grid", "er_directed", "tiny"])
def test_graph_driven_bfs_equals_host_loop(ctx, fusion_knobs, gen):
    """BFS levels as one CUDA graph (device push/pull decisions) against the
    host-driven loop: same levels, same iteration count and variant sequence."""
    old = gg.tuning_get("graph")
    if gen == "rmat":
        og, sym = O.rmat(15, 16 << 15, seed=64), True
    elif gen == "grid":
        og, sym = O.grid(150, 90, seed=7, del_bp=200), True
    elif gen == "er_directed":
        og, sym = O.er(20000, 8.0, seed=3, dangling_bp=200, symmetric=False), False
    else:
        og, sym = O.from_edges(5, [(0, 1), (1, 2)]), True
    g = ctx.upload(og.off, og.adj, symmetric=sym)
    gg.tuning_set("persistent", 0)
    roots = [0, int(np.argmax(og.outdeg())), og.n - 1]
    try:
        for r in roots:
            res = {}
            for mode in (0, 1):
                gg.tuning_set("graph", mode)
                st = gg.RunStats()
                lv = g.bfs_level(r, opts=gg.default_opts(collect=True), stats=st)
                res[mode] = (lv, st)
            ref = O.bfs_level(og, r)
            assert np.array_equal(res[0][0], ref) and np.array_equal(res[1][0], ref), (gen, r)
            s0, s1 = res[0][1], res[1][1]
            assert s0.iterations == s1.iterations
            k = min(s0.iterations, gg.MAX_ITERS)
            assert [s0.variant[i] for i in range(k)] == [s1.variant[i] for i in range(k)]
            assert [s0.nactv[i] for i in range(k)] == [s1.nactv[i] for i in range(k)]
            assert s0.edges_reached == s1.edges_reached
    finally:
        gg.tuning_set("graph", old)
    g.close()


@pytest.mark.parametrize("gen", ["rmat", "er_directed", "grid"])
def test_graph_bfs_handoff_to_device_driven(ctx, fusion_knobs, gen):
    """A graph-driven BFS handed over to the device-driven traversal after
    k iterations (after a push: a list-only frontier; after a pull: a
    bitmap-only one) gives the oracle's levels and the host loop's
    iteration count, per-iteration frontier sizes and reached edges."""
    old = {k: gg.tuning_get(k) for k in ("graph", "graph_handoff", "persistent")}
    if gen == "rmat":
        og, sym = O.rmat(15, 16 << 15, seed=65), True
    elif gen == "er_directed":
        og, sym = O.er(30000, 6.0, seed=4, dangling_bp=200, symmetric=False), False
    else:
        og, sym = O.grid(70, 40, seed=8, del_bp=300), True
    g = ctx.upload(og.off, og.adj, symmetric=sym)
    r = int(np.argmax(og.outdeg()))
    ref = O.bfs_level(og, r)
    try:
        gg.tuning_set("persistent", 0)
        gg.tuning_set("graph", 0)
        s0 = gg.RunStats()
        assert np.array_equal(g.bfs_level(r, opts=gg.default_opts(collect=True), stats=s0), ref)
        k0 = min(s0.iterations, gg.MAX_ITERS)
        gg.tuning_set("graph", 1)
        for h in (1, 2, 3, 4, 7, 0):
            gg.tuning_set("graph_handoff", h)
            st = gg.RunStats()
            lv = g.bfs_level(r, opts=gg.default_opts(collect=True), stats=st)
            assert np.array_equal(lv, ref), (gen, h)
            assert st.iterations == s0.iterations, (gen, h)
            assert [st.nactv[i] for i in range(k0)] == [s0.nactv[i] for i in range(k0)], (gen, h)
            assert [st.variant[i] for i in range(k0)] == [s0.variant[i] for i in range(k0)], (gen, h)
            assert st.edges_reached == s0.edges_reached and st.vertices_reached == s0.vertices_reached
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)
    g.close()


@pytest.mark.parametrize("unroll", [1, 2, 3])
@pytest.mark.parametrize("pdl", [0, 1])
@pytest.mark.parametrize("gen", ["rmat", "er_directed", "grid"])
def test_graph_loop_shapes_exact(ctx, fusion_knobs, gen, pdl, unroll):
    """The graph-driven BFS loop with its chain of kernels copied 1-3 times
    per loop iteration (knob graph_unroll: a run ends in any copy, the later
    copies then do nothing) and with the chain's kernels joined by
    programmatic edges or plain ones (knob graph_pdl): the oracle's levels
    and the host loop's iteration count, frontier sizes and variants, with
    and without the hand-over to the device-driven traversal."""
    knobs = ("graph", "graph_handoff", "persistent", "graph_unroll", "graph_pdl", "graph_flat")
    old = {k: gg.tuning_get(k) for k in knobs}
    if gen == "rmat":
        og, sym = O.rmat(15, 16 << 15, seed=66), True
    elif gen == "er_directed":
        og, sym = O.er(30000, 6.0, seed=5, dangling_bp=200, symmetric=False), False
    else:
        og, sym = O.grid(70, 40, seed=9, del_bp=300), True
    g = ctx.upload(og.off, og.adj, symmetric=sym)
    deg = og.outdeg()
    nz = np.flatnonzero(deg)
    roots = [int(np.argmax(deg)), int(nz[len(nz) // 2])]
    try:
        gg.tuning_set("persistent", 0)
        gg.tuning_set("graph", 0)
        want = {}
        for r in roots:
            s0 = gg.RunStats()
            lv = g.bfs_level(r, opts=gg.default_opts(collect=True), stats=s0)
            assert np.array_equal(lv, O.bfs_level(og, r))
            want[r] = (lv, s0)
        gg.tuning_set("graph", 1)
        gg.tuning_set("graph_flat", 1)
        gg.tuning_set("graph_pdl", pdl)
        gg.tuning_set("graph_unroll", unroll)
        for h in (0, 3, 32):
            gg.tuning_set("graph_handoff", h)
            for r in roots:
                ref, s0 = want[r]
                k0 = min(s0.iterations, gg.MAX_ITERS)
                for _ in range(2):
                    st = gg.RunStats()
                    lv = g.bfs_level(r, opts=gg.default_opts(collect=True), stats=st)
                    assert np.array_equal(lv, ref), (gen, h, r)
                    assert st.iterations == s0.iterations, (gen, h, r)
                    assert [st.nactv[i] for i in range(k0)] == [s0.nactv[i] for i in range(k0)], (gen, h, r)
                    assert [st.variant[i] for i in range(k0)] == [s0.variant[i] for i in range(k0)], (gen, h, r)
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)
    g.close()


@pytest.mark.parametrize("gen", ["rmat", "er_directed", "grid", "chain"])
def test_small_frontier_kernel_equals_cooperative(ctx, fusion_knobs, gen):
    """Device-driven BFS levels with the one-CTA small-frontier kernel on and
    off: the oracle's levels, and the same iteration count, per-iteration
    frontier sizes and reached counts.  R-MAT and ER frontiers outgrow the
    kernel's shared-memory queue (hand-back to the cooperative kernel, also in
    the middle of a level); the grid and the chain stay in it throughout."""
    old = {k: gg.tuning_get(k) for k in ("small_frontier", "graph", "graph_handoff")}
    if gen == "rmat":
        og, sym = O.rmat(15, 16 << 15, seed=66), True
    elif gen == "er_directed":
        og, sym = O.er(40000, 12.0, seed=5, dangling_bp=200, symmetric=False), False
    elif gen == "grid":
        og, sym = O.grid(160, 120, seed=9, del_bp=300), True
    else:
        og, sym = O.from_edges(3000, [(i, i + 1) for i in range(2999)]), True
    g = ctx.upload(og.off, og.adj, symmetric=sym)
    deg = og.outdeg()
    roots = [0, int(np.argmax(deg)), int(np.flatnonzero(deg)[-1])]
    try:
        gg.tuning_set("persistent", 1)
        gg.tuning_set("graph", 0)
        # the cluster may take over from the second level on (by default only
        # after 32), so that short R-MAT / ER runs go in and out of it
        gg.tuning_set("graph_handoff", 1)
        for r in roots:
            ref = O.bfs_level(og, r)
            res = {}
            for sf in (0, 1):
                gg.tuning_set("small_frontier", sf)
                st = gg.RunStats()
                lv = g.bfs_level(r, opts=gg.default_opts(collect=True), stats=st)
                assert np.array_equal(lv, ref), (gen, r, sf)
                res[sf] = st
            s0, s1 = res[0], res[1]
            assert s0.iterations == s1.iterations
            k = min(s0.iterations, gg.MAX_ITERS)
            assert [s0.nactv[i] for i in range(k)] == [s1.nactv[i] for i in range(k)], (gen, r)
            assert [s0.nacte[i] for i in range(k)] == [s1.nacte[i] for i in range(k)], (gen, r)
            assert s0.edges_reached == s1.edges_reached and s0.vertices_reached == s1.vertices_reached
            if gen in ("grid", "chain"):  # small from the second level on: the cluster kernel ran
                assert s1.kernels > s0.kernels, (gen, r, s0.kernels, s1.kernels)
    finally:
        for k, v in old.items():
            gg.tuning_set(k, v)
    g.close()


def test_cc_hooking_repeated_long_chains(ctx, fusion_knobs):
    """Hooking's final pass writes every label once; repeated runs on long
    chains (deep trees) must always give the canonical labels."""
    gg.tuning_set("persistent", 4)
    gg.tuning_set("cc_hook", 1)
    n = 200000
    edges = [(i, i + 1) for i in range(n - 1) if i % 50000 != 49999]  # four long paths
    og = O.from_edges(n, edges)
    g = ctx.upload(og.off, og.adj)
    ref = O.cc(og)
    for _ in range(25):
        assert np.array_equal(g.cc(), ref)
    g.close()
