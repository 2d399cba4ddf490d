"""Batched traversals on the GPU against the oracle: multi-source BFS levels
bit-exact per root, personalized PageRank (bfloat16 storage, float32 sums)
within stated L1 of the float64 oracle, and BFS / CC over a disjoint union of
many small graphs bit-exact per part."""
import numpy as np
import pytest

from graptor_b200 import gg
from oracle import batch_oracle as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# PPR, per seed, L1 over all vertices (each seed's ranks sum to <= 1):
# bfloat16 keeps 8 significant bits; against the float64 oracle the error is
# the storage rounding, against the bfloat16 restatement only summation order
# (an occasional one-ulp flip of a stored value).
PPR_L1_VS_F64 = 2e-2
PPR_L1_VS_BF16_EMUL = 2e-3


def upload(ctx, g, symmetric=True):
    return ctx.upload(g.off, g.adj, symmetric)


def nonisolated(g, k, seed):
    nz = np.flatnonzero(np.diff(g.off))
    return np.random.default_rng(seed).choice(nz, size=k, replace=len(nz) < k)


@pytest.mark.parametrize("k", [1, 7, 64])
def test_msbfs_rmat(ctx, k):
    g = O.rmat(12, 1 << 16, 21)
    G = upload(ctx, g)
    roots = nonisolated(g, k, k)
    st = gg.RunStats()
    L = gg.msbfs(G, roots, stats=st)
    ref = B.msbfs_levels(g, roots)
    assert np.array_equal(L, ref)
    assert st.edges_reached == sum(O.reached_edges(g, ref[:, i]) for i in range(k))
    assert st.iterations == int(ref[ref <= g.n].max()) + 1
    G.close()


def test_msbfs_repeated_and_isolated_roots(ctx):
    g = O.from_edges(40, [(i, i + 1) for i in range(30)] + [(31, 32)])
    G = upload(ctx, g)
    roots = [0, 0, 39, 31, 15, 30, 39]  # 39 is isolated, 0 repeats
    L = gg.msbfs(G, roots)
    assert np.array_equal(L, B.msbfs_levels(g, roots))
    G.close()


def test_msbfs_grid_many_levels(ctx):
    # long diameter: both push and pull iterations, many barriers
    g = O.grid(40, 50, 4, del_bp=300)
    G = upload(ctx, g)
    roots = nonisolated(g, 64, 1)
    st = gg.RunStats()
    L = gg.msbfs(G, roots, stats=st)
    assert np.array_equal(L, B.msbfs_levels(g, roots))
    used = {st.variant[i] for i in range(min(st.iterations, gg.MAX_ITERS))}
    assert used <= {gg.VAR_PUSH_DENSE, gg.VAR_PULL_DENSE}
    G.close()


def test_msbfs_rejects_bad_arguments(ctx):
    g = O.rmat(6, 300, 1)
    G = upload(ctx, g)
    with pytest.raises(gg.GGError):
        gg.msbfs(G, np.arange(65))
    with pytest.raises(gg.GGError):
        gg.msbfs(G, [g.n])
    G.close()


@pytest.mark.parametrize("k", [1, 37, 128])
def test_ppr_rmat(ctx, k):
    g = O.rmat(12, 1 << 16, 33)
    G = upload(ctx, g)
    seeds = nonisolated(g, k, 100 + k)
    st = gg.RunStats()
    x = gg.ppr(G, seeds, alpha=0.15, iters=20, stats=st)
    x64 = B.ppr_f64(g, seeds, 0.15, 20)
    xb = B.ppr_bf16(g, seeds, 0.15, 20)
    err64 = np.abs(x - x64).sum(0)
    errb = np.abs(x - xb).sum(0)
    assert err64.max() < PPR_L1_VS_F64, err64.max()
    assert errb.max() < PPR_L1_VS_BF16_EMUL, errb.max()
    assert st.iterations == 20 and st.total_ms > 0
    G.close()


def test_ppr_heavy_rows_and_sinks(ctx):
    # a star (hub in-degree far above the heavy-row threshold) plus a
    # directed sink: exercises the chunked hub gather and the leak rule
    n = 3000
    edges = [(0, i) for i in range(1, n - 1)] + [(n - 2, n - 1)]
    g = O.from_edges(n, edges)
    gd = O.from_edges(n, edges + [(5, n - 1)], symmetric=False)
    for graph, sym in ((g, True), (gd, False)):
        G = upload(ctx, graph, sym)
        seeds = [0, 1, n - 2, n - 1]
        x = gg.ppr(G, seeds, alpha=0.2, iters=15)
        err = np.abs(x - B.ppr_f64(graph, seeds, 0.2, 15)).sum(0)
        assert err.max() < PPR_L1_VS_F64, err
        G.close()


def test_ppr_zero_iterations_is_teleport(ctx):
    g = O.rmat(8, 2000, 2)
    G = upload(ctx, g)
    x = gg.ppr(G, [3, 9], iters=0)
    e = np.zeros((g.n, 2), dtype=np.float32)
    e[3, 0] = e[9, 1] = 1
    assert np.array_equal(x, e)
    G.close()


def small_graph_family(count, seed, lo=6, hi=12):
    """Graphs of log-uniform size in [2^lo, 2^hi]: R-MAT (edge factor 8-32)
    and 2-D grids, plus an edgeless graph."""
    rng = np.random.default_rng(seed)
    parts = []
    for i in range(count):
        lg = rng.uniform(lo, hi)
        if i % 2 == 0:
            scale = int(round(lg))
            ef = int(rng.integers(8, 33))
            parts.append(O.rmat(scale, ef << scale, 500 + i))
        else:
            side = max(2, int(2 ** (lg / 2)))
            parts.append(O.grid(side, int(2 ** lg) // side, 700 + i, del_bp=100))
    parts.append(O.from_edges(17, []))
    return parts


def test_union_bfs_and_cc_per_part(ctx):
    parts = small_graph_family(41, 3)
    Gs = [upload(ctx, p) for p in parts]
    U, base = gg.graph_union(ctx, Gs)
    ou, obase = B.union(parts)
    assert np.array_equal(base, obase)
    off, adj = U.download()
    assert np.array_equal(off, ou.off) and np.array_equal(adj, ou.adj)
    # BFS from vertex 0 of every part, one launch
    st = gg.RunStats()
    lv = gg.bfs_level_multi(U, base[:-1], stats=st)
    cc = U.cc()
    for i, p in enumerate(parts):
        a, b = int(base[i]), int(base[i + 1])
        ref = O.bfs_level(p, 0)
        got = lv[a:b].copy()
        got[got == U.n + 1] = p.n + 1   # unreached: n+1 of the union vs of the part
        assert np.array_equal(got, ref), i
        assert np.array_equal(cc[a:b] - a, O.cc(p)), i
    assert st.iterations == max(int(O.bfs_level(p, 0)[O.bfs_level(p, 0) <= p.n].max()) for p in parts) + 1
    for G in Gs:
        G.close()
    U.close()


def test_batch_bfs_cc_one_graph_launch(ctx):
    """BFS from every part's vertex 0 and CC of the union, submitted as one
    CUDA graph launch: per-part levels and labels equal the oracle's, twice
    in a row."""
    parts = small_graph_family(41, 5)
    Gs = [upload(ctx, p) for p in parts]
    U, base = gg.graph_union(ctx, Gs)
    for _ in range(2):
        bs, cs = gg.RunStats(), gg.RunStats()
        lv, lb, glaunch, kernels = gg.batch_bfs_cc(U, base[:-1], bfs_stats=bs, cc_stats=cs)
        assert glaunch == 1 and kernels > 2
        assert bs.iterations >= 1 and cs.iterations >= 1
        for i, p in enumerate(parts):
            a, b = int(base[i]), int(base[i + 1])
            got = lv[a:b].copy()
            got[got == U.n + 1] = p.n + 1
            assert np.array_equal(got, O.bfs_level(p, 0)), i
            assert np.array_equal(lb[a:b] - a, O.cc(p)), i
    for G in Gs:
        G.close()
    U.close()


def test_bfs_level_multi_single_root_matches_bfs_level(ctx):
    g = O.rmat(11, 1 << 15, 8)
    G = upload(ctx, g)
    r = int(nonisolated(g, 1, 2)[0])
    assert np.array_equal(gg.bfs_level_multi(G, [r, r]), G.bfs_level(r))
    G.close()
