"""The batched-traversal oracle on the CPU: known answers and invariants."""
import numpy as np

from oracle import batch_oracle as B
from oracle import oracle as O


def test_msbfs_levels_stack_single_root_runs():
    g = O.rmat(10, 1 << 13, 5)
    roots = [0, 3, 3, 100]
    L = B.msbfs_levels(g, roots)
    assert L.shape == (g.n, 4)
    for i, r in enumerate(roots):
        assert np.array_equal(L[:, i], O.bfs_level(g, r))


def test_ppr_two_vertex_closed_form():
    # 0 <-> 1: x0 = a + (1-a) x1, x1 = (1-a) x0  =>  x0 = a / (1 - (1-a)^2)
    g = O.from_edges(2, [(0, 1)])
    a = 0.15
    x = B.ppr_f64(g, [0], alpha=a, iters=400)
    x0 = a / (1 - (1 - a) ** 2)
    assert abs(x[0, 0] - x0) < 1e-12
    assert abs(x[1, 0] - (1 - a) * x0) < 1e-12


def test_ppr_mass_conserved_without_sinks():
    g = O.grid(12, 13, 3)
    seeds = [0, 5, 77]
    x = B.ppr_f64(g, seeds, iters=30)
    assert np.allclose(x.sum(0), 1.0, atol=1e-12)
    assert (x >= 0).all()


def test_ppr_sink_leaks_mass():
    # directed 0 -> 1, vertex 1 has no out-edges: its mass is not passed on
    g = O.from_edges(2, [(0, 1)], symmetric=False)
    x = B.ppr_f64(g, [0], alpha=0.5, iters=5)
    assert x[0, 0] == 0.5 and x[1, 0] == 0.25


def test_bf16_round_ties_to_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9], dtype=np.float32)
    r = B.bf16_round(v)
    assert r[0] == 1.0
    assert r[1] == 1.0               # tie -> even (mantissa 0)
    assert r[2] == 1.0 + 2 ** -6     # tie -> even (rounds up)
    assert r[3] == 1.0


def test_ppr_bf16_close_to_f64():
    g = O.rmat(10, 1 << 14, 9)
    deg = np.diff(g.off)
    seeds = np.flatnonzero(deg)[:8]
    x64 = B.ppr_f64(g, seeds, iters=20)
    xb = B.ppr_bf16(g, seeds, iters=20)
    assert np.abs(xb - x64).sum(0).max() < 2e-2


def test_union_layout():
    parts = [O.rmat(6, 200, 1), O.grid(3, 4, 2), O.from_edges(5, []), O.rmat(5, 90, 3)]
    u, base = B.union(parts)
    assert list(base) == [0, 64, 76, 81, 113]
    assert u.m == sum(p.m for p in parts)
    for i, p in enumerate(parts):
        lab = O.cc(u)[base[i]:base[i + 1]] - base[i]
        assert np.array_equal(lab, O.cc(p))


def test_multi_root_bfs_over_union_is_per_part_bfs():
    """The oracle's multi-root BFS (the checker of the one-launch union
    batch) equals each part's own BFS from its first vertex."""
    parts = [O.rmat(8, 2000, seed=i) for i in range(4)] + [O.grid(9, 13, seed=2, del_bp=500),
                                                           O.from_edges(5, [(1, 2)])]
    u, base = B.union(parts)
    lv = O.bfs_level_multi(u, base[:-1])
    for i, p in enumerate(parts):
        a, b = int(base[i]), int(base[i + 1])
        got = lv[a:b].copy()
        got[got == u.n + 1] = p.n + 1
        assert np.array_equal(got, O.bfs_level(p, 0)), i
    # duplicate roots count once
    assert np.array_equal(O.bfs_level_multi(u, [0, 0, 3]), O.bfs_level_multi(u, [3, 0]))
