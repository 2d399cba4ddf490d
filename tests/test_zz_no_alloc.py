"""gg_bfs_level_noalloc: BFS levels for callers that cannot let the library
allocate device memory (fixed memory budgets, no implicit synchronisation
from cudaMalloc/cudaFree, hosts that forbid allocation by plug-ins).  The
caller brings the graph and the output; the traversal's queues live in a
fixed device array of the library.

The tests call the entry point through the C ABI and check its levels
against the allocating entry point gg_bfs_level and the oracle on the same
graph, on two calls in a row (the second call reuses the shared scratch array
the first one left behind), on a larger graph followed by a smaller one (the
clearing of the shared array between calls is enough), and check that graphs
above the size limit and adjacency entries out of range are refused, with a
valid call still correct afterwards.
"""
import ctypes as C

import numpy as np
import pytest

from graptor_b200 import gg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _noalloc():
    f = gg.lib().gg_bfs_level_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int), C.c_char_p, C.c_size_t]
    return f


def _run(ctx, g, root, out):
    """One no-alloc call on g's device CSR into the I32 property out."""
    off_d, adj_d, _, _ = g.device_ptrs()
    err = C.create_string_buffer(256)
    it = C.c_int()
    ctx.sync()
    s = _noalloc()(off_d, adj_d, g.n, root, out.device_ptr(), ctx.stream(), C.byref(it), err, 256)
    assert s == gg.GG_OK, err.value
    ctx.sync()
    assert it.value >= 1
    return out.download()


def test_noalloc_matches_bfs_level_twice():
    ctx = gg.Context(0)
    try:
        og = O.rmat(16, 16 << 16, seed=41)
        g = ctx.upload(og.off, og.adj)
        out = g.prop(gg.I32)
        root0, _ = g.max_degree_vertex()
        for root in (root0, 12345):  # two calls in a row
            got = _run(ctx, g, root, out)
            assert np.array_equal(got, g.bfs_level(root))  # the allocating entry point
            assert np.array_equal(got, O.bfs_level(og, root))
    finally:
        ctx.close()


def test_noalloc_large_then_small_graph():
    ctx = gg.Context(0)
    try:
        big = O.rmat(19, 16 << 19, seed=43)   # about 2^19 vertices, deep queues
        small = O.grid(37, 41, seed=5)         # long, thin frontiers
        gb = ctx.upload(big.off, big.adj)
        gs = ctx.upload(small.off, small.adj)
        ob, os_ = gb.prop(gg.I32), gs.prop(gg.I32)
        rb, _ = gb.max_degree_vertex()
        got_b = _run(ctx, gb, rb, ob)
        assert np.array_equal(got_b, gb.bfs_level(rb))
        got_s = _run(ctx, gs, 0, os_)
        assert np.array_equal(got_s, gs.bfs_level(0))
        assert np.array_equal(got_s, O.bfs_level(small, 0))
    finally:
        ctx.close()


def test_noalloc_rejects_graphs_above_limit():
    f = _noalloc()
    err = C.create_string_buffer(256)
    n = (1 << 20) + 1
    s = f(C.c_void_p(16), C.c_void_p(16), n, 0, C.c_void_p(16), None, None, err, 256)
    assert s == gg.GG_ERR_ARG
    assert b"exceeds" in err.value


def test_noalloc_rejects_out_of_range_adjacency_then_recovers():
    torch = pytest.importorskip("torch")
    ctx = gg.Context(0)
    try:
        # 4 vertices, a path 0-1-2-3 whose vertex 2 also names vertex 9 (>= n);
        # every offset is inside adj, so the kernel reads only valid entries
        n = 4
        off = torch.tensor([0, 1, 3, 6, 7], dtype=torch.int64, device="cuda:0")
        adj = torch.tensor([1, 0, 2, 1, 3, 9, 2], dtype=torch.int32, device="cuda:0")
        lvl = torch.empty(n, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        f = _noalloc()
        err = C.create_string_buffer(256)
        it = C.c_int()
        s = f(off.data_ptr(), adj.data_ptr(), n, 0, lvl.data_ptr(), None, C.byref(it), err, 256)
        torch.cuda.synchronize()
        assert s == gg.GG_ERR_ARG
        assert b"adjacency entry >= n" in err.value
        # a valid call afterwards: the error flag does not stick
        og = O.rmat(12, 16 << 12, seed=44)
        g = ctx.upload(og.off, og.adj)
        out = g.prop(gg.I32)
        root, _ = g.max_degree_vertex()
        assert np.array_equal(_run(ctx, g, root, out), g.bfs_level(root))
    finally:
        ctx.close()
