"""gg_bfs_level_noalloc: BFS levels for callers that cannot let the library
allocate device memory (fixed memory budgets, no implicit synchronisation
from cudaMalloc/cudaFree, hosts that forbid allocation by plug-ins).  The
caller brings the graph and the output; the traversal's queues live in a
fixed device array of the library.

The test calls the entry point through the C ABI and checks its levels
against the allocating entry point gg_bfs_level on the same graph, on two
calls in a row (the second call reuses the shared scratch array the first
one left behind), and checks that graphs above the size limit are refused.
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


def test_noalloc_matches_bfs_level_twice():
    ctx = gg.Context(0)
    try:
        og = O.rmat(16, 16 << 16, seed=41)
        g = ctx.upload(og.off, og.adj)
        off_d, adj_d, _, _ = g.device_ptrs()
        out = g.prop(gg.I32)
        f = _noalloc()
        err = C.create_string_buffer(256)
        it = C.c_int()
        root0, _ = g.max_degree_vertex()
        for root in (root0, 12345):  # two calls in a row
            ctx.sync()
            s = f(off_d, adj_d, g.n, root, out.device_ptr(), ctx.stream(), C.byref(it), err, 256)
            assert s == gg.GG_OK, err.value
            ctx.sync()
            want = g.bfs_level(root)  # the allocating entry point
            got = out.download()
            assert np.array_equal(got, want)
            assert it.value >= 1
    finally:
        ctx.close()


def test_noalloc_rejects_graphs_above_limit():
    f = _noalloc()
    err = C.create_string_buffer(256)
    n = (1 << 20) + 1
    s = f(C.c_void_p(16), C.c_void_p(16), n, 0, C.c_void_p(16), None, None, err, 256)
    assert s == gg.GG_ERR_ARG
    assert b"exceeds" in err.value
