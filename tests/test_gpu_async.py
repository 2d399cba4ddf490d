"""gg_bfs_level_host_async: BFS levels delivered to host memory with the copy
running behind the next call.  Each call's host buffer, read once the next
call (or the wait) has returned, equals the oracle's levels and the
synchronous entry point's, with page-locked and with pageable buffers."""
import numpy as np
import pytest

from graptor_b200 import gg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pinned", [True, False])
def test_async_levels_match_each_call(ctx, pinned):
    torch = pytest.importorskip("torch")
    og = O.rmat(15, 16 << 15, seed=71)
    g = ctx.upload(og.off, og.adj)
    deg = og.outdeg()
    roots = [int(r) for r in np.random.default_rng(3).choice(np.flatnonzero(deg), 7, replace=False)]
    roots.append(int(np.flatnonzero(deg == 0)[0]) if (deg == 0).any() else 0)  # an isolated root
    if pinned:
        bufs = [torch.empty(g.n, dtype=torch.int32, pin_memory=True).numpy() for _ in range(2)]
    else:
        bufs = [np.empty(g.n, dtype=np.int32) for _ in range(2)]
    prev = None
    for k, r in enumerate(roots):
        st = gg.RunStats()
        g.bfs_level_host_async(r, out=bufs[k % 2], stats=st)
        assert st.iterations >= 1
        if prev is not None:  # the previous call's copy has landed
            pk, pr = prev
            assert np.array_equal(bufs[pk % 2], O.bfs_level(og, pr)), pr
        prev = (k, r)
    g.bfs_level_host_wait()
    pk, pr = prev
    assert np.array_equal(bufs[pk % 2], O.bfs_level(og, pr))
    assert np.array_equal(bufs[pk % 2], g.bfs_level(pr))
    g.bfs_level_host_wait()  # nothing pending: returns at once
    g.close()
