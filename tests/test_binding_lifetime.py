"""CPU test of the ctypes binding's handle lifetimes: destroying a context
first destroys its graphs and their properties/frontiers, and no C call
reaches a destroyed context afterwards (checked against a fake library)."""
import ctypes as C
import gc

import pytest

from graptor_b200 import gg


class FakeLib:
    def __init__(self):
        self.live_ctx, self.live = set(), {}
        self.log = []
        self.next = 100

    def _new(self, kind, parent, out):
        self.next += 1
        self.live[self.next] = (kind, parent)
        out._obj.value = self.next
        return 0

    def gg_ctx_create(self, dev, out):
        self.next += 1
        self.live_ctx.add(self.next)
        out._obj.value = self.next
        return 0

    def _check_parent_alive(self, h):
        kind, parent = self.live[h]
        while kind != "ctx":
            if parent in self.live_ctx:
                return
            kind, parent = self.live.get(parent, ("dead", None))
            if kind == "dead":
                raise AssertionError("call on a handle whose context is gone")

    def gg_ctx_destroy(self, h):
        h = h.value if hasattr(h, "value") else h
        self.log.append(("ctx_destroy", h))
        assert all(p != h for (_, p) in self.live.values()), "graph outlived its context"
        self.live_ctx.discard(h)
        return 0

    def gg_graph_upload(self, ctx, n, m, off, adj, sym, out):
        return self._new("graph", ctx.value, out)

    def gg_graph_info(self, h, n, m, sym):
        n._obj.value, m._obj.value, sym._obj.value = 4, 0, 1
        return 0

    def gg_graph_destroy(self, h):
        h = h.value
        assert all(p != h for (_, p) in self.live.values()), "prop/frontier outlived its graph"
        self._check_parent_alive(h)
        del self.live[h]
        self.log.append(("graph_destroy", h))
        return 0

    def gg_prop_create(self, g, dt, out):
        return self._new("prop", g.value, out)

    def gg_frontier_create(self, g, out):
        return self._new("frontier", g.value, out)

    def gg_prop_destroy(self, h):
        self._check_parent_alive(h.value)
        del self.live[h.value]
        return 0

    gg_frontier_destroy = gg_prop_destroy

    def gg_last_error(self, h):
        return b""

    def gg_status_string(self, s):
        return b"X"


@pytest.fixture
def fake(monkeypatch):
    f = FakeLib()
    monkeypatch.setattr(gg, "lib", lambda: f)
    return f


def _ptr(v):
    import numpy as np
    return np.zeros(v, dtype=np.uint64)


def test_ctx_close_destroys_children_first(fake):
    import numpy as np
    ctx = gg.Context(0)
    g = ctx.upload(np.zeros(5, dtype=np.uint64), np.zeros(0, dtype=np.uint32))
    p, f = g.prop(gg.I32), g.frontier()
    ctx.close()  # must destroy p, f, g before the context
    assert not fake.live and not fake.live_ctx
    del p, f, g
    gc.collect()  # later finalisers must not call into the destroyed context


def test_garbage_collection_any_order(fake):
    import numpy as np
    ctx = gg.Context(0)
    g = ctx.upload(np.zeros(5, dtype=np.uint64), np.zeros(0, dtype=np.uint32))
    props = [g.prop(gg.F32) for _ in range(3)]
    del g
    gc.collect()
    assert len(fake.live) == 4  # still referenced through props
    props[0].close()
    del props
    gc.collect()
    ctx.close()
    assert not fake.live and not fake.live_ctx
