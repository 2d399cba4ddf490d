"""Ingest with cleaning on the device: duplicates and self-loops dropped,
optional symmetrisation, from host or device edge lists and from dirty .bin
files; the CSR must equal the oracle's cleaned graph exactly."""
import os

import numpy as np
import pytest

from graptor_b200 import gg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def dirty_edges(n, k, seed):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, k, dtype=np.int64)
    dst = rng.integers(0, n, k, dtype=np.int64)
    # duplicates and self-loops on purpose
    src = np.concatenate([src, src[:k // 4], np.arange(0, n, 7)])
    dst = np.concatenate([dst, dst[:k // 4], np.arange(0, n, 7)])
    return src, dst


@pytest.mark.parametrize("sym", [True, False])
def test_from_edges_host(ctx, sym):
    n = 3000
    src, dst = dirty_edges(n, 20000, 1)
    g = ctx.from_edges(n, src, dst, symmetrise=sym)
    ref = O.from_edges(n, np.stack([src, dst], 1), symmetric=sym)
    off, adj = g.download()
    assert g.symmetric == sym
    assert np.array_equal(off, ref.off) and np.array_equal(adj, ref.adj)
    assert np.array_equal(g.bfs_level(0), O.bfs_level(ref, 0))
    g.close()


def test_from_edges_device_and_bad_ids(ctx):
    torch = pytest.importorskip("torch")
    n = 5000
    src, dst = dirty_edges(n, 40000, 2)
    ts = torch.tensor(src.astype(np.int32), device="cuda").contiguous()
    td = torch.tensor(dst.astype(np.int32), device="cuda").contiguous()
    torch.cuda.synchronize()
    g = ctx.from_edges(n, (ts.data_ptr(), len(src)), (td.data_ptr(), len(dst)), symmetrise=True, device=True)
    ref = O.from_edges(n, np.stack([src, dst], 1), symmetric=True)
    off, adj = g.download()
    assert np.array_equal(off, ref.off) and np.array_equal(adj, ref.adj)
    g.close()
    td[5] = n + 3  # out of range: reported, not written anywhere
    torch.cuda.synchronize()
    with pytest.raises(gg.GGError):
        ctx.from_edges(n, (ts.data_ptr(), len(src)), (td.data_ptr(), len(dst)), device=True)
    with pytest.raises(gg.GGError):
        ctx.from_edges(10, [1, 2], [3, 10])


def test_read_bin_clean(ctx, tmp_path):
    n = 2000
    src, dst = dirty_edges(n, 15000, 3)
    order = np.lexsort((dst, src))
    s_, d_ = src[order], dst[order]
    off = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(off, s_ + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    path = os.path.join(tmp_path, "dirty.bin")
    with open(path, "wb") as f:
        np.array([2, 1, n, len(s_), 4, 8, 0, 0], dtype=np.uint64).tofile(f)
        off[:-1].tofile(f)
        d_.astype(np.uint32).tofile(f)
    g = ctx.read_bin_clean(path, symmetrise=True)
    ref = O.from_edges(n, np.stack([src, dst], 1), symmetric=True)
    o2, a2 = g.download()
    assert np.array_equal(o2, ref.off) and np.array_equal(a2, ref.adj)
    assert np.array_equal(g.cc(), O.cc(ref))
    g.close()
