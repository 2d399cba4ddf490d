"""Accelerated (delta) PageRank (the reference's bench/APRv.C) on the
library: the contribution gather over all in-edges or over the in-edges from
the frontier only (ADD_GATHER with a source frontier), vertex passes with
predicated updates, and the active set written as a dense logical array that
becomes the next frontier.

The oracle's float restatement (oracle.c orc_apr) is pinned to the
reference's own APRv build through the golden fixtures' apr_* keys: the same
iteration count, ranks within float rounding of the sums' order."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
L1_BAR = 2e-6  # float32 ranks, summed in another order


def _fixtures():
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if "customfp" not in p)


def _graph(z):
    if "off" in z:
        return O.Graph(int(z["n"]), z["off"], z["adj"])
    return O.rmat(int(z["scale"]), int(z["nedges"]), seed=int(z["seed"]))


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_apr_restatement_matches_reference_fixture(path):
    z = np.load(path)
    x, it, l1 = O.apr(_graph(z))
    assert it == int(z["apr_iters"])
    assert np.abs(x - z["apr_x"]).sum() <= L1_BAR
    assert l1[-1] < 1e-7 or it == 100


@pytest.mark.skipif(not O.ref_available("APRv"), reason="reference APRv not built")
def test_apr_restatement_matches_reference_build(tmp_path):
    g = O.er(4096, 5.0, seed=51)  # a multiple of the layout's vector length: no padding
    p = str(tmp_path / "g.bin")
    O.write_bin(g, p)
    xr, its = O.ref_apr(p, str(tmp_path / "x.txt"))
    x, it, _ = O.apr(g)
    assert it == its and np.abs(x - xr).sum() <= L1_BAR


@pytest.mark.gpu
@pytest.mark.parametrize("accum_f64", [0, 1])
def test_gather_with_source_frontier(ctx, accum_f64):
    """y[d] += sum of contrib[s] over in-edges from the frontier's vertices."""
    from graptor_b200 import gg
    og = O.rmat(14, 16 << 14, seed=52)
    g = ctx.upload(og.off, og.adj)
    rng = np.random.default_rng(5)
    c = rng.random(og.n).astype(np.float32)
    y0 = rng.random(og.n).astype(np.float32)
    act = np.flatnonzero(rng.random(og.n) < 0.1).astype(np.uint32)
    cp, yp = g.prop(gg.F32), g.prop(gg.F32)
    cp.upload(c)
    yp.upload(y0)
    F = g.frontier()
    F.set_list(act)
    g.edgemap(gg.EmapDesc(relax=gg.RELAX_ADD_GATHER, a=yp.h, src=cp.h, accum_f64=accum_f64,
                          record=gg.RECORD_NONE), F)
    mask = np.zeros(og.n, dtype=bool)
    mask[act] = True
    csc = og.transpose()
    dst = np.repeat(np.arange(og.n), np.diff(csc.off.astype(np.int64)))
    keep = mask[csc.adj]
    want = y0.astype(np.float64)
    np.add.at(want, dst[keep], c[csc.adj[keep]].astype(np.float64))
    got = yp.download().astype(np.float64)
    assert np.allclose(got, want, rtol=2e-6, atol=0)
    untouched = np.ones(og.n, dtype=bool)
    untouched[dst[keep]] = False
    assert np.array_equal(got[untouched], y0[untouched].astype(np.float64))
    g.close()
