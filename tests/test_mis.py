"""Maximal independent set (the reference's bench/MISv.C) on the library's
edgemap: the MIS relation on uint8 states with the frontier as destination
filter and the undecided destinations recorded, then the vertex pass over the
frontier (conditionally in -> in, undecided -> conditionally in).

The rounds settle on the greedy set in priority order; the oracle's
restatement (oracle.c orc_mis) is pinned to the reference's own MISv build
(oracle/harness/ref_mis.C, whose priorities are its layout's vertex ids)
through the golden fixtures' mis_* keys.  The GPU runs (vertex ids as
priorities) must equal the restatement state for state."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _fixtures():
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if "customfp" not in p)


def _graph(z):
    if "off" in z:
        return O.Graph(int(z["n"]), z["off"], z["adj"])
    return O.rmat(int(z["scale"]), int(z["nedges"]), seed=int(z["seed"]))


def independent_and_maximal(g, st):
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.off.astype(np.int64)))
    dst = g.adj.astype(np.int64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    conflict = int(((st[src] == 3) & (st[dst] == 3)).sum())
    has_in = np.zeros(g.n, dtype=bool)
    np.logical_or.at(has_in, src, st[dst] == 3)
    missing = int(((st != 3) & ~has_in).sum())
    return conflict == 0 and missing == 0 and bool(np.isin(st, [2, 3]).all())


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_mis_restatement_matches_reference_fixture(path):
    z = np.load(path)
    g = _graph(z)
    st = O.mis(g, z["mis_remap"])
    assert np.array_equal(st, z["mis_state"])
    assert independent_and_maximal(g, st)


def test_mis_restatement_rejects_bad_priorities():
    g = O.rmat(6, 4 << 6, seed=1)
    with pytest.raises(RuntimeError):
        O.mis(g, np.zeros(g.n, dtype=np.uint32))


@pytest.mark.skipif(not O.ref_available("ref_mis"), reason="reference MISv harness not built")
@pytest.mark.parametrize("threads", [1, 8])
def test_mis_restatement_matches_reference_build(tmp_path, threads):
    for k, g in enumerate([O.rmat(11, 8 << 11, seed=41), O.grid(24, 50, seed=42, del_bp=400),
                           O.er(2500, 5.0, seed=43)]):
        p = str(tmp_path / f"g{k}.bin")
        O.write_bin(g, p)
        st, remap, _ = O.ref_mis(p, str(tmp_path / f"mis{k}"), threads=threads)
        assert np.array_equal(st, O.mis(g, remap))


# ---------------------------------------------------------------------------
# GPU, through the C ABI
# ---------------------------------------------------------------------------
def _state_program(gg, st):
    """MISv.C:284-312: conditionally in -> in, out stays out, else
    conditionally in."""
    P = [(gg.VM_LOAD, 0), (gg.VM_CONST, 1), (gg.VM_EQ, 0), (gg.VM_CONST, 3),
         (gg.VM_LOAD, 0), (gg.VM_CONST, 2), (gg.VM_EQ, 0), (gg.VM_CONST, 2), (gg.VM_CONST, 1),
         (gg.VM_SELECT, 0), (gg.VM_SELECT, 0), (gg.VM_STORE, 0)]
    d = gg.VmapDesc()
    d.ncode = len(P)
    for i, (c, a) in enumerate(P):
        d.code[i], d.arg[i] = c, a
    d.props[0] = st.h
    d.consts[0], d.consts[1], d.consts[2], d.consts[3] = 0.0, 1.0, 2.0, 3.0
    return d


def mis_gpu(ctx, og):
    from graptor_b200 import gg
    g = ctx.upload(og.off, og.adj)
    st = g.prop(gg.U8)
    st.fill(1)  # conditionally in
    F, out = g.frontier(), g.frontier()
    F.set_all()
    prog = _state_program(gg, st)
    rounds = 0
    while F.counts()[0]:
        d = gg.EmapDesc(relax=gg.RELAX_MIS_U8, a=st.h, dst_filter=gg.FILTER_IN_FRONTIER,
                        record=gg.RECORD_EQ_ZERO)
        g.edgemap(d, F, out)
        g.vertexmap(prog, F)
        F, out = out, F
        rounds += 1
        if rounds > og.n + 1:
            raise RuntimeError("no convergence")
    s = st.download()
    g.close()
    return s, rounds


@pytest.mark.gpu
@pytest.mark.parametrize("gen", ["rmat", "grid", "er", "edgecases"])
def test_mis_edgemap_matches_oracle(ctx, gen):
    og = {"rmat": lambda: O.rmat(15, 16 << 15, seed=44), "grid": lambda: O.grid(100, 120, seed=45, del_bp=200),
          "er": lambda: O.er(50000, 6.0, seed=46),
          "edgecases": lambda: O.Graph(int(np.load(os.path.join(GOLDEN, "edgecases32.npz"))["n"]),
                                       np.load(os.path.join(GOLDEN, "edgecases32.npz"))["off"],
                                       np.load(os.path.join(GOLDEN, "edgecases32.npz"))["adj"])}[gen]()
    st, rounds = mis_gpu(ctx, og)
    assert np.array_equal(st, O.mis(og))
    assert independent_and_maximal(og, st) and rounds >= 1


@pytest.mark.gpu
def test_mis_relax_contract(ctx):
    from graptor_b200 import gg
    og = O.rmat(8, 8 << 8, seed=1)
    g = ctx.upload(og.off, og.adj)
    bad = g.prop(gg.U32)
    with pytest.raises(gg.GGError) as e:
        g.edgemap(gg.EmapDesc(relax=gg.RELAX_MIS_U8, a=bad.h, record=gg.RECORD_NONE))
    assert e.value.status == gg.GG_ERR_ARG
    st = g.prop(gg.U8)
    F = g.frontier()
    F.set_single(0)
    with pytest.raises(gg.GGError) as e:  # a source frontier is not the relation's filter
        g.edgemap(gg.EmapDesc(relax=gg.RELAX_MIS_U8, a=st.h, record=gg.RECORD_NONE), F)
    assert e.value.status == gg.GG_ERR_UNSUPPORTED
    g.close()
