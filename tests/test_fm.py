"""Flajolet-Martin neighbourhood estimation (the reference's bench/FMv.C) on
the library's edgemap / vertexmap: a[d] |= b[s] relax with the all-ones
destination filter, record a[d] != prev[d], and the estimate pass as one
vertex program with let-temporaries and uint32 bit operations.

The oracle's restatement (oracle.c orc_fm) is pinned to the reference's own
FMv build (oracle/harness/ref_fm.C) through the golden fixtures' fm_* keys:
final bit masks bit for bit, iteration counts, frontier sizes and deffG.
The GPU runs through the C ABI (every traversal variant) must give the same
masks, frontier sizes and running sums."""
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


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_fm_restatement_matches_reference_fixture(path):
    z = np.load(path)
    g = _graph(z)
    init = O.fm_draws(int(z["fm_padded"]))[z["fm_remap"]]
    mask, nhm, nactv, deffg = O.fm(g, init)
    assert np.array_equal(mask, z["fm_mask"])
    assert len(nhm) == int(z["fm_iters"])
    # the layout's padding vertices are active in the first iteration only
    assert int(z["fm_nactv"][0]) - int(nactv[0]) == int(z["fm_padded"]) - g.n
    assert np.array_equal(nactv[1:], z["fm_nactv"][1:])
    assert abs(deffg - float(z["fm_deffg"])) <= 1e-5 * max(1.0, abs(float(z["fm_deffg"])))


def test_fm_draws_are_geometric():
    d = O.fm_draws(1 << 16)
    assert (d & (d - 1) == 0).all()  # one bit (or none) per mask
    frac = [float(np.mean(d == (1 << i))) for i in range(4)]
    for i, f in enumerate(frac):
        assert abs(f - 2.0 ** -(i + 1)) < 0.01, frac
    assert np.array_equal(O.fm_draws(100), O.fm_draws(1000)[:100])  # one draw per vertex, in order


@pytest.mark.skipif(not O.ref_available("ref_fm"), reason="reference FMv harness not built")
@pytest.mark.parametrize("gen", ["rmat", "grid", "er"])
def test_fm_restatement_matches_reference_build(tmp_path, gen):
    g = {"rmat": lambda: O.rmat(11, 8 << 11, seed=21), "grid": lambda: O.grid(24, 50, seed=22, del_bp=400),
         "er": lambda: O.er(2500, 3.0, seed=23)}[gen]()
    p = str(tmp_path / "g.bin")
    O.write_bin(g, p)
    mask, remap, iters, deffg, nactv, padded = O.ref_fm(p, str(tmp_path / "fm"))
    m2, nhm, na2, dg2 = O.fm(g, O.fm_draws(padded)[remap])
    assert np.array_equal(mask, m2) and iters == len(nhm)
    assert np.array_equal(nactv[1:], na2[1:])
    assert abs(deffg - dg2) <= 1e-5 * max(1.0, abs(deffg))


# ---------------------------------------------------------------------------
# GPU, through the C ABI
# ---------------------------------------------------------------------------
def _estimate_program(gg, mask, prev, est):
    """FMv.C:386-412 as a vertex program: old = est; new = 2^(lowest zero
    bit of mask) / 0.77351 (mask 0: 2^32-1); prev = mask; est = float(new);
    reduce += new - old."""
    P = [(gg.VM_LOAD, 2), (gg.VM_TSET, 0),                                   # old_est
         (gg.VM_CONST, 0),                                                   # 1/phi
         (gg.VM_LOAD, 0), (gg.VM_CONST, 1), (gg.VM_NE, 0),                   # mask != 0
         (gg.VM_LOAD, 0), (gg.VM_NOT, 0),                                    # ~m
         (gg.VM_LOAD, 0), (gg.VM_NOT, 0), (gg.VM_LOAD, 0), (gg.VM_NOT, 0),
         (gg.VM_CONST, 2), (gg.VM_SUB, 0), (gg.VM_TOU32, 0),                 # ~m - 1
         (gg.VM_AND, 0), (gg.VM_XOR, 0),                                     # lowest set bit of ~m
         (gg.VM_CONST, 3), (gg.VM_SELECT, 0), (gg.VM_MUL, 0), (gg.VM_TSET, 1),
         (gg.VM_LOAD, 0), (gg.VM_STORE, 1),                                  # prev = mask
         (gg.VM_TGET, 1), (gg.VM_TOF32, 0), (gg.VM_STORE, 2),                # est = float(new)
         (gg.VM_TGET, 1), (gg.VM_TGET, 0), (gg.VM_SUB, 0), (gg.VM_REDUCE_ADD, 0)]
    d = gg.VmapDesc()
    d.ncode = len(P)
    for i, (c, a) in enumerate(P):
        d.code[i], d.arg[i] = c, a
    d.props[0], d.props[1], d.props[2] = mask.h, prev.h, est.h
    d.consts[0], d.consts[1], d.consts[2], d.consts[3] = 1.0 / 0.77351, 0.0, 1.0, 4294967295.0
    d.nreduce = 1
    return d


def fm_gpu(ctx, og, variant):
    from graptor_b200 import gg
    g = ctx.upload(og.off, og.adj)
    mask, prev, est = g.prop(gg.U32), g.prop(gg.U32), g.prop(gg.F32)
    init = O.fm_draws(og.n)
    mask.upload(init)
    prev.upload(init)
    est.fill(0.0)
    F, out = g.frontier(), g.frontier()
    F.set_all()
    prog = _estimate_program(gg, mask, prev, est)
    accum, nhm, nactv = 0.0, [], []
    while F.counts()[0]:
        nactv.append(F.counts()[0])
        d = gg.EmapDesc(relax=gg.RELAX_OR_U32, a=mask.h, src=prev.h, dst_filter=gg.FILTER_NE_CONST,
                        dst_filter_prop=mask.h, dst_filter_k=0xFFFFFFFF, record=gg.RECORD_NE_PREV,
                        prev=prev.h, variant=variant)
        g.edgemap(d, F, out)
        if out.counts()[0]:
            accum += float(g.vertexmap(prog, out)[0])
        nhm.append(np.float32(accum))
        F, out = out, F
        if len(nactv) > 4096:
            raise RuntimeError("no convergence")
    m = mask.download()
    g.close()
    return m, np.array(nhm, dtype=np.float32), np.array(nactv, dtype=np.uint64)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["auto", "push_sparse", "pull_dense", "push_dense"])
@pytest.mark.parametrize("gen", ["rmat", "grid"])
def test_fm_edgemap_matches_oracle(ctx, gen, variant):
    from graptor_b200 import gg
    og = O.rmat(14, 16 << 14, seed=31) if gen == "rmat" else O.grid(80, 90, seed=32, del_bp=300)
    v = {"auto": gg.VAR_AUTO, "push_sparse": gg.VAR_PUSH_SPARSE, "pull_dense": gg.VAR_PULL_DENSE,
         "push_dense": gg.VAR_PUSH_DENSE}[variant]
    mask, nhm, nactv = fm_gpu(ctx, og, v)
    m2, nhm2, na2, _ = O.fm(og, O.fm_draws(og.n))
    assert np.array_equal(mask, m2)
    assert np.array_equal(nactv, na2)
    # the sums run in another order on the device: float32 running sums agree to rounding
    assert np.allclose(nhm, nhm2, rtol=1e-6, atol=0)


@pytest.mark.gpu
def test_fm_or_relax_needs_uint32_source(ctx):
    from graptor_b200 import gg
    og = O.rmat(8, 8 << 8, seed=1)
    g = ctx.upload(og.off, og.adj)
    a, f = g.prop(gg.U32), g.prop(gg.F32)
    d = gg.EmapDesc(relax=gg.RELAX_OR_U32, a=a.h, src=f.h, record=gg.RECORD_NONE)
    with pytest.raises(gg.GGError) as e:
        g.edgemap(d)
    assert e.value.status == gg.GG_ERR_ARG
    d = gg.EmapDesc(relax=gg.RELAX_OR_U32, a=a.h, src=None, record=gg.RECORD_NONE)
    with pytest.raises(gg.GGError):
        g.edgemap(d)
    g.close()
