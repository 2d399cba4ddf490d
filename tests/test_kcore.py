"""k-core decomposition (the reference's bench/KC_bucket.C) on the library's
edgemap: the count of every vertex starts at its degree; for floors
k = 0, 1, 2, ... the vertices whose count is k are peeled and count their
neighbours down towards k (relax COUNT_DOWN with floor k, record AT_FLOOR,
KC_bucket.C:343-380), until no count reaches k.

The oracle's restatement (oracle.c orc_kcore, a sequential bucket peel) is
pinned to the reference's own KC_bucket build through the golden fixtures'
kc key and, where the build is present, on fresh graphs; the GPU runs must
equal it vertex for vertex under every traversal variant.  The reference
gives isolated vertices coreness 1 when fewer than n/2 vertices have a
degree above one (its degree-one preprocessing, KC_bucket.C:131-160); the
restatement and the library follow it (the edge-case fixture and the sparse
ER graphs below take that path)."""
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


def is_core_decomposition(g, core):
    """Every vertex of coreness c > 0 has at least c neighbours of coreness
    >= c (it lies in the c-core) and at most c neighbours of coreness > c
    (else it would lie in the (c+1)-core); isolated vertices are left out
    (the reference may give them 1)."""
    deg = np.diff(g.off.astype(np.int64))
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    dst = g.adj.astype(np.int64)
    ge = np.zeros(g.n, dtype=np.int64)
    gt = np.zeros(g.n, dtype=np.int64)
    np.add.at(ge, src, core[dst] >= core[src])
    np.add.at(gt, src, core[dst] > core[src])
    c = core.astype(np.int64)
    live = deg > 0
    return bool(((ge >= c) | ~live).all() and ((gt <= c) | ~live).all() and ((c <= deg) | ~live).all())


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_kcore_restatement_matches_reference_fixture(path):
    z = np.load(path)
    g = _graph(z)
    core, largest = O.kcore(g)
    assert np.array_equal(core, z["kc"])
    assert largest == int(z["kc_largest"])
    assert is_core_decomposition(g, core)


@pytest.mark.skipif(not O.ref_available("KC_bucket"), reason="reference KC_bucket not built")
def test_kcore_restatement_matches_reference_build(tmp_path):
    # vertex counts the reference's layout does not pad (powers of two)
    graphs = [O.rmat(12, 8 << 12, seed=51, a=0.65, b=0.15, c=0.15), O.grid(32, 64, seed=52, del_bp=2500),
              O.er(4096, 1.5, seed=53), O.rmat(11, 1 << 11, seed=54)]
    for k, g in enumerate(graphs):
        p = str(tmp_path / f"g{k}.bin")
        O.write_bin(g, p)
        ref, _ = O.ref_kc(p, str(tmp_path / f"kc{k}.txt"))
        assert np.array_equal(ref, O.kcore(g)[0]), k


def test_kcore_restatement_isolated_vertex_rule():
    # a triangle with a pendant and 28 isolated vertices: 3 of 32 vertices
    # have degree above one, so the reference reports coreness 1 for the
    # isolated ones; with most vertices of higher degree it reports 0
    g = O.from_edges(32, [(0, 1), (1, 2), (2, 0), (0, 3)])
    core, largest = O.kcore(g)
    assert core[:4].tolist() == [2, 2, 2, 1] and (core[4:] == 1).all() and largest == 2
    g = O.from_edges(6, [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 2)])
    core, _ = O.kcore(g)
    assert core.tolist() == [2, 2, 2, 2, 2, 0]


# ---------------------------------------------------------------------------
# GPU, through the C ABI
# ---------------------------------------------------------------------------
def _gen(name):
    return {"rmat16": lambda: O.rmat(16, 16 << 16, seed=55),
            "rmat14_skew": lambda: O.rmat(14, 16 << 14, seed=56, a=0.65, b=0.15, c=0.15),
            "grid": lambda: O.grid(90, 110, seed=57, del_bp=1500),
            "er_sparse": lambda: O.er(20000, 1.4, seed=58),   # most vertices of degree <= 1
            "er": lambda: O.er(30000, 8.0, seed=59)}[name]()


@pytest.mark.gpu
@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_kcore_matches_reference_fixture(ctx, path):
    z = np.load(path)
    og = _graph(z)
    g = ctx.upload(og.off, og.adj)
    core, largest = g.kcore()
    assert np.array_equal(core, z["kc"])
    assert largest == int(z["kc_largest"])
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("gen", ["rmat16", "rmat14_skew", "grid", "er_sparse", "er"])
def test_kcore_every_variant_matches_oracle(ctx, gen):
    from graptor_b200 import gg
    og = _gen(gen)
    want, largest = O.kcore(og)
    g = ctx.upload(og.off, og.adj)
    runs = [gg.default_opts(), gg.default_opts(gg.THRESH_ALWAYS_SPARSE), gg.default_opts(gg.THRESH_ALWAYS_DENSE),
            gg.default_opts(variant=gg.VAR_PUSH_SPARSE), gg.default_opts(variant=gg.VAR_PUSH_MERGE),
            gg.default_opts(variant=gg.VAR_PULL_DENSE), gg.default_opts(variant=gg.VAR_PUSH_DENSE),
            gg.default_opts(collect=True)]
    for opts in runs:
        st = gg.RunStats()
        core, lc = g.kcore(opts=opts, stats=st)
        assert np.array_equal(core, want), (gen, opts.threshold, opts.variant)
        assert lc == largest
        assert st.iterations >= 1 and st.total_ms > 0
    prop = g.prop(gg.U32)
    core, _ = g.kcore(coreness=prop, host=False)
    assert core is None and np.array_equal(prop.download(), want)
    g.close()


def _count_down_step(og, a, active, k):
    """One COUNT_DOWN step on the host: every vertex above the floor k loses
    one per active in-neighbour, not below k."""
    deg = np.diff(og.off.astype(np.int64))
    src = np.repeat(np.arange(og.n, dtype=np.int64), deg)
    dst = og.adj.astype(np.int64)
    takes = np.zeros(og.n, dtype=np.int64)
    np.add.at(takes, dst, active[src])
    a64 = a.astype(np.int64)
    new = np.where(a64 > k, np.maximum(k, a64 - takes), a64)
    return new.astype(np.uint32), (a64 > k) & (new == k), (a64 > k) & (takes > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_count_down_step_semantics(ctx, variant):
    """One edgemap step with COUNT_DOWN from a random frontier on random
    counts: the counts, the AT_FLOOR record (the vertices that reached the
    floor now) and the REDUCTION record (every vertex counted down)."""
    from graptor_b200 import gg
    og = O.rmat(13, 16 << 13, seed=60)
    g = ctx.upload(og.off, og.adj)
    rng = np.random.default_rng(61)
    for k in (0, 3, 17):
        a0 = rng.integers(0, 40, size=og.n).astype(np.uint32)
        active = rng.random(og.n) < 0.3
        want, at_floor, counted = _count_down_step(og, a0, active, k)
        for record, rec_want in ((gg.RECORD_AT_FLOOR, at_floor), (gg.RECORD_REDUCTION, counted)):
            a = g.prop(gg.U32)
            a.upload(a0)
            F, out = g.frontier(), g.frontier()
            F.set_list(np.flatnonzero(active).astype(np.uint32))
            d = gg.EmapDesc(relax=gg.RELAX_COUNT_DOWN_U32, a=a.h, dst_filter=gg.FILTER_GT_CONST, dst_filter_k=k,
                            record=record, variant=variant)
            g.edgemap(d, F, out)
            assert np.array_equal(a.download(), want), (k, record, variant)
            assert np.array_equal(np.sort(out.download()), np.flatnonzero(rec_want)), (k, record, variant)
            F.close()
            out.close()
            a.close()
    g.close()


@pytest.mark.gpu
def test_kcore_contract(ctx):
    from graptor_b200 import gg
    og = O.er(500, 4.0, seed=62, symmetric=False)
    g = ctx.upload(og.off, og.adj, symmetric=False)
    with pytest.raises(gg.GGError) as e:
        g.kcore()
    assert e.value.status == gg.GG_ERR_UNSUPPORTED
    g.close()
    og = O.rmat(8, 8 << 8, seed=63)
    g = ctx.upload(og.off, og.adj)
    with pytest.raises(gg.GGError) as e:
        g.kcore(coreness=g.prop(gg.I32))
    assert e.value.status == gg.GG_ERR_ARG
    a = g.prop(gg.U32)
    F, out = g.frontier(), g.frontier()
    F.set_single(0)
    with pytest.raises(gg.GGError) as e:  # the floor comes with the GT_CONST filter
        g.edgemap(gg.EmapDesc(relax=gg.RELAX_COUNT_DOWN_U32, a=a.h, record=gg.RECORD_AT_FLOOR), F, out)
    assert e.value.status == gg.GG_ERR_ARG
    lv = g.prop(gg.I32)
    with pytest.raises(gg.GGError) as e:  # AT_FLOOR belongs to COUNT_DOWN
        g.edgemap(gg.EmapDesc(relax=gg.RELAX_MIN_PLUS1_I32, a=lv.h, dst_filter=gg.FILTER_GT_CONST, dst_filter_k=1,
                              record=gg.RECORD_AT_FLOOR), F, out)
    assert e.value.status == gg.GG_ERR_UNSUPPORTED
    g.close()
