"""Regenerate the golden fixtures in tests/golden/ from the REFERENCE build.

Each fixture holds a seeded graph (CSR) and the outputs of the reference's own
programs on it, compiled from the reference sources by oracle/Makefile:
  bfs_levels   - BFSLVLv.C per root (harness oracle/harness/ref_bfs.C)
  bfsv_parents - BFSv.C per root (any valid BFS tree; checked, not compared)
  cc           - CCv.C -cc:outfile (canonical min-original-id labels)
  pr           - PRv.C -pr:outfile after pr_iters iterations
  pr_vary_<V>  - PR_vary.C -pr:outfile for VARIANT V (to the 1e-7 residual or
                 100 iterations), with pr_vary_<V>_iters its iteration count:
                 4620 (customfp<6,10> with float sums to 1e-3, then FP32 with
                 double sums), 99 (bfloat16-by-truncation contributions, float
                 sums) and 11 (FP64 throughout)
  fm_*         - FMv.C run by oracle/harness/ref_fm.C: the final bit mask of
                 each vertex (fm_mask), its layout id (fm_remap: the vertex
                 starts with FMv's initial draw number fm_remap[v]), the
                 iteration count, deffG and the frontier size per iteration
                 (fm_nactv; the first counts the layout's padding vertices,
                 fm_padded in all)
  mis_state    - MISv.C run by oracle/harness/ref_mis.C: the final state of
                 each vertex (2 out, 3 in), with mis_remap the layout id of
                 each vertex (MISv's priorities)
  apr_x        - APRv.C -pr:outfile (to sum |delta| < 1e-7 or 100 iterations),
                 with apr_iters its iteration count
  kc           - KC_bucket.C -kc:outfile (coreness of every vertex), with
                 kc_largest the largest
customfp_sweep.npz holds float bit patterns and, per pattern, the codes and
decoded floats of the reference's customfp<6,10> and scustomfp<true,8,7>
conversions (harness oracle/harness/ref_cfp.C).
The config-1 workload (R-MAT scale 16, 2^20 edges) is stored without its CSR
(7 MB): the fixture keeps the CSR's SHA-256 and the generator parameters.

Run (needs the reference tree and `make -C oracle ref`):
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --fm-only  # add / refresh the fm_* keys only
    python tests/golden/make_golden.py --mis-only # add / refresh the mis_* keys only
    python tests/golden/make_golden.py --apr-only # add / refresh the apr_* keys only
    python tests/golden/make_golden.py --kc-only  # add / refresh the kc* keys only
"""
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def csr_sha256(off, adj):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(adj, dtype=np.uint32).tobytes())
    return h.hexdigest()


def roots_for(g, k, seed):
    deg = g.outdeg()
    nz = np.flatnonzero(deg)
    rng = np.random.default_rng(seed)
    r = [int(np.argmax(deg))] + [int(x) for x in rng.choice(nz, size=min(k, len(nz)), replace=False)]
    return sorted(set(r), key=r.index)


PR_VARY = {"4620": "PR_vary", "99": "PR_vary_99", "11": "PR_vary_11"}


def run_reference(g, roots, pr_iters, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    lv = O.ref_bfs(p, roots, out_prefix=os.path.join(tmp, "lv"))
    pa = O.ref_bfs(p, roots, out_prefix=os.path.join(tmp, "pa"), parents=True)
    cc, _ = O.ref_cc(p, os.path.join(tmp, "cc.txt"))
    pr, _ = O.ref_pr(p, os.path.join(tmp, "pr.txt"), maxiter=pr_iters)
    vary = {}
    for v, prog in PR_VARY.items():
        x, _, it = O.ref_pr(p, os.path.join(tmp, "prv.txt"), maxiter=100, prog_name=prog, iterations=True)
        vary[f"pr_vary_{v}"] = x.astype(np.float64)
        vary[f"pr_vary_{v}_iters"] = np.int64(it)
    levels = np.stack([a for _, _, _, a in lv]).astype(np.int32)
    parents = np.stack([a for _, _, _, a in pa]).view(np.uint32)
    return levels, parents, cc.astype(np.uint32), pr, vary


def fm_reference(g, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    mask, remap, iters, deffg, nactv, padded = O.ref_fm(p, os.path.join(tmp, "fm"))
    # sanity: the restatement must agree before a fixture is written
    m2, _, na2, _ = O.fm(g, O.fm_draws(padded)[remap])
    assert np.array_equal(mask, m2) and np.array_equal(nactv[1:], na2[1:])
    return dict(fm_mask=mask, fm_remap=remap, fm_iters=np.int64(iters), fm_deffg=np.float64(deffg),
                fm_nactv=nactv, fm_padded=np.int64(padded))


def mis_reference(g, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    st, remap, _ = O.ref_mis(p, os.path.join(tmp, "mis"))
    assert np.array_equal(st, O.mis(g, remap))  # the restatement must agree
    return dict(mis_state=st, mis_remap=remap)


def apr_reference(g, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    x, its = O.ref_apr(p, os.path.join(tmp, "apr.txt"))
    xo, ito, _ = O.apr(g)
    assert ito == its and np.abs(xo - x).sum() < 1e-5  # the restatement must agree
    return dict(apr_x=x, apr_iters=np.int64(its))


def kc_reference(g, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    core, _ = O.ref_kc(p, os.path.join(tmp, "kc.txt"))
    mine, largest = O.kcore(g)
    assert np.array_equal(core, mine)  # the restatement must agree
    return dict(kc=core, kc_largest=np.int64(largest))


def add_keys(name, tmp, fn):
    path = os.path.join(HERE, name + ".npz")
    d = dict(np.load(path))
    if "off" in d:
        g = O.Graph(int(d["n"]), d["off"], d["adj"])
    else:
        g = O.rmat(int(d["scale"]), int(d["nedges"]), seed=int(d["seed"]))
        assert csr_sha256(g.off, g.adj) == str(d["sha256"]), name
    new = fn(g, tmp)
    d.update(new)
    np.savez_compressed(path, **d)
    print(name, sorted(new))


def save(name, g, roots, pr_iters, tmp, store_csr=True, params=None):
    levels, parents, cc, pr, vary = run_reference(g, roots, pr_iters, tmp)
    vary.update(fm_reference(g, tmp))
    vary.update(mis_reference(g, tmp))
    vary.update(apr_reference(g, tmp))
    vary.update(kc_reference(g, tmp))
    # sanity: the restatement must agree before a fixture is written
    for r, l in zip(roots, levels):
        assert np.array_equal(O.bfs_level(g, r), l), name
    d = dict(n=np.int64(g.n), m=np.int64(g.m), bfs_roots=np.array(roots, dtype=np.uint32),
             bfs_levels=levels, bfsv_parents=parents, cc=cc, pr=pr.astype(np.float64),
             pr_iters=np.int64(pr_iters), sha256=np.array(csr_sha256(g.off, g.adj)), **vary)
    if store_csr:
        d.update(off=g.off, adj=g.adj)
    if params:
        d.update({k: np.array(v) for k, v in params.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(name, g.n, g.m, "roots", roots)


def save_customfp_sweep(tmp):
    """Float bit patterns (special values, every exponent with a few
    mantissas, random patterns) and the reference's conversions of each."""
    rng = np.random.default_rng(2024)
    special = [0x00000000, 0x80000000, 0x3F800000, 0xBF800000, 0x40000000, 0x3FFFFFFF, 0x7F7FFFFF,
               0x7F800000, 0xFF800000, 0x7FC00000, 0x7F800001, 0x00000001, 0x007FFFFF, 0x00800000,
               0x1F800000, 0x20000000, 0x207FFFFF, 0x3F7FFFFF]
    exps = [(e << 23) | int(mt) for e in range(256) for mt in rng.integers(0, 1 << 23, size=8)]
    signs = [x | 0x80000000 for x in exps[::3]]
    rand = [int(x) for x in rng.integers(0, 1 << 32, size=4096, dtype=np.uint64)]
    bits = np.array(special + exps + signs + rand, dtype=np.uint32)
    i, o = os.path.join(tmp, "cfp.in"), os.path.join(tmp, "cfp.out")
    bits.tofile(i)
    subprocess.run([O.ref_prog("ref_cfp"), i, o], check=True)
    ref = np.fromfile(o, dtype=np.uint32).reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "customfp_sweep.npz"), bits=bits, cfp_6_10_code=ref[:, 0],
                        cfp_6_10_dec=ref[:, 1], bf16t_code=ref[:, 2], bf16t_dec=ref[:, 3])
    print("customfp_sweep", len(bits))


def main():
    if not O.ref_available("ref_bfslvl"):
        raise SystemExit("reference build missing: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        only = {"--fm-only": fm_reference, "--mis-only": mis_reference, "--apr-only": apr_reference,
                "--kc-only": kc_reference}
        for flag, fn in only.items():
            if flag in sys.argv:
                for name in ["rmat10_ef8", "rmat12_ef16", "grid20x32_del5pct", "er2000_deg6", "edgecases32",
                             "config1_rmat16"]:
                    add_keys(name, tmp, fn)
                return
        save_customfp_sweep(tmp)
        g = O.rmat(10, 8 << 10, seed=11)
        save("rmat10_ef8", g, roots_for(g, 3, 1), 20, tmp)
        g = O.rmat(12, 16 << 12, seed=12)
        save("rmat12_ef16", g, roots_for(g, 3, 2), 20, tmp)
        g = O.grid(20, 32, seed=13, del_bp=500)
        save("grid20x32_del5pct", g, roots_for(g, 2, 3), 20, tmp)
        g = O.er(2000, 6.0, seed=14)
        save("er2000_deg6", g, roots_for(g, 2, 4), 20, tmp)
        # edge cases: star, path, triangle, isolated vertices, a 2-vertex component
        edges = [(0, i) for i in range(1, 9)] + [(9, 10), (10, 11), (11, 12), (12, 13)] + \
                [(14, 15), (15, 16), (16, 14)] + [(20, 21)]
        g = O.from_edges(32, edges)
        save("edgecases32", g, [0, 9, 13, 14, 20, 22], 20, tmp)
        # config 1: R-MAT scale 16, 2^20 generated edges, root = max-degree vertex
        g = O.rmat(16, 1 << 20, seed=1)
        save("config1_rmat16", g, roots_for(g, 0, 0), 20, tmp, store_csr=False,
             params=dict(scale=16, nedges=1 << 20, seed=1))


if __name__ == "__main__":
    main()
