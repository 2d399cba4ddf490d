"""Regenerate the golden fixtures in tests/golden/ from the REFERENCE build.

Each fixture holds a seeded graph (CSR) and the outputs of the reference's own
programs on it, compiled from the reference sources by oracle/Makefile:
  bfs_levels   - BFSLVLv.C per root (harness oracle/harness/ref_bfs.C)
  bfsv_parents - BFSv.C per root (any valid BFS tree; checked, not compared)
  cc           - CCv.C -cc:outfile (canonical min-original-id labels)
  pr           - PRv.C -pr:outfile after pr_iters iterations
The config-1 workload (R-MAT scale 16, 2^20 edges) is stored without its CSR
(7 MB): the fixture keeps the CSR's SHA-256 and the generator parameters.

Run (needs the reference tree and `make -C oracle ref`):
    python tests/golden/make_golden.py
"""
import hashlib
import os
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


def run_reference(g, roots, pr_iters, tmp):
    p = os.path.join(tmp, "g.bin")
    O.write_bin(g, p)
    lv = O.ref_bfs(p, roots, out_prefix=os.path.join(tmp, "lv"))
    pa = O.ref_bfs(p, roots, out_prefix=os.path.join(tmp, "pa"), parents=True)
    cc, _ = O.ref_cc(p, os.path.join(tmp, "cc.txt"))
    pr, _ = O.ref_pr(p, os.path.join(tmp, "pr.txt"), maxiter=pr_iters)
    levels = np.stack([a for _, _, _, a in lv]).astype(np.int32)
    parents = np.stack([a for _, _, _, a in pa]).view(np.uint32)
    return levels, parents, cc.astype(np.uint32), pr


def save(name, g, roots, pr_iters, tmp, store_csr=True, params=None):
    levels, parents, cc, pr = run_reference(g, roots, pr_iters, tmp)
    # sanity: the restatement must agree before a fixture is written
    for r, l in zip(roots, levels):
        assert np.array_equal(O.bfs_level(g, r), l), name
    d = dict(n=np.int64(g.n), m=np.int64(g.m), bfs_roots=np.array(roots, dtype=np.uint32),
             bfs_levels=levels, bfsv_parents=parents, cc=cc, pr=pr.astype(np.float64),
             pr_iters=np.int64(pr_iters), sha256=np.array(csr_sha256(g.off, g.adj)))
    if store_csr:
        d.update(off=g.off, adj=g.adj)
    if params:
        d.update({k: np.array(v) for k, v in params.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(name, g.n, g.m, "roots", roots)


def main():
    if not O.ref_available("ref_bfslvl"):
        raise SystemExit("reference build missing: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
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
