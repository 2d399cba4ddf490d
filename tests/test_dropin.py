"""The reference's own analytics sources (bench/BFSLVLv.C, bench/BFSv.C),
unmodified, compiled against this library's Graptor-compatible headers
(graptor_b200/dropin/Makefile) and run on the GPU: their levels must equal
the oracle's and their parents must form a valid BFS tree."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "graptor_b200", "dropin", "_build")


def _prog(name):
    p = os.path.join(BUILD, name)
    if not os.path.exists(p):
        pytest.skip(f"drop-in build {name} absent (needs the reference sources at build time)")
    return p


def _run(prog, binpath, roots, prefix):
    r = subprocess.run([prog, binpath, prefix] + [str(x) for x in roots], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return {int(x): np.fromfile(f"{prefix}.{x}.i32", dtype=np.int32) for x in roots}


@pytest.mark.parametrize("gen", ["rmat", "grid"])
def test_reference_bfslvlv_source_on_gpu(tmp_path, gen):
    g = O.rmat(14, 16 << 14, seed=51) if gen == "rmat" else O.grid(60, 80, seed=3, del_bp=300)
    p = str(tmp_path / "g.bin")
    O.write_bin(g, p)
    deg = g.outdeg()
    roots = [int(np.argmax(deg)), int(np.flatnonzero(deg)[7]), int(np.flatnonzero(deg == 0)[0])
             if (deg == 0).any() else 1]
    out = _run(_prog("bfslvl"), p, roots, str(tmp_path / "lv"))
    for r in roots:
        assert np.array_equal(out[r], O.bfs_level(g, r))


def test_reference_bfsv_source_on_gpu(tmp_path):
    g = O.rmat(13, 16 << 13, seed=52)
    p = str(tmp_path / "g.bin")
    O.write_bin(g, p)
    roots = [0, 17]
    out = _run(_prog("bfsv"), p, roots, str(tmp_path / "pa"))
    for r in roots:
        lv = O.bfs_level(g, r)
        assert O.check_parents(g, r, out[r].view(np.uint32), lv) == 0
