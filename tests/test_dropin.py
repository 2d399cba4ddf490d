"""The reference's own analytics sources (bench/BFSLVLv.C, BFSv.C, CCv.C,
PRv.C, PR_vary.C), unmodified, compiled against this library's
Graptor-compatible headers with the reference's own bench/driver.C as their
main() (graptor_b200/dropin/Makefile) and run on the GPU: BFS levels equal the
oracle's, BFS parents form a valid BFS tree, CC labels equal the reference
build's bit for bit, PageRank ranks are within the stated L1 of the reference
build's, and every program's own validate() passes."""
import glob
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


GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden_graphs():
    return [os.path.basename(p)[:-4] for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
            if "config1" not in p and "customfp" not in p]


def _graph_file(tmp_path, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = O.Graph(int(z["n"]), z["off"], z["adj"])
    p = str(tmp_path / "g.bin")
    O.write_bin(g, p)
    return z, g, p


def _driver(prog, args):
    """Runs a drop-in program through the reference's driver main()."""
    r = subprocess.run([_prog(prog)] + args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (prog, r.stdout[-1000:], r.stderr[-2000:])
    assert "Running :" in r.stdout, r.stdout[-1000:]
    return r


@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_ccv_source_on_gpu(tmp_path, name):
    """CCv.C with its driver: canonical labels (-cc:outfile, CCv.C:591-601)
    equal the reference build's; its validate() neighbour check passes."""
    z, g, p = _graph_file(tmp_path, name)
    out = str(tmp_path / "cc.txt")
    r = _driver("CCv", ["-s", "-b", "-rounds", "2", "-cc:outfile", out, p])
    assert "Neighbour check: PASS" in r.stderr, r.stderr[-2000:]
    lab = np.loadtxt(out, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(lab, z["cc"])


@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_prv_source_on_gpu(tmp_path, name):
    """PRv.C with its driver, 20 iterations: ranks within 1e-6 L1 of the
    reference build's PRv."""
    z, g, p = _graph_file(tmp_path, name)
    out = str(tmp_path / "pr.txt")
    _driver("PRv", ["-s", "-b", "-rounds", "1", "-pr:maxiter", str(int(z["pr_iters"])), "-pr:outfile", out, p])
    x = np.loadtxt(out, dtype=np.float64)
    assert np.abs(x - z["pr"]).sum() <= 1e-6


# drop-in program -> (fixture key, L1 bar against the reference build's output)
PR_VARY_PROGS = {"PR_vary": ("4620", 1e-6), "PR_vary_99": ("99", 2e-6), "PR_vary_11": ("11", 1e-11)}


@pytest.mark.parametrize("prog", sorted(PR_VARY_PROGS))
@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_pr_vary_source_on_gpu(tmp_path, name, prog):
    """PR_vary.C with its driver, built for VARIANT 4620 (the default), 99 and
    11: ranks to the 1e-7 residual against the reference build of the same
    variant, iteration counts within one."""
    z, g, p = _graph_file(tmp_path, name)
    key, bar = PR_VARY_PROGS[prog]
    out = str(tmp_path / "prv.txt")
    r = _driver(prog, ["-s", "-b", "-rounds", "1", "-itimes", "-pr:outfile", out, p])
    its = [int(l.split("iterations:")[1].split()[0]) for l in r.stderr.splitlines() if "iterations:" in l]
    assert its and abs(its[-1] - int(z[f"pr_vary_{key}_iters"])) <= 1, (its, int(z[f"pr_vary_{key}_iters"]))
    x = np.loadtxt(out, dtype=np.float64)
    assert np.abs(x - z[f"pr_vary_{key}"]).sum() <= bar


@pytest.mark.parametrize("prog", ["BFSLVLv", "BFSv"])
def test_reference_bfs_sources_with_their_driver(tmp_path, prog):
    """BFSLVLv.C / BFSv.C with the reference's driver main() (no harness):
    runs from -start and its own validate() passes."""
    z, g, p = _graph_file(tmp_path, "rmat12_ef16")
    r = _driver(prog, ["-s", "-b", "-rounds", "2", "-start", str(int(z["bfs_roots"][0])), p])
    assert "FAIL" not in (r.stdout + r.stderr), (r.stdout[-1000:], r.stderr[-1000:])


def _fm_lines(txt):
    head = next(l for l in txt.splitlines() if l.startswith("n ")).split()
    nact = next(l for l in txt.splitlines() if l.startswith("nactv")).split()[1:]
    return int(head[5]), float(head[7]), np.array([int(x) for x in nact], dtype=np.uint64)


@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_fmv_source_on_gpu(tmp_path, name):
    """FMv.C run on the GPU by the fm harness: with the same initial draws in
    vertex order, the final bit masks equal the oracle's bit for bit (the
    oracle is pinned to the reference build), as do the iteration count and
    the frontier sizes; deffG agrees to float rounding of the running sums."""
    z, g, p = _graph_file(tmp_path, name)
    r = subprocess.run([_prog("fm"), p, str(tmp_path / "fm")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    iters, deffg, nactv = _fm_lines(r.stdout)
    mask = np.fromfile(str(tmp_path / "fm.mask"), dtype=np.uint32)
    m2, nhm, na2, dg2 = O.fm(g, O.fm_draws(g.n))
    assert np.array_equal(mask, m2)
    assert iters == len(nhm) and np.array_equal(nactv, na2)
    assert abs(deffg - dg2) <= 1e-4 * max(1.0, abs(dg2))


def test_reference_fmv_with_its_driver(tmp_path):
    """FMv.C with the reference's driver main(): two rounds, each deffG as the
    oracle's."""
    z, g, p = _graph_file(tmp_path, "grid20x32_del5pct")
    r = _driver("FMv", ["-s", "-b", "-rounds", "2", p])
    got = [float(l.split("deffG:")[1]) for l in r.stderr.splitlines() if l.startswith("deffG:")]
    _, _, _, dg = O.fm(g, O.fm_draws(g.n))
    assert len(got) == 2 and all(abs(x - dg) <= 1e-4 * max(1.0, abs(dg)) for x in got), (got, dg)


@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_misv_source_on_gpu(tmp_path, name):
    """MISv.C run on the GPU by the mis harness: its own validate() passes
    and the states equal the oracle's greedy set in vertex-id order (the
    oracle is pinned to the reference build with the reference's priorities)."""
    z, g, p = _graph_file(tmp_path, name)
    out = str(tmp_path / "mis.u8")
    r = subprocess.run([_prog("mis"), p, out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "result: PASS" in r.stderr, r.stderr[-2000:]
    assert np.array_equal(np.fromfile(out, dtype=np.uint8), O.mis(g))


def test_reference_misv_with_its_driver(tmp_path):
    """MISv.C with the reference's driver main(): validate() passes in each round."""
    z, g, p = _graph_file(tmp_path, "rmat12_ef16")
    r = _driver("MISv", ["-s", "-b", "-rounds", "2", p])
    assert r.stderr.count("result: PASS") == 2, r.stderr[-2000:]


@pytest.mark.parametrize("name", _golden_graphs())
def test_reference_aprv_source_on_gpu(tmp_path, name):
    """APRv.C with its driver: ranks within 2e-6 L1 of the reference build's
    APRv, iteration counts within one."""
    z, g, p = _graph_file(tmp_path, name)
    out = str(tmp_path / "apr.txt")
    r = _driver("APRv", ["-s", "-b", "-rounds", "1", "-itimes", "-pr:outfile", out, p])
    its = sum(1 for l in r.stderr.splitlines() if l.startswith("Iteration "))
    assert abs(its - int(z["apr_iters"])) <= 1, (its, int(z["apr_iters"]))
    x = np.loadtxt(out, dtype=np.float64)
    assert np.abs(x - z["apr_x"]).sum() <= 2e-6
