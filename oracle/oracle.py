"""Python handle on the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (built from ``oracle/oracle.c`` by
``oracle/Makefile``) and the reference-built programs under ``oracle/_ref/``.
Only the test suite, the smoke check and the benchmark's CPU-baseline leg
import this module; the GPU library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

# contribution storage formats of orc_pr_vary (must match oracle.c)
F32, F64, BF16, F16, FP8, CFP_6_10, BF16_TRUNC = range(7)

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        u64p = C.POINTER(C.c_uint64)
        u32p = C.POINTER(C.c_uint32)
        L.orc_gen_rmat.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                   C.c_uint64, C.c_int, u32p, u64p,
                                   C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_gen_er.argtypes = [C.c_uint32, C.c_double, C.c_uint32, C.c_uint64, C.c_int,
                                 u32p, u64p, C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_gen_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                   u32p, u64p, C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_transpose.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_write_bin.argtypes = [C.c_char_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p]
        L.orc_read_bin.argtypes = [C.c_char_p, u32p, u64p, C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_bfs_level.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_bfs_level_multi.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        L.orc_reached_edges.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p]
        L.orc_reached_edges.restype = C.c_uint64
        L.orc_check_parents.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                        C.c_void_p, C.c_void_p]
        L.orc_check_parents.restype = C.c_uint64
        L.orc_cc.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_pr_f32.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                 C.c_double, C.c_void_p, C.c_void_p]
        L.orc_pr_f64.argtypes = L.orc_pr_f32.argtypes
        L.orc_pr_vary.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                  C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_pr_vary_staged.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_cfp_from_float.argtypes = [C.c_float, C.c_int, C.c_int, C.c_int]
        L.orc_cfp_from_float.restype = C.c_uint32
        L.orc_cfp_to_float.argtypes = [C.c_uint32, C.c_int, C.c_int, C.c_int]
        L.orc_cfp_to_float.restype = C.c_float
        L.orc_pr_bf16_sr.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                     C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_cfp_convert_bits.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p]
        L.orc_fm.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_int]
        L.orc_fm_deffg.argtypes = [C.c_void_p, C.c_int]
        L.orc_fm_deffg.restype = C.c_float
        L.orc_mis.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mis.restype = C.c_int64
        L.orc_apr.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_kcore.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_kcore.restype = C.c_int64
        L.orc_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


@dataclass
class Graph:
    """Host CSR: off uint64[n+1], adj uint32[m]."""
    n: int
    off: np.ndarray
    adj: np.ndarray

    @property
    def m(self) -> int:
        return int(self.off[-1])

    def outdeg(self) -> np.ndarray:
        return np.diff(self.off).astype(np.uint32)

    def transpose(self) -> "Graph":
        L = lib()
        po, pa = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
        if L.orc_transpose(self.n, _p(self.off), _p(self.adj), C.byref(po), C.byref(pa)):
            raise MemoryError("orc_transpose")
        return _take(self.n, self.m, po, pa)


def _take(n, m, po, pa) -> Graph:
    L = lib()
    off = np.ctypeslib.as_array(po, shape=(n + 1,)).copy()
    adj = np.ctypeslib.as_array(pa, shape=(max(m, 1),))[:m].copy()
    L.orc_free(C.cast(po, C.c_void_p))
    L.orc_free(C.cast(pa, C.c_void_p))
    return Graph(n, off, adj)


def _gen(fn, *args) -> Graph:
    n, m = C.c_uint32(), C.c_uint64()
    po, pa = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    rc = fn(*args, C.byref(n), C.byref(m), C.byref(po), C.byref(pa))
    if rc:
        raise RuntimeError(f"generator failed ({rc})")
    return _take(n.value, m.value, po, pa)


def rmat(scale: int, nedges: int, seed: int, a=0.57, b=0.19, c=0.19, symmetric=True) -> Graph:
    return _gen(lib().orc_gen_rmat, scale, nedges, a, b, c, seed, int(symmetric))


def er(n: int, avgdeg: float, seed: int, dangling_bp: int = 0, symmetric=True) -> Graph:
    return _gen(lib().orc_gen_er, n, avgdeg, dangling_bp, seed, int(symmetric))


def grid(rows: int, cols: int, seed: int, del_bp: int = 0) -> Graph:
    return _gen(lib().orc_gen_grid, rows, cols, del_bp, seed)


def from_edges(n: int, edges, symmetric=True) -> Graph:
    """Small hand-made graphs for edge-case tests (dedup, no self-loops)."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if symmetric and len(e):
        e = np.concatenate([e, e[:, ::-1]])
    e = e[e[:, 0] != e[:, 1]] if len(e) else e
    if len(e):
        e = np.unique(e, axis=0)
    off = np.zeros(n + 1, dtype=np.uint64)
    if len(e):
        np.add.at(off, e[:, 0] + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    adj = e[:, 1].astype(np.uint32) if len(e) else np.zeros(0, dtype=np.uint32)
    return Graph(n, off, adj)


def write_bin(g: Graph, path: str) -> None:
    if lib().orc_write_bin(path.encode(), g.n, g.m, _p(g.off), _p(g.adj)):
        raise OSError(f"write_bin {path}")


def read_bin(path: str) -> Graph:
    n, m = C.c_uint32(), C.c_uint64()
    po, pa = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    rc = lib().orc_read_bin(path.encode(), C.byref(n), C.byref(m), C.byref(po), C.byref(pa))
    if rc:
        raise OSError(f"read_bin {path}: {rc}")
    return _take(n.value, m.value, po, pa)


def bfs_level(g: Graph, root: int) -> np.ndarray:
    lv = np.empty(g.n, dtype=np.int32)
    lib().orc_bfs_level(g.n, _p(g.off), _p(g.adj), root, _p(lv))
    return lv


def bfs_level_multi(g: Graph, roots) -> np.ndarray:
    """BFS levels with every root at level 0 (unreached n + 1)."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    lv = np.empty(g.n, dtype=np.int32)
    if lib().orc_bfs_level_multi(g.n, _p(g.off), _p(g.adj), _p(r), len(r), _p(lv)) < 0:
        raise ValueError("root out of range")
    return lv


def reached_edges(g: Graph, level: np.ndarray) -> int:
    level = np.ascontiguousarray(level, dtype=np.int32)
    return int(lib().orc_reached_edges(g.n, _p(g.off), _p(level)))


def check_parents(g: Graph, root: int, parent: np.ndarray, level: np.ndarray) -> int:
    parent = np.ascontiguousarray(parent, dtype=np.uint32)
    level = np.ascontiguousarray(level, dtype=np.int32)
    return int(lib().orc_check_parents(g.n, _p(g.off), _p(g.adj), root, _p(parent), _p(level)))


def cc(g: Graph) -> np.ndarray:
    lab = np.empty(g.n, dtype=np.uint32)
    lib().orc_cc(g.n, _p(g.off), _p(g.adj), _p(lab))
    return lab


def pagerank(g: Graph, maxiter: int = 20, tol: float = 1e-7, f64: bool = False,
             csc: Graph | None = None):
    """PRv-style power iteration; returns (x, iters, deltas)."""
    csc = csc if csc is not None else g.transpose()
    outdeg = g.outdeg()
    x = np.empty(g.n, dtype=np.float64 if f64 else np.float32)
    deltas = np.zeros(max(maxiter, 1), dtype=np.float64)
    fn = lib().orc_pr_f64 if f64 else lib().orc_pr_f32
    it = fn(g.n, _p(csc.off), _p(csc.adj), _p(outdeg), maxiter, tol, _p(x), _p(deltas))
    return x, it, deltas[:it]


def pagerank_vary(g: Graph, fmt: int, accum_f64: bool, maxiter: int = 100, tol: float = 1e-7,
                  csc: Graph | None = None):
    csc = csc if csc is not None else g.transpose()
    outdeg = g.outdeg()
    x = np.empty(g.n, dtype=np.float32)
    deltas = np.zeros(max(maxiter, 1), dtype=np.float64)
    it = lib().orc_pr_vary(g.n, _p(csc.off), _p(csc.adj), _p(outdeg), fmt, int(accum_f64),
                           maxiter, tol, _p(x), _p(deltas))
    return x, it, deltas[:it]


def pagerank_bf16_sr(g: Graph, stochastic: bool = True, maxiter: int = 100, tol: float = 1e-7,
                     average_last: int = 0, csc: Graph | None = None):
    """BF16 PageRank with stochastic rounding of the contributions and the
    mean of the last `average_last` iterations' ranks (the GPU library's
    extension).  Returns (x, iterations, deltas)."""
    csc = csc if csc is not None else g.transpose()
    outdeg = g.outdeg()
    x = np.empty(g.n, dtype=np.float32)
    deltas = np.zeros(max(maxiter, 1), dtype=np.float64)
    it = lib().orc_pr_bf16_sr(g.n, _p(csc.off), _p(csc.adj), _p(outdeg), int(stochastic), maxiter, tol,
                              average_last, _p(x), _p(deltas))
    return x, it, deltas[:it]


def pagerank_vary_staged(g: Graph, stages, maxiter: int = 100, tol: float = 1e-7, csc: Graph | None = None):
    """PR_vary staged run: stages = [(fmt, accum_f64, tol_k), ...]; the last
    stage runs until `tol`.  Returns (x, iterations, deltas)."""
    csc = csc if csc is not None else g.transpose()
    outdeg = g.outdeg()
    x = np.empty(g.n, dtype=np.float32)
    deltas = np.zeros(max(maxiter, 1), dtype=np.float64)
    f = np.array([s[0] for s in stages], dtype=np.int32)
    a = np.array([int(s[1]) for s in stages], dtype=np.int32)
    t = np.array([s[2] for s in stages], dtype=np.float64)
    it = lib().orc_pr_vary_staged(g.n, _p(csc.off), _p(csc.adj), _p(outdeg), len(stages), _p(f), _p(a), _p(t),
                                  maxiter, tol, _p(x), _p(deltas))
    return x, it, deltas[:it]


def cfp_from_float(f: float, S: int, E: int, M: int) -> int:
    return int(lib().orc_cfp_from_float(f, S, E, M))


def cfp_to_float(c: int, S: int, E: int, M: int) -> float:
    return float(lib().orc_cfp_to_float(c, S, E, M))


def cfp_convert_bits(bits: np.ndarray, S: int, E: int, M: int):
    """Encode the float bit patterns `bits` (uint32) into customfp<S,E,M>
    and decode them again: returns (codes, decoded float bit patterns)."""
    b = np.ascontiguousarray(bits, dtype=np.uint32)
    codes = np.empty_like(b)
    dec = np.empty_like(b)
    lib().orc_cfp_convert_bits(_p(b), len(b), S, E, M, _p(codes), _p(dec))
    return codes, dec


# ---------------------------------------------------------------------------
# The reference's own programs, built from its sources by oracle/Makefile.
# ---------------------------------------------------------------------------

def fm_draws(n: int) -> np.ndarray:
    """FMv's initial bit masks for draws 0..n-1 (oracle/fm_draws.cc: the C++
    standard library's mt19937_64 and uniform_int_distribution, as FMv.C
    draws them)."""
    p = os.path.join(os.path.dirname(LIB_PATH), "liboracle_fm.so")
    if not os.path.exists(p):
        raise RuntimeError(f"oracle library missing: {p} (run make -C oracle)")
    L = C.CDLL(p)
    L.orc_fm_draws.argtypes = [C.c_uint64, C.c_void_p]
    out = np.empty(max(n, 1), dtype=np.uint32)
    L.orc_fm_draws(n, _p(out))
    return out[:n]


def fm(g: Graph, init: np.ndarray, max_iters: int = 4096):
    """Flajolet-Martin neighbourhood estimation as FMv runs it (oracle.c
    orc_fm): returns (final masks, per-iteration running sums as float32,
    per-iteration frontier sizes, effective diameter deffG)."""
    init = np.ascontiguousarray(init, dtype=np.uint32)
    mask = np.empty(max(g.n, 1), dtype=np.uint32)
    nhm = np.zeros(max_iters, dtype=np.float32)
    nactv = np.zeros(max_iters, dtype=np.uint64)
    it = lib().orc_fm(g.n, _p(g.off), _p(g.adj), _p(init), _p(mask), _p(nhm), _p(nactv), max_iters)
    if it < 0:
        raise RuntimeError("orc_fm failed (allocation or iteration cap)")
    return mask[:g.n], nhm[:it], nactv[:it], float(lib().orc_fm_deffg(_p(nhm), it))


def ref_fm(bin_path: str, out_prefix: str, threads: int | None = None):
    """The reference FMv run by oracle/harness/ref_fm.C: returns (final masks
    in original order, layout id of each vertex, iterations, deffG, frontier
    sizes per iteration, padded vertex count)."""
    txt = _run([ref_prog("ref_fm"), bin_path, out_prefix], threads)
    head = next(l for l in txt.splitlines() if l.startswith("n "))
    w = head.split()
    nact = next(l for l in txt.splitlines() if l.startswith("nactv")).split()[1:]
    mask = np.fromfile(out_prefix + ".mask", dtype=np.uint32)
    remap = np.fromfile(out_prefix + ".remap", dtype=np.uint32)
    return mask, remap, int(w[5]), float(w[7]), np.array([int(x) for x in nact], dtype=np.uint64), int(w[3])


def mis(g: Graph, prio: np.ndarray | None = None) -> np.ndarray:
    """MISv's final states (2 out, 3 in): the greedy independent set in
    priority order (vertex ids when prio is None; oracle.c orc_mis)."""
    prio = np.arange(g.n, dtype=np.uint32) if prio is None else np.ascontiguousarray(prio, dtype=np.uint32)
    st = np.empty(max(g.n, 1), dtype=np.uint8)
    if lib().orc_mis(g.n, _p(g.off), _p(g.adj), _p(prio), _p(st)) < 0:
        raise RuntimeError("orc_mis failed (allocation, or prio not a permutation)")
    return st[:g.n]


def ref_mis(bin_path: str, out_path: str, threads: int | None = None):
    """The reference MISv run by oracle/harness/ref_mis.C: returns (states in
    original order, layout id of each vertex, iterations)."""
    txt = _run([ref_prog("ref_mis"), bin_path, out_path], threads)
    w = next(l for l in txt.splitlines() if l.startswith("n ")).split()
    return np.fromfile(out_path, dtype=np.uint8), np.fromfile(out_path + ".remap", dtype=np.uint32), int(w[5])


def apr(g: Graph, maxiter: int = 100, csc: Graph | None = None):
    """APRv's accelerated PageRank (oracle.c orc_apr): returns (x float32,
    iterations, per-iteration sum |delta|)."""
    csc = csc if csc is not None else g.transpose()
    x = np.empty(max(g.n, 1), dtype=np.float32)
    l1 = np.zeros(max(maxiter, 1), dtype=np.float64)
    outdeg = g.outdeg()
    it = lib().orc_apr(g.n, _p(csc.off), _p(csc.adj), _p(outdeg), maxiter, _p(x), _p(l1))
    if it < 0:
        raise RuntimeError("orc_apr failed")
    return x[:g.n], it, l1[:it]


def ref_apr(bin_path: str, out_path: str, maxiter: int = 100, threads: int | None = None):
    """Reference APRv (its driver, -pr:outfile): returns (x float64 in
    original order, iterations)."""
    args = [ref_prog("APRv"), "-s", "-b", "-rounds", "1", "-c", "256", "-pr:maxiter", str(maxiter),
            "-pr:outfile", out_path, "-itimes", bin_path]
    _, err = _run(args, threads, stderr=True)
    x = np.fromfile(out_path, dtype=np.float64, sep=" ")
    n = int(np.fromfile(bin_path, dtype=np.uint64, count=3)[2])
    if len(x) != n:
        raise PaddedGraph(f"reference padded {n} vertices to {len(x)}")
    its = sum(1 for l in err.splitlines() if l.startswith("Iteration "))
    return x, its


def kcore(g: Graph):
    """k-core decomposition (oracle.c orc_kcore, the KC_bucket restatement):
    returns (coreness uint32, largest coreness).  g symmetric."""
    core = np.empty(max(g.n, 1), dtype=np.uint32)
    k = lib().orc_kcore(g.n, _p(g.off), _p(g.adj), _p(core))
    if k < 0:
        raise RuntimeError("orc_kcore failed (allocation)")
    return core[:g.n], int(k)


def ref_kc(bin_path: str, out_path: str, threads: int | None = None):
    """Reference KC_bucket (its driver, -kc:outfile, KC_bucket.C:496-497):
    returns (coreness in original order, seconds of its run()).  The build's
    own validate() stops on an assertion (VL == storedVL, a restriction of
    its vector-length code) after the output is written: a run that wrote
    all n values is taken."""
    args = [ref_prog("KC_bucket"), "-s", "-b", "-rounds", "1", "-c", "256", "-kc:outfile", out_path, bin_path]
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if os.path.exists(out_path):
        os.remove(out_path)
    r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=1800)
    n = int(np.fromfile(bin_path, dtype=np.uint64, count=3)[2])
    core = np.fromfile(out_path, dtype=np.int64, sep=" ") if os.path.exists(out_path) else np.zeros(0)
    if len(core) != n:
        raise RuntimeError(f"KC_bucket wrote {len(core)} of {n} values, rc={r.returncode}: {r.stderr[-1500:]}")
    t = _running_times(r.stdout)
    return core.astype(np.uint32), (t[0] if t else None)


def ref_variant() -> str:
    """Pick the reference build the host CPU can execute (AVX-512 or AVX2)."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        flags = ""
    return "avx512" if " avx512f" in flags and " avx512bw" in flags else "avx2"


def ref_prog(name: str) -> str | None:
    p = os.path.join(REF_DIR, ref_variant(), name)
    return p if os.path.exists(p) else None


def ref_available(name: str = "ref_bfslvl") -> bool:
    return ref_prog(name) is not None


def _run(args, threads: int | None = None, timeout: int = 1800, stderr: bool = False):
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{args[0]} failed rc={r.returncode}: {r.stderr[-2000:]}")
    return (r.stdout, r.stderr) if stderr else r.stdout


class PaddedGraph(RuntimeError):
    """The reference's VEBO layout padded the vertex set (VEBOReorder.h:700-712);
    its PageRank then runs over the padded count and is not comparable."""


def ref_bfs(bin_path: str, roots, out_prefix: str | None = None, parents: bool = False,
            threads: int | None = None, checksums: bool = False):
    """Run the reference BFSLVLv (or BFSv) from each root.

    Returns a list of (root, seconds, reached, per-vertex int32 array or None);
    with checksums=True the last field is the pair of result checksums
    (level_checksums() of the reference's levels) and nothing is written."""
    prog = ref_prog("ref_bfsv" if parents else "ref_bfslvl")
    if prog is None:
        raise RuntimeError("reference BFS harness not built")
    outp = "+" if checksums else (out_prefix or "-")
    txt = _run([prog, bin_path, outp] + [str(r) for r in roots], threads)
    res = []
    for line in txt.splitlines():
        if line.startswith("n "):
            f = line.split()
            if int(f[1]) != int(f[3]):
                raise PaddedGraph(f"reference padded {f[1]} vertices to {f[3]}")
        if not line.startswith("root "):
            continue
        f = line.split()
        r, t, k = int(f[1]), float(f[3]), int(f[5])
        arr = None
        if checksums:
            arr = (int(f[7], 16), int(f[8], 16))
        elif out_prefix:
            arr = np.fromfile(f"{out_prefix}.{r}.i32", dtype=np.int32)
        res.append((r, t, k, arr))
    return res


def _mix64(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def level_checksums(values: np.ndarray):
    """The pair of checksums the reference BFS harness prints for a
    per-vertex int32 result: sum_v (uint32)values[v] * w_k(v) mod 2^64."""
    v = np.ascontiguousarray(values).view(np.uint32).astype(np.uint64)
    idx = np.arange(len(v), dtype=np.uint64)
    out = []
    with np.errstate(over="ignore"):
        for k in (1, 2):
            w = _mix64(idx + np.uint64((k * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF))
            out.append(int(np.sum(v * w, dtype=np.uint64)))
    return tuple(out)


def _running_times(txt: str):
    return [float(l.split(":")[1]) for l in txt.splitlines() if l.startswith("Running")]


def ref_cc(bin_path: str, out_path: str, threads: int | None = None, rounds: int = 1):
    """Reference CCv: returns (labels uint32 in original order, [round seconds])."""
    prog = ref_prog("CCv")
    txt = _run([prog, "-s", "-b", "-rounds", str(rounds), "-c", "256",
                "-cc:outfile", out_path, bin_path], threads)
    lab = np.fromfile(out_path, dtype=np.uint64, sep=" ").astype(np.uint32)
    n = int(np.fromfile(bin_path, dtype=np.uint64, count=3)[2])
    if len(lab) != n:
        raise PaddedGraph(f"reference padded {n} vertices to {len(lab)}")
    return lab, _running_times(txt)


def ref_pr(bin_path: str, out_path: str, maxiter: int = 20, threads: int | None = None,
           prog_name: str = "PRv", symmetric: bool = True, rounds: int = 1, iterations: bool = False):
    """Reference PRv / PR_vary: returns (x float64 array, [round seconds]), and
    with iterations=True also the iteration count of the last round (read from
    the per-iteration report that -itimes enables)."""
    prog = ref_prog(prog_name)
    args = [prog] + (["-s"] if symmetric else []) + [
        "-b", "-rounds", str(rounds), "-c", "256", "-pr:maxiter", str(maxiter),
        "-pr:outfile", out_path] + (["-itimes"] if iterations else []) + [bin_path]
    txt, err = _run(args, threads, stderr=True)
    x = np.fromfile(out_path, dtype=np.float64, sep=" ")
    n = int(np.fromfile(bin_path, dtype=np.uint64, count=3)[2])
    if len(x) != n:
        raise PaddedGraph(f"reference padded {n} vertices to {len(x)}")
    if not iterations:
        return x, _running_times(txt)
    its = [int(l.split("iterations:")[1].split()[0]) for l in err.splitlines() if "iterations:" in l]
    return x, _running_times(txt), (its[-1] if its else None)
