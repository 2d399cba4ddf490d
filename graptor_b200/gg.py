"""ctypes binding of the C ABI in include/gg.h (libgg.so).

This is the FFI a Python caller binds; every call goes through the C ABI
into the CUDA library.  There is no CPU fallback: if libgg.so is missing or no
CUDA device is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgg.so")

# ---- enums (must match include/gg.h) ----
GG_OK, GG_ERR_ARG, GG_ERR_OOM, GG_ERR_CUDA, GG_ERR_TIMEOUT, GG_ERR_UNSUPPORTED, GG_ERR_IO, \
    GG_ERR_STATE, GG_ERR_NOT_FOUND = range(9)
I32, U32, F32, F64, BF16, F16, FP8E4M3, CFP_6_10, BF16_TRUNC, U8 = range(10)
(RELAX_MIN_PLUS1_I32, RELAX_MIN_U32, RELAX_SETIF_U32, RELAX_ADD_GATHER, RELAX_NE_CHECK, RELAX_GAP_CHECK,
 RELAX_AHEAD_CHECK, RELAX_OR_U32, RELAX_MIS_U8, RELAX_COUNT_DOWN_U32) = range(10)
FILTER_NONE, FILTER_GT_CONST, FILTER_NE_ZERO, FILTER_MSB_SET, FILTER_NE_CONST, FILTER_IN_FRONTIER = range(6)
RECORD_NONE, RECORD_REDUCTION, RECORD_NE_PREV, RECORD_EQ_ZERO, RECORD_AT_FLOOR = range(5)
THRESH_DEFAULT, THRESH_FRAC, THRESH_ALWAYS_SPARSE, THRESH_ALWAYS_DENSE, THRESH_LEARNED = range(5)
VAR_AUTO, VAR_PUSH_SPARSE, VAR_PUSH_MERGE, VAR_PULL_DENSE, VAR_PUSH_DENSE, VAR_HOOK = -1, 0, 1, 2, 3, 4
VARIANT_NAMES = {0: "push_sparse", 1: "push_merge", 2: "pull_dense", 3: "push_dense"}
GEN_RMAT, GEN_ER, GEN_GRID = range(3)
(VM_END, VM_LOAD, VM_STORE, VM_CONST, VM_VID, VM_DEGREE, VM_ADD, VM_SUB, VM_MUL, VM_DIV, VM_ABS,
 VM_MIN, VM_MAX, VM_EQ, VM_NE, VM_LT, VM_GT, VM_REDUCE_ADD, VM_TOF32, VM_SELECT, VM_FILTER,
 VM_DUP, VM_AND, VM_OR, VM_XOR, VM_NOT, VM_TOU32, VM_TSET, VM_TGET, VM_LE, VM_GE) = range(31)
MAX_ITERS = 256

NP_DTYPE = {I32: np.int32, U32: np.uint32, F32: np.float32, F64: np.float64, BF16: np.uint16,
            F16: np.float16, FP8E4M3: np.uint8, CFP_6_10: np.uint16, BF16_TRUNC: np.uint16,
            U8: np.uint8}


class GenParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("scale", C.c_int), ("nedges", C.c_uint64), ("a", C.c_double),
                ("b", C.c_double), ("c", C.c_double), ("n", C.c_uint32), ("avgdeg", C.c_double),
                ("rows", C.c_uint32), ("cols", C.c_uint32), ("bp", C.c_uint32),
                ("seed", C.c_uint64), ("symmetric", C.c_int)]


class EmapDesc(C.Structure):
    _fields_ = [("relax", C.c_int), ("a", C.c_void_p), ("src", C.c_void_p), ("src_scale", C.c_float),
                ("accum_f64", C.c_int), ("dst_filter", C.c_int), ("dst_filter_prop", C.c_void_p),
                ("dst_filter_k", C.c_int64), ("src_strong", C.c_int), ("record", C.c_int),
                ("prev", C.c_void_p), ("threshold", C.c_int), ("threshold_k", C.c_int),
                ("variant", C.c_int), ("fusion", C.c_int), ("src_level_sync", C.c_int)]


class EmapStats(C.Structure):
    _fields_ = [("variant", C.c_int), ("nactv_in", C.c_uint64), ("nacte_in", C.c_uint64),
                ("scanned", C.c_uint64), ("nactv_out", C.c_uint64), ("nacte_out", C.c_uint64),
                ("kernel_ms", C.c_double)]


class VmapDesc(C.Structure):
    _fields_ = [("ncode", C.c_int), ("code", C.c_uint8 * 64), ("arg", C.c_uint8 * 64),
                ("props", C.c_void_p * 8), ("consts", C.c_double * 8), ("nreduce", C.c_int)]


class RunStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("total_ms", C.c_double), ("kernels", C.c_uint64),
                ("scanned_edges", C.c_uint64), ("vertices_reached", C.c_uint64),
                ("edges_reached", C.c_uint64), ("variant", C.c_int * MAX_ITERS),
                ("nactv", C.c_uint64 * MAX_ITERS), ("nacte", C.c_uint64 * MAX_ITERS),
                ("scanned", C.c_uint64 * MAX_ITERS), ("delta", C.c_double * MAX_ITERS),
                ("iter_ms", C.c_double * MAX_ITERS), ("kernel_ms", C.c_double * MAX_ITERS)]


class RunOpts(C.Structure):
    _fields_ = [("threshold", C.c_int), ("threshold_k", C.c_int), ("variant", C.c_int),
                ("collect_stats", C.c_int)]


class PrParams(C.Structure):
    _fields_ = [("maxiter", C.c_int), ("tol", C.c_double), ("damping", C.c_float),
                ("contrib_dtype", C.c_int), ("accum_f64", C.c_int), ("renorm_f32", C.c_int),
                ("nstages", C.c_int), ("stage_dtype", C.c_int * 4), ("stage_accum_f64", C.c_int * 4),
                ("stage_tol", C.c_double * 4), ("stochastic", C.c_int), ("average_last", C.c_int)]


EXPORTS = [
    "gg_status_string", "gg_dtype_size", "gg_ctx_create", "gg_ctx_destroy", "gg_ctx_set_stream",
    "gg_ctx_get_stream", "gg_ctx_sync", "gg_last_error", "gg_ctx_launch_count", "gg_graph_upload",
    "gg_graph_read_bin", "gg_graph_write_bin", "gg_graph_generate", "gg_graph_info",
    "gg_graph_download", "gg_graph_device_ptrs", "gg_graph_max_degree_vertex", "gg_graph_destroy",
    "gg_prop_create", "gg_prop_fill", "gg_prop_set", "gg_prop_get", "gg_prop_download",
    "gg_prop_upload", "gg_prop_device_ptr", "gg_prop_destroy", "gg_prop_create_managed", "gg_prop_prefetch",
    "gg_frontier_create",
    "gg_frontier_clear", "gg_frontier_set_single", "gg_frontier_set_all", "gg_frontier_set_list",
    "gg_frontier_counts", "gg_frontier_download", "gg_frontier_destroy", "gg_edgemap",
    "gg_vertexmap", "gg_bfs_level", "gg_bfs_level_host_async", "gg_bfs_level_host_wait",
    "gg_bfs_parent", "gg_cc", "gg_kcore", "gg_pagerank",
    "gg_tuning_set", "gg_tuning_get",
]


class GGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_status_name(status)}: {msg}")
        self.status = status


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libgg.so is not built ({LIB_PATH}); run python -m graptor_b200.build")
    L = C.CDLL(LIB_PATH)
    vp, u64, u32, i32, st = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_int
    L.gg_status_string.restype = C.c_char_p
    L.gg_status_string.argtypes = [st]
    L.gg_dtype_size.restype = C.c_size_t
    L.gg_dtype_size.argtypes = [i32]
    L.gg_last_error.restype = C.c_char_p
    L.gg_last_error.argtypes = [vp]
    L.gg_ctx_launch_count.restype = u64
    L.gg_ctx_launch_count.argtypes = [vp]
    L.gg_ctx_create.argtypes = [i32, C.POINTER(vp)]
    L.gg_ctx_destroy.argtypes = [vp]
    L.gg_ctx_set_stream.argtypes = [vp, vp]
    L.gg_ctx_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.gg_ctx_sync.argtypes = [vp]
    L.gg_graph_upload.argtypes = [vp, u32, u64, vp, vp, i32, C.POINTER(vp)]
    L.gg_graph_read_bin.argtypes = [vp, C.c_char_p, i32, C.POINTER(vp)]
    L.gg_graph_write_bin.argtypes = [vp, C.c_char_p]
    L.gg_graph_generate.argtypes = [vp, C.POINTER(GenParams), C.POINTER(vp)]
    L.gg_graph_info.argtypes = [vp, C.POINTER(u32), C.POINTER(u64), C.POINTER(i32)]
    L.gg_graph_download.argtypes = [vp, vp, vp]
    L.gg_graph_device_ptrs.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.gg_graph_max_degree_vertex.argtypes = [vp, C.POINTER(u32), C.POINTER(u32)]
    L.gg_graph_destroy.argtypes = [vp]
    L.gg_prop_create.argtypes = [vp, i32, C.POINTER(vp)]
    L.gg_prop_fill.argtypes = [vp, vp]
    L.gg_prop_set.argtypes = [vp, u32, vp]
    L.gg_prop_get.argtypes = [vp, u32, vp]
    L.gg_prop_download.argtypes = [vp, vp]
    L.gg_prop_upload.argtypes = [vp, vp]
    L.gg_prop_device_ptr.argtypes = [vp, C.POINTER(vp)]
    L.gg_prop_destroy.argtypes = [vp]
    L.gg_frontier_create.argtypes = [vp, C.POINTER(vp)]
    L.gg_frontier_clear.argtypes = [vp]
    L.gg_frontier_set_single.argtypes = [vp, u32]
    L.gg_frontier_set_all.argtypes = [vp]
    L.gg_frontier_set_list.argtypes = [vp, vp, u64]
    L.gg_frontier_counts.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
    L.gg_frontier_download.argtypes = [vp, vp, u64, C.POINTER(u64)]
    L.gg_frontier_destroy.argtypes = [vp]
    L.gg_edgemap.argtypes = [vp, C.POINTER(EmapDesc), vp, vp, C.POINTER(EmapStats)]
    L.gg_vertexmap.argtypes = [vp, C.POINTER(VmapDesc), vp, vp, vp]
    L.gg_bfs_level.argtypes = [vp, u32, C.POINTER(RunOpts), vp, vp, C.POINTER(RunStats)]
    L.gg_bfs_parent.argtypes = [vp, u32, C.POINTER(RunOpts), vp, vp, C.POINTER(RunStats)]
    L.gg_cc.argtypes = [vp, C.POINTER(RunOpts), vp, vp, C.POINTER(RunStats)]
    L.gg_kcore.argtypes = [vp, C.POINTER(RunOpts), vp, vp, C.POINTER(u32), C.POINTER(RunStats)]
    L.gg_pagerank.argtypes = [vp, C.POINTER(PrParams), vp, vp, C.POINTER(RunStats)]
    L.gg_tuning_set.argtypes = [C.c_char_p, C.c_int64]
    L.gg_tuning_get.argtypes = [C.c_char_p, C.POINTER(C.c_int64)]
    special = ("gg_status_string", "gg_dtype_size", "gg_last_error", "gg_ctx_launch_count")
    for name in EXPORTS:
        if name not in special:
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _status_name(s: int) -> str:
    try:
        return lib().gg_status_string(s).decode()
    except Exception:
        return f"status {s}"


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Context:
    """gg_ctx: one CUDA device + stream."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        self._children = weakref.WeakSet()  # graphs: destroyed before the context
        s = lib().gg_ctx_create(device, C.byref(self.h))
        if s != GG_OK:
            raise GGError(s, "gg_ctx_create failed")

    def check(self, s: int, what: str = ""):
        if s != GG_OK:
            msg = lib().gg_last_error(self.h).decode(errors="replace")
            raise GGError(s, f"{what}: {msg}")

    def close(self):
        """Destroy the context; graphs (and their properties and frontiers)
        created from it are destroyed first, so no handle outlives it."""
        if self.h:
            for g in list(self._children):
                g.close()
            lib().gg_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int):
        self.check(lib().gg_ctx_set_stream(self.h, C.c_void_p(stream_handle)), "set_stream")

    def stream(self) -> int:
        s = C.c_void_p()
        self.check(lib().gg_ctx_get_stream(self.h, C.byref(s)), "get_stream")
        return s.value or 0

    def sync(self):
        self.check(lib().gg_ctx_sync(self.h), "sync")

    @property
    def launches(self) -> int:
        return int(lib().gg_ctx_launch_count(self.h))

    # graph constructors
    def upload(self, off: np.ndarray, adj: np.ndarray, symmetric: bool = True) -> "Graph":
        off = np.ascontiguousarray(off, dtype=np.uint64)
        adj = np.ascontiguousarray(adj, dtype=np.uint32)
        n = len(off) - 1
        h = C.c_void_p()
        self.check(lib().gg_graph_upload(self.h, n, int(off[-1]) if n >= 0 else 0, _p(off), _p(adj),
                                         int(symmetric), C.byref(h)), "gg_graph_upload")
        return Graph(self, h)

    def read_bin(self, path: str, symmetric: bool = True) -> "Graph":
        h = C.c_void_p()
        self.check(lib().gg_graph_read_bin(self.h, path.encode(), int(symmetric), C.byref(h)),
                   "gg_graph_read_bin")
        return Graph(self, h)

    def generate(self, kind: int, seed: int, scale=0, nedges=0, a=0.57, b=0.19, c=0.19, n=0,
                 avgdeg=0.0, rows=0, cols=0, bp=0, symmetric=True) -> "Graph":
        p = GenParams(kind=kind, scale=scale, nedges=nedges, a=a, b=b, c=c, n=n, avgdeg=avgdeg,
                      rows=rows, cols=cols, bp=bp, seed=seed, symmetric=int(symmetric))
        h = C.c_void_p()
        self.check(lib().gg_graph_generate(self.h, C.byref(p), C.byref(h)), "gg_graph_generate")
        return Graph(self, h)

    def rmat(self, scale: int, nedges: int, seed: int, a=0.57, b=0.19, c=0.19, symmetric=True):
        return self.generate(GEN_RMAT, seed, scale=scale, nedges=nedges, a=a, b=b, c=c,
                             symmetric=symmetric)

    def er(self, n: int, avgdeg: float, seed: int, dangling_bp=0, symmetric=True):
        return self.generate(GEN_ER, seed, n=n, avgdeg=avgdeg, bp=dangling_bp, symmetric=symmetric)

    def grid(self, rows: int, cols: int, seed: int, del_bp=0):
        return self.generate(GEN_GRID, seed, rows=rows, cols=cols, bp=del_bp)

    def from_edges(self, n: int, src, dst, symmetrise: bool = True, device: bool = False) -> "Graph":
        """Edge list -> graph, duplicates and self-loops dropped on the device.
        device=True: src / dst are device pointers (ints) to nedges uint32 each,
        with nedges passed as len(src) unless src is an int (then pass (ptr, count))."""
        L = _ingest_lib()
        h = C.c_void_p()
        flags = (INGEST_SYMMETRISE if symmetrise else 0) | (INGEST_DEVICE if device else 0)
        if device:
            (ps, ne), (pd, _) = src, dst
            self.check(L.gg_graph_from_edges(self.h, n, ne, C.c_void_p(ps), C.c_void_p(pd), flags, C.byref(h)),
                       "gg_graph_from_edges")
        else:
            s_ = np.ascontiguousarray(src, dtype=np.uint32)
            d_ = np.ascontiguousarray(dst, dtype=np.uint32)
            assert len(s_) == len(d_)
            self.check(L.gg_graph_from_edges(self.h, n, len(s_), _p(s_) if len(s_) else None,
                                             _p(d_) if len(d_) else None, flags, C.byref(h)), "gg_graph_from_edges")
        return Graph(self, h)

    def read_bin_clean(self, path: str, symmetrise: bool = True) -> "Graph":
        h = C.c_void_p()
        self.check(_ingest_lib().gg_graph_read_bin_clean(self.h, path.encode(),
                                                         INGEST_SYMMETRISE if symmetrise else 0, C.byref(h)),
                   "gg_graph_read_bin_clean")
        return Graph(self, h)


class Graph:
    def __init__(self, ctx: Context, h: C.c_void_p):
        self.ctx, self.h = ctx, h
        self._children = weakref.WeakSet()  # props / frontiers: destroyed before the graph
        ctx._children.add(self)
        n, m, sym = C.c_uint32(), C.c_uint64(), C.c_int()
        ctx.check(lib().gg_graph_info(h, C.byref(n), C.byref(m), C.byref(sym)), "info")
        self.n, self.m, self.symmetric = n.value, m.value, bool(sym.value)

    def close(self):
        if self.h:
            for c in list(self._children):
                c.close()
            if self.ctx.h:
                lib().gg_graph_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def download(self):
        off = np.empty(self.n + 1, dtype=np.uint64)
        adj = np.empty(max(self.m, 1), dtype=np.uint32)
        self.ctx.check(lib().gg_graph_download(self.h, _p(off), _p(adj)), "download")
        return off, adj[: self.m]

    def write_bin(self, path: str):
        self.ctx.check(lib().gg_graph_write_bin(self.h, path.encode()), "write_bin")

    def max_degree_vertex(self):
        v, d = C.c_uint32(), C.c_uint32()
        self.ctx.check(lib().gg_graph_max_degree_vertex(self.h, C.byref(v), C.byref(d)), "maxdeg")
        return v.value, d.value

    def device_ptrs(self):
        ptrs = [C.c_void_p() for _ in range(4)]
        self.ctx.check(lib().gg_graph_device_ptrs(self.h, *[C.byref(p) for p in ptrs]), "ptrs")
        return [p.value for p in ptrs]

    def prop(self, dtype: int) -> "Prop":
        return Prop(self, dtype)

    def frontier(self) -> "Frontier":
        return Frontier(self)

    # analytics
    def bfs_level(self, root: int, level: "Prop" = None, host: bool = True, opts: RunOpts = None,
                  stats: RunStats = None, out: np.ndarray = None):
        if out is not None:
            assert out.dtype == np.int32 and out.size >= self.n and out.flags.c_contiguous
            host = True
        elif host:
            out = np.empty(self.n, dtype=np.int32)
        self.ctx.check(lib().gg_bfs_level(self.h, root, C.byref(opts) if opts else None,
                                          level.h if level else None,
                                          _p(out) if host else None,
                                          C.byref(stats) if stats is not None else None),
                       "gg_bfs_level")
        return out

    def bfs_level_host_async(self, root: int, out: np.ndarray, opts: RunOpts = None, stats: RunStats = None):
        """BFS levels into `out` (int32, n entries, ideally page-locked), the
        copy finishing behind the next call: `out` of call i is complete once
        call i+1 or bfs_level_host_wait() has returned."""
        assert out.dtype == np.int32 and out.size >= self.n and out.flags.c_contiguous
        self.ctx.check(lib().gg_bfs_level_host_async(self.h, root, C.byref(opts) if opts else None, _p(out),
                                                     C.byref(stats) if stats is not None else None),
                       "gg_bfs_level_host_async")
        return out

    def bfs_level_host_wait(self):
        self.ctx.check(lib().gg_bfs_level_host_wait(self.h), "gg_bfs_level_host_wait")

    def bfs_parent(self, root: int, parent: "Prop" = None, host: bool = True,
                   opts: RunOpts = None, stats: RunStats = None):
        out = np.empty(self.n, dtype=np.uint32) if host else None
        self.ctx.check(lib().gg_bfs_parent(self.h, root, C.byref(opts) if opts else None,
                                           parent.h if parent else None,
                                           _p(out) if host else None,
                                           C.byref(stats) if stats is not None else None),
                       "gg_bfs_parent")
        return out

    def cc(self, label: "Prop" = None, host: bool = True, opts: RunOpts = None,
           stats: RunStats = None):
        out = np.empty(self.n, dtype=np.uint32) if host else None
        self.ctx.check(lib().gg_cc(self.h, C.byref(opts) if opts else None,
                                   label.h if label else None, _p(out) if host else None,
                                   C.byref(stats) if stats is not None else None), "gg_cc")
        return out

    def kcore(self, coreness: "Prop" = None, host: bool = True, opts: RunOpts = None,
              stats: RunStats = None):
        """k-core decomposition (KC_bucket): (coreness uint32 per vertex or
        None when host is False, largest coreness)."""
        out = np.empty(self.n, dtype=np.uint32) if host else None
        largest = C.c_uint32()
        self.ctx.check(lib().gg_kcore(self.h, C.byref(opts) if opts else None,
                                      coreness.h if coreness else None, _p(out) if host else None,
                                      C.byref(largest), C.byref(stats) if stats is not None else None),
                       "gg_kcore")
        return out, int(largest.value)

    def pagerank(self, maxiter=20, tol=1e-7, contrib=F32, accum_f64=True, renorm_f32=True,
                 damping=0.85, x: "Prop" = None, host: bool = True, stats: RunStats = None, stages=None,
                 stochastic: bool = False, average_last: int = 0):
        """stages: [(dtype, accum_f64, tol), ...] for a staged run (the last tol is ignored;
        `tol` ends the last stage), e.g. PR_vary VARIANT 4620:
        [(CFP_6_10, False, 1e-3), (F32, True, 0)].  BF16 runs: stochastic rounding of the
        stored contributions, and the mean of the last `average_last` iterations' ranks."""
        p = PrParams(maxiter=maxiter, tol=tol, damping=damping, contrib_dtype=contrib,
                     accum_f64=int(accum_f64), renorm_f32=int(renorm_f32), stochastic=int(stochastic),
                     average_last=int(average_last))
        if stages:
            p.nstages = len(stages)
            for k, (dt, acc, st_tol) in enumerate(stages):
                p.stage_dtype[k], p.stage_accum_f64[k], p.stage_tol[k] = dt, int(acc), st_tol
        if contrib == F64 and host and x is None:
            # the FP64 variant: return the double ranks
            xp = self.prop(F64)
            self.ctx.check(lib().gg_pagerank(self.h, C.byref(p), xp.h, None,
                                             C.byref(stats) if stats is not None else None), "gg_pagerank")
            out = xp.download()
            xp.close()
            return out
        out = np.empty(self.n, dtype=np.float32) if host else None
        self.ctx.check(lib().gg_pagerank(self.h, C.byref(p), x.h if x else None,
                                         _p(out) if host else None,
                                         C.byref(stats) if stats is not None else None),
                       "gg_pagerank")
        return out

    def edgemap(self, desc: EmapDesc, fin: "Frontier" = None, fout: "Frontier" = None,
                stats: bool = False):
        st = EmapStats() if stats else None
        self.ctx.check(lib().gg_edgemap(self.h, C.byref(desc), fin.h if fin else None,
                                        fout.h if fout else None,
                                        C.byref(st) if st is not None else None), "gg_edgemap")
        return st

    def vertexmap(self, desc: VmapDesc, filt: "Frontier" = None, out: "Frontier" = None):
        red = np.zeros(4, dtype=np.float64)
        self.ctx.check(lib().gg_vertexmap(self.h, C.byref(desc), filt.h if filt else None,
                                          out.h if out else None, _p(red)), "gg_vertexmap")
        return red[: desc.nreduce]


class Prop:
    def __init__(self, g: Graph, dtype: int):
        self.g, self.dtype = g, dtype
        self.h = C.c_void_p()
        g.ctx.check(lib().gg_prop_create(g.h, dtype, C.byref(self.h)), "gg_prop_create")
        g._children.add(self)

    def close(self):
        if self.h:
            if self.g.h and self.g.ctx.h:
                lib().gg_prop_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _scalar(self, value):
        return np.array([value], dtype=NP_DTYPE[self.dtype])

    def fill(self, value):
        v = self._scalar(value)
        self.g.ctx.check(lib().gg_prop_fill(self.h, _p(v)), "fill")

    def set(self, vid: int, value):
        v = self._scalar(value)
        self.g.ctx.check(lib().gg_prop_set(self.h, vid, _p(v)), "set")

    def get(self, vid: int):
        v = np.zeros(1, dtype=NP_DTYPE[self.dtype])
        self.g.ctx.check(lib().gg_prop_get(self.h, vid, _p(v)), "get")
        return v[0]

    def download(self) -> np.ndarray:
        a = np.empty(self.g.n, dtype=NP_DTYPE[self.dtype])
        self.g.ctx.check(lib().gg_prop_download(self.h, _p(a)), "download")
        return a

    def upload(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=NP_DTYPE[self.dtype])
        assert a.shape == (self.g.n,)
        self.g.ctx.check(lib().gg_prop_upload(self.h, _p(a)), "upload")

    def device_ptr(self) -> int:
        p = C.c_void_p()
        self.g.ctx.check(lib().gg_prop_device_ptr(self.h, C.byref(p)), "device_ptr")
        return p.value


class Frontier:
    def __init__(self, g: Graph):
        self.g = g
        self.h = C.c_void_p()
        g.ctx.check(lib().gg_frontier_create(g.h, C.byref(self.h)), "gg_frontier_create")
        g._children.add(self)

    def close(self):
        if self.h:
            if self.g.h and self.g.ctx.h:
                lib().gg_frontier_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_single(self, v: int):
        self.g.ctx.check(lib().gg_frontier_set_single(self.h, v), "set_single")

    def set_all(self):
        self.g.ctx.check(lib().gg_frontier_set_all(self.h), "set_all")

    def clear(self):
        self.g.ctx.check(lib().gg_frontier_clear(self.h), "clear")

    def set_list(self, vs):
        a = np.ascontiguousarray(vs, dtype=np.uint32)
        self.g.ctx.check(lib().gg_frontier_set_list(self.h, _p(a) if len(a) else None, len(a)),
                         "set_list")

    def counts(self):
        v, e = C.c_uint64(), C.c_uint64()
        self.g.ctx.check(lib().gg_frontier_counts(self.h, C.byref(v), C.byref(e)), "counts")
        return v.value, e.value

    def download(self) -> np.ndarray:
        k = C.c_uint64()
        self.g.ctx.check(lib().gg_frontier_download(self.h, None, 0, C.byref(k)), "download")
        a = np.empty(max(k.value, 1), dtype=np.uint32)
        self.g.ctx.check(lib().gg_frontier_download(self.h, _p(a), len(a), C.byref(k)), "download")
        return np.sort(a[: k.value])


def tuning_set(name: str, value: int):
    s = lib().gg_tuning_set(name.encode(), int(value))
    if s != GG_OK:
        raise GGError(s, f"gg_tuning_set({name}, {value})")


def tuning_get(name: str) -> int:
    v = C.c_int64()
    s = lib().gg_tuning_get(name.encode(), C.byref(v))
    if s != GG_OK:
        raise GGError(s, f"gg_tuning_get({name})")
    return v.value


def default_opts(threshold=THRESH_DEFAULT, k=0, variant=VAR_AUTO, collect=False) -> RunOpts:
    return RunOpts(threshold=threshold, threshold_k=k, variant=variant, collect_stats=int(collect))


# ---------------------------------------------------------------------------
# Learned variant selector (include/gg_select.h)
# ---------------------------------------------------------------------------
SEL_FEATURES, SEL_VARIANTS, SEL_NPARAMS = 10, 4, 32 * 10 + 32 + 32 * 32 + 32 + 4 * 32 + 4


def _sel_lib():
    L = lib()
    if not getattr(L, "_sel_bound", False):
        vp, fp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int)
        L.gg_selector_create.argtypes = [vp, C.POINTER(vp)]
        L.gg_selector_destroy.argtypes = [vp]
        L.gg_selector_set_params.argtypes = [vp, vp, C.c_int]
        L.gg_selector_get_params.argtypes = [vp, vp, C.c_int]
        L.gg_selector_forward.argtypes = [vp, vp, C.c_int, vp]
        L.gg_selector_loss_grad.argtypes = [vp, vp, vp, vp, C.c_int, fp, vp]
        L.gg_selector_train.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int, C.c_float, fp]
        L.gg_selector_collect.argtypes = [vp, C.c_int, C.c_uint32, C.c_int, vp, vp, C.c_int, ip]
        L.gg_graph_set_selector.argtypes = [vp, vp]
        for n in ["gg_selector_create", "gg_selector_destroy", "gg_selector_set_params",
                  "gg_selector_get_params", "gg_selector_forward", "gg_selector_loss_grad",
                  "gg_selector_train", "gg_selector_collect", "gg_graph_set_selector"]:
            getattr(L, n).restype = C.c_int
        L._sel_bound = True
    return L


def _f32(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float32)
    assert a.shape == shape, (a.shape, shape)
    return a


class Selector:
    """The traversal-variant network: inference, loss gradient, training."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.h = C.c_void_p()
        ctx.check(_sel_lib().gg_selector_create(ctx.h, C.byref(self.h)), "gg_selector_create")
        ctx._children.add(self)

    def close(self):
        if self.h:
            if self.ctx.h:
                _sel_lib().gg_selector_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.empty(SEL_NPARAMS, dtype=np.float32)
        self.ctx.check(_sel_lib().gg_selector_get_params(self.h, _p(p), SEL_NPARAMS), "get_params")
        return p

    @params.setter
    def params(self, p):
        p = _f32(p, (SEL_NPARAMS,))
        self.ctx.check(_sel_lib().gg_selector_set_params(self.h, _p(p), SEL_NPARAMS), "set_params")

    def forward(self, X) -> np.ndarray:
        X = _f32(X, (len(X), SEL_FEATURES))
        out = np.empty((len(X), SEL_VARIANTS), dtype=np.float32)
        self.ctx.check(_sel_lib().gg_selector_forward(self.h, _p(X), len(X), _p(out)), "forward")
        return out

    def loss_grad(self, X, Y, M):
        n = len(X)
        X, Y, M = _f32(X, (n, SEL_FEATURES)), _f32(Y, (n, SEL_VARIANTS)), _f32(M, (n, SEL_VARIANTS))
        loss = C.c_float()
        g = np.empty(SEL_NPARAMS, dtype=np.float32)
        self.ctx.check(_sel_lib().gg_selector_loss_grad(self.h, _p(X), _p(Y), _p(M), n, C.byref(loss), _p(g)),
                       "loss_grad")
        return loss.value, g

    def train(self, X, Y, M, epochs=500, lr=3e-3) -> float:
        n = len(X)
        X, Y, M = _f32(X, (n, SEL_FEATURES)), _f32(Y, (n, SEL_VARIANTS)), _f32(M, (n, SEL_VARIANTS))
        loss = C.c_float()
        self.ctx.check(_sel_lib().gg_selector_train(self.h, _p(X), _p(Y), _p(M), n, epochs, lr, C.byref(loss)),
                       "train")
        return loss.value


def selector_collect(g: "Graph", analytic: int, root: int = 0, max_samples: int = 8, cap: int = 256):
    """Per sampled iteration: features X[k][10], measured log2 us Y[k][4]."""
    X = np.zeros((cap, SEL_FEATURES), dtype=np.float32)
    Y = np.zeros((cap, SEL_VARIANTS), dtype=np.float32)
    k = C.c_int()
    g.ctx.check(_sel_lib().gg_selector_collect(g.h, analytic, root, max_samples, _p(X), _p(Y), cap, C.byref(k)),
                "gg_selector_collect")
    return X[: k.value], Y[: k.value]


def attach_selector(g: "Graph", sel: "Selector | None"):
    """The graph copies the selector's weights as they are now (the selector
    may be retrained or dropped afterwards)."""
    g.ctx.check(_sel_lib().gg_graph_set_selector(g.h, sel.h if sel else None), "gg_graph_set_selector")


# ---------------------------------------------------------------------------
# Batched traversals (include/gg_batch.h)
# ---------------------------------------------------------------------------
MSBFS_MAX_ROOTS, PPR_MAX_SEEDS = 64, 128


def _batch_lib():
    L = lib()
    if not getattr(L, "_batch_bound", False):
        vp, u32 = C.c_void_p, C.c_uint32
        L.gg_msbfs.argtypes = [vp, vp, C.c_int, vp, C.POINTER(RunStats)]
        L.gg_ppr.argtypes = [vp, vp, C.c_int, C.c_float, C.c_int, vp, C.POINTER(RunStats)]
        L.gg_graph_union.argtypes = [vp, vp, C.c_int, C.POINTER(vp), vp]
        L.gg_bfs_level_multi.argtypes = [vp, vp, u32, C.POINTER(RunOpts), vp, vp, C.POINTER(RunStats)]
        L.gg_batch_bfs_cc.argtypes = [vp, vp, u32, vp, vp, vp, vp, C.POINTER(RunStats), C.POINTER(RunStats),
                                      C.POINTER(C.c_int), C.POINTER(C.c_uint64)]
        for n in ["gg_msbfs", "gg_ppr", "gg_graph_union", "gg_bfs_level_multi", "gg_batch_bfs_cc"]:
            getattr(L, n).restype = C.c_int
        L._batch_bound = True
    return L


def msbfs(g: Graph, roots, host: bool = True, stats: RunStats = None):
    """BFS levels from up to 64 roots in one launch: [n][k] int32 (or None)."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    out = np.empty((g.n, len(r)), dtype=np.int32) if host else None
    g.ctx.check(_batch_lib().gg_msbfs(g.h, _p(r), len(r), _p(out) if host else None,
                                      C.byref(stats) if stats is not None else None), "gg_msbfs")
    return out


def ppr(g: Graph, seeds, alpha: float = 0.15, iters: int = 20, host: bool = True, stats: RunStats = None):
    """Personalized PageRank for up to 128 seeds (bfloat16 storage): [n][k] float32."""
    s = np.ascontiguousarray(seeds, dtype=np.uint32)
    out = np.empty((g.n, len(s)), dtype=np.float32) if host else None
    g.ctx.check(_batch_lib().gg_ppr(g.h, _p(s), len(s), alpha, iters, _p(out) if host else None,
                                    C.byref(stats) if stats is not None else None), "gg_ppr")
    return out


def graph_union(ctx: Context, parts):
    """Disjoint union of graphs: (Graph, vertex_base[k+1])."""
    hs = (C.c_void_p * len(parts))(*[p.h.value if isinstance(p.h, C.c_void_p) else p.h for p in parts])
    base = np.empty(len(parts) + 1, dtype=np.uint32)
    h = C.c_void_p()
    ctx.check(_batch_lib().gg_graph_union(ctx.h, hs, len(parts), C.byref(h), _p(base)), "gg_graph_union")
    return Graph(ctx, h), base


def bfs_level_multi(g: Graph, roots, host: bool = True, opts: RunOpts = None, stats: RunStats = None):
    """BFS levels with every root at level 0, one device-driven launch."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    out = np.empty(g.n, dtype=np.int32) if host else None
    g.ctx.check(_batch_lib().gg_bfs_level_multi(g.h, _p(r), len(r), C.byref(opts) if opts else None, None,
                                                _p(out) if host else None,
                                                C.byref(stats) if stats is not None else None),
                "gg_bfs_level_multi")
    return out


def batch_bfs_cc(g: Graph, roots, host: bool = True, bfs_stats: RunStats = None, cc_stats: RunStats = None):
    """BFS levels from every root at once and CC labels, one CUDA graph launch:
    (levels, labels, graph_launches, kernel_launches); arrays None if not host."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    lv = np.empty(g.n, dtype=np.int32) if host else None
    lb = np.empty(g.n, dtype=np.uint32) if host else None
    gl, kl = C.c_int(), C.c_uint64()
    g.ctx.check(_batch_lib().gg_batch_bfs_cc(g.h, _p(r), len(r), None, None, _p(lv) if host else None,
                                             _p(lb) if host else None,
                                             C.byref(bfs_stats) if bfs_stats is not None else None,
                                             C.byref(cc_stats) if cc_stats is not None else None,
                                             C.byref(gl), C.byref(kl)), "gg_batch_bfs_cc")
    return lv, lb, gl.value, kl.value


# ---------------------------------------------------------------------------
# Autotuner (include/gg_tune.h)
# ---------------------------------------------------------------------------
TUNE_BFS, TUNE_CC, TUNE_PR = 1, 2, 4


class TuneResult(C.Structure):
    _fields_ = [("initial_ms", C.c_double), ("best_ms", C.c_double), ("evaluations", C.c_int),
                ("best", C.c_char * 512)]


def _tune_lib():
    L = lib()
    if not getattr(L, "_tune_bound", False):
        L.gg_graph_retune.argtypes = [C.c_void_p]
        L.gg_autotune.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(TuneResult)]
        L.gg_graph_retune.restype = C.c_int
        L.gg_autotune.restype = C.c_int
        L._tune_bound = True
    return L


def graph_retune(g: Graph):
    g.ctx.check(_tune_lib().gg_graph_retune(g.h), "gg_graph_retune")


def autotune(g: Graph, analytics: int = TUNE_BFS | TUNE_CC, roots=(), passes: int = 2, reps: int = 2) -> dict:
    """Coordinate-descent tuning on g; the chosen knobs are set and returned."""
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    res = TuneResult()
    g.ctx.check(_tune_lib().gg_autotune(g.h, analytics, _p(r) if len(r) else None, len(r), passes, reps,
                                        C.byref(res)), "gg_autotune")
    best = dict(kv.split("=") for kv in res.best.decode().split(",") if kv)
    return dict(initial_ms=res.initial_ms, best_ms=res.best_ms, evaluations=res.evaluations,
                knobs={k: int(v) for k, v in best.items()})


# ---------------------------------------------------------------------------
# Ingest with cleaning (gg_graph_from_edges / gg_graph_read_bin_clean)
# ---------------------------------------------------------------------------
INGEST_SYMMETRISE, INGEST_DEVICE = 1, 2


def _ingest_lib():
    L = lib()
    if not getattr(L, "_ingest_bound", False):
        L.gg_graph_from_edges.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int,
                                          C.POINTER(C.c_void_p)]
        L.gg_graph_read_bin_clean.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
        L.gg_graph_from_edges.restype = C.c_int
        L.gg_graph_read_bin_clean.restype = C.c_int
        L._ingest_bound = True
    return L
