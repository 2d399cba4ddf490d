"""CPU oracle of the batched traversals (TEST INFRASTRUCTURE ONLY).

Only the test suite and the benchmark's CPU leg import this module.

* Multi-source BFS: one BFSLVLv level array per root (bench/BFSLVLv.C:165-216
  semantics through the C oracle's orc_bfs_level), stacked as [n][k].
* Personalized PageRank, no reference counterpart (Graptor's PRv.C has a
  uniform teleport vector; here the teleport is the seed's unit vector):
      x_s(0) = e_s,  x_s(t+1) = alpha * e_s + (1 - alpha) * A^T D^-1 x_s(t)
  with D the out-degrees; a vertex without out-edges passes nothing on.
  ppr_f64 is the float64 reference; ppr_bf16 restates the GPU storage
  (bfloat16 ranks and contributions, round to nearest even) with float64
  sums, for a tighter check of the storage path.
* Disjoint union: part i's vertex v becomes base[i] + v.
"""
from __future__ import annotations

import numpy as np

from . import oracle as orc


def msbfs_levels(g: orc.Graph, roots) -> np.ndarray:
    roots = [int(r) for r in roots]
    out = np.empty((g.n, len(roots)), dtype=np.int32)
    for i, r in enumerate(roots):
        out[:, i] = orc.bfs_level(g, r)
    return out


def _csr_matrix(g: orc.Graph):
    import scipy.sparse as sp

    rows = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.off).astype(np.int64))
    return sp.csr_matrix((np.ones(g.m, dtype=np.float64), (rows, g.adj.astype(np.int64))), shape=(g.n, g.n))


def _teleport(n: int, seeds) -> np.ndarray:
    e = np.zeros((n, len(seeds)), dtype=np.float64)
    e[np.asarray(seeds, dtype=np.int64), np.arange(len(seeds))] = 1.0
    return e


def ppr_f64(g: orc.Graph, seeds, alpha: float = 0.15, iters: int = 20) -> np.ndarray:
    A = _csr_matrix(g)
    deg = np.diff(g.off).astype(np.float64)
    inv = np.divide(1.0, deg, out=np.zeros_like(deg), where=deg > 0)[:, None]
    e = _teleport(g.n, seeds)
    x = e.copy()
    for _ in range(iters):
        x = alpha * e + (1.0 - alpha) * (A.T @ (x * inv))
    return x


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def ppr_bf16(g: orc.Graph, seeds, alpha: float = 0.15, iters: int = 20) -> np.ndarray:
    A = _csr_matrix(g)
    deg = np.diff(g.off).astype(np.float32)
    inv = np.divide(np.float32(1.0), deg, out=np.zeros_like(deg), where=deg > 0)[:, None]
    e = _teleport(g.n, seeds).astype(np.float32)
    x = bf16_round(e)
    c = bf16_round(x * inv)
    for _ in range(iters):
        acc = (A.T @ c.astype(np.float64)).astype(np.float32)
        xf = np.float32(1.0 - alpha) * acc + np.float32(alpha) * e
        x = bf16_round(xf)
        c = bf16_round(xf * inv)
    return x


def union(parts) -> tuple[orc.Graph, np.ndarray]:
    base = np.zeros(len(parts) + 1, dtype=np.int64)
    base[1:] = np.cumsum([p.n for p in parts])
    ebase = np.zeros(len(parts) + 1, dtype=np.int64)
    ebase[1:] = np.cumsum([p.m for p in parts])
    off = np.zeros(int(base[-1]) + 1, dtype=np.uint64)
    adj = np.zeros(int(ebase[-1]), dtype=np.uint32)
    for i, p in enumerate(parts):
        off[base[i]:base[i + 1]] = p.off[:-1] + np.uint64(ebase[i])
        adj[ebase[i]:ebase[i + 1]] = p.adj + np.uint32(base[i])
    off[-1] = np.uint64(ebase[-1])
    return orc.Graph(int(base[-1]), off, adj), base.astype(np.uint32)
