"""graptor_b200: B200 (sm_100a) implementation of Graptor's edgemap/vertexmap
hot path (BFS levels / parents, connected components, PageRank).

The product is the CUDA library libgg.so behind the C ABI in include/gg.h and
the C++ operator surface in include/graptor_b200/api.h; ``graptor_b200.gg`` is
its ctypes binding.
"""
from . import gg  # noqa: F401
from .gg import Context, Graph, Prop, Frontier, GGError  # noqa: F401
