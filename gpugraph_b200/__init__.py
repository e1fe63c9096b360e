"""B200-native Gather-Apply-Scatter hot path of MapGraph (BFS, SSSP, CC,
PageRank, batched traversal, differentiable personalised PageRank).

All compute runs in libmapgraph_b200.so (hand-written sm_100a CUDA behind the
C ABI in include/mapgraph_b200.h); importing fails if it is not built.
"""
from ._lib import MapGraphError, default_options, lib  # noqa: F401
from .graph import SSSP_INF, Graph, HostGraph, concat_graphs  # noqa: F401

__all__ = ["Graph", "HostGraph", "concat_graphs", "MapGraphError", "default_options", "SSSP_INF", "lib"]
