"""Python view of the C ABI: host CSR builders and the device graph.

`HostGraph` holds a CSR in numpy arrays (built by the library's seeded
builders or read from Matrix Market). `Graph` is the device-resident graph
(the reference's CsrProblem after FromHostProblem) with one method per GAS
program. Every compute call goes through libmapgraph_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, default_options, lib

SSSP_INF = 100000000  # sssp::INIT_VALUE (Algorithms/SSSP/sssp.h:43)


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


@dataclass
class HostGraph:
    row_offsets: np.ndarray
    column_indices: np.ndarray
    edge_values: np.ndarray | None = None
    directed: bool = False
    graph_offsets: np.ndarray | None = field(default=None)

    @property
    def nodes(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def edges(self) -> int:
        return int(self.column_indices.shape[0])

    def out_degree(self) -> np.ndarray:
        return np.diff(self.row_offsets).astype(np.int64)

    @staticmethod
    def _from_c(h: _lib.HostCsr) -> "HostGraph":
        n, m = int(h.nodes), int(h.edges)
        ro = np.ctypeslib.as_array(h.row_offsets, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(h.column_indices, shape=(max(m, 1),))[:m].copy()
        vals = None
        if bool(h.edge_values):
            vals = np.ctypeslib.as_array(h.edge_values, shape=(max(m, 1),))[:m].copy()
        directed = bool(h.directed)
        lib.mg_host_csr_free(C.byref(h))
        return HostGraph(ro, col, vals, directed)

    def _to_c(self) -> _lib.HostCsr:
        h = _lib.HostCsr()
        h.nodes, h.edges = self.nodes, self.edges
        h.row_offsets = self.row_offsets.ctypes.data_as(_lib.I32P)
        h.column_indices = self.column_indices.ctypes.data_as(_lib.I32P)
        h.edge_values = self.edge_values.ctypes.data_as(_lib.I32P) if self.edge_values is not None else None
        h.directed = int(self.directed)
        return h

    @staticmethod
    def rmat(scale: int, edgefactor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
             symmetrize: bool = True, clean: bool = True) -> "HostGraph":
        h = _lib.HostCsr()
        check(lib.mg_build_rmat(scale, edgefactor, a, b, c, seed, int(symmetrize), int(clean), C.byref(h)),
              "mg_build_rmat")
        return HostGraph._from_c(h)

    @staticmethod
    def road_grid(width: int = 1200, drop_frac: float = 0.02, shortcut_frac: float = 0.005,
                  seed: int = 1) -> "HostGraph":
        h = _lib.HostCsr()
        check(lib.mg_build_road_grid(width, drop_frac, shortcut_frac, seed, C.byref(h)), "mg_build_road_grid")
        return HostGraph._from_c(h)

    @staticmethod
    def read_market(path: str, undirected: bool = False) -> "HostGraph":
        h = _lib.HostCsr()
        check(lib.mg_read_market(str(path).encode(), int(undirected), C.byref(h)), "mg_read_market")
        return HostGraph._from_c(h)

    @staticmethod
    def read_csv(path: str, fmt: str = "adjacency", undirected: bool = True) -> "HostGraph":
        """CSV graph as the reference's csv_graph_reader reads it: fmt "adjacency" for rows
        "src,dst:val,...", "edges" for rows "src,dst,val"; ids renumbered in sorted order."""
        h = _lib.HostCsr()
        f = {"adjacency": 0, "edges": 1}[fmt]
        check(lib.mg_read_csv(str(path).encode(), f, int(undirected), C.byref(h)), "mg_read_csv")
        return HostGraph._from_c(h)

    def with_weights(self, lo: int, hi: int, seed: int = 1) -> "HostGraph":
        """Symmetric uint32 weights w(u,v)=w(v,u) in [lo, hi] (a copy of self)."""
        g = HostGraph(self.row_offsets.copy(), self.column_indices.copy(), None, self.directed, self.graph_offsets)
        h = g._to_c()
        h.edge_values = None
        check(lib.mg_build_weights(C.byref(h), lo, hi, seed), "mg_build_weights")
        m = g.edges
        g.edge_values = np.ctypeslib.as_array(h.edge_values, shape=(max(m, 1),))[:m].copy()
        # only the weights array was allocated by the library
        h2 = _lib.HostCsr()
        h2.edge_values = h.edge_values
        lib.mg_host_csr_free(C.byref(h2))
        return g

    def transpose(self) -> "HostGraph":
        h = self._to_c()
        out = _lib.HostCsr()
        check(lib.mg_host_csr_transpose(C.byref(h), C.byref(out)), "mg_host_csr_transpose")
        return HostGraph._from_c(out)

    def max_degree_vertex(self) -> int:
        d = self.out_degree()
        return int(np.argmax(d))  # ties -> lowest id


def concat_graphs(graphs: list[HostGraph]) -> HostGraph:
    """Concatenates independent graphs into one CSR with global vertex ids."""
    offs = np.zeros(len(graphs) + 1, dtype=np.int64)
    for i, g in enumerate(graphs):
        offs[i + 1] = offs[i] + g.nodes
    ro_parts, col_parts = [np.zeros(1, dtype=np.int64)], []
    ebase = 0
    for i, g in enumerate(graphs):
        ro_parts.append(g.row_offsets[1:].astype(np.int64) + ebase)
        col_parts.append(g.column_indices.astype(np.int64) + offs[i])
        ebase += g.edges
    ro = np.concatenate(ro_parts).astype(np.int32)
    col = np.concatenate(col_parts).astype(np.int32) if col_parts else np.zeros(0, np.int32)
    return HostGraph(ro, col, None, False, offs)


class Graph:
    """Device-resident graph: the reference's CsrProblem after FromHostProblem."""

    def __init__(self, host: HostGraph, directed: bool | None = None, value_type: str | None = None,
                 float_values: np.ndarray | None = None):
        self.host = host
        self.directed = host.directed if directed is None else directed
        self._g = C.c_void_p()
        self.nodes, self.edges = host.nodes, host.edges
        if host.graph_offsets is not None:
            check(lib.mg_graph_create_batch(_ptr(host.row_offsets), _ptr(host.column_indices), host.nodes,
                                            host.edges, _ptr(np.ascontiguousarray(host.graph_offsets, np.int64)),
                                            len(host.graph_offsets) - 1, None, C.byref(self._g)),
                  "mg_graph_create_batch")
            return
        vals, vt = None, _lib.MG_VAL_NONE
        if float_values is not None:
            vals, vt = np.ascontiguousarray(float_values, np.float32), _lib.MG_VAL_F32
        elif host.edge_values is not None:
            vals, vt = np.ascontiguousarray(host.edge_values, np.int32), _lib.MG_VAL_I32
        self._vals = vals
        check(lib.mg_graph_create(_ptr(host.row_offsets), _ptr(host.column_indices), _ptr(vals), vt, host.nodes,
                                  host.edges, int(self.directed), None, C.byref(self._g)), "mg_graph_create")

    def close(self) -> None:
        if self._g:
            lib.mg_graph_destroy(self._g)
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._g

    # ------------------------------------------------------------ programs --
    def _run(self, fn, name, out, *args, opts=None):
        st = _lib.Stats()
        o = opts if opts is not None else default_options()
        check(fn(self._g, *args, _ptr(out) if isinstance(out, np.ndarray) else out, C.byref(st), C.byref(o)), name)
        return out, st.as_dict()

    def bfs(self, src: int, **kw):
        out = np.empty(self.nodes, np.int32)
        return self._run(lib.mg_bfs, "mg_bfs", out, int(src), opts=default_options(**kw))

    def bfs_pred(self, src: int, **kw):
        """Depths and predecessors (pred_extract's rule: the largest in-neighbour one level up, else -1)."""
        depths = np.empty(self.nodes, np.int32)
        preds = np.empty(self.nodes, np.int32)
        st = _lib.Stats()
        check(lib.mg_bfs_pred(self._g, int(src), _ptr(depths), _ptr(preds), C.byref(st),
                              C.byref(default_options(**kw))), "mg_bfs_pred")
        return depths, preds, st.as_dict()

    def bfs_roots(self, srcs, **kw):
        s = np.ascontiguousarray(srcs, np.int32)
        out = np.empty(self.nodes, np.int32)
        return self._run(lib.mg_bfs_roots, "mg_bfs_roots", out, _ptr(s), len(s), opts=default_options(**kw))

    def bfs_multi(self, srcs, **kw):
        s = np.ascontiguousarray(srcs, np.int32)
        out = np.empty((len(s), self.nodes), np.int32)
        return self._run(lib.mg_bfs_multi, "mg_bfs_multi", out, _ptr(s), len(s), opts=default_options(**kw))

    def bfs_batch(self, local_srcs, **kw):
        s = np.ascontiguousarray(local_srcs, np.int32)
        out = np.empty(self.nodes, np.int32)
        return self._run(lib.mg_bfs_batch, "mg_bfs_batch", out, _ptr(s), opts=default_options(**kw))

    def sssp(self, src: int, **kw):
        out = np.empty(self.nodes, np.int32)
        return self._run(lib.mg_sssp, "mg_sssp", out, int(src), opts=default_options(**kw))

    def sssp_multi(self, srcs, **kw):
        s = np.ascontiguousarray(srcs, np.int32)
        out = np.empty((len(s), self.nodes), np.int32)
        return self._run(lib.mg_sssp_multi, "mg_sssp_multi", out, _ptr(s), len(s), opts=default_options(**kw))

    def cc(self, **kw):
        out = np.empty(self.nodes, np.int32)
        return self._run(lib.mg_cc, "mg_cc", out, opts=default_options(**kw))

    def pagerank(self, damping: float = 0.85, tolerance: float = 1e-6, iter_num: int = 100, **kw):
        """Normalised PageRank (FP32 ranks, FP64 norms); stops at L1 residual <= tolerance or iter_num."""
        out = np.empty(self.nodes, np.float32)
        return self._run(lib.mg_pagerank, "mg_pagerank", out,
                         opts=default_options(damping=damping, tolerance=tolerance, iter_num=iter_num, **kw))

    def pagerank_gas(self, tolerance: float = 0.01, **kw):
        out = np.empty(self.nodes, np.float32)
        return self._run(lib.mg_pagerank_gas, "mg_pagerank_gas", out, opts=default_options(tolerance=tolerance, **kw))
