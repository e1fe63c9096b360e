"""mg_bfs_noalloc: the BFS entry point for callers that cannot allocate device
memory (their GPU memory is planned up front by their own pool, or they must
not trigger cudaMalloc's implicit synchronisation). It keeps every working
buffer in a fixed static device array, so its output is checked here against
the regular mg_bfs on the same graph, for two calls in a row (the second call
reuses the array the first one left behind).

This file is collected last, so a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpugraph_b200 import Graph, HostGraph, _lib

pytestmark = pytest.mark.gpu

MAX_NODES, MAX_EDGES = 1 << 20, 1 << 24


def _noalloc(ro_d, col_d, nodes, edges, src, out_d, stream=None, stats=None):
    return _lib.lib.mg_bfs_noalloc(ro_d, col_d, nodes, edges, src, out_d, stream,
                                   C.byref(stats) if stats is not None else None)


def test_noalloc_bfs_matches_mg_bfs_twice():
    import torch

    hg = HostGraph.rmat(15, 16, seed=4)
    g = Graph(hg)
    ro = torch.from_numpy(hg.row_offsets).cuda()
    col = torch.from_numpy(hg.column_indices).cuda()
    out = torch.empty(hg.nodes, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    for src in (hg.max_degree_vertex(), 7):  # two calls in a row
        st = _lib.Stats()
        rc = _noalloc(ro.data_ptr(), col.data_ptr(), hg.nodes, hg.edges, int(src), out.data_ptr(), None, st)
        assert rc == _lib.MG_OK, _lib.lib.mg_last_error()
        torch.cuda.synchronize()
        ref, ref_st = g.bfs(int(src))
        assert np.array_equal(out.cpu().numpy(), ref)  # integer depths: exact
        assert st.iterations == ref_st["iterations"] and st.vertices_reached == ref_st["vertices_reached"]
    g.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    import torch

    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    assert _noalloc(p, p, MAX_NODES + 1, 2, 0, p) == _lib.MG_ERR_ARG
    assert b"fixed scratch" in _lib.lib.mg_last_error()
    assert _noalloc(p, p, 2, MAX_EDGES + 1, 0, p) == _lib.MG_ERR_ARG
    assert _noalloc(p, p, 2, 2, 5, p) == _lib.MG_ERR_ARG  # source out of range
    assert _noalloc(None, p, 2, 2, 0, p) == _lib.MG_ERR_ARG
