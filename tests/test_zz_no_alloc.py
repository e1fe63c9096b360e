"""mg_bfs_noalloc: the BFS entry point for callers that cannot allocate device
memory (their GPU memory is planned up front by their own pool, or they must
not trigger cudaMalloc's implicit synchronisation). It keeps every working
buffer in a fixed static device array, so its output is checked here against
the regular mg_bfs on the same graph, for two calls in a row (the second call
reuses the array the first one left behind), near the documented size limits,
and on edge cases; the defining property, that a call allocates nothing, is
checked through the device's free-memory figure.

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


def _device_copy(hg):
    import torch

    ro = torch.from_numpy(hg.row_offsets).cuda()
    col = torch.from_numpy(hg.column_indices if hg.edges else np.zeros(1, np.int32)).cuda()
    out = torch.empty(hg.nodes, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    return ro, col, out


def _check_against_mg_bfs(hg, sources):
    import torch

    g = Graph(hg)
    ro, col, out = _device_copy(hg)
    for src in sources:  # calls in a row, each reusing what the previous one left in the array
        st = _lib.Stats()
        rc = _noalloc(ro.data_ptr(), col.data_ptr(), hg.nodes, hg.edges, int(src), out.data_ptr(), None, st)
        assert rc == _lib.MG_OK, _lib.lib.mg_last_error()
        torch.cuda.synchronize()
        ref, ref_st = g.bfs(int(src))
        assert np.array_equal(out.cpu().numpy(), ref)  # integer depths: exact
        assert st.iterations == ref_st["iterations"]
        assert st.vertices_reached == ref_st["vertices_reached"]
        assert st.edges_traversed == int(hg.out_degree()[ref >= 0].sum())
    g.close()


def test_noalloc_bfs_matches_mg_bfs_twice():
    hg = HostGraph.rmat(15, 16, seed=4)
    _check_against_mg_bfs(hg, (hg.max_degree_vertex(), 7))


def test_noalloc_near_its_size_limits():
    # 2^20 nodes (the limit) and about 16.1M of the 16.8M allowed edges
    hg = HostGraph.rmat(20, 8, seed=3)
    assert hg.nodes == MAX_NODES and MAX_EDGES - 1_000_000 < hg.edges <= MAX_EDGES
    _check_against_mg_bfs(hg, (hg.max_degree_vertex(), 12345))


def test_noalloc_edge_cases():
    # a single vertex without edges, and an isolated source beside a component
    one = HostGraph(np.array([0, 0], np.int32), np.zeros(0, np.int32))
    _check_against_mg_bfs(one, (0, 0))
    hg = HostGraph.rmat(12, 4, seed=31)
    iso = np.flatnonzero(hg.out_degree() == 0)
    assert iso.size > 0
    _check_against_mg_bfs(hg, (int(iso[0]), hg.max_degree_vertex()))


def test_noalloc_call_allocates_nothing():
    import torch

    hg = HostGraph.rmat(16, 16, seed=8)
    ro, col, out = _device_copy(hg)
    src = hg.max_degree_vertex()
    assert _noalloc(ro.data_ptr(), col.data_ptr(), hg.nodes, hg.edges, src, out.data_ptr()) == _lib.MG_OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(ro.data_ptr(), col.data_ptr(), hg.nodes, hg.edges, src, out.data_ptr()) == _lib.MG_OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    import torch

    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    assert _noalloc(p, p, MAX_NODES + 1, 2, 0, p) == _lib.MG_ERR_ARG
    assert b"fixed scratch" in _lib.lib.mg_last_error()
    assert _noalloc(p, p, 2, MAX_EDGES + 1, 0, p) == _lib.MG_ERR_ARG
    assert _noalloc(p, p, 2, 2, 5, p) == _lib.MG_ERR_ARG  # source out of range
    assert _noalloc(None, p, 2, 2, 0, p) == _lib.MG_ERR_ARG
