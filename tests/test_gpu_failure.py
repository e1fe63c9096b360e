"""Failure detection without faulting the GPU: device-side waits end at their
spin limit with MG_ERR_TIMEOUT and the context stays usable; bad arguments are
rejected on the host before any launch."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpugraph_b200 import Graph, HostGraph, MapGraphError, _lib

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives():
    ms = C.c_double()
    st = _lib.lib.mg_selftest_wait_timeout(2000, C.byref(ms))
    assert st == _lib.MG_ERR_TIMEOUT
    assert ms.value < 2000.0  # ended by the limit, not by a hang
    # the context is still usable: a traversal right after gives exact results
    hg = HostGraph.rmat(12, 8, seed=3)
    g = Graph(hg)
    s = hg.max_degree_vertex()
    assert np.array_equal(g.bfs(s)[0], oracle.bfs(hg.row_offsets, hg.column_indices, s))


def test_tiny_spin_limit_in_a_real_run_reports_or_succeeds():
    # With spin_limit = 1 any look-back wait that has to spin reports
    # MG_ERR_TIMEOUT instead of waiting; runs that never spin succeed. Either
    # way the call returns and the next call on the same graph is exact.
    hg = HostGraph.rmat(14, 16, seed=4)
    g = Graph(hg)
    s = hg.max_degree_vertex()
    try:
        g.bfs(s, spin_limit=1, ordered_frontier=1, direction=_lib.MG_DIR_PUSH)
    except MapGraphError as e:
        assert e.status == _lib.MG_ERR_TIMEOUT
    assert np.array_equal(g.bfs(s)[0], oracle.bfs(hg.row_offsets, hg.column_indices, s))


def test_selftest_argument_check():
    assert _lib.lib.mg_selftest_wait_timeout(0, None) == _lib.MG_ERR_ARG
