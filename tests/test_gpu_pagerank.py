"""GPU PageRank (FP32 ranks and sums, FP64 norms) against the FP64 oracle.

The stated error bound: L1(r_fp32 - r_fp64) <= 1e-6 at the same iteration
count (the L1 norm of a rank vector is 1), plus the stop iteration agreeing
with the FP64 run of the same stopping rule to within one iteration."""
import numpy as np
import pytest

import oracle
from gpugraph_b200 import Graph, HostGraph

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _check(hg, directed, tol=1e-6, max_iter=100):
    t = hg.transpose() if directed else hg
    g = Graph(hg, directed=directed)
    r, st = g.pagerank(tolerance=tol, iter_num=max_iter)
    it = st["iterations"]
    ref_same, _, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 0.0, it)
    ref_stop, it_ref, res_ref = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, tol,
                                                     max_iter)
    l1 = float(np.abs(r.astype(np.float64) - ref_same).sum())
    mx = float(np.abs(r.astype(np.float64) - ref_same).max())
    assert l1 <= L1_TOL, (l1, mx, it)
    assert abs(it - it_ref) <= 1, (it, it_ref)
    assert abs(float(r.astype(np.float64).sum()) - 1.0) < 1e-4
    if st["converged"]:
        assert st["residual"] <= tol
    return r, st, l1, mx


@pytest.mark.parametrize("scale,ef,seed", [(14, 16, 1), (16, 8, 2), (12, 32, 3)])
def test_pagerank_directed_rmat(scale, ef, seed):
    hg = HostGraph.rmat(scale, ef, seed=seed, symmetrize=False)
    assert (np.diff(hg.row_offsets) == 0).any()  # has dangling vertices
    _check(hg, True)


@pytest.mark.parametrize("extra", [1, 2, 3])
def test_pagerank_vertex_count_not_a_multiple_of_four(extra):
    # isolated vertices appended (dangling, no in-edges): the last 32-vertex
    # group of the pull is partial and the vertex count is not a multiple of 4
    base = HostGraph.rmat(12, 8, seed=21, symmetrize=False)
    ro = np.concatenate([base.row_offsets, np.full(extra, base.row_offsets[-1], np.int32)])
    hg = HostGraph(ro, base.column_indices)
    assert hg.nodes % 4 == extra
    _check(hg, True)


def test_pagerank_road_grid_symmetric():
    hg = HostGraph.road_grid(300, 0.02, 0.005, seed=3)
    _check(hg, False)


def test_pagerank_iteration_cap_and_no_edges():
    hg = HostGraph.rmat(12, 8, seed=5, symmetrize=False)
    g = Graph(hg, directed=True)
    r, st = g.pagerank(tolerance=0.0, iter_num=7)
    assert st["iterations"] == 7 and not st["converged"]
    t = hg.transpose()
    ref, _, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 0.0, 7)
    assert np.abs(r - ref).sum() <= L1_TOL
    empty = HostGraph(np.zeros(5, np.int32), np.zeros(0, np.int32))
    ge = Graph(empty, directed=True)
    r, st = ge.pagerank()
    assert np.allclose(r, 0.25) and st["iterations"] == 1 and st["converged"]


def test_pagerank_deterministic_and_graph_equals_host_loop():
    hg = HostGraph.rmat(15, 16, seed=9, symmetrize=False)
    g = Graph(hg, directed=True)
    a, _ = g.pagerank()
    b, _ = g.pagerank()
    c, _ = g.pagerank(use_cuda_graph=0)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
