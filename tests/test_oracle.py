"""Pins the oracle (CPU restatement in oracle/mg_oracle.c) against the golden
vectors produced by the reference's own CPUBFS/CPUSSSP/CPUCC/CPUPR, and against
the reference functions themselves where oracle/_ref is built."""
import numpy as np
import pytest

from conftest import fixture_names, host_graph_from_fixture, load_fixture

import oracle
from gpugraph_b200 import HostGraph

FIXTURES = fixture_names()


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden(name):
    fx = load_fixture(name)
    g = host_graph_from_fixture(fx)
    ex = fx["expected"]
    for s in fx["sources"]:
        assert oracle.bfs(g.row_offsets, g.column_indices, s).tolist() == ex["bfs"][str(s)]
        assert oracle.sssp(g.row_offsets, g.column_indices, g.edge_values, s).tolist() == ex["sssp"][str(s)]
        assert oracle.sssp(g.row_offsets, g.column_indices, g.edge_values, s, "array").tolist() == ex["sssp"][str(s)]
    assert oracle.cc(g.row_offsets, g.column_indices).tolist() == ex["cc"]


def test_known_answers_small_mtx():
    # Known answers: the reference CPU code's outputs on smallRegressionGraphs/small.mtx from vertex 0.
    fx = load_fixture("mtx_small.json")
    assert fx["expected"]["bfs"]["0"] == [0, 1, 1, 1, 2, 2, 2]
    assert fx["expected"]["sssp"]["0"] == [0, 1, 4, 1, 2, 2, 2]
    assert fx["expected"]["cc"] == [0, 1, 1, 3, 4, 5, 6]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_against_reference_functions(seed):
    if oracle.ref() is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    g = HostGraph.rmat(11, 8, seed=seed, symmetrize=(seed != 3)).with_weights(1, 1000, seed=seed)
    t = g.transpose()
    for s in (0, g.max_degree_vertex(), 77):
        assert np.array_equal(oracle.bfs(g.row_offsets, g.column_indices, s),
                              oracle.ref_bfs(g.row_offsets, g.column_indices, s))
        assert np.array_equal(oracle.sssp(g.row_offsets, g.column_indices, g.edge_values, s),
                              oracle.ref_sssp(g.row_offsets, g.column_indices, g.edge_values, s))
    assert np.array_equal(oracle.cc(g.row_offsets, g.column_indices), oracle.ref_cc(g.row_offsets, g.column_indices))
    r = oracle.ref_pr(g.row_offsets, g.column_indices, t.row_offsets, t.column_indices)
    assert np.isfinite(r).all() and (r >= 0.15 - 1e-6).all()


def test_multi_root_bfs_is_min_over_roots():
    g = HostGraph.rmat(10, 8, seed=4)
    roots = [3, 99, 512]
    both = oracle.bfs(g.row_offsets, g.column_indices, roots)
    per = [oracle.bfs(g.row_offsets, g.column_indices, r) for r in roots]
    per = np.stack([np.where(p < 0, 1 << 30, p) for p in per]).min(0)
    per = np.where(per == 1 << 30, -1, per)
    assert np.array_equal(both, per)


def test_cc_push_equals_sweep_on_symmetric_graphs():
    g = HostGraph.rmat(11, 4, seed=8)
    assert np.array_equal(oracle.cc(g.row_offsets, g.column_indices), oracle.cc(g.row_offsets, g.column_indices, "push"))


def test_cc_push_directed_semantics():
    # 0 -> 1 -> 2, 3 -> 2 : min id with a path to v
    ro = np.array([0, 1, 2, 2, 3], np.int32)
    col = np.array([1, 2, 2], np.int32)
    assert oracle.cc(ro, col, "push").tolist() == [0, 0, 0, 3]


def test_pagerank_fp64_matches_dense_solve():
    g = HostGraph.rmat(8, 8, seed=2, symmetrize=False)
    t = g.transpose()
    n = g.nodes
    r, it, res = oracle.pagerank_fp64(g.row_offsets, t.row_offsets, t.column_indices, 0.85, 1e-13, 1000)
    assert res <= 1e-13 and abs(r.sum() - 1) < 1e-12
    od = np.diff(g.row_offsets)
    M = np.zeros((n, n))
    src = np.repeat(np.arange(n), od)
    np.add.at(M, (g.column_indices, src), 1.0 / od[src])
    M[:, od == 0] = 1.0 / n  # dangling mass spread uniformly
    A = np.eye(n) - 0.85 * M
    x = np.linalg.solve(A, np.full(n, 0.15 / n))
    assert np.abs(x - r).sum() < 1e-10


def test_pr_gas_restatement_close_to_reference_cpupr():
    if oracle.ref() is None:
        pytest.skip("oracle/_ref not built")
    g = HostGraph.rmat(10, 8, seed=11, symmetrize=False)
    t = g.transpose()
    od = np.diff(g.row_offsets).astype(np.int32)
    mine, _ = oracle.pr_gas(g.row_offsets, g.column_indices, t.row_offsets, t.column_indices, od, 0.01)
    ref = oracle.ref_pr(g.row_offsets, g.column_indices, t.row_offsets, t.column_indices)
    rel = np.linalg.norm(mine - ref) / np.linalg.norm(ref)
    assert rel < 0.1  # the reference's own check (PageRank.cu:305-315, tol default 0.1)


def test_bfs_pred_known_answer_directed():
    # 0->1, 0->2, 1->3, 2->3, 3->4, 5->0. From 0: depths [0, 1, 1, 2, 3, -1]. pred_extract's
    # rule takes the largest in-neighbour one level up; the root's unreached in-neighbour 5
    # (depth -1) also satisfies depth[v] - depth[u] == 1, as in the reference's arithmetic.
    ro = np.array([0, 2, 3, 4, 5, 5, 6], np.int32)
    col = np.array([1, 2, 3, 3, 4, 0], np.int32)
    g = HostGraph(ro, col, directed=True)
    t = g.transpose()
    d = oracle.bfs(ro, col, 0)
    assert d.tolist() == [0, 1, 1, 2, 3, -1]
    assert oracle.bfs_pred(t.row_offsets, t.column_indices, d).tolist() == [5, 0, 0, 2, 3, -1]


@pytest.mark.parametrize("seed", [1, 2])
def test_bfs_pred_is_a_bfs_tree(seed):
    # Graph500-style checks: every reached non-root vertex has a predecessor that is an
    # in-neighbour one level up, and it is the largest such in-neighbour.
    g = HostGraph.rmat(12, 8, seed=seed)
    src = g.max_degree_vertex()
    d = oracle.bfs(g.row_offsets, g.column_indices, src)
    p = oracle.bfs_pred(g.row_offsets, g.column_indices, d)
    assert p[src] == -1 and (p[d < 0] == -1).all()
    for v in np.flatnonzero(d > 0):
        nb = g.column_indices[g.row_offsets[v]:g.row_offsets[v + 1]]
        up = nb[d[nb] == d[v] - 1]
        assert len(up) > 0 and p[v] == up.max()
