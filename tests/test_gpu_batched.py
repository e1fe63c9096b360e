"""GPU parity of the batched traversals: the 64-bit mask-frontier BFS/SSSP must
equal independent per-source runs bit for bit, and the multi-graph batch must
equal one BFS per graph."""
import numpy as np
import pytest

import oracle
from gpugraph_b200 import SSSP_INF, Graph, HostGraph, MapGraphError, _lib, concat_graphs

pytestmark = pytest.mark.gpu

DIRS = [_lib.MG_DIR_AUTO, _lib.MG_DIR_PUSH, _lib.MG_DIR_PULL]


def seeded_sources(hg, n, seed=1):
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(np.diff(hg.row_offsets) > 0)
    return rng.choice(cand, size=n, replace=False).astype(np.int32)


@pytest.mark.parametrize("scale,ef,nsrc", [(14, 16, 64), (12, 8, 17), (10, 4, 1)])
def test_bfs_multi_rmat(scale, ef, nsrc):
    hg = HostGraph.rmat(scale, ef, seed=scale)
    g = Graph(hg)
    srcs = seeded_sources(hg, nsrc)
    ref = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in srcs])
    for d in DIRS:
        out, st = g.bfs_multi(srcs, direction=d)
        assert np.array_equal(out, ref), d
        reached = ref >= 0
        deg = hg.out_degree()
        assert st["vertices_reached"] == int(reached.sum())
        assert st["edges_traversed"] == int((reached * deg[None, :]).sum())


# direction policies of a deep traversal: push and pull levels before and past
# the 16 levels whose masks the level stack keeps; the last one flips between
# push and pull whenever the frontier grows or shrinks
ROAD_MODES = [dict(direction=d) for d in DIRS] + [dict(direction=_lib.MG_DIR_AUTO, alpha_multi=1e9, beta=0.5)]


@pytest.mark.parametrize("mode", ROAD_MODES)
def test_bfs_multi_road_grid_and_duplicate_sources(mode):
    hg = HostGraph.road_grid(150, 0.02, 0.005, seed=5)
    g = Graph(hg)
    srcs = np.array([0, 11249, 22499, 0, 500] + list(range(1000, 1059)), np.int32)  # 64, with a duplicate
    out, st = g.bfs_multi(srcs, **mode)
    ref = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in srcs])
    assert np.array_equal(out, ref)
    assert st["iterations"] >= int(ref.max())
    if mode.get("beta") == 0.5:
        assert st["push_iterations"] > 2 and st["pull_iterations"] > 2


def test_bfs_multi_directed():
    hg = HostGraph.rmat(12, 8, seed=21, symmetrize=False)
    g = Graph(hg, directed=True)
    srcs = seeded_sources(hg, 40, seed=3)
    ref = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in srcs])
    for d in DIRS:
        assert np.array_equal(g.bfs_multi(srcs, direction=d)[0], ref), d


def test_bfs_multi_runs_in_a_row():
    # runs on one graph in a row, with a run cut short by iter_num and a batched
    # SSSP (which shares the frontier mask arrays) in between
    hg = HostGraph.rmat(13, 16, seed=12).with_weights(1, 20, seed=12)
    g = Graph(hg)
    a, b = seeded_sources(hg, 64, seed=1), seeded_sources(hg, 40, seed=2)
    ref_a = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in a])
    ref_b = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in b])
    for _ in range(2):
        assert np.array_equal(g.bfs_multi(a)[0], ref_a)
        assert np.array_equal(g.bfs_multi(b)[0], ref_b)
    cut, st = g.bfs_multi(a, iter_num=2)
    assert st["iterations"] == 2 and not st["converged"]
    assert np.array_equal(np.where(cut >= 0, cut, ref_a), ref_a) and (cut == -1).sum() > (ref_a == -1).sum()
    assert np.array_equal(g.bfs_multi(b)[0], ref_b)
    g.sssp_multi(a)
    assert np.array_equal(g.bfs_multi(a)[0], ref_a)


@pytest.mark.parametrize("extra", [1, 2, 3])
def test_multi_vertex_count_not_a_multiple_of_four(extra):
    # an R-MAT graph with 1-3 isolated vertices appended: the results leave in
    # [nsrc][V] rows that do not start 16-byte aligned, and the last 32-vertex
    # group and the last step of the transpose's CTAs are partial
    base = HostGraph.rmat(11, 8, seed=17).with_weights(1, 30, seed=17)
    ro = np.concatenate([base.row_offsets, np.full(extra, base.row_offsets[-1], np.int32)])
    hg = HostGraph(ro, base.column_indices, base.edge_values)
    assert hg.nodes % 4 == extra
    g = Graph(hg)
    srcs = np.concatenate([seeded_sources(hg, 20, seed=extra), [hg.nodes - 1]]).astype(np.int32)
    ref = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in srcs])
    for d in DIRS:
        assert np.array_equal(g.bfs_multi(srcs, direction=d)[0], ref), d
    out, _ = g.sssp_multi(srcs)
    for k in (0, 7, len(srcs) - 1):
        assert np.array_equal(out[k], oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, srcs[k])), k


def test_bfs_multi_host_loop_equals_graph_loop():
    hg = HostGraph.rmat(13, 16, seed=2)
    g = Graph(hg)
    srcs = seeded_sources(hg, 64)
    a, _ = g.bfs_multi(srcs, use_cuda_graph=1)
    b, _ = g.bfs_multi(srcs, use_cuda_graph=0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("scale,hi,nsrc", [(13, 64, 64), (11, 1000, 9)])
def test_sssp_multi_rmat(scale, hi, nsrc):
    hg = HostGraph.rmat(scale, 16, seed=scale).with_weights(1, hi, seed=4)
    g = Graph(hg)
    srcs = seeded_sources(hg, nsrc, seed=2)
    out, st = g.sssp_multi(srcs)
    for k, s in enumerate(srcs):
        assert np.array_equal(out[k], oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, s)), k
    single, _ = g.sssp(int(srcs[0]))
    assert np.array_equal(single, out[0])


def test_sssp_multi_road_grid_unreachable():
    hg = HostGraph.road_grid(120, 0.3, 0.0, seed=8).with_weights(1, 1000, seed=8)  # 30% dropped: islands
    g = Graph(hg)
    srcs = np.arange(0, 14400, 225, dtype=np.int32)[:64]
    out, _ = g.sssp_multi(srcs)
    for k in (0, 17, 63):
        ref = oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, srcs[k])
        assert np.array_equal(out[k], ref)
    assert (out == SSSP_INF).any()


def test_multi_argument_errors():
    hg = HostGraph.rmat(8, 4, seed=1)
    g = Graph(hg)
    with pytest.raises(MapGraphError) as e:
        g.bfs_multi(np.arange(65, dtype=np.int32))
    assert e.value.status == _lib.MG_ERR_ARG
    with pytest.raises(MapGraphError) as e:
        g.bfs_multi(np.array([0, 1 << 20], np.int32))
    assert e.value.status == _lib.MG_ERR_ARG
    with pytest.raises(MapGraphError) as e:
        g.sssp_multi(np.array([0], np.int32))
    assert e.value.status == _lib.MG_ERR_UNSUPPORTED


def test_graph_batch_bfs():
    rng = np.random.default_rng(7)
    graphs = [HostGraph.rmat(int(s), 8, seed=100 + i) for i, s in enumerate(rng.integers(6, 12, size=24))]
    big = concat_graphs(graphs)
    g = Graph(big)
    local = np.array([h.max_degree_vertex() for h in graphs], np.int32)
    out, st = g.bfs_batch(local)
    for i, h in enumerate(graphs):
        b, e = big.graph_offsets[i], big.graph_offsets[i + 1]
        assert np.array_equal(out[b:e], oracle.bfs(h.row_offsets, h.column_indices, local[i])), i
    with pytest.raises(MapGraphError):
        g.bfs_batch(np.full(24, 1 << 20, np.int32))


def test_multi_isolated_sources_and_edge_free_graph():
    # sources with no out-edges finish at level 0 while the others keep expanding; an
    # edge-free graph ends after the first level for every source
    hg = HostGraph.rmat(12, 4, seed=31).with_weights(1, 50, seed=31)
    iso = np.flatnonzero(hg.out_degree() == 0)
    assert iso.size >= 8
    srcs = np.concatenate([iso[:8], seeded_sources(hg, 56, seed=9)]).astype(np.int32)
    g = Graph(hg)
    ref = np.stack([oracle.bfs(hg.row_offsets, hg.column_indices, s) for s in srcs])
    for d in DIRS:
        assert np.array_equal(g.bfs_multi(srcs, direction=d)[0], ref), d
    out, _ = g.sssp_multi(srcs)
    for k in (0, 7, 8, 63):
        assert np.array_equal(out[k], oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, srcs[k])), k
    for k in range(8):
        assert (out[k] == SSSP_INF).sum() == hg.nodes - 1 and out[k][srcs[k]] == 0
    n = 300
    empty = HostGraph(np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    ge = Graph(empty)
    s = np.array([0, 299, 5, 5], np.int32)
    bo, _ = ge.bfs_multi(s)
    so, _ = ge.sssp_multi(s)
    for k, v in enumerate(s):
        exp = np.full(n, -1, np.int32)
        exp[v] = 0
        assert np.array_equal(bo[k], exp)
        exp_s = np.full(n, SSSP_INF, np.int32)
        exp_s[v] = 0
        assert np.array_equal(so[k], exp_s)


@pytest.mark.parametrize("nsrc", [64, 20])
def test_sssp_multi_directed_duplicates_zero_weights(nsrc):
    # 64 sources run the dense relaxation mode, 20 the sparse one; duplicated sources and
    # zero-weight edges must give each row the single-source distances
    hg = HostGraph.rmat(12, 8, seed=41, symmetrize=False).with_weights(0, 9, seed=41)
    assert (hg.edge_values == 0).any()
    g = Graph(hg, directed=True)
    base = seeded_sources(hg, nsrc - 4, seed=5)
    srcs = np.concatenate([base, base[:4]]).astype(np.int32)
    out, _ = g.sssp_multi(srcs)
    for k, s in enumerate(srcs):
        assert np.array_equal(out[k], oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, s)), k
    assert np.array_equal(out[:4], out[nsrc - 4:])


def test_graph_batch_with_trivial_graphs():
    # single-vertex, edge-free and path graphs mixed with R-MAT graphs in one batch
    one = HostGraph(np.array([0, 0], np.int32), np.zeros(0, np.int32))
    bare = HostGraph(np.zeros(6, np.int32), np.zeros(0, np.int32))
    path = HostGraph(np.array([0, 1, 3, 5, 6], np.int32), np.array([1, 0, 2, 1, 3, 2], np.int32))
    graphs = [one, HostGraph.rmat(9, 8, seed=3), bare, path, one, HostGraph.rmat(7, 4, seed=4), path]
    big = concat_graphs(graphs)
    g = Graph(big)
    local = np.array([0, graphs[1].max_degree_vertex(), 4, 0, 0, 3, 2], np.int32)
    out, _ = g.bfs_batch(local)
    for i, h in enumerate(graphs):
        b, e = big.graph_offsets[i], big.graph_offsets[i + 1]
        assert np.array_equal(out[b:e], oracle.bfs(h.row_offsets, h.column_indices, local[i])), i


def test_bfs_multi_deeper_than_16bit_depth_rows():
    # a path of 66,000 vertices: depths past 65,534 do not fit the 16-bit depth rows
    # the batched BFS keeps, so the run is redone with 32-bit rows; a shallower
    # source set on the same graph stays on the 16-bit rows
    n = 66000
    ro = np.concatenate([[0], np.cumsum([1] + [2] * (n - 2) + [1])]).astype(np.int32)
    col = np.empty(ro[-1], np.int32)
    for v in range(n):
        nb = [u for u in (v - 1, v + 1) if 0 <= u < n]
        col[ro[v]:ro[v + 1]] = nb
    hg = HostGraph(ro, col, None)
    g = Graph(hg)
    for srcs in (np.array([0, n - 1, n // 2], np.int32), np.array([n // 2, n // 2 + 7], np.int32)):
        out, st = g.bfs_multi(srcs, direction=_lib.MG_DIR_PUSH)
        ref = np.stack([oracle.bfs(ro, col, s) for s in srcs])
        assert np.array_equal(out, ref)
        assert st["iterations"] >= int(ref.max())
    assert int(oracle.bfs(ro, col, 0).max()) == n - 1

