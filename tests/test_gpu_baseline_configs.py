"""Parity of the CUDA path against the oracle at the full benchmark sizes.

Every benchmarked configuration, on the same seeded inputs the benchmark uses:
  1. plain BFS on undirected R-MAT scale 16 (edgefactor 16) from the hub;
  2. SSSP from 8 seeded sources (weights [1, 64]) and CC on undirected R-MAT 22;
  3. FP32 PageRank on directed R-MAT 23 and on the 1200x1200 road grid, against
     the FP64 oracle at the same iteration count;
  4. 64-source batched BFS and SSSP on R-MAT 22 and on the road grid (weights
     [1, 1000]), every source row, and all 256 graphs of the many-graph batch;
  5. personalised PageRank on directed R-MAT 20 (32 teleport vectors) against an
     FP64 sparse power iteration, and its gradients against FP64 central finite
     differences and a dense FP64 autograd reference on a 1,024-vertex subgraph
     induced from that graph.
BFS depths, SSSP distances and CC labels must be bit-exact. The oracle runs the
sources in parallel in spawned processes (oracle/pool.py).
"""
import numpy as np
import pytest

import oracle
from gpugraph_b200 import Graph, HostGraph, _lib, concat_graphs
from oracle import pool

pytestmark = pytest.mark.gpu

SEED = 1
NSRC = 64
PR_L1_TOL = 1e-6      # FP32 PageRank vs FP64, same iteration count
PPR_L1_TOL = 2e-5     # per teleport column, FP32 PPR (tolerance 1e-7) vs FP64
DIRS = [_lib.MG_DIR_AUTO, _lib.MG_DIR_PUSH, _lib.MG_DIR_PULL]


def seeded_sources(hg, n, seed=SEED):
    """n distinct seeded vertices with out-degree > 0, ascending (the benchmark's choice)."""
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(np.diff(hg.row_offsets) > 0)
    return np.sort(rng.choice(cand, size=n, replace=False)).astype(np.int32)


def _first_mismatch(a, b):
    bad = np.argwhere(a != b)
    return None if bad.size == 0 else (tuple(bad[0]), int(len(bad)))


@pytest.fixture(scope="module")
def rmat22():
    hg = HostGraph.rmat(22, 16, seed=SEED).with_weights(1, 64, seed=SEED)
    g = Graph(hg)
    srcs = seeded_sources(hg, NSRC)
    yield hg, g, srcs
    g.close()


@pytest.fixture(scope="module")
def rmat22_oracle(rmat22):
    hg, _, srcs = rmat22
    bfs, _ = pool.run_sources("bfs", hg.row_offsets, hg.column_indices, srcs)
    sssp, _ = pool.run_sources("sssp", hg.row_offsets, hg.column_indices, srcs, weights=hg.edge_values)
    return bfs, sssp


@pytest.fixture(scope="module")
def road1200():
    hg = HostGraph.road_grid(1200, 0.02, 0.005, seed=SEED).with_weights(1, 1000, seed=SEED)
    g = Graph(hg)
    yield hg, g, seeded_sources(hg, NSRC)
    g.close()


# ------------------------------------------------------------ config 1 --
def test_config1_rmat16_bfs_from_hub():
    hg = HostGraph.rmat(16, 16, seed=SEED)
    assert hg.nodes == 65536
    g = Graph(hg)
    s = hg.max_degree_vertex()
    ref = oracle.bfs(hg.row_offsets, hg.column_indices, s)
    for d in DIRS:
        depths, st = g.bfs(s, direction=d)
        assert np.array_equal(depths, ref), (d, _first_mismatch(depths, ref))
        assert st["edges_traversed"] == int(hg.out_degree()[ref >= 0].sum())
    g.close()


# ------------------------------------------------------------ config 2 --
def test_config2_rmat22_sssp_eight_sources(rmat22, rmat22_oracle):
    hg, g, srcs = rmat22
    _, ref = rmat22_oracle
    assert hg.nodes == 1 << 22 and hg.edges > 120_000_000
    for k in range(8):
        dist, st = g.sssp(int(srcs[k]))
        assert np.array_equal(dist, ref[k]), (k, _first_mismatch(dist, ref[k]))
        assert st["converged"] == 1


def test_config2_rmat22_cc(rmat22):
    hg, g, _ = rmat22
    labels, _ = g.cc()
    ref = oracle.cc(hg.row_offsets, hg.column_indices)
    assert np.array_equal(labels, ref), _first_mismatch(labels, ref)
    gen, _ = g.cc(generic_engine=1)  # the GAS cc program through the generic engine
    assert np.array_equal(gen, ref), _first_mismatch(gen, ref)


# ------------------------------------------------------------ config 4 --
def test_config4_rmat22_bfs_batched64(rmat22, rmat22_oracle):
    hg, g, srcs = rmat22
    ref, _ = rmat22_oracle
    out, st = g.bfs_multi(srcs)
    assert np.array_equal(out, ref), _first_mismatch(out, ref)
    reached = ref >= 0
    assert st["vertices_reached"] == int(reached.sum())
    assert st["edges_traversed"] == int(np.dot(reached.sum(0, dtype=np.int64), hg.out_degree()))
    # the plain engine (one source at a time) on a few of the same sources
    for k in (0, 21, 42, 63):
        d, _ = g.bfs(int(srcs[k]))
        assert np.array_equal(d, ref[k]), k


def test_config4_rmat22_sssp_batched64(rmat22, rmat22_oracle):
    hg, g, srcs = rmat22
    _, ref = rmat22_oracle
    out, st = g.sssp_multi(srcs)
    assert np.array_equal(out, ref), _first_mismatch(out, ref)
    assert st["converged"] == 1


def test_config4_road1200_batched64(road1200):
    hg, g, srcs = road1200
    assert hg.nodes == 1_440_000
    ref_b, _ = pool.run_sources("bfs", hg.row_offsets, hg.column_indices, srcs)
    ref_s, _ = pool.run_sources("sssp", hg.row_offsets, hg.column_indices, srcs, weights=hg.edge_values)
    out_b, _ = g.bfs_multi(srcs)
    assert np.array_equal(out_b, ref_b), _first_mismatch(out_b, ref_b)
    out_s, _ = g.sssp_multi(srcs)
    assert np.array_equal(out_s, ref_s), _first_mismatch(out_s, ref_s)
    for k in (0, 63):
        assert np.array_equal(g.sssp(int(srcs[k]))[0], ref_s[k]), k
        assert np.array_equal(g.bfs(int(srcs[k]))[0], ref_b[k]), k


def test_config4_256_graph_batch_every_graph():
    rng = np.random.default_rng(SEED)
    graphs = [HostGraph.rmat(int(s), 8, seed=1000 + i) for i, s in enumerate(rng.integers(10, 17, size=256))]
    big = concat_graphs(graphs)
    g = Graph(big)
    local = np.array([h.max_degree_vertex() for h in graphs], np.int32)
    out, st = g.bfs_batch(local)
    edges = 0
    for i, h in enumerate(graphs):
        b, e = big.graph_offsets[i], big.graph_offsets[i + 1]
        ref = oracle.bfs(h.row_offsets, h.column_indices, local[i])
        assert np.array_equal(out[b:e], ref), (i, _first_mismatch(out[b:e], ref))
        edges += int(h.out_degree()[ref >= 0].sum())
    assert st["edges_traversed"] == edges
    g.close()


# ------------------------------------------------------------ config 3 --
@pytest.mark.parametrize("which", ["rmat23_directed", "road1200"])
def test_config3_pagerank_fp32_vs_fp64(which):
    if which == "rmat23_directed":
        hg, directed = HostGraph.rmat(23, 16, seed=SEED, symmetrize=False), True
    else:
        hg, directed = HostGraph.road_grid(1200, 0.02, 0.005, seed=SEED), False
    g = Graph(hg, directed=directed)
    r, st = g.pagerank(damping=0.85, tolerance=1e-6, iter_num=100)
    g.close()
    t = hg.transpose() if directed else hg
    it = st["iterations"]
    ref, _, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 0.0, it)
    diff = np.abs(r.astype(np.float64) - ref)
    l1, mx = float(diff.sum()), float(diff.max())
    print(f"{which}: iterations {it} residual {st['residual']:.3e} L1 {l1:.3e} max-abs {mx:.3e}")
    assert l1 <= PR_L1_TOL, (l1, mx)
    _, it_ref, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 1e-6, 100)
    assert abs(it - it_ref) <= 1 and st["converged"] == 1


# ------------------------------------------------------------ config 5 --
D = 0.85


def _ppr_inputs(hg, nvec, rng, support=100):
    w = rng.lognormal(0.0, 1.0, size=hg.edges)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    rowsum = np.bincount(src, weights=w, minlength=hg.nodes)
    w = w / rowsum[src]
    T = np.zeros((hg.nodes, nvec))
    for c in range(nvec):
        T[rng.choice(hg.nodes, size=min(support, hg.nodes), replace=False), c] = 1.0 / min(support, hg.nodes)
    return src, w, T


def test_config5_ppr_forward_rmat20_vs_fp64_power_iteration():
    torch = pytest.importorskip("torch")
    sp = pytest.importorskip("scipy.sparse")
    from gpugraph_b200.ppr import ppr

    hg = HostGraph.rmat(20, 16, seed=SEED, symmetrize=False)
    g = Graph(hg, directed=True)
    src, w, T = _ppr_inputs(hg, 32, np.random.default_rng(SEED))
    R = ppr(g, torch.tensor(w, dtype=torch.float32, device="cuda"),
            torch.tensor(T, dtype=torch.float32, device="cuda"), damping=D, tol=1e-7)
    R = R.double().cpu().numpy()
    g.close()
    PT = sp.csr_matrix((w, (hg.column_indices.astype(np.int64), src)), shape=(hg.nodes, hg.nodes))
    # (1) every column: the FP64 residual of the FP32 result bounds its error,
    #     ||R - R*||_1 <= ||R - (1-d)T - d P^T R||_1 / (1 - d)
    res = np.abs(R - (1 - D) * T - D * (PT @ R)).sum(0)
    bound = res / (1 - D)
    print(f"ppr rmat20: max per-column residual bound {bound.max():.3e}")
    assert bound.max() <= PPR_L1_TOL, float(bound.max())
    # (2) four columns: against an FP64 power iteration run to convergence
    cols = [0, 9, 22, 31]
    X = (1 - D) * T[:, cols]
    for _ in range(400):
        Xn = (1 - D) * T[:, cols] + D * (PT @ X)
        delta = np.abs(Xn - X).sum(0).max()
        X = Xn
        if delta < 1e-13:
            break
    err = np.abs(R[:, cols] - X).sum(0)
    print(f"ppr rmat20: per-column L1 vs FP64 power iteration {err}")
    assert err.max() <= PPR_L1_TOL, err


def _induced_subgraph(hg, keep):
    """CSR of the subgraph induced by the sorted vertex set `keep`, ids renumbered in
    order (rows stay sorted), plus the original edge id of every kept edge."""
    n = hg.nodes
    new_id = np.full(n, -1, np.int64)
    new_id[keep] = np.arange(len(keep))
    src = np.repeat(np.arange(n), np.diff(hg.row_offsets))
    m = (new_id[src] >= 0) & (new_id[hg.column_indices] >= 0)
    eid = np.flatnonzero(m)
    s, d = new_id[src[eid]], new_id[hg.column_indices[eid]]
    ro = np.zeros(len(keep) + 1, np.int64)
    np.add.at(ro, s + 1, 1)
    return HostGraph(np.cumsum(ro).astype(np.int32), d.astype(np.int32), None, directed=True), s, eid


def test_config5_ppr_gradients_on_induced_scale10_subgraph():
    torch = pytest.importorskip("torch")
    from gpugraph_b200.ppr import ppr

    big = HostGraph.rmat(20, 16, seed=SEED, symmetrize=False)
    deg = big.out_degree() + np.bincount(big.column_indices, minlength=big.nodes)
    keep = np.sort(np.argsort(-deg, kind="stable")[:1024])  # the dense core of the scale-20 graph
    hg, src, _ = _induced_subgraph(big, keep)
    assert hg.nodes == 1024 and hg.edges > 10_000
    rng = np.random.default_rng(SEED + 1)
    w = rng.lognormal(0.0, 1.0, size=hg.edges)
    rowsum = np.bincount(src, weights=w, minlength=hg.nodes)
    w = w / rowsum[src]
    _, _, T = _ppr_inputs(hg, 32, rng)
    Cm = rng.standard_normal((hg.nodes, 32))
    g = Graph(hg, directed=True)
    wt = torch.tensor(w, dtype=torch.float32, device="cuda", requires_grad=True)
    Tt = torch.tensor(T, dtype=torch.float32, device="cuda", requires_grad=True)
    (ppr(g, wt, Tt, damping=D, tol=1e-7) * torch.tensor(Cm, dtype=torch.float32, device="cuda")).sum().backward()
    gw, gT = wt.grad.double().cpu(), Tt.grad.double().cpu()
    g.close()

    n = hg.nodes
    idx = (torch.as_tensor(src), torch.as_tensor(hg.column_indices.astype(np.int64)))
    Ct = torch.tensor(Cm)

    def loss(wv, Tv):
        P = torch.zeros((n, n), dtype=torch.float64).index_put(idx, wv, accumulate=True)
        return (torch.linalg.solve(torch.eye(n, dtype=torch.float64) - D * P.T, (1 - D) * Tv) * Ct).sum()

    w64 = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    T64 = torch.tensor(T, dtype=torch.float64, requires_grad=True)
    loss(w64, T64).backward()
    rel_w = float((gw - w64.grad).norm() / w64.grad.norm())
    rel_t = float((gT - T64.grad).norm() / T64.grad.norm())
    print(f"ppr subgraph: relative gradient error vs dense FP64 autograd: edges {rel_w:.2e} teleport {rel_t:.2e}")
    assert rel_w < 1e-4 and rel_t < 1e-4
    h = 1e-6
    bw, bT = torch.tensor(w, dtype=torch.float64), torch.tensor(T, dtype=torch.float64)
    with torch.no_grad():
        for e in rng.choice(hg.edges, size=6, replace=False):
            wp, wm = bw.clone(), bw.clone()
            wp[e] += h
            wm[e] -= h
            fd = float(loss(wp, bT) - loss(wm, bT)) / (2 * h)
            assert abs(fd - float(gw[e])) <= 1e-3 * max(1.0, abs(fd)), (e, fd, float(gw[e]))
        for v, c in zip(rng.integers(0, n, 4), rng.integers(0, 32, 4)):
            Tp, Tm = bT.clone(), bT.clone()
            Tp[v, c] += h
            Tm[v, c] -= h
            fd = float(loss(bw, Tp) - loss(bw, Tm)) / (2 * h)
            assert abs(fd - float(gT[v, c])) <= 1e-3 * max(1.0, abs(fd)), (v, c, fd, float(gT[v, c]))
