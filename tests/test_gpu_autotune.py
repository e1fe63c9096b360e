"""The autotuner times real candidates on the GPU and returns options that keep
results exact."""
import json

import numpy as np
import pytest

import oracle
from gpugraph_b200 import Graph, HostGraph
from gpugraph_b200.autotune import autotune

pytestmark = pytest.mark.gpu


def test_autotune_bfs_multi_and_sssp(tmp_path):
    hg = HostGraph.rmat(14, 16, seed=2).with_weights(1, 64, seed=2)
    g = Graph(hg)
    rng = np.random.default_rng(0)
    srcs = rng.choice(np.flatnonzero(np.diff(hg.row_offsets) > 0), 64, replace=False).astype(np.int32)
    rec = tmp_path / "tuning.json"
    best, report = autotune(g, "bfs_multi", srcs, record=str(rec))
    assert best["tile_items"] in (1024, 2048) and 2 <= best["ctas_per_sm"] <= 5
    assert len(report["trials"]) >= 8 and report["best_ms"] > 0
    assert len(json.loads(rec.read_text())) == 1
    out, _ = g.bfs_multi(srcs, **best)
    for k in (0, 63):
        assert np.array_equal(out[k], oracle.bfs(hg.row_offsets, hg.column_indices, srcs[k]))
    best_s, _ = autotune(g, "sssp", srcs[:2])
    d, _ = g.sssp(int(srcs[0]), **best_s)
    assert np.array_equal(d, oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, srcs[0]))
    best_b, _ = autotune(g, "bfs", srcs[:4])
    assert np.array_equal(g.bfs(int(srcs[1]), **best_b)[0], oracle.bfs(hg.row_offsets, hg.column_indices, srcs[1]))


def test_autotune_pagerank_and_ppr():
    import torch

    from gpugraph_b200.ppr import ppr

    hg = HostGraph.rmat(13, 8, seed=5, symmetrize=False)
    g = Graph(hg, directed=True)
    best, report = autotune(g, "pagerank")
    assert 2 <= best["ctas_per_sm"] <= 8 and len(report["trials"]) == 7
    t = hg.transpose()
    r, st = g.pagerank(ctas_per_sm=best["ctas_per_sm"])
    ref, _, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 0.0, st["iterations"])
    assert np.abs(r - ref).sum() <= 1e-6
    srcs = np.array([0, 5, 77, 4000], np.int32)
    best_p, report_p = autotune(g, "ppr", srcs)
    assert 2 <= best_p["ctas_per_sm"] <= 8 and len(report_p["trials"]) == 7
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    w = 1.0 / np.diff(hg.row_offsets)[src]
    T = np.zeros((hg.nodes, 4), np.float32)
    T[srcs, np.arange(4)] = 1.0
    wt = torch.tensor(w, dtype=torch.float32, device="cuda")
    Tt = torch.tensor(T, device="cuda")
    a = ppr(g, wt, Tt)
    b = ppr(g, wt, Tt, ctas_per_sm=best_p["ctas_per_sm"])
    assert torch.allclose(a, b, atol=1e-6)
