"""Differentiable personalised PageRank: forward against a dense FP64 solve,
gradients against FP64 central finite differences on a scale-10 subgraph and
against a dense torch FP64 autograd reference."""
import numpy as np
import pytest

from gpugraph_b200 import Graph, HostGraph

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

D = 0.85


def _setup(scale=10, ef=16, nvec=32, seed=0):
    from gpugraph_b200.ppr import ppr  # noqa: F401

    hg = HostGraph.rmat(scale, ef, seed=seed + 3, symmetrize=False)
    g = Graph(hg, directed=True)
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 1.0, size=hg.edges)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    rowsum = np.bincount(src, weights=w, minlength=hg.nodes)
    w = w / rowsum[src]  # row-normalised
    T = np.zeros((hg.nodes, nvec))
    for c in range(nvec):
        pick = rng.choice(hg.nodes, size=min(100, hg.nodes), replace=False)
        T[pick, c] = 1.0 / len(pick)
    C = rng.standard_normal((hg.nodes, nvec))
    return hg, g, src, w, T, C


def _dense_solve(hg, src, w, T):
    n = hg.nodes
    P = torch.zeros((n, n), dtype=torch.float64)
    P.index_put_((torch.as_tensor(src), torch.as_tensor(hg.column_indices.astype(np.int64))),
                 torch.as_tensor(w), accumulate=True)
    A = torch.eye(n, dtype=torch.float64) - D * P.T
    return torch.linalg.solve(A, (1 - D) * T), P


@pytest.mark.parametrize("nvec", [32, 5, 12, 40, 64])
def test_ppr_forward_matches_dense_fp64(nvec):
    # nvec % 4 == 0 runs the 16-byte-row kernel (4 or 2 chunks per warp), other
    # counts the column-per-lane kernel; nvec > 32 takes two columns per lane
    from gpugraph_b200.ppr import ppr

    hg, g, src, w, T, _ = _setup(nvec=nvec)
    R_ref, _ = _dense_solve(hg, src, w, torch.as_tensor(T))
    R = ppr(g, torch.tensor(w, dtype=torch.float32, device="cuda"), torch.tensor(T, dtype=torch.float32,
                                                                               device="cuda"))
    err = (R.double().cpu() - R_ref).abs()
    assert err.sum(0).max() < 2e-5, float(err.sum(0).max())  # per-column L1


def test_ppr_gradients_vs_dense_autograd_and_finite_differences():
    from gpugraph_b200.ppr import ppr

    hg, g, src, w, T, Cm = _setup()
    wt = torch.tensor(w, dtype=torch.float32, device="cuda", requires_grad=True)
    Tt = torch.tensor(T, dtype=torch.float32, device="cuda", requires_grad=True)
    Ct = torch.tensor(Cm, dtype=torch.float32, device="cuda")
    loss = (ppr(g, wt, Tt) * Ct).sum()
    loss.backward()
    gw, gT = wt.grad.double().cpu(), Tt.grad.double().cpu()

    # dense torch FP64 reference gradient: edge weights enter P at (src, dst)
    w64 = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    T64 = torch.tensor(T, dtype=torch.float64, requires_grad=True)
    n = hg.nodes
    P = torch.zeros((n, n), dtype=torch.float64).index_put(
        (torch.as_tensor(src), torch.as_tensor(hg.column_indices.astype(np.int64))), w64, accumulate=True)
    R64 = torch.linalg.solve(torch.eye(n, dtype=torch.float64) - D * P.T, (1 - D) * T64)
    L64 = (R64 * torch.tensor(Cm)).sum()
    L64.backward()
    rel_w = (gw - w64.grad).norm() / w64.grad.norm()
    rel_t = (gT - T64.grad).norm() / T64.grad.norm()
    assert rel_w < 1e-4 and rel_t < 1e-4, (float(rel_w), float(rel_t))

    # FP64 central finite differences on a few coordinates
    rng = np.random.default_rng(5)

    def L_of(wv, Tv):
        Pm = torch.zeros((n, n), dtype=torch.float64).index_put(
            (torch.as_tensor(src), torch.as_tensor(hg.column_indices.astype(np.int64))), wv, accumulate=True)
        Rm = torch.linalg.solve(torch.eye(n, dtype=torch.float64) - D * Pm.T, (1 - D) * Tv)
        return float((Rm * torch.tensor(Cm)).sum())

    h = 1e-6
    base_w, base_T = torch.tensor(w, dtype=torch.float64), torch.tensor(T, dtype=torch.float64)
    for e in rng.choice(hg.edges, size=6, replace=False):
        wp, wm = base_w.clone(), base_w.clone()
        wp[e] += h
        wm[e] -= h
        fd = (L_of(wp, base_T) - L_of(wm, base_T)) / (2 * h)
        assert abs(fd - float(gw[e])) <= 1e-3 * max(1.0, abs(fd)), (e, fd, float(gw[e]))
    for (v, c) in zip(rng.integers(0, n, 4), rng.integers(0, T.shape[1], 4)):
        Tp, Tm = base_T.clone(), base_T.clone()
        Tp[v, c] += h
        Tm[v, c] -= h
        fd = (L_of(base_w, Tp) - L_of(base_w, Tm)) / (2 * h)
        assert abs(fd - float(gT[v, c])) <= 1e-3 * max(1.0, abs(fd)), (v, c, fd, float(gT[v, c]))


@pytest.mark.parametrize("nvec", [40, 7])
def test_ppr_gradients_other_column_counts(nvec):
    # two columns per lane (nvec > 32, 16-byte rows) and the column-per-lane
    # kernel (nvec = 7) against the dense FP64 autograd gradient
    from gpugraph_b200.ppr import ppr

    hg, g, src, w, T, Cm = _setup(nvec=nvec, seed=2)
    wt = torch.tensor(w, dtype=torch.float32, device="cuda", requires_grad=True)
    Tt = torch.tensor(T, dtype=torch.float32, device="cuda", requires_grad=True)
    (ppr(g, wt, Tt) * torch.tensor(Cm, dtype=torch.float32, device="cuda")).sum().backward()
    w64 = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    T64 = torch.tensor(T, dtype=torch.float64, requires_grad=True)
    n = hg.nodes
    P = torch.zeros((n, n), dtype=torch.float64).index_put(
        (torch.as_tensor(src), torch.as_tensor(hg.column_indices.astype(np.int64))), w64, accumulate=True)
    R64 = torch.linalg.solve(torch.eye(n, dtype=torch.float64) - D * P.T, (1 - D) * T64)
    (R64 * torch.tensor(Cm)).sum().backward()
    rel_w = (wt.grad.double().cpu() - w64.grad).norm() / w64.grad.norm()
    rel_t = (Tt.grad.double().cpu() - T64.grad).norm() / T64.grad.norm()
    assert rel_w < 1e-4 and rel_t < 1e-4, (float(rel_w), float(rel_t))


def test_ppr_rejects_symmetric_graph_and_host_pointers():
    from gpugraph_b200 import MapGraphError
    from gpugraph_b200.ppr import ppr

    hg = HostGraph.rmat(8, 4, seed=1)
    g = Graph(hg)  # symmetric
    with pytest.raises(MapGraphError):
        ppr(g, torch.ones(hg.edges, device="cuda"), torch.ones((hg.nodes, 4), device="cuda"))
    gd = Graph(HostGraph.rmat(8, 4, seed=1, symmetrize=False), directed=True)
    with pytest.raises(TypeError):
        ppr(gd, torch.ones(gd.edges), torch.ones((gd.nodes, 4)))
