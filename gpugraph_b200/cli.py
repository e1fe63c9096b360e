"""Command-line driver mirroring the reference's algorithm drivers
(Algorithms/{BFS,SSSP,CC,PageRank}/*.cu main(): -g graph.mtx, -o output,
-s sources file, -p "k=v k=v", -c config file; Algorithms/SSSP/sssp.cu:185-265).

    python -m gpugraph_b200.cli bfs -g graph.mtx -s srcs.txt -o out.txt
    python -m gpugraph_b200.cli sssp --rmat 20 -p "src=0 direction=push"
    python -m gpugraph_b200.cli bfs_multi --rmat 22 --nsrc 64 --repeat 3
    python -m gpugraph_b200.cli ppr --rmat 20 --directed --nsrc 32

Parameters (-p / -c) use the reference's knob names where they exist:
src, directed, iter_num, threshold, tol (PageRank), plus direction
(auto|push|pull), alpha, beta, use_cuda_graph, ctas_per_sm. Unknown keys are
an error (the reference dereferences end() on them, Algorithms/BFS/config.cpp:66-72).
Synthetic inputs: --rmat SCALE [--ef 16 --seed 1 --directed] or --grid WIDTH.
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

from . import Graph, HostGraph
from ._lib import MG_DIR_AUTO, MG_DIR_PULL, MG_DIR_PUSH

KNOWN = {"src", "directed", "iter_num", "threshold", "tol", "direction", "alpha", "beta", "alpha_multi",
         "use_cuda_graph", "ctas_per_sm", "run_CPU", "weights", "csv_format"}
DIRS = {"auto": MG_DIR_AUTO, "push": MG_DIR_PUSH, "pull": MG_DIR_PULL}


def parse_params(text: str) -> dict:
    out = {}
    for tok in text.split():
        if "=" not in tok:
            raise SystemExit(f"bad parameter '{tok}' (expected key=value)")
        k, v = tok.split("=", 1)
        if k not in KNOWN:
            raise SystemExit(f"unknown parameter '{k}'; known: {sorted(KNOWN)}")
        out[k] = v
    return out


def options_from(params: dict) -> dict:
    kw = {}
    if "iter_num" in params:
        kw["iter_num"] = int(params["iter_num"])
    if "threshold" in params:
        kw["threshold"] = int(params["threshold"])
    if "direction" in params:
        kw["direction"] = DIRS[params["direction"]]
    for k in ("alpha", "beta", "alpha_multi"):
        if k in params:
            kw[k] = float(params[k])
    for k in ("use_cuda_graph", "ctas_per_sm"):
        if k in params:
            kw[k] = int(params[k])
    return kw


def run_ppr(g: Graph, hg: HostGraph, nvec: int, seed: int, tol: float, options: dict | None = None):
    """Differentiable personalised PageRank, forward and backward of the loss
    <C, R>: lognormal(0, 1) edge weights normalised per row, nvec teleport
    vectors each uniform over 100 seeded vertices, C ~ N(0, 1). Returns the
    ranks [V, nvec] and device time / iteration counts of both passes."""
    import torch

    from .ppr import ppr

    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 1.0, size=hg.edges)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    w = w / np.bincount(src, weights=w, minlength=hg.nodes)[src]
    k = min(100, hg.nodes)
    tele = np.zeros((hg.nodes, nvec), np.float32)
    for c in range(nvec):
        tele[rng.choice(hg.nodes, k, replace=False), c] = 1.0 / k
    wt = torch.tensor(w, dtype=torch.float32, device="cuda", requires_grad=True)
    tt = torch.tensor(tele, device="cuda", requires_grad=True)
    cm = torch.tensor(rng.standard_normal((hg.nodes, nvec)), dtype=torch.float32, device="cuda")
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    r = ppr(g, wt, tt, tol=tol, **{k: v for k, v in (options or {}).items() if k == "use_cuda_graph"})
    e1.record()
    (r * cm).sum().backward()
    e2.record()
    torch.cuda.synchronize()
    fwd, total = e0.elapsed_time(e1), e0.elapsed_time(e2)
    print(f"ppr: {nvec} vectors, forward {fwd:.3f} ms, backward {total - fwd:.3f} ms", file=sys.stderr)
    st = {"device_ms": total, "iterations": 0, "push_iterations": 0, "pull_iterations": 0,
          "edges_traversed": 0}
    return r.detach().cpu().numpy(), st


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="gpugraph_b200.cli")
    ap.add_argument("algo", choices=["bfs", "bfs_multi", "sssp", "sssp_multi", "cc", "pagerank", "pagerank_gas",
                                     "ppr"])
    ap.add_argument("-g", "--graph")
    ap.add_argument("-o", "--output")
    ap.add_argument("-s", "--sources")
    ap.add_argument("-p", "--params", default="")
    ap.add_argument("-c", "--config")
    ap.add_argument("--rmat", type=int)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--directed", action="store_true")
    ap.add_argument("--grid", type=int)
    ap.add_argument("--nsrc", type=int, default=64)
    ap.add_argument("--repeat", type=int, default=1)
    args = ap.parse_args(argv)
    params = {}
    if args.config:
        with open(args.config) as f:
            params.update(parse_params(" ".join(ln.split("#")[0] for ln in f)))
    params.update(parse_params(args.params))
    kw = options_from(params)

    if args.graph:
        directed = params.get("directed", "1") != "0"
        if args.graph.endswith(".csv"):
            # the reference's BFS driver reads CSV graphs as undirected adjacency rows (bfs.cu:519-520)
            hg = HostGraph.read_csv(args.graph, params.get("csv_format", "adjacency"), undirected=not directed)
        else:
            hg = HostGraph.read_market(args.graph, undirected=not directed)
    elif args.rmat:
        hg = HostGraph.rmat(args.rmat, args.ef, seed=args.seed, symmetrize=not args.directed)
    elif args.grid:
        hg = HostGraph.road_grid(args.grid, seed=args.seed)
    else:
        raise SystemExit("give -g FILE, --rmat SCALE or --grid WIDTH")
    if args.algo.startswith("sssp") and (hg.edge_values is None or "weights" in params):
        lo, hi = (1, 64) if "weights" not in params else map(int, params["weights"].split(":"))
        hg = hg.with_weights(lo, hi, seed=args.seed)
    g = Graph(hg, directed=hg.directed)
    if args.sources:
        srcs = np.loadtxt(args.sources, dtype=np.int64, ndmin=1).astype(np.int32)
    elif "src" in params:
        srcs = np.array([int(params["src"])], np.int32)
    elif args.algo.endswith("_multi"):
        rng = np.random.default_rng(args.seed)
        cand = np.flatnonzero(np.diff(hg.row_offsets) > 0)
        srcs = np.sort(rng.choice(cand, size=min(args.nsrc, len(cand)), replace=False)).astype(np.int32)
    else:
        srcs = np.array([hg.max_degree_vertex()], np.int32)

    print(f"graph: {hg.nodes} nodes, {hg.edges} directed edges", file=sys.stderr)
    result = None
    for rep in range(args.repeat):
        t0 = time.perf_counter()
        if args.algo == "bfs":
            result, st = g.bfs(int(srcs[0]), **kw)
        elif args.algo == "bfs_multi":
            result, st = g.bfs_multi(srcs, **kw)
        elif args.algo == "sssp":
            result, st = g.sssp(int(srcs[0]), **kw)
        elif args.algo == "sssp_multi":
            result, st = g.sssp_multi(srcs, **kw)
        elif args.algo == "cc":
            result, st = g.cc(**kw)
        elif args.algo == "pagerank":
            result, st = g.pagerank(**({"tolerance": float(params["tol"])} if "tol" in params else {}), **kw)
        elif args.algo == "ppr":
            result, st = run_ppr(g, hg, args.nsrc, args.seed, float(params.get("tol", 1e-7)), kw)
        else:
            result, st = g.pagerank_gas(tolerance=float(params.get("tol", 0.01)), **kw)
        wall = (time.perf_counter() - t0) * 1e3
        teps = st["edges_traversed"] / (st["device_ms"] * 1e-3) / 1e6 if st["device_ms"] else 0.0
        # the reference prints "Kernel time took", "visited edges", "M-Edges / sec" (README:67-75)
        print(f"[{rep}] Kernel time took: {st['device_ms']:.4f} ms  Wall time took: {wall:.4f} ms  "
              f"iterations: {st['iterations']} (push {st['push_iterations']}, pull {st['pull_iterations']})  "
              f"visited edges: {st['edges_traversed']}  M-Edges / sec: {teps:.1f}")
    if args.output and result is not None:
        np.savetxt(args.output, np.asarray(result).reshape(-1), fmt="%.9g" if result.dtype.kind == "f" else "%d")
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
