"""Generates tests/golden/*.json from the reference's own CPU functions.

Run in a checkout where the reference tree is present (oracle/_ref is built
from it by oracle/build_ref.sh; both read its location from $MG_REFERENCE):

    MG_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Each fixture stores a small graph (derived CSR arrays, not the reference's
files) together with the outputs of CPUBFS / CPUSSSP / CPUCC / CPUPR on it, so
a machine without the reference tree can check parity against them. R-MAT fixtures store only a SHA-256 of the CSR the seeded builder
must reproduce, plus the expected outputs.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from gpugraph_b200 import HostGraph  # noqa: E402

OUT = Path(__file__).resolve().parent
# the reference checkout: $MG_REFERENCE, as for oracle/build_ref.sh
REF_GRAPHS = Path(os.environ.get("MG_REFERENCE", "/root/reference")) / "smallRegressionGraphs"


def csr_sha(g: HostGraph) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.row_offsets, np.int32).tobytes())
    h.update(np.ascontiguousarray(g.column_indices, np.int32).tobytes())
    if g.edge_values is not None:
        h.update(np.ascontiguousarray(g.edge_values, np.int32).tobytes())
    return h.hexdigest()


def outputs(g: HostGraph, srcs: list[int]) -> dict:
    t = g.transpose()
    res = {"bfs": {}, "sssp": {}}
    for s in srcs:
        res["bfs"][str(s)] = oracle.ref_bfs(g.row_offsets, g.column_indices, s).tolist()
        if g.edge_values is not None:
            res["sssp"][str(s)] = oracle.ref_sssp(g.row_offsets, g.column_indices, g.edge_values, s).tolist()
    res["cc"] = oracle.ref_cc(g.row_offsets, g.column_indices).tolist()
    res["pr_ref"] = [float(x) for x in oracle.ref_pr(g.row_offsets, g.column_indices, t.row_offsets, t.column_indices)]
    return res


def main() -> None:
    if oracle.ref() is None:
        oracle.build()
    assert oracle.ref() is not None, "oracle/_ref could not be built (reference tree missing?)"
    for name in ("small", "trivialGraph", "chesapeake"):
        g = HostGraph.read_market(str(REF_GRAPHS / f"{name}.mtx"), undirected=False)
        srcs = list(range(g.nodes)) if g.nodes <= 8 else [0, 1, 5, g.max_degree_vertex()]
        fx = {
            "source": f"smallRegressionGraphs/{name}.mtx read as directed (ReadMarketStream + FromCoo)",
            "nodes": g.nodes, "edges": g.edges,
            "row_offsets": g.row_offsets.tolist(), "column_indices": g.column_indices.tolist(),
            "edge_values": g.edge_values.tolist(),
            "sources": srcs,
            "expected": outputs(g, srcs),
        }
        (OUT / f"mtx_{name}.json").write_text(json.dumps(fx))
    for scale, ef, seed, sym in ((10, 16, 1, True), (11, 8, 7, True), (10, 16, 3, False)):
        g = HostGraph.rmat(scale, ef, seed=seed, symmetrize=sym).with_weights(1, 64, seed=seed)
        srcs = [g.max_degree_vertex(), 1, 17]
        fx = {
            "source": f"mg_build_rmat(scale={scale}, edgefactor={ef}, seed={seed}, symmetrize={int(sym)}, clean=1)"
                      f" + mg_build_weights(1, 64, seed={seed})",
            "scale": scale, "edgefactor": ef, "seed": seed, "symmetrize": sym,
            "nodes": g.nodes, "edges": g.edges, "csr_sha256": csr_sha(g),
            "sources": srcs,
            "expected": outputs(g, srcs),
        }
        (OUT / f"rmat_s{scale}_ef{ef}_seed{seed}_{'sym' if sym else 'dir'}.json").write_text(json.dumps(fx))
    print("wrote", sorted(p.name for p in OUT.glob("*.json")))


if __name__ == "__main__":
    main()
