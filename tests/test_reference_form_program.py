"""GAS Programs written in the reference's form (host Initialize and
extractResult, device functors; tests/cpp/reference_form_programs.cu) build
against include/ alone, link against libmapgraph_b200.so and run through the
reference's driver calls (CsrProblem::FromHostProblem,
EnactorVertexCentric::EnactIterativeSearch, CsrProblem::ExtractResults):
SSSP bit-exact against the oracle on symmetric and directed graphs, and BFS
over out- and in-edges (EXPAND_ALL_EDGES) against the oracle's BFS of the
graph's undirected view."""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from gpugraph_b200 import HostGraph

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "gpugraph_b200"


def build(tmp_path) -> Path:
    so = tmp_path / "libreference_form_programs.so"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    "--expt-relaxed-constexpr", "-shared", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
                    str(ROOT / "tests/cpp/reference_form_programs.cu"), "-L", str(LIBDIR), "-lmapgraph_b200",
                    "-Xlinker", f"-rpath={LIBDIR}", "-o", str(so)], check=True, capture_output=True)
    return so


def load(so):
    lib = C.CDLL(str(so), mode=os.RTLD_NOW)  # every engine symbol resolves against the library
    P = C.c_void_p
    lib.rf_run_sssp.argtypes = [C.c_int, C.c_int, P, P, P, C.c_int, C.c_int, C.c_int, P]
    lib.rf_run_bfs_all.argtypes = [C.c_int, C.c_int, P, P, C.c_int, C.c_int, C.c_int, P]
    return lib


def test_reference_form_programs_build_against_include_only(tmp_path):
    lib = load(build(tmp_path))
    assert hasattr(lib, "rf_run_sssp") and hasattr(lib, "rf_run_bfs_all")


def _p(a):
    return a.ctypes.data


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["rmat_sym", "rmat_directed", "road"])
def test_reference_form_sssp_matches_oracle(tmp_path, kind):
    lib = load(build(tmp_path))
    if kind == "rmat_sym":
        hg = HostGraph.rmat(14, 16, seed=3).with_weights(1, 64, seed=3)
    elif kind == "rmat_directed":
        hg = HostGraph.rmat(13, 8, seed=4, symmetrize=False).with_weights(1, 1000, seed=4)
    else:
        hg = HostGraph.road_grid(100, 0.02, 0.005, seed=5).with_weights(1, 1000, seed=5)
    for src in (hg.max_degree_vertex(), 3):
        out = np.empty(hg.nodes, np.int32)
        # two enacts on one problem: the Program's lists persist, Initialize resets them
        rc = lib.rf_run_sssp(hg.nodes, hg.edges, _p(hg.row_offsets), _p(hg.column_indices), _p(hg.edge_values),
                             int(hg.directed), int(src), 2, _p(out))
        assert rc == 0, rc
        assert np.array_equal(out, oracle.sssp(hg.row_offsets, hg.column_indices, hg.edge_values, src)), src


@pytest.mark.gpu
def test_reference_form_bfs_over_all_edges(tmp_path):
    lib = load(build(tmp_path))
    hg = HostGraph.rmat(13, 4, seed=9, symmetrize=False)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    key = np.unique(np.concatenate([src * hg.nodes + hg.column_indices, hg.column_indices * hg.nodes + src]))
    u, v = key // hg.nodes, key % hg.nodes
    ro = np.concatenate([[0], np.cumsum(np.bincount(u, minlength=hg.nodes))]).astype(np.int32)
    for s in (hg.max_degree_vertex(), int(np.argmin(hg.out_degree()))):
        out = np.empty(hg.nodes, np.int32)
        rc = lib.rf_run_bfs_all(hg.nodes, hg.edges, _p(hg.row_offsets), _p(hg.column_indices), 1, int(s), 1,
                                _p(out))
        assert rc == 0, rc
        assert np.array_equal(out, oracle.bfs(ro, v.astype(np.int32), s)), s
