"""A GAS Program written outside the library (tests/cpp/user_program.cu), to the
reference's Program contract, compiles against the engine headers, links
against libmapgraph_b200.so and runs through mg::run_gas: the in-, out- and
all-edge gathers that the bundled programs do not use, bit-exact against numpy."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gpugraph_b200 import Graph, HostGraph, _lib

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "gpugraph_b200"


def build_user_lib(tmp_path) -> Path:
    so = tmp_path / "libuser_program.so"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    "--expt-relaxed-constexpr", "-shared", "-Xcompiler", "-fPIC", "-I", str(LIBDIR / "csrc"),
                    "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/user_program.cu"), "-L", str(LIBDIR),
                    "-lmapgraph_b200", f"-Xlinker", f"-rpath={LIBDIR}", "-o", str(so)], check=True,
                   capture_output=True)
    return so


def test_user_program_builds_against_engine_headers(tmp_path):
    so = build_user_lib(tmp_path)
    assert hasattr(C.CDLL(str(so)), "user_nbr_sum")


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [1, 0])
def test_user_program_gathers_in_out_all(tmp_path, use_graph):
    import torch

    lib = C.CDLL(str(build_user_lib(tmp_path)))
    lib.user_nbr_sum.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(_lib.Options)]
    hg = HostGraph.rmat(12, 8, seed=3, symmetrize=False)
    g = Graph(hg, directed=True)
    rng = np.random.default_rng(0)
    val = rng.integers(-1000, 1000, size=hg.nodes).astype(np.int32)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    dst = hg.column_indices
    want = {1: np.bincount(dst, weights=val[src], minlength=hg.nodes),   # in-neighbours u -> v
            2: np.bincount(src, weights=val[dst], minlength=hg.nodes)}   # out-neighbours v -> w
    want[3] = want[1] + want[2]
    d_val = torch.tensor(val, device="cuda")
    d_out = torch.full((hg.nodes,), -7, dtype=torch.int32, device="cuda")
    o = _lib.default_options(use_cuda_graph=use_graph)
    for gd in (1, 2, 3):
        assert lib.user_nbr_sum(g.handle, d_val.data_ptr(), d_out.data_ptr(), gd, C.byref(o)) == 0
        assert np.array_equal(d_out.cpu().numpy(), want[gd].astype(np.int32)), gd
    g.close()
