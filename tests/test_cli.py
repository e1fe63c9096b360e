"""The command-line driver (gpugraph_b200.cli): parameter parsing on the CPU,
every algorithm end to end on the GPU, with BFS / SSSP / CC outputs written
with -o and compared against the oracle (the reference drivers' -o files)."""
import numpy as np
import pytest

import oracle
from gpugraph_b200 import HostGraph, _lib, cli


def test_parse_params_known_and_unknown_keys():
    p = cli.parse_params("src=5 direction=pull iter_num=7 use_cuda_graph=0")
    assert p == {"src": "5", "direction": "pull", "iter_num": "7", "use_cuda_graph": "0"}
    kw = cli.options_from(p)
    assert kw == {"iter_num": 7, "direction": _lib.MG_DIR_PULL, "use_cuda_graph": 0}
    with pytest.raises(SystemExit):
        cli.parse_params("bogus=1")
    with pytest.raises(SystemExit):
        cli.parse_params("src")


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_cli_outputs_match_oracle(algo, tmp_path):
    out = tmp_path / f"{algo}.txt"
    assert cli.main([algo, "--rmat", "10", "--ef", "8", "-o", str(out), "-p", "src=3"]) == 0
    got = np.loadtxt(out, dtype=np.int64)
    hg = HostGraph.rmat(10, 8, seed=1)
    if algo == "bfs":
        ref = oracle.bfs(hg.row_offsets, hg.column_indices, 3)
    elif algo == "sssp":
        hw = hg.with_weights(1, 64, seed=1)  # the CLI's default weights for SSSP
        ref = oracle.sssp(hw.row_offsets, hw.column_indices, hw.edge_values, 3)
    else:
        ref = oracle.cc(hg.row_offsets, hg.column_indices)
    assert np.array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    ["bfs_multi", "--rmat", "10", "--nsrc", "8"],
    ["sssp_multi", "--rmat", "10", "--nsrc", "8"],
    ["pagerank", "--rmat", "10", "--directed"],
    ["pagerank_gas", "--rmat", "10"],
    ["ppr", "--rmat", "10", "--directed", "--nsrc", "4", "-p", "use_cuda_graph=0"],
    ["bfs", "--grid", "40", "-p", "direction=push use_cuda_graph=0", "--repeat", "2"],
])
def test_cli_runs_every_algorithm(args):
    assert cli.main(args) == 0
