"""Host-side tests of the C ABI (no GPU needed): exported symbols, option
defaults, builders, argument validation and error reporting."""
import ctypes as C
import hashlib
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import fixture_names, host_graph_from_fixture, load_fixture

import gpugraph_b200 as gg
from gpugraph_b200 import HostGraph, MapGraphError, _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "mapgraph_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 25
    so = C.CDLL(str(_lib.LIB_PATH))
    for n in names:
        assert hasattr(so, n), f"{n} declared in mapgraph_b200.h but not exported"
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_abi_version_and_status_strings():
    assert _lib.lib.mg_abi_version() == 1
    assert _lib.lib.mg_status_string(_lib.MG_ERR_TIMEOUT) == b"MG_ERR_TIMEOUT"
    assert _lib.lib.mg_status_string(12345) == b"MG_ERR_UNKNOWN"


def test_options_defaults():
    o = gg.default_options()
    assert o.struct_size == C.sizeof(_lib.Options)
    assert o.iter_num > 1000 and o.use_cuda_graph == 1 and o.direction == _lib.MG_DIR_AUTO
    assert o.damping == pytest.approx(0.85) and o.spin_limit > 0
    with pytest.raises(TypeError):
        gg.default_options(no_such_knob=1)


def _sha(g):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.row_offsets, np.int32).tobytes())
    h.update(np.ascontiguousarray(g.column_indices, np.int32).tobytes())
    if g.edge_values is not None:
        h.update(np.ascontiguousarray(g.edge_values, np.int32).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", [n for n in fixture_names() if n.startswith("rmat")])
def test_rmat_builder_reproduces_golden_csr(name):
    fx = load_fixture(name)
    g = host_graph_from_fixture(fx)
    assert (g.nodes, g.edges) == (fx["nodes"], fx["edges"])
    assert _sha(g) == fx["csr_sha256"]


def test_rmat_symmetric_clean():
    g = gg.HostGraph.rmat(12, 16, seed=5)
    t = g.transpose()
    assert np.array_equal(g.row_offsets, t.row_offsets) and np.array_equal(g.column_indices, t.column_indices)
    src = np.repeat(np.arange(g.nodes), np.diff(g.row_offsets))
    assert not np.any(src == g.column_indices), "self-loop survived"
    for v in range(0, g.nodes, 97):
        row = g.column_indices[g.row_offsets[v]:g.row_offsets[v + 1]]
        assert np.all(np.diff(row) > 0), "row not strictly increasing (duplicate or unsorted)"
    # seeded: same seed -> same bytes, other seed -> other graph
    assert _sha(gg.HostGraph.rmat(12, 16, seed=5)) == _sha(g)
    assert _sha(gg.HostGraph.rmat(12, 16, seed=6)) != _sha(g)


def test_rmat_directed_has_no_reverse_requirement():
    g = gg.HostGraph.rmat(11, 16, seed=3, symmetrize=False)
    assert g.directed and g.edges <= 16 * 2048


def test_road_grid_shape():
    g = gg.HostGraph.road_grid(100, 0.02, 0.005, seed=2)
    assert g.nodes == 10000
    lattice = 2 * 100 * 99
    kept_und = g.edges // 2
    # about 2% dropped, plus about 0.5% shortcuts
    assert 0.96 * lattice < kept_und < 1.0 * lattice
    t = g.transpose()
    assert np.array_equal(g.column_indices, t.column_indices)


def test_weights_symmetric_and_in_range():
    g = gg.HostGraph.rmat(10, 8, seed=1).with_weights(1, 1000, seed=9)
    w = g.edge_values
    assert w.min() >= 1 and w.max() <= 1000
    src = np.repeat(np.arange(g.nodes), np.diff(g.row_offsets))
    d = {(int(u), int(v)): int(x) for u, v, x in zip(src, g.column_indices, w)}
    for (u, v), x in list(d.items())[:5000]:
        assert d[(v, u)] == x


def test_market_reader_errors(tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate integer general\n3 3 2\n1 2 1\n")
    with pytest.raises(gg.MapGraphError) as e:
        gg.HostGraph.read_market(str(bad))
    assert e.value.status == _lib.MG_ERR_IO
    with pytest.raises(gg.MapGraphError):
        gg.HostGraph.read_market(str(tmp_path / "missing.mtx"))
    ok = tmp_path / "ok.mtx"
    ok.write_text("%%MatrixMarket matrix coordinate integer general\n3 3 3\n1 2 5\n2 3 1\n1 2 5\n")
    g = gg.HostGraph.read_market(str(ok))
    assert g.row_offsets.tolist() == [0, 2, 3, 3]  # duplicates kept, like FromCoo
    assert g.column_indices.tolist() == [1, 1, 2] and g.edge_values.tolist() == [5, 5, 1]
    und = gg.HostGraph.read_market(str(ok), undirected=True)
    assert und.edges == 6


def _create(ro, col, nodes, edges, vals=None, vt=0):
    g = C.c_void_p()
    st = _lib.lib.mg_graph_create(ro.ctypes.data if ro is not None else None,
                                  col.ctypes.data if col is not None else None,
                                  vals.ctypes.data if vals is not None else None, vt, nodes, edges, 0, None,
                                  C.byref(g))
    return st, g


def test_graph_create_validates_before_touching_the_device():
    ro = np.array([0, 1, 2], np.int32)
    col = np.array([1, 5], np.int32)  # 5 out of range
    st, _ = _create(ro, col, 2, 2)
    assert st == _lib.MG_ERR_ARG and b"out of range" in _lib.lib.mg_last_error()
    st, _ = _create(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32), 2, 1)
    assert st == _lib.MG_ERR_ARG
    st, _ = _create(ro, None, 2, 2)
    assert st == _lib.MG_ERR_ARG
    st, _ = _create(ro, np.array([1, 0], np.int32), 2, 2, None, 99)
    assert st == _lib.MG_ERR_ARG
    st, _ = _create(np.array([1, 2, 2], np.int32), np.array([1, 0], np.int32), 2, 2)
    assert st == _lib.MG_ERR_ARG


def test_graph_create_without_gpu_reports_cuda_error(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    ro = np.array([0, 1, 2], np.int32)
    col = np.array([1, 0], np.int32)
    st, g = _create(ro, col, 2, 2)
    assert st == _lib.MG_ERR_CUDA and not g.value


def test_null_graph_arguments():
    out = np.zeros(4, np.int32)
    st = _lib.lib.mg_bfs(None, 0, out.ctypes.data, None, None)
    assert st == _lib.MG_ERR_ARG
    assert _lib.lib.mg_graph_destroy(None) == _lib.MG_OK
    assert _lib.lib.mg_graph_info(None, None, None, None, None) == _lib.MG_ERR_ARG


def test_kernel_launch_counter_resets():
    _lib.lib.mg_kernel_launches(1)
    assert _lib.lib.mg_kernel_launches(0) == 0


def test_csv_reader_adjacency_rows(tmp_path):
    # csv_graph_reader::read: "src,dst:val,..." rows; ids 10, 20, 30, 40 -> 0..3 in sorted
    # order; a lone "40" row still makes a vertex; a cell without ':' takes its own
    # number as the value; undirected appends the reversed edges; CSR sorted by (row, col).
    p = tmp_path / "g.csv"
    p.write_text("20,10:5,30:7\n10,30:2\n\n40\n30,20\n")
    g = HostGraph.read_csv(str(p), "adjacency", undirected=False)
    assert g.nodes == 4 and g.directed
    assert g.row_offsets.tolist() == [0, 1, 3, 4, 4]
    assert g.column_indices.tolist() == [2, 0, 2, 1]
    assert g.edge_values.tolist() == [2, 5, 7, 20]
    u = HostGraph.read_csv(str(p), "adjacency", undirected=True)
    assert not u.directed and u.edges == 8
    assert u.row_offsets.tolist() == [0, 2, 5, 8, 8]
    assert u.column_indices.tolist() == [1, 2, 0, 2, 2, 0, 1, 1]


def test_csv_reader_edge_rows_and_errors(tmp_path):
    # csv_graph_reader::read2: "src,dst,val" rows, duplicates kept
    p = tmp_path / "e.csv"
    p.write_text("7,3,1\n3,9,4\n7,3,2\n")
    g = HostGraph.read_csv(str(p), "edges", undirected=False)
    assert g.nodes == 3
    assert g.row_offsets.tolist() == [0, 1, 3, 3]
    assert g.column_indices.tolist() == [2, 0, 0] and g.edge_values.tolist() == [4, 1, 2]
    bad = tmp_path / "bad.csv"
    bad.write_text("1,2\n")
    with pytest.raises(MapGraphError):
        HostGraph.read_csv(str(bad), "edges")
    with pytest.raises(MapGraphError):
        HostGraph.read_csv(str(tmp_path / "missing.csv"))
