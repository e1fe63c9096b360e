"""bench.py on the CPU: the reference arm builds its input with the oracle's
generator and never loads the product library, and both arms pick the same
sources."""
import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

import oracle
from gpugraph_b200 import HostGraph, replicas

ROOT = Path(__file__).resolve().parents[1]


def _sha(ro, col):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ro, np.int32).tobytes())
    h.update(np.ascontiguousarray(col, np.int32).tobytes())
    return h.hexdigest()


def test_oracle_rmat_equals_product_builder_at_bench_scale():
    # the reference arm's R-MAT 22 input is byte-identical to the native arm's
    ro, col = oracle.rmat(22, 16, seed=1)
    hg = HostGraph.rmat(22, 16, seed=1)
    assert _sha(ro, col) == _sha(hg.row_offsets, hg.column_indices)


def test_oracle_rmat_equals_product_builder_small_and_directed():
    for scale, ef, seed, sym in ((1, 1, 3, True), (8, 4, 2, False), (12, 16, 7, True), (14, 8, 1, False)):
        ro, col = oracle.rmat(scale, ef, seed=seed, symmetrize=sym)
        hg = HostGraph.rmat(scale, ef, seed=seed, symmetrize=sym)
        assert _sha(ro, col) == _sha(hg.row_offsets, hg.column_indices), (scale, ef, seed, sym)


def test_both_arms_pick_the_same_sources():
    sys.path.insert(0, str(ROOT))
    import bench

    hg = HostGraph.rmat(14, 16, seed=1)
    assert np.array_equal(bench.pick_sources(hg.row_offsets, 64), replicas.source_block(hg.row_offsets, 64))


def test_reference_arm_never_loads_the_product_library():
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '12', '--steps', '1', "
            "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('LOADED' if ('libmapgraph_b200' in maps or 'gpugraph_b200' in sys.modules) else 'CLEAN')")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "CLEAN"
    rec = json.loads(lines[-2])
    assert rec["impl"] == "reference" and rec["metric"].startswith("BFS aggregate GTEPS, batched 64-source")
    assert rec["value"] > 0 and rec["e2e"]["h2d_bytes_per_step"] == 0
