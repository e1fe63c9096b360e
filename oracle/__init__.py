"""ORACLE -- test infrastructure only.

ctypes access to (1) the plain-C restatement of the reference's CPU algorithms
(oracle/libmg_oracle.so, from mg_oracle.c) and (2) the reference's own CPU
functions compiled from its sources (oracle/_ref/libref_cpu.so, from
build_ref.sh), when present. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this package, and only to check results or as
the timed CPU baseline; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmg_oracle.so"
REF_PATH = HERE / "_ref" / "libref_cpu.so"
SSSP_INF = 100000000

_P = C.c_void_p
_I64 = C.c_int64


def build() -> None:
    """Compiles the restatement (gcc) and, where the reference tree exists, oracle/_ref."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def _load():
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    lib.oracle_bfs.argtypes = [_I64, _P, _P, _P, C.c_int32, _P]
    lib.oracle_sssp_array.argtypes = [_I64, _P, _P, _P, C.c_int32, _P]
    lib.oracle_sssp_heap.argtypes = [_I64, _P, _P, _P, C.c_int32, _P]
    lib.oracle_cc_sweep.argtypes = [_I64, _P, _P, _P]
    lib.oracle_cc_push.argtypes = [_I64, _P, _P, _P]
    lib.oracle_pr_gas.argtypes = [_I64, _P, _P, _P, _P, _P, C.c_float, C.c_int32, _P, _P]
    lib.oracle_pagerank_fp64.argtypes = [_I64, _P, _P, _P, C.c_double, C.c_double, C.c_int32, _P, _P, _P]
    lib.oracle_bfs_pred.argtypes = [_I64, _P, _P, _P, _P]
    lib.oracle_build_rmat.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                      C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_int32)),
                                      C.POINTER(C.POINTER(C.c_int32)), C.POINTER(_I64)]
    lib.oracle_free.argtypes = [_P]
    return lib


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def ref():
    """The reference's own CPU functions, or None when oracle/_ref was not built."""
    global _ref
    if _ref is None and REF_PATH.exists():
        r = C.CDLL(str(REF_PATH))
        r.ref_cpubfs.argtypes = [_I64, _I64, _P, _P, C.c_int32, _P]
        r.ref_cpusssp.argtypes = [_I64, _I64, _P, _P, _P, C.c_int32, _P]
        r.ref_cpucc.argtypes = [_I64, _I64, _P, _P, _P]
        r.ref_cpupr.argtypes = [_I64, _I64, _P, _P, _P, _P, _P]
        _ref = r
    return _ref


def _p(a):
    return a.ctypes.data


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ----------------------------------------------------------- restatement --
def bfs(ro, col, srcs) -> np.ndarray:
    ro, col = _c32(ro), _c32(col)
    s = _c32(np.atleast_1d(srcs))
    out = np.empty(len(ro) - 1, np.int32)
    assert lib().oracle_bfs(len(ro) - 1, _p(ro), _p(col), _p(s), len(s), _p(out)) == 0
    return out


def bfs_pred(coff, crow, depth) -> np.ndarray:
    """Predecessors from BFS depths by pred_extract's rule (coff/crow: in-lists)."""
    coff, crow, depth = _c32(coff), _c32(crow), _c32(depth)
    out = np.empty(len(coff) - 1, np.int32)
    assert lib().oracle_bfs_pred(len(coff) - 1, _p(coff), _p(crow), _p(depth), _p(out)) == 0
    return out


def sssp(ro, col, w, src, method: str = "heap") -> np.ndarray:
    ro, col, w = _c32(ro), _c32(col), _c32(w)
    out = np.empty(len(ro) - 1, np.int32)
    fn = lib().oracle_sssp_heap if method == "heap" else lib().oracle_sssp_array
    assert fn(len(ro) - 1, _p(ro), _p(col), _p(w), int(src), _p(out)) == 0
    return out


def cc(ro, col, method: str = "sweep") -> np.ndarray:
    ro, col = _c32(ro), _c32(col)
    out = np.empty(len(ro) - 1, np.int32)
    fn = lib().oracle_cc_sweep if method == "sweep" else lib().oracle_cc_push
    assert fn(len(ro) - 1, _p(ro), _p(col), _p(out)) == 0
    return out


def pr_gas(ro, col, coff, crow, outdeg, tol=0.01, max_iter=1 << 30):
    ro, col, coff, crow, od = map(_c32, (ro, col, coff, crow, outdeg))
    out = np.empty(len(ro) - 1, np.float32)
    it = C.c_int32(0)
    assert lib().oracle_pr_gas(len(ro) - 1, _p(ro), _p(col), _p(coff), _p(crow), _p(od), tol, max_iter, _p(out),
                               C.byref(it)) == 0
    return out, it.value


def pagerank_fp64(ro, coff, crow, damping=0.85, tol=1e-6, max_iter=100):
    ro, coff, crow = _c32(ro), _c32(coff), _c32(crow)
    out = np.empty(len(ro) - 1, np.float64)
    it, res = C.c_int32(0), C.c_double(0)
    assert lib().oracle_pagerank_fp64(len(ro) - 1, _p(ro), _p(coff), _p(crow), damping, tol, max_iter, _p(out),
                                      C.byref(it), C.byref(res)) == 0
    return out, it.value, res.value


def rmat(scale, edgefactor=16, seed=1, symmetrize=True, a=0.57, b=0.19, c=0.19):
    """Seeded R-MAT CSR (row_offsets, column_indices) built without the product
    library: the same bytes as gpugraph_b200.HostGraph.rmat (asserted by tests)."""
    ro_p, col_p, m = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), _I64(0)
    assert lib().oracle_build_rmat(scale, edgefactor, a, b, c, seed, int(symmetrize), 1, C.byref(ro_p),
                                   C.byref(col_p), C.byref(m)) == 0
    n = 1 << scale
    try:
        ro = np.ctypeslib.as_array(ro_p, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(col_p, shape=(max(m.value, 1),))[:m.value].copy()
    finally:
        lib().oracle_free(C.cast(ro_p, _P))
        lib().oracle_free(C.cast(col_p, _P))
    return ro, col


# --------------------------------------------------- reference functions --
def ref_bfs(ro, col, src):
    ro, col = _c32(ro), _c32(col)
    out = np.empty(len(ro) - 1, np.int32)
    ref().ref_cpubfs(len(ro) - 1, len(col), _p(ro), _p(col), int(src), _p(out))
    return out


def ref_sssp(ro, col, w, src):
    ro, col, w = _c32(ro), _c32(col), _c32(w)
    out = np.empty(len(ro) - 1, np.int32)
    ref().ref_cpusssp(len(ro) - 1, len(col), _p(ro), _p(col), _p(w), int(src), _p(out))
    return out


def ref_cc(ro, col):
    ro, col = _c32(ro), _c32(col)
    out = np.empty(len(ro) - 1, np.int32)
    ref().ref_cpucc(len(ro) - 1, len(col), _p(ro), _p(col), _p(out))
    return out


def ref_pr(ro, col, coff, crow):
    ro, col, coff, crow = map(_c32, (ro, col, coff, crow))
    out = np.empty(len(ro) - 1, np.float32)
    ref().ref_cpupr(len(ro) - 1, len(col), _p(ro), _p(col), _p(coff), _p(crow), _p(out))
    return out
