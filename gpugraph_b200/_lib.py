"""ctypes binding of the C ABI declared in include/mapgraph_b200.h.

The shared library is loaded from this package directory; importing this
module fails loudly when it has not been built (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmapgraph_b200.so"

MG_OK, MG_ERR_ARG, MG_ERR_OOM, MG_ERR_OVERFLOW, MG_ERR_TIMEOUT, MG_ERR_CUDA, MG_ERR_UNSUPPORTED, MG_ERR_IO = range(8)
MG_VAL_NONE, MG_VAL_I32, MG_VAL_F32 = 0, 1, 2
MG_DIR_AUTO, MG_DIR_PUSH, MG_DIR_PULL = 0, 1, 2


class Options(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("outputs_on_device", C.c_int32),
        ("stream", C.c_void_p),
        ("iter_num", C.c_int32),
        ("direction", C.c_int32),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("use_cuda_graph", C.c_int32),
        ("threshold", C.c_int32),
        ("damping", C.c_double),
        ("tolerance", C.c_double),
        ("spin_limit", C.c_int64),
        ("tile_items", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("compute_stats", C.c_int32),
        ("pad0", C.c_int32),
        ("alpha_multi", C.c_double),
        ("ordered_frontier", C.c_int32),
        ("generic_engine", C.c_int32),
        ("reserved", C.c_int32 * 2),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("push_iterations", C.c_int32),
        ("pull_iterations", C.c_int32),
        ("converged", C.c_int32),
        ("vertices_reached", C.c_int64),
        ("edges_traversed", C.c_int64),
        ("device_ms", C.c_double),
        ("residual", C.c_double),
        ("reserved", C.c_int64 * 4),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class HostCsr(C.Structure):
    _fields_ = [
        ("nodes", C.c_int64),
        ("edges", C.c_int64),
        ("row_offsets", C.POINTER(C.c_int32)),
        ("column_indices", C.POINTER(C.c_int32)),
        ("edge_values", C.POINTER(C.c_int32)),
        ("directed", C.c_int32),
    ]


P = C.c_void_p
I32P = C.POINTER(C.c_int32)
OPTP = C.POINTER(Options)
STP = C.POINTER(Stats)
CSRP = C.POINTER(HostCsr)

# name -> (restype, argtypes); this table is also the list of exported symbols
# that the header declares.
SIGNATURES = {
    "mg_options_init": (None, [OPTP]),
    "mg_last_error": (C.c_char_p, []),
    "mg_status_string": (C.c_char_p, [C.c_int]),
    "mg_abi_version": (C.c_int, []),
    "mg_kernel_launches": (C.c_int64, [C.c_int]),
    "mg_profile_enable": (C.c_int, [C.c_int]),
    "mg_profile_read": (C.c_int, [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                  C.POINTER(C.c_uint64)]),
    "mg_selftest_wait_timeout": (C.c_int, [C.c_int64, C.POINTER(C.c_double)]),
    "mg_graph_create": (C.c_int, [P, P, P, C.c_int32, C.c_int64, C.c_int64, C.c_int32, OPTP, C.POINTER(P)]),
    "mg_graph_create_batch": (C.c_int, [P, P, C.c_int64, C.c_int64, P, C.c_int32, OPTP, C.POINTER(P)]),
    "mg_graph_destroy": (C.c_int, [P]),
    "mg_graph_info": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int64)]),
    "mg_bfs": (C.c_int, [P, C.c_int32, P, STP, OPTP]),
    "mg_bfs_pred": (C.c_int, [P, C.c_int32, P, P, STP, OPTP]),
    "mg_bfs_roots": (C.c_int, [P, P, C.c_int32, P, STP, OPTP]),
    "mg_bfs_multi": (C.c_int, [P, P, C.c_int32, P, STP, OPTP]),
    "mg_bfs_batch": (C.c_int, [P, P, P, STP, OPTP]),
    "mg_sssp": (C.c_int, [P, C.c_int32, P, STP, OPTP]),
    "mg_sssp_multi": (C.c_int, [P, P, C.c_int32, P, STP, OPTP]),
    "mg_cc": (C.c_int, [P, P, STP, OPTP]),
    "mg_pagerank": (C.c_int, [P, P, STP, OPTP]),
    "mg_pagerank_gas": (C.c_int, [P, P, STP, OPTP]),
    "mg_ppr_forward": (C.c_int, [P, P, P, C.c_int32, P, STP, OPTP]),
    "mg_ppr_backward": (C.c_int, [P, P, P, P, C.c_int32, P, P, STP, OPTP]),
    "mg_bfs_noalloc": (C.c_int, [P, P, C.c_int64, C.c_int64, C.c_int32, P, P, STP]),
    "mg_autotune": (C.c_int, [P, C.c_int32, P, C.c_int32, OPTP, C.c_char_p, C.c_int64]),
    "mg_build_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int32,
                                C.c_int32, CSRP]),
    "mg_build_road_grid": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_uint64, CSRP]),
    "mg_build_weights": (C.c_int, [CSRP, C.c_uint32, C.c_uint32, C.c_uint64]),
    "mg_read_market": (C.c_int, [C.c_char_p, C.c_int32, CSRP]),
    "mg_read_csv": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, CSRP]),
    "mg_host_csr_transpose": (C.c_int, [CSRP, CSRP]),
    "mg_host_csr_free": (None, [CSRP]),
}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python gpugraph_b200/build.py` "
            "(there is no CPU fallback for the GAS hot path)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class MapGraphError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = lib.mg_last_error().decode(errors="replace")
        super().__init__(f"{where}: {lib.mg_status_string(status).decode()} ({msg})")


def check(status: int, where: str) -> None:
    if status != MG_OK:
        raise MapGraphError(status, where)


def profile_read() -> dict:
    """Per-kernel profile accumulated since mg_profile_enable(1): name -> (ms, launches, bytes)."""
    out = {}
    for k in range(13):
        name, ms, n, b = C.c_char_p(), C.c_double(), C.c_int64(), C.c_uint64()
        check(lib.mg_profile_read(k, C.byref(name), C.byref(ms), C.byref(n), C.byref(b)), "mg_profile_read")
        if n.value:
            out[name.value.decode()] = (ms.value, n.value, b.value)
    return out


def default_options(**kw) -> Options:
    o = Options()
    lib.mg_options_init(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o
