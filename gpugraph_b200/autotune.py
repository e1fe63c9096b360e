"""Autotuner front end: mg_autotune over the C ABI, with results recorded per GPU.

    from gpugraph_b200.autotune import autotune
    opts, report = autotune(graph, "bfs_multi", srcs, record="tuning.json")
    depths, stats = graph.bfs_multi(srcs, **opts)
"""
from __future__ import annotations

import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check, default_options, lib

KINDS = {"bfs": 0, "bfs_multi": 1, "sssp": 2, "cc": 3, "pagerank": 4, "ppr": 5}
TUNED = ("tile_items", "ctas_per_sm", "alpha", "alpha_multi", "beta")


def gpu_name() -> str:
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "--id=0"],
                             capture_output=True, text=True, timeout=10).stdout.strip()
        return out or "unknown-gpu"
    except Exception:
        return "unknown-gpu"


def autotune(graph, kind: str, srcs=None, record: str | None = None, **start) -> tuple[dict, dict]:
    """Returns (best option values, trial report). `start` seeds the search."""
    o = default_options(**start)
    s = np.ascontiguousarray(srcs if srcs is not None else [0], np.int32)
    buf = C.create_string_buffer(1 << 16)
    check(lib.mg_autotune(graph.handle, KINDS[kind], s.ctypes.data, len(s), C.byref(o), buf, len(buf)),
          "mg_autotune")
    best = {k: getattr(o, k) for k in TUNED}
    report = json.loads(buf.value.decode())
    if record:
        p = Path(record)
        data = json.loads(p.read_text()) if p.exists() else {}
        key = f"{gpu_name()}|{kind}|V={graph.nodes}|E={graph.edges}"
        data[key] = {"best": best, "best_ms": report["best_ms"], "trials": len(report["trials"])}
        p.write_text(json.dumps(data, indent=1, sort_keys=True))
    return best, report
