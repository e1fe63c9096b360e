"""ORACLE -- test infrastructure only.

Runs the oracle (or the reference's own CPU functions from oracle/_ref) for many
sources at once in spawned worker processes, one source per task. The graph
arrays go to a temporary directory as .npy files that every worker maps
read-only; each worker writes its result row straight into a shared [n][V]
memory-mapped output and reports the CPU seconds of its traversal alone
(measured inside the worker, so process start-up is not counted). Used by the
parity tests at full benchmark sizes and by bench.py's CPU baseline; the
product path never imports it.

Processes are started with the `spawn` method, so a pool may be created after
the parent has used the GPU.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import shutil
import tempfile
import time
from pathlib import Path

import numpy as np

KINDS = ("bfs", "sssp", "ref_bfs", "ref_sssp")


def _work(task):
    tmp, kind, row, src = task
    import oracle

    d = Path(tmp)
    ro = np.load(d / "ro.npy", mmap_mode="r")
    col = np.load(d / "col.npy", mmap_mode="r")
    w = np.load(d / "w.npy", mmap_mode="r") if kind in ("sssp", "ref_sssp") else None
    t0 = time.perf_counter()
    if kind == "bfs":
        res = oracle.bfs(ro, col, src)
    elif kind == "ref_bfs":
        res = oracle.ref_bfs(ro, col, src)
    elif kind == "sssp":
        res = oracle.sssp(ro, col, w, src)
    else:
        res = oracle.ref_sssp(ro, col, w, src)
    dt = time.perf_counter() - t0
    out = np.load(d / f"out{row[0]}.npy", mmap_mode="r+")
    out[row[1]] = res
    out.flush()
    return row[1], dt


def default_procs() -> int:
    return max(1, len(os.sched_getaffinity(0)))


class SourceRunner:
    """A worker pool over one graph: `with SourceRunner(ro, col, w) as r: r.run("bfs", sources)`."""

    def __init__(self, row_offsets, column_indices, weights=None, procs: int | None = None):
        self.n = len(row_offsets) - 1
        self.tmp = Path(tempfile.mkdtemp(prefix="mg_oracle_pool_"))
        np.save(self.tmp / "ro.npy", np.ascontiguousarray(row_offsets, np.int32))
        np.save(self.tmp / "col.npy", np.ascontiguousarray(column_indices, np.int32))
        if weights is not None:
            np.save(self.tmp / "w.npy", np.ascontiguousarray(weights, np.int32))
        self.procs = max(1, procs or default_procs())
        self.pool = mp.get_context("spawn").Pool(self.procs) if self.procs > 1 else None
        self.calls = 0

    def run(self, kind: str, sources):
        """Result rows [len(sources)][V] (int32) and the seconds each source took."""
        if kind not in KINDS:
            raise ValueError(kind)
        sources = [int(s) for s in np.atleast_1d(sources)]
        call = self.calls
        self.calls += 1
        path = self.tmp / f"out{call}.npy"
        out = np.lib.format.open_memmap(path, mode="w+", dtype=np.int32, shape=(len(sources), self.n))
        del out
        tasks = [(str(self.tmp), kind, (call, r), s) for r, s in enumerate(sources)]
        secs = [0.0] * len(sources)
        it = self.pool.imap_unordered(_work, tasks) if self.pool else map(_work, tasks)
        for r, dt in it:
            secs[r] = dt
        res = np.array(np.load(path, mmap_mode="r"))
        path.unlink()
        return res, secs

    def close(self):
        if self.pool:
            self.pool.close()
            self.pool.join()
            self.pool = None
        shutil.rmtree(self.tmp, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_sources(kind: str, row_offsets, column_indices, sources, weights=None, procs: int | None = None):
    """Oracle result for every source: an int32 array [len(sources)][V], plus the
    CPU seconds each source took."""
    n = len(np.atleast_1d(sources))
    with SourceRunner(row_offsets, column_indices, weights, min(procs or default_procs(), max(n, 1))) as r:
        return r.run(kind, sources)
