"""Benchmark of the B200 GAS hot path (one JSON line on rank 0).

Workload (R-MAT scale 22, edgefactor 16, A/B/C/D = .57/.19/.19/.05, seed 1,
symmetrised, self-loops and duplicates removed, int32 CSR; uint32 weights in
[1, 64]): a step is one batched BFS from 64 seeded sources (the 64-bit mask
frontier, mg_bfs_multi). value = aggregate GTEPS = sum over sources of the
out-degrees of the vertices each source reaches, divided by the step time.
With N GPUs every rank runs its own block of 64 sources (weak scaling, no
source run twice, no collective on the data path; gpugraph_b200/replicas.py).
Alongside, in sub_results (one GPU): every other benchmarked configuration
(plain BFS on R-MAT 16 from the hub, the 64 sources as 64 single-source runs,
8 single-source SSSP runs, batched 64-source SSSP, CC, PageRank on R-MAT 23
and the road grid, batched BFS/SSSP on the road grid, the 256-graph batch and
differentiable PPR), each with the fraction of the HBM roofline its kernels
reach by their device-counted algorithmic bytes.

--impl reference times the reference's own CPU BFS (CPUBFS, compiled from the
reference sources into oracle/_ref, or the oracle restatement when that is
absent) on the same graph and sources, one source per host core, and builds
its input with the oracle's generator: it never loads the product library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE, EDGEFACTOR, SEED = 22, 16, 1
NSRC = 64


def metric_name(scale: int) -> str:
    return f"BFS aggregate GTEPS, batched 64-source (mask frontier) on R-MAT scale {scale}"


def workload(scale: int) -> str:
    return (f"R-MAT scale {scale} edgefactor {EDGEFACTOR} A/B/C/D .57/.19/.19/.05 seed {SEED}, symmetrised, "
            f"cleaned, int32 CSR; batched BFS from {NSRC} seeded sources (64-bit mask frontier)")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def pick_sources(row_offsets, n, seed=SEED):
    """n distinct seeded vertices with out-degree > 0, ascending (one rank's sources)."""
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(np.diff(row_offsets) > 0)
    return np.sort(rng.choice(cand, size=n, replace=False)).astype(np.int32)


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int = 0, period_ms: int = 20):
        self.dev = device_index
        self.period_ms = period_ms
        self.proc = None
        self.lines: list[tuple[float, str]] = []  # (host arrival time, csv line)
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.time() + 5.0
            while not self.lines and time.time() < t_end:  # sampler is live before timing starts
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0: float, t1: float):
        """Host times bracketing the timed region."""
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines, widened = [ln for _, ln in self.lines], 0
        if self.window:
            # samples taken during the timed region (one sampling period of slack
            # for the arrival delay); widen only if the region was shorter than a period
            for slack in (self.period_ms / 1000.0, 0.25, 0.5):
                t0, t1 = self.window[0] - 0.0, self.window[1] + slack
                sel = [ln for t, ln in self.lines if t0 <= t <= t1]
                if sel:
                    lines, widened = sel, int(slack * 1000)
                    break
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "window_slack_ms": widened, "period_ms": self.period_ms}


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes (read + write) of `kernel` at the bench workload, from
    the committed ncu summary profiles/<kernel>__<workload>.md (line
    'traffic_bytes_per_launch: N')."""
    found = sorted((ROOT / "profiles").glob(f"{kernel}__*.md"))
    if not found:
        return None
    for ln in found[0].read_text().splitlines():
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled(fn, peak: float) -> tuple[dict, dict]:
    """One run of fn with per-kernel profiling on: the level loops run host-driven,
    every launch is bracketed by CUDA events on its stream, and the kernels count
    their algorithmic bytes on the device. Returns the run's roofline summary (all
    kernels, and the kernel kind with the most time) and the raw profile."""
    import torch

    from gpugraph_b200 import _lib

    _lib.lib.mg_profile_enable(1)
    try:
        fn()
        torch.cuda.synchronize()
        prof = _lib.profile_read()
    finally:
        _lib.lib.mg_profile_enable(0)
    ms = sum(v[0] for v in prof.values())
    byts = sum(v[2] for v in prof.values())
    out = {"algorithmic_GB": byts / 1e9, "kernel_ms": ms,
           "achieved_GBps": byts / (ms * 1e-3) / 1e9 if ms else None,
           "frac": byts / (ms * 1e-3) / 1e9 / peak if ms else None}
    kernels = {k: v for k, v in prof.items() if k != "other"}
    if kernels:
        dom = max(kernels, key=lambda k: kernels[k][0])
        kms, n, kb = kernels[dom]
        out["dominant"] = {"kernel": dom, "ms": kms, "launches": n, "GB": kb / 1e9,
                           "frac": kb / (kms * 1e-3) / 1e9 / peak if kms else None}
    return out, prof


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time_events(fn, stream, reps=3):
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


# ------------------------------------------------------------- native arm --
def run_native(args, world: int):
    import torch

    import gpugraph_b200 as gg
    from gpugraph_b200 import _lib, replicas

    lib = _lib.lib
    rank = replicas.rank()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.device("cuda")
    peak, peak_kind = measured_peak_hbm()
    t0 = time.time()
    hg = gg.HostGraph.rmat(args.scale, EDGEFACTOR, seed=SEED).with_weights(1, 64, seed=SEED)
    log(f"[bench] rank {rank}: graph V={hg.nodes} E={hg.edges} built in {time.time() - t0:.1f}s")
    srcs = replicas.source_block(hg.row_offsets, NSRC, seed=SEED)  # this rank's own 64 sources
    g = gg.Graph(hg)
    out_dev = torch.empty((NSRC, hg.nodes), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    graphs = 0 if args.no_cuda_graph else 1
    base_opts = dict(outputs_on_device=1, stream=stream.cuda_stream, compute_stats=0, use_cuda_graph=graphs)
    st = _lib.Stats()
    src_arr = np.ascontiguousarray(srcs)
    # launch shape and direction factors from the library's autotuner, on this graph and these
    # sources (untimed); the default options are timed beside them in sub_results
    tuned = {}
    if not args.no_autotune:
        from gpugraph_b200.autotune import autotune

        tuned, _ = autotune(g, "bfs_multi", src_arr, **base_opts)
    o_multi = _lib.default_options(**dict(base_opts, **tuned))
    o_default = _lib.default_options(**base_opts)

    def multi_step(opts=o_multi):
        _lib.check(lib.mg_bfs_multi(g.handle, src_arr.ctypes.data, NSRC, out_dev.data_ptr(), None, opts),
                   "mg_bfs_multi")

    # TEPS numerator (once, outside timing)
    o_stats = _lib.default_options(**dict(base_opts, compute_stats=1))
    _lib.check(lib.mg_bfs_multi(g.handle, src_arr.ctypes.data, NSRC, out_dev.data_ptr(), st, o_stats), "stats")
    teps_edges = int(st.edges_traversed)
    reached_total = int(st.vertices_reached)
    levels_multi = (st.iterations, st.push_iterations, st.pull_iterations)

    for _ in range(args.warmup):
        multi_step()
    torch.cuda.synchronize()
    lib.mg_kernel_launches(1)
    ev0, ev1 = _events()
    with ClockSampler(torch.cuda.current_device()) as clk:
        replicas.barrier()
        torch.cuda.synchronize()
        h0 = time.time()
        ev0.record(stream)
        for _ in range(args.steps):
            multi_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark(h0, time.time())
        replicas.barrier()
    launches = int(lib.mg_kernel_launches(1))
    # N replicas: the units all ranks processed over the slowest rank's device time
    rate, step_s = replicas.aggregate_rate(teps_edges, ev0.elapsed_time(ev1) / args.steps * 1e-3, str(dev))
    value = rate / 1e9
    sub = {"bfs_batched64": {"gteps_this_rank": teps_edges / (ev0.elapsed_time(ev1) / args.steps * 1e-3) / 1e9,
                             "ms": step_s * 1e3, "levels": levels_multi, "vertices_reached": reached_total,
                             "autotuned_options": tuned}}
    if tuned:
        dms = _time_events(lambda: multi_step(o_default), stream, max(3, min(args.steps, 10)))
        sub["bfs_batched64"]["default_options_ms"] = dms

    # ---- end to end through the C ABI with host buffers (pinned), one call per step
    host_out = torch.empty((NSRC, hg.nodes), dtype=torch.int32, pin_memory=True)
    o_host = _lib.default_options(stream=stream.cuda_stream, compute_stats=0, use_cuda_graph=graphs, **tuned)
    src_pinned = torch.from_numpy(src_arr.copy()).pin_memory()
    _lib.check(lib.mg_bfs_multi(g.handle, src_pinned.data_ptr(), NSRC, host_out.data_ptr(), None, o_host), "e2e")
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 5))
    replicas.barrier()
    ev0.record(stream)
    for _ in range(e2e_steps):
        _lib.check(lib.mg_bfs_multi(g.handle, src_pinned.data_ptr(), NSRC, host_out.data_ptr(), None, o_host), "e2e")
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_rate, e2e_s = replicas.aggregate_rate(teps_edges, ev0.elapsed_time(ev1) / e2e_steps * 1e-3, str(dev))
    e2e = {"value": e2e_rate / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": NSRC * 4,
           "d2h_bytes_per_step": NSRC * hg.nodes * 4, "ms_per_step": e2e_s * 1e3}

    # ---- live roofline of the dominant kernel (profiled pass, host-driven loop)
    summ, prof = profiled(multi_step, peak)
    kernels = {k: v for k, v in prof.items() if k != "other"}
    roofline = None
    if kernels:
        dom = max(kernels, key=lambda k: kernels[k][0])
        ms, n, byts = kernels[dom]
        achieved = byts / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": ncu_traffic(dom), "peak_source": peak_kind,
                    "launches": n, "bytes_per_launch": byts / max(n, 1), "ms_per_launch": ms / max(n, 1),
                    "path_frac_all_kernels": summ["frac"],
                    "kernels": {k: {"ms": v[0], "launches": v[1], "GB": v[2] / 1e9} for k, v in prof.items()}}

    # ---- the 256-graph batch, its graphs sharded over the ranks
    sub.update(graph_batch(dev, stream, peak))

    if world == 1 and not args.quick:
        sub.update(single_gpu_configs(args, hg, g, srcs, out_dev, teps_edges, reached_total, value, stream, peak))
        sub.update(extra_configs(dev, stream, peak))

    res = {"value": value, "ms_per_step": step_s * 1e3, "launches": launches, "sub": sub, "e2e": e2e, "tuned": tuned,
           "roofline": roofline, "clocks": clk.summary(), "V": hg.nodes, "E": hg.edges,
           "teps_edges_this_rank": teps_edges}
    g.close()
    return res, hg, srcs


def graph_batch(dev, stream, peak) -> dict:
    """256 independent R-MAT graphs (scales U{10..16}, edgefactor 8), one BFS each in
    the same launches (mg_bfs_batch); with N ranks each rank runs its share."""
    import ctypes as C

    import torch

    import gpugraph_b200 as gg
    import oracle
    from gpugraph_b200 import _lib, replicas

    lib = _lib.lib
    rng = np.random.default_rng(SEED)
    todo = replicas.shard(list(enumerate(rng.integers(10, 17, size=256))))
    graphs = [gg.HostGraph.rmat(int(s), 8, seed=1000 + i) for i, s in todo]
    big = gg.concat_graphs(graphs)
    gb = gg.Graph(big)
    local = np.array([h.max_degree_vertex() for h in graphs], np.int32)
    dep = torch.empty(big.nodes, dtype=torch.int32, device=dev)
    st = _lib.Stats()
    os_ = _lib.default_options(outputs_on_device=1, compute_stats=1, stream=stream.cuda_stream)
    o = _lib.default_options(outputs_on_device=1, compute_stats=0, stream=stream.cuda_stream)
    _lib.check(lib.mg_bfs_batch(gb.handle, local.ctypes.data, dep.data_ptr(), C.byref(st), C.byref(os_)), "batch")
    teps = int(st.edges_traversed)
    replicas.barrier()
    bms = _time_events(lambda: _lib.check(lib.mg_bfs_batch(gb.handle, local.ctypes.data, dep.data_ptr(), None,
                                                           C.byref(o)), "batch"), stream)
    rate, slow = replicas.aggregate_rate(teps, bms * 1e-3, str(dev))
    d = dep.cpu().numpy()
    ok = all(np.array_equal(d[big.graph_offsets[i]:big.graph_offsets[i + 1]],
                            oracle.bfs(graphs[i].row_offsets, graphs[i].column_indices, local[i]))
             for i in (0, len(graphs) // 2, len(graphs) - 1))
    roof, _ = profiled(lambda: _lib.check(lib.mg_bfs_batch(gb.handle, local.ctypes.data, dep.data_ptr(), None,
                                                           C.byref(o)), "batch"), peak)
    gb.close()
    return {"bfs_256_graph_batch": {"gteps": rate / 1e9, "ms": slow * 1e3, "graphs_this_rank": len(graphs),
                                    "V_this_rank": big.nodes, "E_this_rank": big.edges, "spot_check_equal": ok,
                                    "roofline": roof}}


def single_gpu_configs(args, hg, g, srcs, out_dev, teps_edges, reached_total, batched_gteps, stream, peak) -> dict:
    """Plain engine on the same sources, config 1 (R-MAT 16 from the hub), SSSP, CC."""
    import torch

    import gpugraph_b200 as gg
    from gpugraph_b200 import _lib

    lib = _lib.lib
    dev = out_dev.device
    sub = {}
    graphs = 0 if args.no_cuda_graph else 1
    base = dict(outputs_on_device=1, stream=stream.cuda_stream, compute_stats=0, use_cuda_graph=graphs)
    o_single = _lib.default_options(**base)
    o_push = _lib.default_options(**dict(base, direction=_lib.MG_DIR_PUSH))
    one = torch.empty(hg.nodes, dtype=torch.int32, device=dev)
    st1 = _lib.Stats()

    # ---- plain engine: the same 64 sources one at a time
    for s in srcs[:4]:
        _lib.check(lib.mg_bfs(g.handle, int(s), one.data_ptr(), None, o_single), "mg_bfs")
    torch.cuda.synchronize()
    dev_sum = 0.0
    ev0, ev1 = _events()
    ev0.record(stream)
    for s in srcs:
        _lib.check(lib.mg_bfs(g.handle, int(s), one.data_ptr(), st1, o_single), "mg_bfs")
        dev_sum += float(st1.device_ms)
    ev1.record(stream)
    torch.cuda.synchronize()
    single_ms = ev0.elapsed_time(ev1)
    single_gteps = teps_edges / (single_ms * 1e-3) / 1e9
    parity = True
    for k in (0, NSRC // 2, NSRC - 1):
        _lib.check(lib.mg_bfs(g.handle, int(srcs[k]), one.data_ptr(), None, o_single), "mg_bfs")
        parity &= bool(torch.equal(one, out_dev[k]))
    # bytes actually moved: device-counted algorithmic bytes of what the kernels did
    # (a bottom-up level counts the in-edges it inspected, not every edge) over kernel time
    roof_auto, _ = profiled(lambda: _lib.check(lib.mg_bfs(g.handle, int(srcs[0]), one.data_ptr(), None, o_single),
                                               "mg_bfs"), peak)
    roof_push, _ = profiled(lambda: _lib.check(lib.mg_bfs(g.handle, int(srcs[0]), one.data_ptr(), None, o_push),
                                               "mg_bfs"), peak)
    path_bytes = 8 * teps_edges + 20 * reached_total
    sub["bfs_single_x64"] = {
        "gteps": single_gteps, "ms_total": single_ms, "ms_per_source": single_ms / NSRC, "device_ms_sum": dev_sum,
        "gteps_device_only": teps_edges / (dev_sum * 1e-3) / 1e9 if dev_sum else None,
        "teps_formula_bytes": path_bytes,
        "teps_formula_frac": path_bytes / (single_ms * 1e-3) / 1e9 / peak,
        "roofline_direction_optimising": roof_auto, "roofline_push_only": roof_push}
    sub["batched_over_single"] = batched_gteps / single_gteps
    sub["batched_over_single_device_only"] = (batched_gteps / (teps_edges / (dev_sum * 1e-3) / 1e9)
                                              if dev_sum else None)
    sub["batched_equals_single_spot_check"] = parity

    # ---- config 1: plain BFS on R-MAT 16 from the hub
    h16 = gg.HostGraph.rmat(16, 16, seed=SEED)
    g16 = gg.Graph(h16)
    hub = h16.max_degree_vertex()
    d16 = torch.empty(h16.nodes, dtype=torch.int32, device=dev)
    o16 = _lib.default_options(**dict(base, compute_stats=1))
    _lib.check(lib.mg_bfs(g16.handle, hub, d16.data_ptr(), st1, o16), "bfs16")
    e16 = int(st1.edges_traversed)
    ms16 = _time_events(lambda: _lib.check(lib.mg_bfs(g16.handle, hub, d16.data_ptr(), None, o_single), "bfs16"),
                        stream, 20)
    roof16, _ = profiled(lambda: _lib.check(lib.mg_bfs(g16.handle, hub, d16.data_ptr(), None, o_single), "bfs16"),
                         peak)
    sub["bfs_rmat16_hub"] = {"ms": ms16, "gteps": e16 / (ms16 * 1e-3) / 1e9, "levels": int(st1.iterations),
                             "roofline": roof16}
    g16.close()

    # ---- config 2: 8 single-source SSSP runs, CC; config 4: batched SSSP
    o_s = _lib.default_options(**dict(base, compute_stats=1))
    sssp_edges, sssp_ms = 0, 0.0
    for s in srcs[:8]:
        _lib.check(lib.mg_sssp(g.handle, int(s), one.data_ptr(), st1, o_s), "mg_sssp")
        sssp_edges += int(st1.edges_traversed)
        sssp_ms += float(st1.device_ms)
    roof_s, _ = profiled(lambda: _lib.check(lib.mg_sssp(g.handle, int(srcs[0]), one.data_ptr(), None, o_single),
                                            "mg_sssp"), peak)
    sub["sssp_single_x8"] = {"gteps": sssp_edges / (sssp_ms * 1e-3) / 1e9, "ms_per_source": sssp_ms / 8,
                             "roofline": roof_s}
    src_arr = np.ascontiguousarray(srcs)
    o_multi = _lib.default_options(**base)
    _lib.check(lib.mg_sssp_multi(g.handle, src_arr.ctypes.data, NSRC, out_dev.data_ptr(), st1, o_s), "sssp_multi")
    mst = int(st1.edges_traversed)
    mms = _time_events(lambda: _lib.check(lib.mg_sssp_multi(g.handle, src_arr.ctypes.data, NSRC, out_dev.data_ptr(),
                                                            None, o_multi), "sssp_multi"), stream, 2)
    roof_ms, _ = profiled(lambda: _lib.check(lib.mg_sssp_multi(g.handle, src_arr.ctypes.data, NSRC,
                                                               out_dev.data_ptr(), None, o_multi), "sssp_multi"), peak)
    sub["sssp_batched64"] = {"gteps": mst / (mms * 1e-3) / 1e9, "ms": mms, "levels": int(st1.iterations),
                             "over_single": (mst / mms) / (sssp_edges / sssp_ms), "roofline": roof_ms}
    lab = torch.empty(hg.nodes, dtype=torch.int32, device=dev)
    _lib.check(lib.mg_cc(g.handle, lab.data_ptr(), st1, o_multi), "mg_cc")
    cms = _time_events(lambda: _lib.check(lib.mg_cc(g.handle, lab.data_ptr(), None, o_multi), "mg_cc"), stream)
    roof_cc, _ = profiled(lambda: _lib.check(lib.mg_cc(g.handle, lab.data_ptr(), None, o_multi), "mg_cc"), peak)
    sub["cc"] = {"gedges_per_s": hg.edges / (cms * 1e-3) / 1e9, "ms": cms, "iterations": int(st1.iterations),
                 "roofline": roof_cc}
    return sub


def extra_configs(dev, stream, peak) -> dict:
    """PageRank (directed R-MAT 23 and the road grid), batched BFS/SSSP on the road
    grid and differentiable PPR."""
    import ctypes as C

    import torch

    import gpugraph_b200 as gg
    import oracle
    from gpugraph_b200 import _lib

    lib = _lib.lib
    out = {}
    st = _lib.Stats()
    # PageRank: FP32 ranks vs the FP64 oracle at the same iteration count
    for name, mk, directed in (("pagerank_rmat23", lambda: gg.HostGraph.rmat(23, 16, seed=SEED, symmetrize=False), True),
                               ("pagerank_road1200", lambda: gg.HostGraph.road_grid(1200, 0.02, 0.005, seed=SEED),
                                False)):
        hg = mk()
        g = gg.Graph(hg, directed=directed)
        r = torch.empty(hg.nodes, dtype=torch.float32, device=dev)
        o = _lib.default_options(outputs_on_device=1, iter_num=100, tolerance=1e-6, stream=stream.cuda_stream)
        f = lambda: _lib.check(lib.mg_pagerank(g.handle, r.data_ptr(), C.byref(st), C.byref(o)), "mg_pagerank")
        ms = _time_events(f, stream)
        it = int(st.iterations)
        roof, _ = profiled(f, peak)
        t = hg.transpose() if directed else hg
        ref, _, _ = oracle.pagerank_fp64(hg.row_offsets, t.row_offsets, t.column_indices, 0.85, 0.0, it)
        diff = np.abs(r.cpu().numpy().astype(np.float64) - ref)
        out[name] = {"gedges_per_s": hg.edges * it / (ms * 1e-3) / 1e9, "ms": ms, "iterations": it,
                     "residual": float(st.residual), "l1_vs_fp64": float(diff.sum()), "maxabs_vs_fp64": float(diff.max()),
                     "V": hg.nodes, "E": hg.edges, "roofline": roof}
        g.close()
    # batched 64-source BFS / SSSP on the road grid (uint32 weights in [1, 1000])
    hg = gg.HostGraph.road_grid(1200, 0.02, 0.005, seed=SEED).with_weights(1, 1000, seed=SEED)
    g = gg.Graph(hg)
    srcs = pick_sources(hg.row_offsets, NSRC)
    buf = torch.empty((NSRC, hg.nodes), dtype=torch.int32, device=dev)
    one = torch.empty(hg.nodes, dtype=torch.int32, device=dev)
    o = _lib.default_options(outputs_on_device=1, compute_stats=0, stream=stream.cuda_stream)
    os_ = _lib.default_options(outputs_on_device=1, compute_stats=1, stream=stream.cuda_stream)
    for algo, multi, single in (("bfs", lib.mg_bfs_multi, lib.mg_bfs), ("sssp", lib.mg_sssp_multi, lib.mg_sssp)):
        _lib.check(multi(g.handle, srcs.ctypes.data, NSRC, buf.data_ptr(), C.byref(st), C.byref(os_)), algo)
        teps = int(st.edges_traversed)
        call = lambda: _lib.check(multi(g.handle, srcs.ctypes.data, NSRC, buf.data_ptr(), None, C.byref(o)), algo)
        mms = _time_events(call, stream, 2)
        sms = _time_events(lambda: [_lib.check(single(g.handle, int(s), one.data_ptr(), None, C.byref(o)), algo)
                                    for s in srcs[:8]], stream, 1) / 8 * NSRC
        roof, _ = profiled(call, peak)
        out[f"{algo}_road1200_batched64"] = {"gteps": teps / (mms * 1e-3) / 1e9, "ms": mms,
                                             "single_x64_ms_est": sms, "batched_over_single": sms / mms,
                                             "roofline": roof}
    g.close()
    # differentiable PPR: directed R-MAT 20, lognormal row-normalised weights, 32 teleport columns
    from gpugraph_b200.ppr import ppr

    rng = np.random.default_rng(SEED)
    hg = gg.HostGraph.rmat(20, 16, seed=SEED, symmetrize=False)
    g = gg.Graph(hg, directed=True)
    w = rng.lognormal(0.0, 1.0, size=hg.edges)
    src = np.repeat(np.arange(hg.nodes), np.diff(hg.row_offsets))
    w = w / np.bincount(src, weights=w, minlength=hg.nodes)[src]
    T = np.zeros((hg.nodes, 32), np.float32)
    for c in range(32):
        T[rng.choice(hg.nodes, 100, replace=False), c] = 0.01
    wt = torch.tensor(w, dtype=torch.float32, device=dev, requires_grad=True)
    Tt = torch.tensor(T, device=dev, requires_grad=True)
    Cm = torch.randn((hg.nodes, 32), device=dev)

    def fb():
        wt.grad = None
        Tt.grad = None
        (ppr(g, wt, Tt) * Cm).sum().backward()

    fbms = _time_events(fb, stream, 2)
    fwd = lambda: ppr(g, wt.detach(), Tt.detach())
    fms = _time_events(fwd, stream, 2)
    roof, _ = profiled(fwd, peak)
    out["ppr_rmat20_32vec"] = {"forward_ms": fms, "forward_backward_ms": fbms, "V": hg.nodes, "E": hg.edges,
                               "roofline_forward": roof}
    g.close()
    return out


# ---------------------------------------------------------- reference arm --
def cpu_bfs_steps(ro, col, srcs, cores: int, steps: int, warmup: int = 0):
    """The reference's CPU BFS (CPUBFS from oracle/_ref, else the oracle port) on
    `cores` sources per step, one source per worker process and core. Returns the
    per-step GTEPS (edges of the sources' reached vertices over the slowest
    worker's traversal time: the workers run concurrently) and what ran."""
    import oracle
    from oracle import pool

    kind = "ref_bfs" if oracle.ref() is not None else "bfs"
    deg = np.diff(ro).astype(np.int64)
    vals, secs = [], []
    with pool.SourceRunner(ro, col, procs=cores) as runner:
        for step in range(warmup + steps):
            sample = np.roll(srcs, -step * cores)[:cores]
            res, t = runner.run(kind, sample)
            if step >= warmup:
                edges = int(sum(deg[r >= 0].sum() for r in res))
                vals.append(edges / max(t) / 1e9)
                secs.append(max(t))
    return vals, {"kind": "reference" if kind == "ref_bfs" else "port", "sources_per_step": cores,
                  "step_seconds": secs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--quick", action="store_true", help="headline, e2e, roofline and the graph batch only")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cuda-graph", action="store_true",
                    help="launch the same level kernels host-driven (for ncu launch lists)")
    ap.add_argument("--no-autotune", action="store_true", help="time the headline with the default options")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch under torch.distributed.run
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={29500 + os.getpid() % 1000}", __file__] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    if args.gpus != world:
        log(f"[bench] --gpus {args.gpus} but WORLD_SIZE={world}: running {world} rank(s)")
    cores = len(os.sched_getaffinity(0))
    metric = metric_name(args.scale)
    config = {"workload": workload(args.scale), "nsrc_per_rank": NSRC,
              "l2": "inputs larger than L2 (CSR > 0.5 GB, per-source state 1 GB)",
              "parallelism": f"replicas x{world}, disjoint source blocks" if world > 1 else "single GPU"}
    cpu_cores = max(1, min(cores, NSRC))

    if args.impl == "reference":
        if rank != 0:
            return
        import oracle  # the oracle's own generator: the product library is never loaded here

        ro, col = oracle.rmat(args.scale, EDGEFACTOR, seed=SEED)
        srcs = pick_sources(ro, NSRC)
        vals, info = cpu_bfs_steps(ro, col, srcs, cpu_cores, max(1, args.steps), args.warmup)
        v = statistics.median(vals)
        # n_gpus is the launch's N (the arm runs on rank 0's host cores; cpu_baseline.cores says how many)
        line = {"impl": "reference", "metric": metric, "value": v, "unit": "GTEPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "int32",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": cpu_cores, "kind": info["kind"],
                                 "sample": f"each step: CPUBFS from {cpu_cores} of the 64 sources, one per core in "
                                           f"spawned processes, edges of the reached vertices over the slowest "
                                           f"traversal; median over steps"},
                "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime

        import torch

        # each rank on its own GPU before NCCL sets up its communicator
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        res, hg, srcs = run_native(args, world)
        if rank == 0:
            cpu = None
            if not args.no_cpu_baseline:
                vals, info = cpu_bfs_steps(hg.row_offsets, hg.column_indices, srcs, cpu_cores, 1)
                cpu = {"value": vals[0], "unit": "GTEPS", "cores": cpu_cores, "kind": info["kind"],
                       "sample": f"CPUBFS from {cpu_cores} of rank 0's 64 sources, one per core, concurrent; "
                                 f"slowest traversal {info['step_seconds'][0]:.1f}s"}
            line = {
                "impl": "native", "metric": metric, "value": res["value"], "unit": "GTEPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic", "config": dict(config, options=res["tuned"] or "defaults"),
                "e2e": res["e2e"], "roofline": res["roofline"],
                "cpu_baseline": cpu, "gpu_launches": res["launches"], "clocks": res["clocks"],
                "sub_results": res["sub"],
                "graph": {"V": res["V"], "E": res["E"], "teps_edges_rank0": res["teps_edges_this_rank"]},
            }
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
