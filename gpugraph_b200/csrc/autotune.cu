// Autotuner for the level-loop launch parameters: the expand thresholds, tile
// shapes and direction-switch factors, chosen on the caller's graph.
// The reference fixes them at compile time (KernelPolicy<..., 200>, CTA/warp
// gather thresholds 512/32: GASengine/enactor_vertex_centric.cuh:3934-3970).
//
// Search, by coordinate descent on the caller's graph and sources, timing each
// candidate with the library's own CUDA events (mg_stats.device_ms, median of
// three runs): expand tile (1024 or 2048 items) x persistent CTAs per SM
// (2..5), then the push->pull factor (alpha, or alpha_multi for the batched
// BFS), then the pull->push factor (beta); for PageRank and PPR, the CTAs per
// SM of their SpMV over a fixed number of iterations. The best options are
// written back to *inout; a JSON report of every trial goes to report (if given).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "graph.cuh"
#include "host_util.h"

namespace mg {
namespace {

struct Trial {
  mg_options o;
  double ms;
};

// Inputs of the PPR trials: row-normalised uniform weights and one-hot teleport
// columns (device buffers owned by the tuner).
struct PprInputs {
  float *w = nullptr, *tele = nullptr;
};

int time_once(mg_graph *g, int32_t kind, const int32_t *srcs, int32_t nsrc, const mg_options &o, void *out,
              const PprInputs &pi, double *ms) {
  mg_stats st;
  int rc = MG_OK;
  double total = 0.0;
  if (kind == MG_TUNE_PAGERANK) {
    rc = mg_pagerank(g, (float *)out, &st, &o);
    total = st.device_ms;
  } else if (kind == MG_TUNE_PPR) {
    rc = mg_ppr_forward(g, pi.w, pi.tele, nsrc, (float *)out, &st, &o);
    total = st.device_ms;
  } else if (kind == MG_TUNE_BFS) {
    for (int i = 0; i < nsrc && rc == MG_OK; ++i) {
      rc = mg_bfs(g, srcs[i], (int32_t *)out, &st, &o);
      total += st.device_ms;
    }
  } else if (kind == MG_TUNE_BFS_MULTI) {
    rc = mg_bfs_multi(g, srcs, nsrc, (int32_t *)out, &st, &o);
    total = st.device_ms;
  } else if (kind == MG_TUNE_SSSP) {
    for (int i = 0; i < nsrc && rc == MG_OK; ++i) {
      rc = mg_sssp(g, srcs[i], (int32_t *)out, &st, &o);
      total += st.device_ms;
    }
  } else {
    rc = mg_cc(g, (int32_t *)out, &st, &o);
    total = st.device_ms;
  }
  *ms = total;
  return rc;
}

int measure(mg_graph *g, int32_t kind, const int32_t *srcs, int32_t nsrc, const mg_options &o, void *out,
            const PprInputs &pi, double *ms) {
  double t[3];
  for (int r = 0; r < 3; ++r) {
    int rc = time_once(g, kind, srcs, nsrc, o, out, pi, &t[r]);
    if (rc != MG_OK) return rc;
  }
  std::sort(t, t + 3);
  *ms = t[1];
  return MG_OK;
}

}  // namespace
}  // namespace mg

using namespace mg;

extern "C" int mg_autotune(mg_graph *g, int32_t kind, const int32_t *srcs, int32_t nsrc, mg_options *inout,
                           char *report, int64_t report_len) {
  clear_error();
  if (!g || !inout) return set_error(MG_ERR_ARG, "graph/options is NULL");
  if (kind < MG_TUNE_BFS || kind > MG_TUNE_PPR) return set_error(MG_ERR_ARG, "unknown tuning kind");
  const bool need_srcs = kind != MG_TUNE_CC && kind != MG_TUNE_PAGERANK;
  if (need_srcs && (!srcs || nsrc < 1 || nsrc > 64)) return set_error(MG_ERR_ARG, "need 1..64 sources");
  for (int32_t i = 0; need_srcs && i < nsrc; ++i)
    if (srcs[i] < 0 || srcs[i] >= g->nodes) return set_error(MG_ERR_ARG, "source out of range");
  if (kind == MG_TUNE_SSSP && !g->csr.wgt) return set_error(MG_ERR_UNSUPPORTED, "SSSP needs edge weights");
  if (kind == MG_TUNE_PPR && !g->directed) return set_error(MG_ERR_UNSUPPORTED, "PPR needs a directed graph");
  // one device result buffer for the trials ([nsrc][V] for the batched BFS, [V][nsrc] for PPR)
  const bool per_src = kind == MG_TUNE_BFS_MULTI || kind == MG_TUNE_PPR;
  const size_t bytes = (size_t)g->nodes * 4 * (per_src ? (size_t)nsrc : 1);
  void *out = nullptr;
  cudaError_t e = cudaMalloc(&out, bytes);
  if (e != cudaSuccess) return cuda_status(e, "autotune buffer");
  PprInputs pi;
  if (kind == MG_TUNE_PPR) {
    const int64_t V = g->nodes, E = g->edges;
    std::vector<int32_t> ro((size_t)V + 1);
    std::vector<float> w((size_t)std::max<int64_t>(E, 1)), tele((size_t)V * nsrc, 0.f);
    e = cudaMemcpy(ro.data(), g->csr.row_offsets, ro.size() * 4, cudaMemcpyDeviceToHost);
    for (int64_t v = 0; e == cudaSuccess && v < V; ++v)
      for (int32_t k = ro[v]; k < ro[v + 1]; ++k) w[k] = 1.f / (float)(ro[v + 1] - ro[v]);
    for (int32_t c = 0; c < nsrc; ++c) tele[(size_t)srcs[c] * nsrc + c] = 1.f;
    if (e == cudaSuccess) e = cudaMalloc(&pi.w, w.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&pi.tele, tele.size() * 4);
    if (e == cudaSuccess) e = cudaMemcpy(pi.w, w.data(), w.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pi.tele, tele.data(), tele.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(out);
      cudaFree(pi.w);
      cudaFree(pi.tele);
      return cuda_status(e, "autotune PPR inputs");
    }
  }
  mg_options base = *inout;
  base.outputs_on_device = 1;
  base.compute_stats = 0;
  if (kind == MG_TUNE_PAGERANK || kind == MG_TUNE_PPR) {
    base.iter_num = 20;  // a fixed amount of work per trial
    base.tolerance = 0.0;
  }
  std::vector<Trial> trials;
  auto eval = [&](const mg_options &o, double *ms) -> int {
    int rc = measure(g, kind, srcs, nsrc, o, out, pi, ms);
    if (rc == MG_OK) trials.push_back({o, *ms});
    return rc;
  };
  mg_options best = base;
  double best_ms = 1e300;
  int rc = MG_OK;
  // 0) SpMV kernels: CTAs per SM only
  if (kind == MG_TUNE_PAGERANK || kind == MG_TUNE_PPR) {
    for (int cps : {2, 3, 4, 5, 6, 7, 8}) {
      mg_options o = best;
      o.ctas_per_sm = cps;
      double ms;
      if ((rc = eval(o, &ms)) != MG_OK) break;
      if (ms < best_ms) best_ms = ms, best = o;
    }
  }
  // 1) tile x CTAs per SM
  for (int tile : {1024, 2048}) {
    if (kind == MG_TUNE_PAGERANK || kind == MG_TUNE_PPR) break;
    for (int cps : {2, 3, 4, 5}) {
      mg_options o = best;
      o.tile_items = tile;
      o.ctas_per_sm = cps;
      double ms;
      if ((rc = eval(o, &ms)) != MG_OK) break;
      if (ms < best_ms) best_ms = ms, best = o;
    }
    if (rc != MG_OK) break;
  }
  // 2) push -> pull factor, 3) pull -> push factor (traversals with direction switching)
  if (rc == MG_OK && (kind == MG_TUNE_BFS || kind == MG_TUNE_BFS_MULTI)) {
    const std::vector<double> alphas = kind == MG_TUNE_BFS ? std::vector<double>{5, 10, 15, 25, 40}
                                                           : std::vector<double>{1.5, 3, 5, 10, 20};
    mg_options cur = best;
    for (double a : alphas) {
      mg_options o = cur;
      (kind == MG_TUNE_BFS ? o.alpha : o.alpha_multi) = a;
      double ms;
      if ((rc = eval(o, &ms)) != MG_OK) break;
      if (ms < best_ms) best_ms = ms, best = o;
    }
    cur = best;
    for (double b : {6.0, 12.0, 18.0, 30.0}) {
      if (rc != MG_OK) break;
      mg_options o = cur;
      o.beta = b;
      double ms;
      if ((rc = eval(o, &ms)) != MG_OK) break;
      if (ms < best_ms) best_ms = ms, best = o;
    }
  }
  cudaFree(out);
  cudaFree(pi.w);
  cudaFree(pi.tele);
  if (rc != MG_OK) return rc;
  best.outputs_on_device = inout->outputs_on_device;
  best.compute_stats = inout->compute_stats;
  best.iter_num = inout->iter_num;
  best.tolerance = inout->tolerance;
  *inout = best;
  if (report && report_len > 0) {
    std::string js = "{\"kind\":" + std::to_string(kind) + ",\"best_ms\":" + std::to_string(best_ms) + ",\"trials\":[";
    for (size_t i = 0; i < trials.size(); ++i) {
      char buf[256];
      snprintf(buf, sizeof(buf),
               "%s{\"tile_items\":%d,\"ctas_per_sm\":%d,\"alpha\":%g,\"alpha_multi\":%g,\"beta\":%g,\"ms\":%.5f}",
               i ? "," : "", trials[i].o.tile_items, trials[i].o.ctas_per_sm, trials[i].o.alpha,
               trials[i].o.alpha_multi, trials[i].o.beta, trials[i].ms);
      js += buf;
    }
    js += "]}";
    const size_t n = std::min<size_t>(js.size(), (size_t)report_len - 1);
    memcpy(report, js.data(), n);
    report[n] = '\0';
  }
  return MG_OK;
}
