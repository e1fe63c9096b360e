#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../host_util.h"
#include "driver.cuh"
#include "engine.cuh"

namespace mg {

constexpr size_t kMaxCachedLoops = 64;
constexpr int kLevelsPerIteration = 4;

int read_ctl(mg_graph *g, cudaStream_t s, Ctl *out) {
  cudaError_t e = cudaMemcpyAsync(g->host_ctl, g->ws.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) memcpy(out, g->host_ctl, sizeof(Ctl));
  return cuda_status(e, "control block read");
}

// ---------------------------------------------------------------- profiler --
namespace {
const char *kKernelNames[kNumKernelKinds] = {"frontier_scan",   "expand_contract", "bfs_pull",
                                             "multi_bfs_pull",  "multi_bfs_apply", "frontier_convert",
                                             "multi_sssp_expand", "pagerank_pull", "gather",
                                             "apply",           "ppr",             "cc",
                                             "other"};
struct Profiler {
  bool on = false;
  std::vector<std::pair<int, cudaEvent_t>> marks;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  double ms[kNumKernelKinds] = {0};
  int64_t launches[kNumKernelKinds] = {0};
  unsigned long long bytes[kNumKernelKinds] = {0};
  cudaEvent_t next_event() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
};
thread_local Profiler g_prof;
}  // namespace

bool prof_on() { return g_prof.on; }

void prof_mark(cudaStream_t s, int kid) {
  if (!g_prof.on) return;
  cudaEvent_t e = g_prof.next_event();
  cudaEventRecord(e, s);
  g_prof.marks.push_back({kid, e});
}

void prof_flush(cudaStream_t s, const unsigned long long *kbytes) {
  if (!g_prof.on) return;
  cudaEvent_t end = g_prof.next_event();
  cudaEventRecord(end, s);
  cudaEventSynchronize(end);
  for (size_t i = 0; i < g_prof.marks.size(); ++i) {
    cudaEvent_t b = g_prof.marks[i].second;
    cudaEvent_t e = (i + 1 < g_prof.marks.size()) ? g_prof.marks[i + 1].second : end;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b, e);
    const int k = g_prof.marks[i].first;
    g_prof.ms[k] += ms;
    g_prof.launches[k] += 1;
  }
  g_prof.marks.clear();
  g_prof.used = 0;
  if (kbytes)
    for (int k = 0; k < kNumKernelKinds; ++k) g_prof.bytes[k] += kbytes[k];
}

int prepare_run(mg_graph *g, cudaStream_t s) {
  if (g->epochs_used < (1ull << 27)) return MG_OK;
  cudaError_t e = cudaMemsetAsync(g->ws.status, 0, g->ws.status_cap * 8, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.ctl, 0, sizeof(Ctl), s);
  g->epochs_used = 0;
  return cuda_status(e, "status reset");
}

void finish_run(mg_graph *g, uint32_t levels) { g->epochs_used += 4ull * ((uint64_t)levels + 2); }

static int build_graph(mg_graph *g, cudaStream_t s, const LevelBody &body, LoopCache *lc) {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphCreate(&graph, 0);
  cudaGraphConditionalHandle h = 0;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t cnode;
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams &params = *reinterpret_cast<cudaGraphNodeParams *>(raw);
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = h;
  params.conditional.type = cudaGraphCondTypeWhile;
  params.conditional.size = 1;
  if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, graph, nullptr, 0, &params);
  if (e == cudaSuccess) {
    cudaGraph_t bodyg = params.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      // four levels per iteration of the WHILE node (a node iteration costs
      // about as much as four empty kernels): when a level ends the loop, the
      // later copies' kernels return at once, as in the host-driven loop
      for (int k = 0; k < kLevelsPerIteration; ++k) body(s, h, 1);
      cudaGraph_t captured = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(s, &captured);
      e = (e2 != cudaSuccess) ? e2 : cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    return cuda_status(e, "level-loop graph capture");
  }
  lc->graph = graph;
  lc->exec = exec;
  (void)g;
  return MG_OK;
}

int run_level_loop(mg_graph *g, cudaStream_t s, const std::string &key, int kernels_per_level, const LevelBody &body,
                   bool use_graph, LoopResult *res, const std::function<void(cudaStream_t)> *epilogue) {
  cudaError_t e = cudaEventRecord(g->ev0, s);
  if (e != cudaSuccess) return cuda_status(e, "event record");
  bool graphed = false;
  if (use_graph && !prof_on()) {
    auto it = g->loops.find(key);
    if (it == g->loops.end() && g->loops.size() >= kMaxCachedLoops) {
      // bound the cache (keys include argument hashes): drop every cached
      // graph; the ones still in use are rebuilt on their next run
      for (auto &kv : g->loops) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
      }
      g->loops.clear();
    }
    if (it == g->loops.end()) {
      LoopCache lc;
      lc.kernels_per_level = kernels_per_level;
      if (build_graph(g, s, body, &lc) == MG_OK) {
        it = g->loops.emplace(key, lc).first;
      } else {
        clear_error();  // fall back to host-driven launches of the same kernels
      }
    }
    if (it != g->loops.end()) {
      e = cudaGraphLaunch(it->second.exec, s);
      if (e != cudaSuccess) return cuda_status(e, "graph launch");
      graphed = true;
    }
  }
  if (!graphed) {
    // Host-driven loop: a few levels per control-block check; levels after the
    // end are no-ops because every kernel returns when ctl->active == 0.
    for (;;) {
      for (int k = 0; k < 4; ++k) {
        body(s, 0, 0);
        count_launch(kernels_per_level);
      }
      int st = launch_check("level kernels");
      if (st != MG_OK) return st;
      Ctl c;
      if ((st = read_ctl(g, s, &c)) != MG_OK) return st;
      if (!c.active) break;
    }
  }
  e = cudaEventRecord(g->ev1, s);
  if (e != cudaSuccess) return cuda_status(e, "event record");
  if (epilogue) {
    (*epilogue)(s);
    int st = launch_check("loop epilogue");
    if (st != MG_OK) return st;
  }
  int st = read_ctl(g, s, &res->ctl);
  if (st != MG_OK) return st;
  prof_flush(s, res->ctl.kbytes);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, g->ev0, g->ev1);
  res->ms = ms;
  res->used_graph = graphed;
  if (graphed) {
    // every iteration of the WHILE node launches all its level copies
    const int64_t iters = std::max<int64_t>(1, ((int64_t)res->ctl.level + kLevelsPerIteration - 1) /
                                                   kLevelsPerIteration);
    count_launch((int64_t)kernels_per_level * kLevelsPerIteration * iters);
  }
  return MG_OK;
}

}  // namespace mg

extern "C" {

int mg_profile_enable(int enable) {
  mg::g_prof.on = enable != 0;
  mg::g_prof.marks.clear();
  mg::g_prof.used = 0;
  for (int k = 0; k < mg::kNumKernelKinds; ++k) {
    mg::g_prof.ms[k] = 0;
    mg::g_prof.launches[k] = 0;
    mg::g_prof.bytes[k] = 0;
  }
  return MG_OK;
}

int mg_profile_read(int32_t kind, const char **name, double *total_ms, int64_t *launches, uint64_t *bytes) {
  if (kind < 0 || kind >= mg::kNumKernelKinds) return mg::set_error(MG_ERR_ARG, "kernel kind out of range");
  if (name) *name = mg::kKernelNames[kind];
  if (total_ms) *total_ms = mg::g_prof.ms[kind];
  if (launches) *launches = mg::g_prof.launches[kind];
  if (bytes) *bytes = (uint64_t)mg::g_prof.bytes[kind];
  return MG_OK;
}

}  // extern "C"
