// The generic GAS level loop for any Program written to the reference's
// contract (GASengine/enactor_vertex_centric.cuh:3269-3924, EnactIterativeSearch):
// gather -> apply -> post_apply -> frontier scan -> expand/contract -> level end,
// run as one CUDA graph per (Program, launch shape). A new Program drops in by
// including this header in its own .cu, filling GasArgs<P> from base_args<P>()
// plus its VertexType/EdgeType arrays, putting its initial frontier in queue 0
// and calling run_gas<P>() (tests/cpp/user_program.cu is such a file).
#pragma once
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <typeinfo>

#include "../algo_util.cuh"
#include "driver.cuh"
#include "engine.cuh"

namespace mg {

constexpr int kGasVTS = 4;  // frontier entries per thread in the scan
constexpr int kGasVT = 8;   // items per thread in the expand (NV = 2048)

template <class P>
GasArgs<P> base_args(mg_graph *g) {
  Workspace &w = g->ws;
  GasArgs<P> a;
  // zeroed first, so the bytes of the struct (padding included) identify the
  // arguments when run_gas keys its cached CUDA graph on them
  memset(static_cast<void *>(&a), 0, sizeof(a));
  a.g = g->csr;
  a.queue0 = w.queue[0];
  a.queue1 = w.queue[1];
  a.scan = w.scan;
  a.part = w.part;
  a.status = w.status;
  a.bm0 = w.bm[0];
  a.bm1 = w.bm[1];
  a.changed = w.changed;
  a.gather_tmp = reinterpret_cast<typename P::GatherType *>(w.gather_tmp);
  a.gather_res = reinterpret_cast<typename P::GatherType *>(w.vbuf[1]);
  a.ctl = w.ctl;
  a.expand_in = P::expandOverEdges() == EXPAND_IN_EDGES ? 1 : P::expandOverEdges() == EXPAND_ALL_EDGES ? 2 : 0;
  a.gather_dir = (int32_t)P::gatherOverEdges();
  return a;
}

// Generic level loop for a Program: gather -> apply -> post_apply -> scan ->
// expand/contract -> level end. n0 = initial frontier size (already in queue 0).
template <class P>
int run_gas(mg_graph *g, const GasArgs<P> &a, uint32_t n0, const mg_options *o, const char *name, LoopResult *res) {
  // NO_EXPAND_EDGES ends the run after one gather/apply round (nothing enters
  // the next frontier); EXPAND_ALL_EDGES expands out-edges and in-edges.
  cudaStream_t s = run_stream(g, o);
  const int grid = persistent_grid(g, o, 4);
  // Every level of a traversal settles at least one vertex, so V + 2 levels bound
  // the device loop even if a Program never empties its frontier.
  const uint32_t max_iter = (uint32_t)std::min<int64_t>(o->iter_num > 0 ? o->iter_num : 0, g->nodes + 2);
  cudaError_t e = cudaMemsetAsync(g->ws.bm[0], 0, g->ws.words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.bm[1], 0, g->ws.words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.changed, 0, (size_t)g->nodes, s);
  int st = cuda_status(e, "gas init");
  if (st != MG_OK) return st;
  k_ctl_init<<<1, 32, 0, s>>>(a.ctl, n0, max_iter, (unsigned long long)o->spin_limit, MODE_QUEUE, ctl_flags(o));
  count_launch();
  const bool expand = P::expandOverEdges() != NO_EXPAND_EDGES;
  const bool gather = P::gatherOverEdges() != NO_GATHER_EDGES;
  const bool apply = P::applyOverEdges() != NO_APPLY_VERTICES;
  const bool post = P::postApplyOverEdges() != NO_POST_APPLY_VERTICES;
  const int apply_all = P::applyOverEdges() == APPLY_ALL;
  const int post_all = P::postApplyOverEdges() == POST_APPLY_ALL;
  const int kpl = 1 + (expand ? 2 : 0) + (gather ? 1 : 0) + (apply ? 1 : 0) + (post ? 1 : 0);
  // expand tile: 1024 or 2048 items (mg_options.tile_items; 0 = 2048)
  const bool small_tiles = o->tile_items > 0 && o->tile_items <= 1024;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    if (gather) MG_LAUNCH(KID_GATHER, ss, k_gather<P><<<grid, kNT, 0, ss>>>(a));
    if (apply) MG_LAUNCH(KID_APPLY, ss, k_apply<P><<<grid, kNT, 0, ss>>>(a, apply_all, gather ? 1 : 0));
    if (post) MG_LAUNCH(KID_APPLY, ss, k_post_apply<P><<<grid, kNT, 0, ss>>>(a, post_all));
    if (expand && small_tiles) {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kGasVTS, 4><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_expand<P, 4><<<grid, kNT, 0, ss>>>(a)));
    } else if (expand) {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kGasVTS, kGasVT><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_expand<P, kGasVT><<<grid, kNT, 0, ss>>>(a)));
    }
    MG_LAUNCH(KID_OTHER, ss, k_level_end<<<1, 32, 0, ss>>>(a.ctl, h, use_h));
  };
  // The CUDA graph bakes in the kernels' arguments: key it on the Program type
  // and on the argument bytes (a Program's own arrays can change between runs).
  uint64_t h = 1469598103934665603ull;  // FNV-1a
  const unsigned char *bytes = reinterpret_cast<const unsigned char *>(&a);
  for (size_t i = 0; i < sizeof(a); ++i) h = (h ^ bytes[i]) * 1099511628211ull;
  char tag[32];
  snprintf(tag, sizeof(tag), "/%016llx", (unsigned long long)h);
  st = run_level_loop(g, s,
                      std::string(name) + "/" + typeid(P).name() + tag + "/" + std::to_string(grid) +
                          (small_tiles ? "/t1024" : "/t2048"),
                      kpl, body, o->use_cuda_graph != 0, res);
  if (st != MG_OK) return st;
  finish_run(g, res->ctl.level);
  if (res->ctl.error)
    return set_error(res->ctl.error, std::string(name) + ": device reported " + mg_status_string(res->ctl.error));
  return MG_OK;
}

}  // namespace mg
