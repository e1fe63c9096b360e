// SSSP, CC and the reference PageRank program, each run by the generic GAS
// engine (gas/engine.cuh) with the Program from gas/programs.cuh.
// Replaces EnactorVertexCentric::EnactIterativeSearch
// (GASengine/enactor_vertex_centric.cuh:3269-3924) for these programs.
#include <cuda_runtime.h>

#include <algorithm>

#include <string>
#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"
#include "gas/programs.cuh"

namespace mg {

constexpr int kVTS = 4;
constexpr int kVT = 8;

template <class P>
GasArgs<P> base_args(mg_graph *g) {
  Workspace &w = g->ws;
  GasArgs<P> a;
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
  a.expand_in = (P::expandOverEdges() == EXPAND_IN_EDGES) ? 1 : 0;
  a.gather_dir = (int32_t)P::gatherOverEdges();
  return a;
}

__global__ void k_fill_u32(uint32_t *p, uint32_t v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// Generic level loop for a Program: gather -> apply -> post_apply -> scan ->
// expand/contract -> level end. n0 = initial frontier size (already in queue 0).
template <class P>
int run_gas(mg_graph *g, const GasArgs<P> &a, uint32_t n0, const mg_options *o, const char *name, LoopResult *res) {
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
  const bool gather = P::gatherOverEdges() != NO_GATHER_EDGES;
  const bool apply = P::applyOverEdges() != NO_APPLY_VERTICES;
  const bool post = P::postApplyOverEdges() != NO_POST_APPLY_VERTICES;
  const int apply_all = P::applyOverEdges() == APPLY_ALL;
  const int post_all = P::postApplyOverEdges() == POST_APPLY_ALL;
  const int kpl = 3 + (gather ? 1 : 0) + (apply ? 1 : 0) + (post ? 1 : 0);
  // expand tile: 1024 or 2048 items (mg_options.tile_items; 0 = 2048)
  const bool small_tiles = o->tile_items > 0 && o->tile_items <= 1024;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    if (gather) MG_LAUNCH(KID_GATHER, ss, k_gather<P><<<grid, kNT, 0, ss>>>(a));
    if (apply) MG_LAUNCH(KID_APPLY, ss, k_apply<P><<<grid, kNT, 0, ss>>>(a, apply_all, gather ? 1 : 0));
    if (post) MG_LAUNCH(KID_APPLY, ss, k_post_apply<P><<<grid, kNT, 0, ss>>>(a, post_all));
    if (small_tiles) {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kVTS, 4><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_expand<P, 4><<<grid, kNT, 0, ss>>>(a)));
    } else {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kVTS, kVT><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_expand<P, kVT><<<grid, kNT, 0, ss>>>(a)));
    }
    MG_LAUNCH(KID_OTHER, ss, k_level_end<<<1, 32, 0, ss>>>(a.ctl, h, use_h));
  };
  st = run_level_loop(g, s, std::string(name) + "/" + std::to_string(grid) + (small_tiles ? "/t1024" : "/t2048"),
                      kpl, body, o->use_cuda_graph != 0, res);
  if (st != MG_OK) return st;
  finish_run(g, res->ctl.level);
  if (res->ctl.error)
    return set_error(res->ctl.error, std::string(name) + ": device reported " + mg_status_string(res->ctl.error));
  return MG_OK;
}

static void fill_stats(mg_stats *stats, const LoopResult &res) {
  if (!stats) return;
  stats->iterations = (int32_t)res.ctl.level;
  stats->push_iterations = (int32_t)res.ctl.level;
  stats->pull_iterations = 0;
  stats->converged = (res.ctl.frontier_size == 0) ? 1 : 0;
  stats->device_ms = res.ms;
  stats->vertices_reached = 0;
  stats->edges_traversed = 0;
}

static const mg_options *opts_or_default(const mg_options *o, mg_options *d) {
  if (o) return o;
  mg_options_init(d);
  return d;
}

}  // namespace mg

using namespace mg;

extern "C" {

int mg_sssp(mg_graph *g, int32_t src, int32_t *dists, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (!g->csr.wgt) return set_error(MG_ERR_UNSUPPORTED, "SSSP needs int32 edge weights (value_type MG_VAL_I32)");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  std::vector<int32_t> roots;
  int st = check_sources(g, &src, 1, &roots);
  if (st != MG_OK) return st;
  cudaStream_t s = run_stream(g, o);
  if ((st = prepare_run(g, s)) != MG_OK) return st;
  using P = programs::sssp;
  GasArgs<P> a = base_args<P>(g);
  a.vl.nodes = a.el.nodes = (int)g->nodes;
  a.vl.edges = a.el.edges = (int)g->edges;
  a.vl.d_dists = g->ws.vbuf[0];
  a.vl.d_dists_out = g->ws.vbuf[1];
  a.el.d_weights = g->csr.wgt;
  const int V = (int)g->nodes;
  // sssp::Initialize (sssp.h:73-166): dists = INIT except the source, frontier = {src}.
  k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.d_dists, P::INIT_VALUE, V);
  k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.d_dists_out, P::INIT_VALUE, V);
  k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(a.gather_tmp, P::INIT_VALUE, V);
  count_launch(3);
  const int32_t zero = 0;
  cudaError_t e = cudaMemcpyAsync(a.vl.d_dists + src, &zero, 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(a.vl.d_dists_out + src, &zero, 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->ws.queue[0], &src, 4, cudaMemcpyHostToDevice, s);
  if ((st = cuda_status(e, "sssp init")) != MG_OK) return st;
  LoopResult res;
  if ((st = run_gas<P>(g, a, 1, o, "sssp", &res)) != MG_OK) return st;
  fill_stats(stats, res);
  if (stats && want_stats(o)) {
    if ((st = reach_stats(g, s, a.vl.d_dists, P::INIT_VALUE, 1, 1, &stats->vertices_reached, &stats->edges_traversed)) !=
        MG_OK)
      return st;
  }
  return copy_out(s, dists, a.vl.d_dists, (size_t)V * 4, o->outputs_on_device != 0);
}

int mg_cc(mg_graph *g, int32_t *labels, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK) return st;
  using P = programs::cc;
  GasArgs<P> a = base_args<P>(g);
  a.vl.nodes = a.el.nodes = (int)g->nodes;
  a.vl.edges = a.el.edges = (int)g->edges;
  a.vl.d_dists = g->ws.vbuf[0];
  a.vl.d_dists_out = g->ws.vbuf[1];
  const int V = (int)g->nodes;
  // cc::Initialize (cc.h:87-140): labels = ids, frontier = every vertex.
  k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.d_dists, V);
  k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.d_dists_out, V);
  k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(g->ws.queue[0], V);
  k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(a.gather_tmp, P::INIT_VALUE, V);
  count_launch(4);
  LoopResult res;
  if ((st = run_gas<P>(g, a, (uint32_t)V, o, "cc", &res)) != MG_OK) return st;
  fill_stats(stats, res);
  if (stats) {
    stats->vertices_reached = g->nodes;
    stats->edges_traversed = g->edges;
  }
  return copy_out(s, labels, a.vl.d_dists, (size_t)V * 4, o->outputs_on_device != 0);
}

}  // extern "C"

namespace mg {

// Reference out-degree for the PageRank program (PageRank.h:141-161): row
// degree, plus the column degree when the graph is undirected.
__global__ void k_pr_ref_outdeg(const int32_t *ro, const int32_t *co, int sym, int32_t *out, int32_t V) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    int32_t d = ro[v + 1] - ro[v];
    if (sym) d += co[v + 1] - co[v];
    out[v] = d;
  }
}

__global__ void k_fill_f32(float *p, float v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace mg

extern "C" int mg_pagerank_gas(mg_graph *g, float *ranks, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK) return st;
  if (!g->ref_outdeg && (st = device_alloc(g, (void **)&g->ref_outdeg, (size_t)g->nodes * 4)) != MG_OK) return st;
  using P = programs::pagerank;
  GasArgs<P> a = base_args<P>(g);
  a.vl.nodes = a.el.nodes = (int)g->nodes;
  a.vl.edges = a.el.edges = (int)g->edges;
  a.vl.d_dists = reinterpret_cast<float *>(g->ws.vbuf[0]);
  a.vl.d_num_out_edge = g->ref_outdeg;
  a.vl.tolerance = (float)o->tolerance;
  const int V = (int)g->nodes;
  k_pr_ref_outdeg<<<g->num_sms * 4, 256, 0, s>>>(g->csr.row_offsets, g->csr.csc_offsets, g->directed ? 0 : 1,
                                                 g->ref_outdeg, V);
  k_fill_f32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.d_dists, 0.15f, V);
  k_fill_f32<<<g->num_sms * 4, 256, 0, s>>>(reinterpret_cast<float *>(a.gather_tmp), 0.0f, V);
  k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(g->ws.queue[0], V);
  count_launch(4);
  LoopResult res;
  if ((st = run_gas<P>(g, a, (uint32_t)V, o, "pagerank_gas", &res)) != MG_OK) return st;
  fill_stats(stats, res);
  if (stats) {
    stats->vertices_reached = g->nodes;
    stats->edges_traversed = (int64_t)g->edges;
  }
  return copy_out(s, ranks, a.vl.d_dists, (size_t)V * 4, o->outputs_on_device != 0);
}
