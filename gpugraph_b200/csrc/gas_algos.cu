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
#include "gas/run_gas.cuh"

namespace mg {

int cc_union_find(mg_graph *g, int32_t *labels, mg_stats *stats, const mg_options *o);  // cc.cu
int sssp_fused(mg_graph *g, int32_t src, int32_t *dists, mg_stats *stats, const mg_options *o);  // sssp.cu

__global__ void k_fill_u32(uint32_t *p, uint32_t v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
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
  if (!dists) return set_error(MG_ERR_ARG, "dists is NULL");
  if (!o->generic_engine) return sssp_fused(g, src, dists, stats, o);  // sssp.cu
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
  if (!labels) return set_error(MG_ERR_ARG, "labels is NULL");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  // symmetric graph: the same labels in one union-find pass (cc.cu)
  if (!g->directed && !o->generic_engine) return cc_union_find(g, labels, stats, o);
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
