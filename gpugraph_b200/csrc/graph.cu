// Device graph construction and working-set management.
// Replaces CsrProblem::FromHostProblem (GASengine/csr_problem.cuh:512-839),
// the CSC build it runs with thrust (util.cuh:55-126) and CsrProblem::Reset
// (csr_problem.cuh:845-1045): queues are sized exactly (a frontier is a set of
// distinct vertices, so V entries suffice), allocated once per graph and reused.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "graph.cuh"
#include "host_util.h"

namespace mg {

int cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return MG_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return set_error(MG_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
  }
  return set_error(MG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int launch_check(const char *what) { return cuda_status(cudaGetLastError(), what); }

int device_alloc(mg_graph *g, void **p, size_t bytes) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_status(e, "cudaMalloc");
  }
  g->allocations.push_back(*p);
  g->device_bytes += bytes;
  return MG_OK;
}

cudaStream_t run_stream(mg_graph *g, const mg_options *o) {
  return (o && o->stream) ? (cudaStream_t)o->stream : g->stream;
}

// Largest tile sizes used by the level-loop kernels (items per expand tile and
// frontier entries per scan tile are both >= 1024).
static constexpr size_t kMinTile = 1024;

int ensure_workspace(mg_graph *g) {
  Workspace &w = g->ws;
  if (w.ctl) return MG_OK;
  const size_t V = (size_t)g->nodes, E = (size_t)g->edges;
  w.words = (V + 31) / 32 + 4;
  w.part_cap = (V + E) / kMinTile + 8;
  w.status_cap = (V + E) / kMinTile + 64;
  int st;
#define MG_ALLOC(ptr, bytes)                                   \
  if ((st = device_alloc(g, (void **)&(ptr), (bytes))) != MG_OK) \
    return st;
  MG_ALLOC(w.queue[0], V * 4);
  MG_ALLOC(w.queue[1], V * 4);
  MG_ALLOC(w.scan, (V + 1) * 4);
  MG_ALLOC(w.part, w.part_cap * 4);
  MG_ALLOC(w.status, w.status_cap * 8);
  MG_ALLOC(w.bm[0], w.words * 4);
  MG_ALLOC(w.bm[1], w.words * 4);
  MG_ALLOC(w.visited, w.words * 4);
  MG_ALLOC(w.changed, V);
  MG_ALLOC(w.gather_tmp, V * 4);
  MG_ALLOC(w.vbuf[0], V * 4);
  MG_ALLOC(w.vbuf[1], V * 4);
  MG_ALLOC(w.ctl, sizeof(Ctl));
#undef MG_ALLOC
  cudaError_t e = cudaMemsetAsync(w.status, 0, w.status_cap * 8, g->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w.ctl, 0, sizeof(Ctl), g->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w.bm[0], 0, w.words * 4, g->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w.bm[1], 0, w.words * 4, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  return cuda_status(e, "workspace init");
}

int ensure_multi(mg_graph *g) {
  const size_t V = (size_t)g->nodes;
  int st;
  for (int i = 0; i < 3; ++i)
    if (!g->mask[i] && (st = device_alloc(g, (void **)&g->mask[i], V * 8)) != MG_OK) return st;
  if (!g->multi_out) {
    if ((st = device_alloc(g, (void **)&g->multi_out, V * 64 * 4)) != MG_OK) return st;
    g->multi_bytes = V * 64 * 4;
  }
  if (!g->multi_stk_bm &&
      (st = device_alloc(g, (void **)&g->multi_stk_bm, (size_t)kMsStackLevels * ((V + 31) / 32) * 4)) != MG_OK)
    return st;
  if (g->ms_nheavy < 0) {
    // the long in-lists, longest first (the pull kernel deals them to warps in
    // this order, back and forth, so each warp gets a similar share)
    std::vector<int32_t> off(V + 1);
    cudaError_t e = cudaMemcpy(off.data(), g->csr.csc_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost);
    if ((st = cuda_status(e, "in-list lengths")) != MG_OK) return st;
    std::vector<int32_t> heavy;
    for (size_t v = 0; v < V; ++v)
      if (off[v + 1] - off[v] > kMsHeavyList) heavy.push_back((int32_t)v);
    std::stable_sort(heavy.begin(), heavy.end(),
                     [&](int32_t x, int32_t y) { return off[x + 1] - off[x] > off[y + 1] - off[y]; });
    if ((st = device_alloc(g, (void **)&g->ms_heavy, std::max<size_t>(heavy.size(), 1) * 4)) != MG_OK) return st;
    if (!heavy.empty()) {
      e = cudaMemcpy(g->ms_heavy, heavy.data(), heavy.size() * 4, cudaMemcpyHostToDevice);
      if ((st = cuda_status(e, "long in-lists upload")) != MG_OK) return st;
    }
    g->ms_nheavy = (int32_t)heavy.size();
  }
  return MG_OK;
}

}  // namespace mg

using namespace mg;

namespace {

// Copy of the in-lists with every list ordered by descending out-degree of the
// neighbour (ties by id), for the bottom-up kernels only: a high-degree
// neighbour is the likeliest to be in the frontier, so their early exit comes
// after fewer probes, and the hubs' frontier entries stay hot in cache. The
// order of a list does not change which vertices a pull level finds.
int upload_pull_rows(mg_graph *g, const int32_t *in_off, const int32_t *in_rows, const int32_t *row_offsets) {
  const int64_t V = g->nodes, E = g->edges;
  int st = device_alloc(g, (void **)&g->csr.pull_rows, (size_t)E * 4 + 64);
  if (st != MG_OK || E == 0) return st;
  std::vector<int32_t> pull(in_rows, in_rows + E);
  host_parallel_for(V, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t v = b; v < e; ++v)
      std::sort(pull.data() + in_off[v], pull.data() + in_off[v + 1], [&](int32_t x, int32_t y) {
        const int32_t dx = row_offsets[x + 1] - row_offsets[x], dy = row_offsets[y + 1] - row_offsets[y];
        return dx != dy ? dx > dy : x < y;
      });
  });
  return cuda_status(cudaMemcpy(g->csr.pull_rows, pull.data(), (size_t)E * 4, cudaMemcpyHostToDevice),
                     "pull list upload");
}

int create_common(const int32_t *row_offsets, const int32_t *col, const void *vals, int32_t value_type, int64_t nodes,
                  int64_t edges, int32_t directed, mg_graph **out) {
  if (!out) return set_error(MG_ERR_ARG, "out is NULL");
  *out = nullptr;
  std::string why = validate_csr(nodes, edges, row_offsets, col);
  if (!why.empty()) return set_error(MG_ERR_ARG, why);
  if (value_type != MG_VAL_NONE && value_type != MG_VAL_I32 && value_type != MG_VAL_F32)
    return set_error(MG_ERR_ARG, "unknown value_type");
  if (value_type != MG_VAL_NONE && !vals && edges > 0) return set_error(MG_ERR_ARG, "edge_values is NULL");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    cudaGetLastError();
    return set_error(MG_ERR_CUDA, "no CUDA device available");
  }
  mg_graph *g = new mg_graph();
  cudaGetDevice(&g->device);
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device);
  g->nodes = nodes;
  g->edges = edges;
  g->directed = directed ? 1 : 0;
  int st = MG_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&g->host_ctl, sizeof(Ctl));
  if ((st = cuda_status(e, "stream/event setup")) != MG_OK) {
    mg_graph_destroy(g);
    return st;
  }
  const size_t V = (size_t)nodes, E = (size_t)edges;
  // Row offsets padded to a multiple of 4 entries plus one spare 16-byte chunk.
  const size_t ro_n = ((V + 1 + 3) & ~(size_t)3) + 4;
  DevCsr &c = g->csr;
  c.V = (int32_t)nodes;
  c.E = (int32_t)edges;
  std::vector<int32_t> ro_pad(ro_n, (int32_t)edges);
  memcpy(ro_pad.data(), row_offsets, (V + 1) * 4);
  if ((st = device_alloc(g, (void **)&c.row_offsets, ro_n * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&c.col, E * 4 + 64)) != MG_OK) {
    mg_graph_destroy(g);
    return st;
  }
  e = cudaMemcpy(c.row_offsets, ro_pad.data(), ro_n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && E) e = cudaMemcpy(c.col, col, E * 4, cudaMemcpyHostToDevice);
  if ((st = cuda_status(e, "graph upload")) != MG_OK) {
    mg_graph_destroy(g);
    return st;
  }
  if (value_type == MG_VAL_I32 || value_type == MG_VAL_F32) {
    // 4-byte values either way (the reference also copies edge values as 4-byte
    // words, csr_problem.cuh:706-741); F32 values are stored bit-exactly.
    if ((st = device_alloc(g, (void **)&c.wgt, E * 4 + 64)) != MG_OK) {
      mg_graph_destroy(g);
      return st;
    }
    e = E ? cudaMemcpy(c.wgt, vals, E * 4, cudaMemcpyHostToDevice) : cudaSuccess;
    if ((st = cuda_status(e, "edge value upload")) != MG_OK) {
      mg_graph_destroy(g);
      return st;
    }
  }
  if (directed) {
    std::vector<int32_t> t_off(ro_n, (int32_t)edges), t_rows(E ? E : 1), t_eid(E ? E : 1);
    host_transpose(nodes, edges, row_offsets, col, t_off.data(), t_rows.data(), t_eid.data());
    if ((st = device_alloc(g, (void **)&c.csc_offsets, ro_n * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&c.csc_rows, E * 4 + 64)) != MG_OK ||
        (st = device_alloc(g, (void **)&c.csc_eid, E * 4 + 64)) != MG_OK) {
      mg_graph_destroy(g);
      return st;
    }
    e = cudaMemcpy(c.csc_offsets, t_off.data(), ro_n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && E) e = cudaMemcpy(c.csc_rows, t_rows.data(), E * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && E) e = cudaMemcpy(c.csc_eid, t_eid.data(), E * 4, cudaMemcpyHostToDevice);
    if ((st = cuda_status(e, "transpose upload")) != MG_OK ||
        (st = upload_pull_rows(g, t_off.data(), t_rows.data(), row_offsets)) != MG_OK) {
      mg_graph_destroy(g);
      return st;
    }
  } else {
    // Symmetric graph: the in-edges of v are its out-edges; the CSR entry of
    // (v,u) stands for the in-edge (u,v) (edge values are symmetric).
    c.csc_offsets = c.row_offsets;
    c.csc_rows = c.col;
    c.csc_eid = nullptr;
    if ((st = upload_pull_rows(g, row_offsets, col, row_offsets)) != MG_OK) {
      mg_graph_destroy(g);
      return st;
    }
  }
  if ((st = ensure_workspace(g)) != MG_OK) {
    mg_graph_destroy(g);
    return st;
  }
  *out = g;
  return MG_OK;
}

}  // namespace

extern "C" {

int mg_graph_create(const int32_t *row_offsets, const int32_t *column_indices, const void *edge_values,
                    int32_t value_type, int64_t nodes, int64_t edges, int32_t directed, const mg_options *opts,
                    mg_graph **out) {
  (void)opts;
  clear_error();
  return create_common(row_offsets, column_indices, edge_values, value_type, nodes, edges, directed, out);
}

int mg_graph_create_batch(const int32_t *row_offsets, const int32_t *column_indices, int64_t nodes, int64_t edges,
                          const int64_t *graph_offsets, int32_t ngraphs, const mg_options *opts, mg_graph **out) {
  (void)opts;
  clear_error();
  if (!graph_offsets || ngraphs < 1) return set_error(MG_ERR_ARG, "graph_offsets/ngraphs");
  if (graph_offsets[0] != 0 || graph_offsets[ngraphs] != nodes)
    return set_error(MG_ERR_ARG, "graph_offsets must run from 0 to nodes");
  for (int i = 0; i < ngraphs; ++i)
    if (graph_offsets[i + 1] <= graph_offsets[i]) return set_error(MG_ERR_ARG, "every graph needs >= 1 vertex");
  std::string why = validate_csr(nodes, edges, row_offsets, column_indices);
  if (!why.empty()) return set_error(MG_ERR_ARG, why);
  // Edges must stay inside their graph.
  for (int i = 0; i < ngraphs; ++i) {
    const int64_t b = graph_offsets[i], e = graph_offsets[i + 1];
    for (int64_t j = row_offsets[b]; j < row_offsets[e]; ++j)
      if (column_indices[j] < b || column_indices[j] >= e)
        return set_error(MG_ERR_ARG, "edge leaves its graph in batch graph " + std::to_string(i));
  }
  int st = create_common(row_offsets, column_indices, nullptr, MG_VAL_NONE, nodes, edges, 0, out);
  if (st != MG_OK) return st;
  (*out)->graph_offsets.assign(graph_offsets, graph_offsets + ngraphs + 1);
  return MG_OK;
}

int mg_graph_destroy(mg_graph *g) {
  if (!g) return MG_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  for (auto &kv : g->loops) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  for (void *p : g->allocations) cudaFree(p);
  if (g->host_ctl) cudaFreeHost(g->host_ctl);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return MG_OK;
}

int mg_graph_info(const mg_graph *g, int64_t *nodes, int64_t *edges, int32_t *directed, int64_t *device_bytes) {
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (nodes) *nodes = g->nodes;
  if (edges) *edges = g->edges;
  if (directed) *directed = g->directed;
  if (device_bytes) *device_bytes = (int64_t)g->device_bytes;
  return MG_OK;
}

}  // extern "C"
