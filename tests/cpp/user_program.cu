// A GAS Program written outside the library, to the reference's Program
// contract (typedefs, INIT_VALUE, policy selectors, device functors; see
// Algorithms/PageRank/PageRank.h for the reference's own pull program), built
// against the engine headers and run by mg::run_gas. It exercises the gather
// directions the bundled programs do not use: for every vertex v,
//   out[v] = sum of val[u] over the in-, out- or all neighbours u of v
// (GATHER_IN_EDGES / GATHER_OUT_EDGES / GATHER_ALL_EDGES), one gather/apply round
// over all vertices and no expansion (NO_EXPAND_EDGES).
#include <cuda_runtime.h>
#include <stdint.h>

#include "gas/run_gas.cuh"
#include "graph.cuh"

namespace {

template <GatherEdges GD>
struct nbr_sum {
  typedef int DataType;
  typedef int MiscType;
  typedef int GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = 0;
  static const bool allow_duplicates = true;
  struct VertexType {
    const int *d_val;
    int *d_out;
    int nodes;
  };
  struct EdgeType {
    int nodes;
  };
  static SrcVertex srcVertex() { return ALL; }
  static GatherEdges gatherOverEdges() { return GD; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static PostApplyVertices postApplyOverEdges() { return NO_POST_APPLY_VERTICES; }
  static ExpandEdges expandOverEdges() { return NO_EXPAND_EDGES; }
  struct gather_edge {
    __device__ void operator()(const int, const int, const int nbr, VertexType &vl, EdgeType &, int &out) {
      out = vl.d_val[nbr];
    }
  };
  struct gather_sum {
    __device__ int operator()(int l, int r) { return l + r; }
  };
  struct apply {
    __device__ void operator()(const int v, const int, const int g, VertexType &vl, EdgeType &, char &changed) {
      vl.d_out[v] = g;
      changed = 0;
    }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, int *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return false; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int, const int, const int, VertexType &, EdgeType &,
                               int &frontier, int &) {
      frontier = -1;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &, VertexType &, EdgeType &, int *, int &) {}
  };
};

template <GatherEdges GD>
int run(mg_graph *g, const int32_t *d_val, int32_t *d_out, const mg_options *o) {
  using P = nbr_sum<GD>;
  int st = mg::ensure_workspace(g);
  if (st != MG_OK) return st;
  cudaStream_t s = mg::run_stream(g, o);
  if ((st = mg::prepare_run(g, s)) != MG_OK) return st;
  mg::GasArgs<P> a = mg::base_args<P>(g);
  a.vl.d_val = d_val;
  a.vl.d_out = d_out;
  a.vl.nodes = a.el.nodes = (int)g->nodes;
  // srcVertex() == ALL: every vertex starts in the frontier
  mg::k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(a.queue0, g->nodes);
  mg::LoopResult res;
  st = mg::run_gas<P>(g, a, (uint32_t)g->nodes, o, "user_nbr_sum", &res);
  if (st != MG_OK) return st;
  return mg::cuda_status(cudaStreamSynchronize(s), "user program");
}

}  // namespace

// dir: 1 = in-neighbours, 2 = out-neighbours, 3 = both (the GatherEdges values).
extern "C" int user_nbr_sum(mg_graph *g, const int32_t *d_val, int32_t *d_out, int32_t dir, const mg_options *o) {
  if (!g || !d_val || !d_out || !o) return MG_ERR_ARG;
  switch (dir) {
    case GATHER_IN_EDGES:
      return run<GATHER_IN_EDGES>(g, d_val, d_out, o);
    case GATHER_OUT_EDGES:
      return run<GATHER_OUT_EDGES>(g, d_val, d_out, o);
    case GATHER_ALL_EDGES:
      return run<GATHER_ALL_EDGES>(g, d_val, d_out, o);
    default:
      return MG_ERR_ARG;
  }
}
