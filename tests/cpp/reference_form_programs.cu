// Two GAS Programs written the way the reference writes its Programs (a host
// Initialize that allocates and fills the vertex/edge lists and the initial
// frontier, device functors, a host extractResult), compiled against include/
// only and run through the reference's driver calls (CsrProblem,
// EnactorVertexCentric, ExtractResults):
//   - rf_sssp: Bellman-Ford relaxation with an atomicMin contract, the shape of
//     the reference's SSSP Program (Algorithms/SSSP/sssp.h:34-393);
//   - rf_bfs_all: BFS levels over out- and in-edges (EXPAND_ALL_EDGES), i.e. BFS
//     of the undirected view of a directed graph.
#include <cstdio>
#include <vector>

#include <mapgraph_b200_gas.cuh>

namespace {

struct rf_sssp {
  typedef int DataType;
  typedef DataType MiscType;
  typedef DataType GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = 100000000;
  static const bool allow_duplicates = true;

  struct VertexType {
    int nodes, edges;
    DataType *d_dists_out, *d_dists;
    VertexType() : nodes(0), edges(0), d_dists_out(NULL), d_dists(NULL) {}
  };
  struct EdgeType {
    int nodes, edges;
    DataType *d_weights;
    EdgeType() : nodes(0), edges(0), d_weights(NULL) {}
  };

  static void Initialize(const int, const int nodes, const int edges, int num_srcs, int *srcs, int *, int *, int *,
                         int *, int *d_edge_values, VertexType &vl, EdgeType &el, int *d_frontier_keys[3],
                         MiscType *d_frontier_values[3]) {
    vl.nodes = el.nodes = nodes;
    vl.edges = el.edges = edges;
    if (!vl.d_dists) cudaMalloc((void **)&vl.d_dists, sizeof(DataType) * nodes);
    if (!vl.d_dists_out) cudaMalloc((void **)&vl.d_dists_out, sizeof(DataType) * nodes);
    if (!el.d_weights) cudaMalloc((void **)&el.d_weights, sizeof(DataType) * (edges > 0 ? edges : 1));
    if (edges > 0) cudaMemcpy(el.d_weights, d_edge_values, sizeof(DataType) * edges, cudaMemcpyDeviceToDevice);
    std::vector<DataType> init(nodes, INIT_VALUE);
    for (int i = 0; i < num_srcs; ++i) init[srcs[i]] = 0;
    cudaMemcpy(vl.d_dists, init.data(), sizeof(DataType) * nodes, cudaMemcpyHostToDevice);
    cudaMemcpy(vl.d_dists_out, init.data(), sizeof(DataType) * nodes, cudaMemcpyHostToDevice);
    cudaMemcpy(d_frontier_keys[0], srcs, sizeof(int) * num_srcs, cudaMemcpyHostToDevice);
    cudaMemcpy(d_frontier_keys[1], srcs, sizeof(int) * num_srcs, cudaMemcpyHostToDevice);
    std::vector<MiscType> zero(num_srcs, 0);
    cudaMemcpy(d_frontier_values[0], zero.data(), sizeof(MiscType) * num_srcs, cudaMemcpyHostToDevice);
  }

  static SrcVertex srcVertex() { return SINGLE; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static PostApplyVertices postApplyOverEdges() { return POST_APPLY_FRONTIER; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }

  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, GatherType &) {}
  };
  struct gather_sum {
    __device__ GatherType operator()(const GatherType &a, const GatherType &b) { return a + b; }
  };
  // the best candidate distance contract() left in gather_tmp, kept if smaller
  struct apply {
    __device__ void operator()(const int v, const int iteration, GatherType best, VertexType &vl, EdgeType &,
                               char &changed) {
      const int cur = vl.d_dists[v];
      const int nv = best < cur ? best : cur;
      changed = (iteration == 0 || nv != cur) ? 1 : 0;
      vl.d_dists_out[v] = nv;
    }
  };
  struct post_apply {
    __device__ void operator()(const int v, VertexType &vl, EdgeType &, GatherType *gather_tmp) {
      vl.d_dists[v] = vl.d_dists_out[v];
      gather_tmp[v] = INIT_VALUE;
    }
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char changed, VertexType &, EdgeType &) { return changed == 1; }
  };
  // enqueue the neighbour when the edge improves it; the candidate rides along
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int v, const int nbr, const int eid, VertexType &vl,
                               EdgeType &el, int &frontier, int &misc) {
      const int cand = vl.d_dists[v] + el.d_weights[eid];
      frontier = cand < vl.d_dists[nbr] ? nbr : -1;
      misc = cand;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &v, VertexType &, EdgeType &, GatherType *gather_tmp, int &misc) {
      atomicMin(&gather_tmp[v], misc);
    }
  };

  static void extractResult(VertexType &vl, DataType *h_output) {
    cudaMemcpy(h_output, vl.d_dists, sizeof(DataType) * vl.nodes, cudaMemcpyDeviceToHost);
  }
};

struct rf_bfs_all {
  typedef int DataType;
  typedef DataType MiscType;
  typedef DataType GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = -1;
  static const bool allow_duplicates = true;

  struct VertexType {
    int nodes, edges;
    int *d_labels;
    VertexType() : nodes(0), edges(0), d_labels(NULL) {}
  };
  struct EdgeType {
    int nodes, edges;
    EdgeType() : nodes(0), edges(0) {}
  };

  static void Initialize(const int, const int nodes, const int edges, int num_srcs, int *srcs, int *, int *, int *,
                         int *, int *, VertexType &vl, EdgeType &el, int *d_frontier_keys[3], MiscType *[3]) {
    vl.nodes = el.nodes = nodes;
    vl.edges = el.edges = edges;
    if (!vl.d_labels) cudaMalloc((void **)&vl.d_labels, sizeof(int) * nodes);
    std::vector<int> init(nodes, INIT_VALUE);
    for (int i = 0; i < num_srcs; ++i) init[srcs[i]] = 0;
    cudaMemcpy(vl.d_labels, init.data(), sizeof(int) * nodes, cudaMemcpyHostToDevice);
    cudaMemcpy(d_frontier_keys[0], srcs, sizeof(int) * num_srcs, cudaMemcpyHostToDevice);
  }

  static SrcVertex srcVertex() { return SINGLE; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return NO_APPLY_VERTICES; }
  static PostApplyVertices postApplyOverEdges() { return NO_POST_APPLY_VERTICES; }
  static ExpandEdges expandOverEdges() { return EXPAND_ALL_EDGES; }

  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, GatherType &) {}
  };
  struct gather_sum {
    __device__ GatherType operator()(const GatherType &a, const GatherType &) { return a; }
  };
  struct apply {
    __device__ void operator()(const int, const int, GatherType, VertexType &, EdgeType &, char &changed) {
      changed = 1;
    }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, GatherType *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int, const int nbr, const int, VertexType &vl,
                               EdgeType &, int &frontier, int &) {
      frontier = vl.d_labels[nbr] == INIT_VALUE ? nbr : -1;
    }
  };
  // the first claim of an unlabelled vertex labels it with the next depth
  struct contract {
    __device__ void operator()(const int iteration, int &v, VertexType &vl, EdgeType &, GatherType *, int &) {
      if (atomicCAS(&vl.d_labels[v], INIT_VALUE, iteration + 1) != INIT_VALUE) v = -1;
    }
  };

  static void extractResult(VertexType &vl, DataType *h_output) {
    cudaMemcpy(h_output, vl.d_labels, sizeof(int) * vl.nodes, cudaMemcpyDeviceToHost);
  }
};

// A driver written the reference's way: FromHostProblem, EnactIterativeSearch,
// ExtractResults; `runs` enacts in a row on the same problem.
template <class P>
int drive(int nodes, int edges, const int *h_ro, const int *h_col, const int *h_val, int directed, int src,
          int runs, int *h_out) {
  mapgraph::CsrProblem<P> problem;
  int st = problem.FromHostProblem(false, nodes, edges, h_col, h_ro, h_val, NULL, NULL, 1, directed);
  if (st != MG_OK) return st;
  mapgraph::EnactorVertexCentric<P> enactor;
  for (int r = 0; r < runs; ++r) {
    st = enactor.EnactIterativeSearch(problem, h_ro, directed, 1, &src, 1 << 30, 0);
    if (st != MG_OK) return st;
  }
  return problem.ExtractResults(h_out);
}

}  // namespace

extern "C" int rf_run_sssp(int nodes, int edges, const int *h_ro, const int *h_col, const int *h_w, int directed,
                           int src, int runs, int *h_out) {
  return drive<rf_sssp>(nodes, edges, h_ro, h_col, h_w, directed, src, runs, h_out);
}

extern "C" int rf_run_bfs_all(int nodes, int edges, const int *h_ro, const int *h_col, int directed, int src,
                              int runs, int *h_out) {
  return drive<rf_bfs_all>(nodes, edges, h_ro, h_col, NULL, directed, src, runs, h_out);
}
