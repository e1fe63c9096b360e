// The four bundled GAS programs, re-expressed against the engine's Program
// contract. Device functor signatures and policy selectors follow the
// reference programs one to one; VertexType/EdgeType hold device pointers into
// the graph's working set instead of arrays cudaMalloc'ed by Initialize.
#pragma once
#include <stdint.h>

#include "enums.h"

namespace mg {
namespace programs {

// BFS depth labels (Algorithms/BFS/bfs.h:28-298). The reference leaves contract
// empty and culls with the engine's best-effort bitmask; here contract performs
// the visited test-and-set and writes the label, which is the single-GPU
// MapGraph BFS contract (commented out at bfs.h:261-284).
struct bfs {
  typedef int DataType;
  typedef DataType MiscType;
  typedef DataType GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const DataType INIT_VALUE = -1;
  static const bool allow_duplicates = true;
  static const bool track_next_edges = true;  // direction heuristic needs next-frontier edges

  struct VertexType {
    int *d_labels;
    uint32_t *d_visited;
    int nodes;
    int edges;
  };
  struct EdgeType {
    int nodes;
    int edges;
  };
  static SrcVertex srcVertex() { return SINGLE; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return NO_APPLY_VERTICES; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }
  static PostApplyVertices postApplyOverEdges() { return NO_POST_APPLY_VERTICES; }

  struct gather_sum {
    __device__ GatherType operator()(GatherType l, GatherType r) { return l > r ? l : r; }
  };
  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, GatherType &nv) { nv = -1; }
  };
  struct apply {
    __device__ void operator()(const int, const int, GatherType, VertexType &, EdgeType &, char &changed) { changed = 1; }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, GatherType *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int, const int neighbor_id_in, const int, VertexType &,
                               EdgeType &, int &frontier, int &) {
      frontier = neighbor_id_in;
    }
  };
  struct contract {
    __device__ void operator()(const int iteration, int &vertex_id, VertexType &vl, EdgeType &, GatherType *, int &) {
      const uint32_t bit = 1u << (vertex_id & 31);
      uint32_t *w = vl.d_visited + (vertex_id >> 5);
      if (*(volatile uint32_t *)w & bit) {
        vertex_id = -1;
        return;
      }
      if (atomicOr(w, bit) & bit) {
        vertex_id = -1;
        return;
      }
      vl.d_labels[vertex_id] = iteration + 1;
    }
  };
};

// Bellman-Ford frontier relaxation (Algorithms/SSSP/sssp.h:34-393).
struct sssp {
  typedef int DataType;
  typedef DataType MiscType;
  typedef DataType GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = 100000000;
  static const bool allow_duplicates = true;
  // expand_vertex(changed) is false only for frontier vertices whose apply()
  // found no improvement; their relaxations cannot improve anything, so the
  // engine may skip their adjacency (same fixpoint, less work).
  static const bool skip_unchanged_vertices = true;

  struct VertexType {
    int nodes;
    int edges;
    DataType *d_dists_out;
    DataType *d_dists;
  };
  struct EdgeType {
    int nodes;
    int edges;
    DataType *d_weights;
  };
  static SrcVertex srcVertex() { return SINGLE; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static PostApplyVertices postApplyOverEdges() { return POST_APPLY_FRONTIER; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }

  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, GatherType &) {}
  };
  struct gather_sum {
    __device__ GatherType operator()(const GatherType &l, const GatherType &r) { return l + r; }
  };
  struct apply {
    __device__ void operator()(const int vertex_id, const int iteration, GatherType gathervalue, VertexType &vl,
                               EdgeType &, char &changed) {
      const int oldvalue = vl.d_dists[vertex_id];
      const int newvalue = min(oldvalue, gathervalue);
      changed = (iteration == 0) ? 1 : (oldvalue != newvalue);
      vl.d_dists_out[vertex_id] = newvalue;
    }
  };
  struct post_apply {
    __device__ void operator()(const int vertex_id, VertexType &vl, EdgeType &, GatherType *gather_tmp) {
      vl.d_dists[vertex_id] = vl.d_dists_out[vertex_id];
      gather_tmp[vertex_id] = INIT_VALUE;
    }
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char changed, VertexType &, EdgeType &) { return changed == 1; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int, const int vertex_id, const int neighbor_id_in, const int edge_id,
                               VertexType &vl, EdgeType &el, int &frontier, int &misc_value) {
      const int src_dist = vl.d_dists[vertex_id];
      const int dst_dist = vl.d_dists[neighbor_id_in];
      const int edge_value = el.d_weights[edge_id];
      frontier = (dst_dist > src_dist + edge_value) ? neighbor_id_in : -1;
      misc_value = src_dist + edge_value;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &vertex_id, VertexType &, EdgeType &, GatherType *gather_tmp,
                               int &misc_value) {
      atomicMin(&gather_tmp[vertex_id], misc_value);
    }
  };
};

// Min-label connected components (Algorithms/CC/cc.h:32-349).
struct cc {
  typedef int DataType;
  typedef DataType MiscType;
  typedef DataType GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = 100000000;
  static const bool allow_duplicates = true;
  static const bool skip_unchanged_vertices = true;  // iteration 0 marks every vertex changed

  struct VertexType {
    int nodes;
    int edges;
    DataType *d_dists_out;
    DataType *d_dists;
  };
  struct EdgeType {
    int nodes;
    int edges;
  };
  static SrcVertex srcVertex() { return ALL; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static PostApplyVertices postApplyOverEdges() { return POST_APPLY_FRONTIER; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }

  struct gather_edge {
    __device__ void operator()(const int, const int, const int, VertexType &, EdgeType &, GatherType &) {}
  };
  struct gather_sum {
    __device__ GatherType operator()(const GatherType &, const GatherType &) { return 0; }
  };
  struct apply {
    __device__ void operator()(const int vertex_id, const int iteration, GatherType gathervalue, VertexType &vl,
                               EdgeType &, char &changed) {
      const int oldvalue = vl.d_dists[vertex_id];
      const int newvalue = min(oldvalue, gathervalue);
      changed = (iteration == 0) ? 1 : (oldvalue != newvalue);
      vl.d_dists_out[vertex_id] = newvalue;
    }
  };
  struct post_apply {
    __device__ void operator()(const int vertex_id, VertexType &vl, EdgeType &, GatherType *gather_tmp) {
      vl.d_dists[vertex_id] = vl.d_dists_out[vertex_id];
      gather_tmp[vertex_id] = INIT_VALUE;
    }
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char changed, VertexType &, EdgeType &) { return changed == 1; }
  };
  struct expand_edge {
    __device__ void operator()(const bool changed, const int iteration, const int vertex_id, const int neighbor_id_in,
                               const int, VertexType &vl, EdgeType &, int &frontier, int &misc_value) {
      const int src_dist = vl.d_dists[vertex_id];
      const int dst_dist = vl.d_dists[neighbor_id_in];
      frontier = ((changed || iteration == 0) && dst_dist > src_dist) ? neighbor_id_in : -1;
      misc_value = src_dist;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &vertex_id, VertexType &, EdgeType &, GatherType *gather_tmp,
                               int &misc_value) {
      atomicMin(&gather_tmp[vertex_id], misc_value);
    }
  };
};

// The reference PageRank program (Algorithms/PageRank/PageRank.h:33-409):
// unnormalised rank = 0.15 + 0.85 * sum over in-edges of rank[u]/outdeg[u];
// a vertex stays active while |delta| >= tolerance (reference 0.01).
struct pagerank {
  typedef float DataType;
  typedef int MiscType;
  typedef float GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static constexpr DataType INIT_VALUE = 0.0f;
  static const bool allow_duplicates = false;

  struct VertexType {
    int nodes;
    int edges;
    DataType *d_dists;
    int *d_num_out_edge;
    float tolerance;
  };
  struct EdgeType {
    int nodes;
    int edges;
  };
  static SrcVertex srcVertex() { return ALL; }
  static GatherEdges gatherOverEdges() { return GATHER_IN_EDGES; }
  static ApplyVertices applyOverEdges() { return APPLY_FRONTIER; }
  static PostApplyVertices postApplyOverEdges() { return POST_APPLY_FRONTIER; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }

  struct gather_edge {
    __device__ void operator()(const int, const int, const int neighbor_id_in, VertexType &vl, EdgeType &,
                               GatherType &new_value) {
      const DataType nb_dist = vl.d_dists[neighbor_id_in];
      new_value = nb_dist / (DataType)vl.d_num_out_edge[neighbor_id_in];
    }
  };
  struct gather_sum {
    __device__ GatherType operator()(const GatherType &l, const GatherType &r) { return l + r; }
  };
  struct apply {
    __device__ void operator()(const int vertex_id, const int, GatherType gathervalue, VertexType &vl, EdgeType &,
                               char &changed) {
      const DataType oldvalue = vl.d_dists[vertex_id];
      const DataType newvalue = 0.15f + (1.0f - 0.15f) * gathervalue;
      changed = (fabsf(oldvalue - newvalue) < vl.tolerance) ? 0 : 1;
      vl.d_dists[vertex_id] = newvalue;
    }
  };
  struct post_apply {
    __device__ void operator()(const int, VertexType &, EdgeType &, GatherType *) {}
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char changed, VertexType &, EdgeType &) { return changed; }
  };
  struct expand_edge {
    __device__ void operator()(const bool changed, const int, const int, const int neighbor_id_in, const int,
                               VertexType &, EdgeType &, int &frontier, int &) {
      if (changed) frontier = neighbor_id_in;
    }
  };
  struct contract {
    __device__ void operator()(const int, int &, VertexType &, EdgeType &, GatherType *, int &) {}
  };
};

}  // namespace programs
}  // namespace mg
