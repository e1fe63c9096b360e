// mapgraph_b200.hpp -- C++ host API with the reference's names over the C ABI.
//
// The reference's drivers (Algorithms/{BFS,SSSP,CC,PageRank}/*.cu) use
//   CsrProblem<Program,...>::FromHostProblem(...)      GASengine/csr_problem.cuh:512-524
//   EnactorVertexCentric<...>::EnactIterativeSearch(...) GASengine/enactor_vertex_centric.cuh:3269
//   CsrProblem::ExtractResults(h_values)               GASengine/csr_problem.cuh:433-458
// This header keeps those names, argument meanings and the cudaError_t-style
// "return a status, do not throw" behaviour, so a driver written against the
// reference ports by changing includes. The four bundled Programs are tags
// (mapgraph::bfs, sssp, cc, pagerank) served by the library's specialised
// kernels. Any other Program -- a struct written in the reference's form, with
// Initialize, the device functors and extractResult -- runs through the same
// CsrProblem / EnactorVertexCentric calls once its translation unit (compiled
// by nvcc) includes mapgraph_b200_gas.cuh, which instantiates the generic GAS
// engine for it.
#ifndef MAPGRAPH_B200_HPP
#define MAPGRAPH_B200_HPP

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "mapgraph_b200.h"

namespace mapgraph {

// Program tags with the reference's result types and unreached values.
struct bfs {
  typedef int DataType;
  static const int INIT_VALUE = -1;
};
struct sssp {
  typedef int DataType;
  static const int INIT_VALUE = 100000000;
};
struct cc {
  typedef int DataType;
};
struct pagerank {  // the reference PageRank program (unnormalised, |delta| threshold)
  typedef float DataType;
};

// The device-resident graph (reference: CsrProblem after FromHostProblem).
// MARK_PREDECESSORS (the reference's template flag, GASengine/problem_type.cuh)
// makes single-source BFS runs also produce predecessors for ExtractPreds.
template <class Program, bool MARK_PREDECESSORS = false>
class CsrProblem {
 public:
  CsrProblem() {
    mg_options_init(&opts_);
    // the reference PageRank program's change threshold (Algorithms/PageRank/register.h)
    if (std::is_same<Program, pagerank>::value) opts_.tolerance = 0.01;
  }
  ~CsrProblem() { mg_graph_destroy(g_); }
  CsrProblem(const CsrProblem &) = delete;
  CsrProblem &operator=(const CsrProblem &) = delete;

  // Same argument order as the reference; h_row_indices / h_column_offsets (the
  // host transpose) and num_gpus are accepted and ignored: the transpose is
  // built by the library and the path is single-GPU.
  int FromHostProblem(bool /*stream_from_host*/, int nodes, int edges, const int *h_column_indices,
                      const int *h_row_offsets, const int *h_edge_values, const int * /*h_row_indices*/,
                      const int * /*h_column_offsets*/, int /*num_gpus*/, int directed) {
    mg_graph_destroy(g_);
    g_ = nullptr;
    program_state_.reset();
    nodes_ = nodes;
    return mg_graph_create(h_row_offsets, h_column_indices, h_edge_values,
                           h_edge_values ? MG_VAL_I32 : MG_VAL_NONE, nodes, edges, directed, &opts_, &g_);
  }

  // Copies the last run's per-vertex result (reference: ExtractResults).
  int ExtractResults(typename Program::DataType *h_values) const {
    if (result_.empty()) return MG_ERR_ARG;
    std::copy(result_.begin(), result_.end(), h_values);
    return MG_OK;
  }

  // Copies the last run's predecessors (BFS with MARK_PREDECESSORS; the
  // reference's CsrProblem::ExtractPreds, as called at Algorithms/BFS/bfs.cu:1063).
  int ExtractPreds(int *h_preds) const {
    if (preds_.empty()) return MG_ERR_ARG;
    std::copy(preds_.begin(), preds_.end(), h_preds);
    return MG_OK;
  }

  mg_graph *graph() const { return g_; }
  mg_options &options() { return opts_; }
  int nodes() const { return nodes_; }
  std::vector<typename Program::DataType> &result() { return result_; }
  std::vector<int> &preds() { return preds_; }
  const mg_stats &stats() const { return stats_; }
  mg_stats &stats() { return stats_; }
  // State a Program in the reference's form keeps between runs (its VertexType
  // and EdgeType, whose arrays its Initialize allocates once); owned here, set
  // by the engine in mapgraph_b200_gas.cuh.
  std::shared_ptr<void> &program_state() { return program_state_; }

 private:
  // program_state_ is declared first so that it is released last, after the
  // graph (its release may free device memory the graph's last run used)
  std::shared_ptr<void> program_state_;
  mg_graph *g_ = nullptr;
  mg_options opts_;
  int nodes_ = 0;
  std::vector<typename Program::DataType> result_;
  std::vector<int> preds_;
  mg_stats stats_{};
};

namespace detail {
// Runs a Program written in the reference's form through the generic GAS
// engine. Defined in mapgraph_b200_gas.cuh: a translation unit that enacts such
// a Program includes that header (the bundled tags below do not need it).
template <class Program, bool M>
struct ProgramRunner;
template <class Program, bool M>
int run(CsrProblem<Program, M> &p, int num_srcs, const int *srcs) {
  return ProgramRunner<Program, M>::run(p, num_srcs, srcs);
}

template <bool M>
int run(CsrProblem<bfs, M> &p, int num_srcs, const int *srcs) {
  p.result().resize((size_t)p.nodes());
  if (M && num_srcs == 1) {
    p.preds().resize((size_t)p.nodes());
    return mg_bfs_pred(p.graph(), srcs[0], p.result().data(), p.preds().data(), &p.stats(), &p.options());
  }
  return num_srcs == 1 ? mg_bfs(p.graph(), srcs[0], p.result().data(), &p.stats(), &p.options())
                       : mg_bfs_roots(p.graph(), srcs, num_srcs, p.result().data(), &p.stats(), &p.options());
}
template <bool M>
int run(CsrProblem<sssp, M> &p, int num_srcs, const int *srcs) {
  if (num_srcs != 1) return MG_ERR_UNSUPPORTED;  // the reference validates single-source runs only
  p.result().resize((size_t)p.nodes());
  return mg_sssp(p.graph(), srcs[0], p.result().data(), &p.stats(), &p.options());
}
template <bool M>
int run(CsrProblem<cc, M> &p, int, const int *) {
  p.result().resize((size_t)p.nodes());
  return mg_cc(p.graph(), p.result().data(), &p.stats(), &p.options());
}
template <bool M>
int run(CsrProblem<pagerank, M> &p, int, const int *) {
  p.result().resize((size_t)p.nodes());
  return mg_pagerank_gas(p.graph(), p.result().data(), &p.stats(), &p.options());
}
}  // namespace detail

// Reference: EnactorVertexCentric<CsrProblem, Program, INSTRUMENT>.
template <class Program>
class EnactorVertexCentric {
 public:
  // Same argument meaning as the reference's 7-argument call used by the
  // drivers (Algorithms/SSSP/sssp.cu:397-398): iter_num caps the GAS
  // iterations; threshold is the reference's expand switch (kept for API
  // compatibility: the load-balanced expand needs no threshold).
  template <bool M>
  int EnactIterativeSearch(CsrProblem<Program, M> &problem, const int * /*h_row_offsets*/, int /*directed*/,
                           int num_srcs, const int *srcs, int iter_num, int threshold) {
    if (iter_num > 0) problem.options().iter_num = iter_num;
    problem.options().threshold = threshold;
    return detail::run(problem, num_srcs, srcs);
  }
};

inline std::string LastError() { return mg_last_error(); }

}  // namespace mapgraph

#endif  // MAPGRAPH_B200_HPP
