// mapgraph_b200_gas.cuh -- runs GAS Programs written in the reference's form.
//
// A Program written for the reference engine is a struct with the typedefs
// (DataType, MiscType, GatherType, VertexId, SizeT), INIT_VALUE,
// allow_duplicates, the policy selectors (srcVertex, gatherOverEdges,
// applyOverEdges, postApplyOverEdges, expandOverEdges), a host
// Initialize(directed, nodes, edges, num_srcs, srcs, d_row_offsets,
// d_column_indices, d_column_offsets, d_row_indices, d_edge_values,
// vertex_list, edge_list, d_frontier_keys[3], d_frontier_values[3]), the device
// functors gather_edge / gather_sum / apply / post_apply / expand_vertex /
// expand_edge / contract, and a host extractResult(vertex_list, h_output)
// (Algorithms/SSSP/sssp.h:34-393 is the reference's SSSP written that way).
// Such a Program runs unchanged through the reference's driver calls:
//
//   #include <mapgraph_b200_gas.cuh>
//   mapgraph::CsrProblem<MyProgram> problem;
//   problem.FromHostProblem(false, nodes, edges, h_col, h_ro, h_vals, 0, 0, 1, directed);
//   mapgraph::EnactorVertexCentric<MyProgram> enactor;
//   enactor.EnactIterativeSearch(problem, h_ro, directed, num_srcs, srcs, iter_num, threshold);
//   problem.ExtractResults(h_out);   // filled through MyProgram::extractResult
//
// Compile the translation unit with nvcc for sm_100a with this directory on the
// include path, and link libmapgraph_b200.so. What one enact does, in the
// reference engine's order (GASengine/enactor_vertex_centric.cuh:3975-4095 and
// the level loop at :3386-3630):
//   - the contract/gather scratch is filled with INIT_VALUE and the change flags
//     are cleared;
//   - Program::Initialize is called once per enact with the graph's device CSR
//     (d_row_offsets, d_column_indices), its transpose (d_column_offsets,
//     d_row_indices; the CSR itself on a symmetric graph), the int32 edge values
//     and two frontier key queues of V entries (keys[0] is the initial frontier;
//     keys[2] and the three value arrays are scratch of V entries); the state it
//     builds in vertex_list / edge_list persists for the next enact on the same
//     problem, as the reference's allocate-if-NULL Initialize expects;
//   - the initial frontier holds every vertex when srcVertex() is ALL, else the
//     num_srcs entries Initialize wrote;
//   - the levels run gather -> apply -> post_apply -> expand/contract on the
//     device until the frontier is empty or iter_num levels have run;
//   - extractResult copies the result to the problem's host buffer.
// Initialize and extractResult may use synchronous CUDA calls on the default
// stream: the engine synchronises the device around them. Errors come back as
// the library's MG_* status codes (nothing throws or exits).
#ifndef MAPGRAPH_B200_GAS_CUH
#define MAPGRAPH_B200_GAS_CUH

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <new>

#include "mapgraph_b200.hpp"
// the engine's templates (frontier scan, expand/contract, gather, apply, the
// device-driven level loop), instantiated here for the caller's Program
#include "../gpugraph_b200/csrc/gas/run_gas.cuh"

namespace mapgraph {
namespace detail {

template <class T>
__global__ void k_gas_fill(T *p, T v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// Converts to whatever edge-value pointer type the Program's Initialize declares
// (int* in the reference's BFS/SSSP/CC, DataType* in its PageRank).
struct EdgeValues {
  void *p;
  template <class T>
  operator T *() const {
    return static_cast<T *>(p);
  }
};

// What a problem keeps between enacts of a Program P: its vertex/edge lists and
// the engine-side scratch sized for P's GatherType and MiscType.
template <class P>
struct ProgramState {
  typename P::VertexType vl;
  typename P::EdgeType el;
  typename P::GatherType *gather_tmp = nullptr;  // contract scratch / apply input, V
  typename P::GatherType *gather_res = nullptr;  // gather output, V
  typename P::MiscType *values[3] = {nullptr, nullptr, nullptr};  // frontier values, V each
  int *keys2 = nullptr;                                           // third frontier key queue, V
  void *block = nullptr;

  // One device block for the scratch arrays (256-byte aligned pieces).
  cudaError_t allocate(int64_t V) {
    const size_t n = (size_t)(V > 0 ? V : 1);
    auto round = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t g = round(n * sizeof(typename P::GatherType)), m = round(n * sizeof(typename P::MiscType));
    const size_t k = round(n * sizeof(int));
    cudaError_t e = cudaMalloc(&block, 2 * g + 3 * m + k);
    if (e != cudaSuccess) return e;
    char *b = static_cast<char *>(block);
    gather_tmp = reinterpret_cast<typename P::GatherType *>(b);
    gather_res = reinterpret_cast<typename P::GatherType *>(b + g);
    for (int i = 0; i < 3; ++i) values[i] = reinterpret_cast<typename P::MiscType *>(b + 2 * g + i * m);
    keys2 = reinterpret_cast<int *>(b + 2 * g + 3 * m);
    return cudaSuccess;
  }
  ~ProgramState() {
    if (block) cudaFree(block);
  }
};

// The state lives in zeroed memory, so the padding bytes of the Program's
// vertex/edge lists are zero: the engine keys its cached CUDA graphs on the
// bytes of the kernel arguments, which include those lists.
template <class P>
std::shared_ptr<void> make_program_state() {
  void *mem = std::calloc(1, sizeof(ProgramState<P>));
  if (!mem) return nullptr;
  ProgramState<P> *st = new (mem) ProgramState<P>();
  return std::shared_ptr<void>(st, [](void *q) {
    static_cast<ProgramState<P> *>(q)->~ProgramState<P>();
    std::free(q);
  });
}

template <class P, bool M>
struct ProgramRunner {
  static int run(CsrProblem<P, M> &problem, int num_srcs, const int *srcs) {
    mg_graph *g = problem.graph();
    if (!g) return MG_ERR_ARG;
    if (P::srcVertex() != ALL && (num_srcs < 1 || !srcs)) return MG_ERR_ARG;
    const int64_t V = g->nodes;
    for (int i = 0; P::srcVertex() != ALL && i < num_srcs; ++i)
      if (srcs[i] < 0 || srcs[i] >= V) return MG_ERR_ARG;
    int st = mg::ensure_workspace(g);
    if (st != MG_OK) return st;
    mg_options &o = problem.options();
    cudaStream_t s = mg::run_stream(g, &o);
    if ((st = mg::prepare_run(g, s)) != MG_OK) return st;
    std::shared_ptr<void> &holder = problem.program_state();
    if (!holder) {
      holder = make_program_state<P>();
      if (!holder) return MG_ERR_OOM;
      cudaError_t e = static_cast<ProgramState<P> *>(holder.get())->allocate(V);
      if (e != cudaSuccess) {
        holder.reset();
        return mg::cuda_status(e, "program scratch");
      }
    }
    ProgramState<P> &ps = *static_cast<ProgramState<P> *>(holder.get());
    mg::GasArgs<P> a = mg::base_args<P>(g);
    a.gather_tmp = ps.gather_tmp;
    a.gather_res = ps.gather_res;
    const int grid = g->num_sms * 4;
    k_gas_fill<typename P::GatherType><<<grid, 256, 0, s>>>(ps.gather_tmp, (typename P::GatherType)P::INIT_VALUE, V);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return mg::cuda_status(e, "program init");
    int *keys[3] = {a.queue0, a.queue1, ps.keys2};
    P::Initialize(g->directed ? 1 : 0, (int)V, (int)g->edges, num_srcs, const_cast<int *>(srcs), g->csr.row_offsets,
                  g->csr.col, g->csr.csc_offsets, g->csr.csc_rows, EdgeValues{g->csr.wgt}, ps.vl, ps.el, keys,
                  ps.values);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return mg::cuda_status(e, "Program::Initialize");
    a.vl = ps.vl;
    a.el = ps.el;
    const uint32_t n0 = P::srcVertex() == ALL ? (uint32_t)V : (uint32_t)num_srcs;
    mg::LoopResult res;
    if ((st = mg::run_gas<P>(g, a, n0, &o, "program", &res)) != MG_OK) return st;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return mg::cuda_status(e, "enact");
    problem.result().resize((size_t)V);
    P::extractResult(ps.vl, problem.result().data());
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return mg::cuda_status(e, "Program::extractResult");
    mg_stats &sts = problem.stats();
    std::memset(&sts, 0, sizeof(sts));
    sts.iterations = (int32_t)res.ctl.level;
    sts.push_iterations = (int32_t)res.ctl.push_levels;
    sts.converged = res.ctl.frontier_size == 0 ? 1 : 0;
    sts.device_ms = res.ms;
    return MG_OK;
  }
};

}  // namespace detail
}  // namespace mapgraph

#endif  // MAPGRAPH_B200_GAS_CUH
