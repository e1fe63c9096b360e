// A driver written the way the reference's Algorithms/*/ drivers are
// (FromHostProblem -> EnactIterativeSearch -> ExtractResults), built against
// include/mapgraph_b200.hpp. Prints one line per program: name and results.
// Input: smallRegressionGraphs/small.mtx as a CSR (7 vertices, 11 edges).
#include <cstdio>
#include <vector>

#include "mapgraph_b200.hpp"

static const int kRow[] = {0, 3, 4, 7, 9, 10, 11, 11};
static const int kCol[] = {1, 2, 3, 4, 1, 4, 5, 5, 6, 6, 6};
static const int kVal[] = {1, 4, 1, 1, 1, 1, 1, 1, 1, 1, 1};

template <class P>
static int run(const char *name, const int *vals, int directed, bool print_int) {
  mapgraph::CsrProblem<P> problem;
  int st = problem.FromHostProblem(false, 7, 11, kCol, kRow, vals, nullptr, nullptr, 1, directed);
  if (st != MG_OK) {
    std::printf("%s FromHostProblem failed: %s\n", name, mapgraph::LastError().c_str());
    return st;
  }
  mapgraph::EnactorVertexCentric<P> enactor;
  int src = 0;
  st = enactor.EnactIterativeSearch(problem, kRow, directed, 1, &src, 1 << 30, 0);
  if (st != MG_OK) {
    std::printf("%s EnactIterativeSearch failed: %s\n", name, mapgraph::LastError().c_str());
    return st;
  }
  std::vector<typename P::DataType> out(7);
  problem.ExtractResults(out.data());
  std::printf("%s", name);
  for (auto x : out) {
    if (print_int)
      std::printf(" %d", (int)x);
    else
      std::printf(" %.6f", (double)x);
  }
  std::printf("\n");
  return MG_OK;
}

// BFS with predecessors (MARK_PREDECESSORS), printed as "bfs_pred" + preds.
static int run_pred() {
  mapgraph::CsrProblem<mapgraph::bfs, true> problem;
  int st = problem.FromHostProblem(false, 7, 11, kCol, kRow, nullptr, nullptr, nullptr, 1, 1);
  mapgraph::EnactorVertexCentric<mapgraph::bfs> enactor;
  int src = 0;
  if (st == MG_OK) st = enactor.EnactIterativeSearch(problem, kRow, 1, 1, &src, 1 << 30, 0);
  std::vector<int> preds(7);
  if (st == MG_OK) st = problem.ExtractPreds(preds.data());
  if (st != MG_OK) {
    std::printf("bfs_pred failed: %s\n", mapgraph::LastError().c_str());
    return st;
  }
  std::printf("bfs_pred");
  for (int x : preds) std::printf(" %d", x);
  std::printf("\n");
  return MG_OK;
}

int main() {
  int st = run<mapgraph::bfs>("bfs", nullptr, 1, true);
  st |= run_pred();
  st |= run<mapgraph::sssp>("sssp", kVal, 1, true);
  st |= run<mapgraph::cc>("cc", nullptr, 1, true);
  st |= run<mapgraph::pagerank>("pagerank", nullptr, 1, false);
  return st == MG_OK ? 0 : 1;
}
