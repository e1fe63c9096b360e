// Device-resident graph (the B200 counterpart of CsrProblem::GraphSlice,
// GASengine/csr_problem.cuh:150-354) and its working set.
//
// HBM layout, all int32 unless noted, every array 256-byte aligned:
//   row_offsets[V+1+pad]  CSR offsets (padded with E to a multiple of 4 entries + 4,
//                         so 16-byte reads of any aligned 4-entry piece stay in bounds)
//   col[E+pad]            CSR column indices
//   wgt[E]                int32 edge values (SSSP weights), optional
//   csc_offsets/csc_rows  transposed graph (in-edges); aliases the CSR when the
//                         graph is symmetric
//   csc_eid[E]            CSR edge id of every CSC entry (pull access to edge values)
//   pull_rows[E]          the in-lists again, hubs first (bottom-up BFS only)
//   inv_outdeg[V]         float 1/outdeg (PageRank), built on first use with the
//                         PageRank plan (renumbered in-lists on skewed graphs)
// The working set (queues, scan buffers, bitmaps, look-back status words) is
// allocated once per graph and reused by every run on it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace mg {

// Levels of a batched BFS whose frontier masks are kept (the level stack); the
// [V][64] result buffer holds them ([16][V] u64 = 128 bytes per vertex) beside
// the uint16 depth rows (another 128 bytes per vertex).
constexpr uint32_t kMsStackLevels = 16;
// In-lists longer than this are pulled by a warp of their own in a batched BFS
// pull level (a 32-vertex group holding one would carry most of a warp's work).
constexpr int32_t kMsHeavyList = 512;

struct DevCsr {
  int32_t *row_offsets = nullptr;
  int32_t *col = nullptr;
  int32_t *wgt = nullptr;
  int32_t *csc_offsets = nullptr;
  int32_t *csc_rows = nullptr;
  int32_t *csc_eid = nullptr;
  // In-lists reordered by descending out-degree of the neighbour (ties by id),
  // read only by the bottom-up kernels, whose early exit then comes sooner;
  // shares csc_offsets.
  int32_t *pull_rows = nullptr;
  int32_t V = 0;
  int32_t E = 0;
};

// Working set shared by the level-loop kernels (sizes in elements).
struct Workspace {
  int32_t *queue[2] = {nullptr, nullptr};  // frontier ping-pong, capacity V
  uint32_t *scan = nullptr;                // degree prefix of the frontier, V+1
  int32_t *part = nullptr;                 // expand tile -> first frontier index
  unsigned long long *status = nullptr;    // look-back status words
  uint32_t *bm[2] = {nullptr, nullptr};    // frontier bitmaps (level parity), V/32+1 words
  uint32_t *visited = nullptr;             // visited bitmap, V/32+1 words
  uint8_t *changed = nullptr;              // apply() change flags, V
  int32_t *gather_tmp = nullptr;           // contract/gather scratch (4-byte GatherType), V
  int32_t *vbuf[2] = {nullptr, nullptr};   // program vertex arrays (labels, dists, dists_out)
  Ctl *ctl = nullptr;
  size_t part_cap = 0;
  size_t status_cap = 0;
  size_t words = 0;
  size_t bytes = 0;
};

}  // namespace mg

namespace mg {
// An instantiated level loop (CUDA graph with a WHILE node), cached per graph
// and per loop body so repeated runs only pay cudaGraphLaunch.
struct LoopCache {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels_per_level = 0;
};
}  // namespace mg

struct mg_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  mg::Ctl *host_ctl = nullptr;  // pinned copy of the control block
  std::map<std::string, mg::LoopCache> loops;
  int num_sms = 148;
  int directed = 0;
  int64_t nodes = 0;
  int64_t edges = 0;
  mg::DevCsr csr;
  std::vector<int64_t> graph_offsets;  // batch of graphs: first vertex of each graph
  mg::Workspace ws;
  float *inv_outdeg = nullptr;          // PageRank 1/outdeg (0 for dangling vertices)
  uint8_t *dangling_flags = nullptr;
  int32_t *ref_outdeg = nullptr;        // reference PageRank out-degree (PageRank.h:141-161)
  // Batched (mask-frontier) working set, allocated on first use.
  unsigned long long *mask[3] = {nullptr, nullptr, nullptr};
  // [V][64] int32 per-source results. A batched BFS with 16-bit depths splits
  // it: the first half holds the level stack ([kMsStackLevels][V] u64 frontier
  // masks), the second the [V][64] uint16 depth rows of deeper levels.
  int32_t *multi_out = nullptr;
  uint32_t *multi_stk_bm = nullptr;     // [kMsStackLevels][V/32] valid entries of push-made stack levels
  int32_t *ms_heavy = nullptr;          // vertices with more than kMsHeavyList in-edges, longest first
  int32_t ms_nheavy = -1;               // their number (-1: not built yet)
  int32_t *multi_stage = nullptr;       // [64][V] transposed results on their way to host memory
  size_t multi_bytes = 0;
  // PageRank plan (built on first mg_pagerank): heavy in-lists split into
  // fixed-size chunks whose partial sums are combined in chunk order.
  int32_t *pr_chunk_v = nullptr, *pr_chunk_b = nullptr, *pr_chunk_e = nullptr;
  int32_t *pr_heavy_v = nullptr, *pr_heavy_first = nullptr;
  int32_t pr_nchunks = 0, pr_nheavy = 0;
  int64_t pr_ndangling = 0;
  float *pr_rank[2] = {nullptr, nullptr}, *pr_contrib[2] = {nullptr, nullptr}, *pr_partial = nullptr;
  // The in-lists the PageRank kernels read: on a skewed degree distribution a
  // copy with vertices renumbered by descending out-degree (pr_new_of[v] = the
  // new number of v), otherwise the graph's own CSC (pr_new_of null).
  int32_t *pr_coff = nullptr, *pr_crow = nullptr, *pr_new_of = nullptr;
  // Personalised PageRank: chunk plans over the CSC (forward) and the CSR
  // (adjoint): chunk c covers edges [cb, ce) of vertex cv; cslot >= 0 marks a
  // partial of a split in-list, combined in chunk order by the fix-up pass.
  struct PprPlan {
    int32_t *cv = nullptr, *cb = nullptr, *ce = nullptr, *cslot = nullptr;
    int32_t *mv = nullptr, *mfirst = nullptr;  // split vertices and their first slot
    int32_t nchunks = 0, nmulti = 0, nslots = 0;
  } ppr_plan[2];
  float *ppr_x[2] = {nullptr, nullptr}, *ppr_partial = nullptr;
  float *ppr_rhs = nullptr, *ppr_w = nullptr;  // stable copies of the solve's inputs
  int32_t ppr_cap_nvec = 0;
  size_t device_bytes = 0;
  uint64_t epochs_used = 0;  // look-back epochs consumed since the status words were cleared
  std::vector<void *> allocations;
};

namespace mg {

// Library-internal helpers implemented in graph.cu.
int device_alloc(mg_graph *g, void **p, size_t bytes);
int ensure_workspace(mg_graph *g);
int ensure_multi(mg_graph *g);
cudaStream_t run_stream(mg_graph *g, const mg_options *o);
int cuda_status(cudaError_t e, const char *what);
int launch_check(const char *what);

}  // namespace mg
