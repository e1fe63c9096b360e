/*
 * mapgraph_b200.h -- C ABI of the B200-native Gather-Apply-Scatter (GAS) hot path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes and returns an
 * int status (MG_OK or one of MG_ERR_*). No exception and no exit() crosses this
 * boundary; mg_last_error() returns a human-readable message for the calling
 * thread's most recent failure.
 *
 * The reference (MapGraph 0.3.x) exposes this path as compile-time C++ templates:
 * a Program functor struct, CsrProblem<Program,...> and
 * EnactorVertexCentric<CsrProblem,Program>. Each function below names the
 * reference interface it replaces. Paths are relative to the reference project.
 *
 * Graph ids are int32 (VertexId = SizeT = int in the reference), so nodes and
 * edges must both be < 2^31.
 */
#ifndef MAPGRAPH_B200_H
#define MAPGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MG_ABI_VERSION 1

/* Status codes (the reference returns cudaError_t but in practice calls exit();
 * see GASengine/enactor_vertex_centric.cuh:107-129). */
enum {
  MG_OK = 0,
  MG_ERR_ARG = 1,         /* bad argument: null pointer, out-of-range id, bad size */
  MG_ERR_OOM = 2,         /* device or host allocation failed */
  MG_ERR_OVERFLOW = 3,    /* a device queue would overflow (never silently truncated) */
  MG_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out; context stays usable */
  MG_ERR_CUDA = 5,        /* a CUDA runtime call failed */
  MG_ERR_UNSUPPORTED = 6, /* operation not available for this graph (e.g. no weights) */
  MG_ERR_IO = 7           /* file could not be read or parsed */
};

/* Edge value types for mg_graph_create (reference: CsrGraph::edge_values, Value). */
enum { MG_VAL_NONE = 0, MG_VAL_I32 = 1, MG_VAL_F32 = 2 };

/* Traversal direction policy for BFS (push/pull switching). */
enum { MG_DIR_AUTO = 0, MG_DIR_PUSH = 1, MG_DIR_PULL = 2 };

typedef struct mg_graph mg_graph; /* device-resident CsrProblem (opaque) */

/* Run options. Reference knobs keep their names (Algorithms/BFS/register.h:27-44):
 * iter_num, threshold. Queues are sized exactly, so max_queue_sizing has no
 * counterpart. Zero-valued tuning fields mean "use the autotuned value". */
typedef struct mg_options {
  int32_t struct_size;       /* sizeof(mg_options); set by mg_options_init */
  int32_t outputs_on_device; /* 1: result pointers are device pointers */
  void *stream;              /* cudaStream_t to run on; NULL: the graph's stream */
  int32_t iter_num;          /* maximum number of GAS iterations (levels) */
  int32_t direction;         /* MG_DIR_* (BFS only) */
  double alpha;              /* push->pull when frontier edges > unvisited edges / alpha */
  double beta;               /* pull->push when frontier vertices < nodes / beta */
  int32_t use_cuda_graph;    /* 1: capture the level loop in a CUDA graph */
  int32_t threshold;         /* reference "threshold": frontier size above which the
                                grid-cooperative expand is used (0: always) */
  double damping;            /* PageRank damping (0.85) */
  double tolerance;          /* PageRank L1 stop tolerance */
  int64_t spin_limit;        /* iteration cap of every device-side spin wait */
  int32_t tile_items;        /* items per expand tile (0: autotuned) */
  int32_t ctas_per_sm;       /* persistent CTAs per SM (0: autotuned) */
  int32_t compute_stats;     /* 1: fill mg_stats.edges_traversed (one extra pass) */
  int32_t pad0;
  double alpha_multi;        /* batched BFS: push->pull when the next level's frontier
                                edges exceed edges / alpha_multi */
  int32_t ordered_frontier;  /* 1: next frontiers keep a deterministic order (decoupled
                                look-back); 0: one atomic reservation per tile */
  int32_t generic_engine;    /* 1: mg_sssp / mg_cc run the bundled GAS Program through the
                                generic engine; 0: the specialised kernels (same results) */
  int32_t reserved[2];
} mg_options;

/* Per-run statistics (reference: Statistics::stats_per_iter, GASengine/statistics.h:31-81). */
typedef struct mg_stats {
  int32_t iterations;        /* GAS iterations (BFS levels) executed */
  int32_t push_iterations;   /* iterations run top-down (push) */
  int32_t pull_iterations;   /* iterations run bottom-up (pull) */
  int32_t converged;         /* 1 if the stop criterion was met within iter_num */
  int64_t vertices_reached;  /* vertices with a finite result */
  int64_t edges_traversed;   /* sum of out-degrees of reached vertices (TEPS numerator) */
  double device_ms;          /* CUDA-event time of the device work of this call */
  double residual;           /* PageRank: last L1 residual (FP64 reduction) */
  int64_t reserved[4];
} mg_stats;

/* Host-side CSR produced by the builders below. Memory is owned by the library
 * and released with mg_host_csr_free. */
typedef struct mg_host_csr {
  int64_t nodes;
  int64_t edges;
  int32_t *row_offsets;    /* [nodes+1] */
  int32_t *column_indices; /* [edges] */
  int32_t *edge_values;    /* [edges] or NULL */
  int32_t directed;        /* 0: symmetric (every edge stored both ways) */
} mg_host_csr;

/* ---------------------------------------------------------------- library -- */
/* Fills *opts with the defaults (what a NULL options pointer means). */
void mg_options_init(mg_options *opts);
/* Message of the most recent failure on this thread; the graph and algorithm
 * calls clear it when they start. */
const char *mg_last_error(void);
/* Name of a status code (MG_OK, MG_ERR_ARG, ...). */
const char *mg_status_string(int status);
/* MG_ABI_VERSION of the built library; compare with the header's. */
int mg_abi_version(void);
/* Number of device-side kernel launches issued by this thread since the last reset. */
int64_t mg_kernel_launches(int reset);
/* Per-kernel profiling for this thread (no reference counterpart; the reference
 * has per-CTA clock() statistics, b40c/util/kernel_runtime_stats.cuh:55-86).
 * While enabled, level loops run host-driven and every kernel launch is
 * bracketed by CUDA events; enabling resets the accumulators. */
int mg_profile_enable(int enable);
/* Accumulated time, launch count and algorithmic bytes of kernel kind `kind`
 * (0 <= kind < 13); *name receives a static string. */
int mg_profile_read(int32_t kind, const char **name, double *total_ms, int64_t *launches, uint64_t *bytes);
/* Failure-detection self-test (no reference counterpart; the reference exits
 * on errors, GASengine/enactor_vertex_centric.cuh:107-129): runs the library's
 * bounded device-side wait against a status word nothing publishes. Returns
 * MG_ERR_TIMEOUT when the wait ended at spin_limit as designed. */
int mg_selftest_wait_timeout(int64_t spin_limit, double *elapsed_ms);

/* ----------------------------------------------------------------- graphs -- */
/* Copy a host CSR to the device and build what the hot path needs (out-degrees,
 * the transposed CSC when directed, the working set). Replaces
 * CsrProblem::FromHostProblem (GASengine/csr_problem.cuh:512-839) and the thrust
 * CSC build it calls (util.cuh:55-126). value_type selects how edge_values
 * (may be NULL) is read. */
int mg_graph_create(const int32_t *row_offsets, const int32_t *column_indices,
                    const void *edge_values, int32_t value_type, int64_t nodes,
                    int64_t edges, int32_t directed, const mg_options *opts,
                    mg_graph **out);
/* Same, with a batch of independent graphs concatenated into one CSR:
 * graph_offsets[ngraphs+1] gives each graph's first vertex (vertex ids in
 * column_indices are global). Used by mg_bfs_batch. */
int mg_graph_create_batch(const int32_t *row_offsets, const int32_t *column_indices,
                          int64_t nodes, int64_t edges, const int64_t *graph_offsets,
                          int32_t ngraphs, const mg_options *opts, mg_graph **out);
/* Free all device memory of the graph (GraphSlice::~GraphSlice, csr_problem.cuh:234-353). */
int mg_graph_destroy(mg_graph *g);
/* Vertex and edge counts, directedness and device bytes held by the graph. */
int mg_graph_info(const mg_graph *g, int64_t *nodes, int64_t *edges, int32_t *directed,
                  int64_t *device_bytes);

/* ------------------------------------------------------------ algorithms -- */
/* BFS depths from one source, -1 = unreachable. Replaces
 * EnactorVertexCentric::EnactIterativeSearch (enactor_vertex_centric.cuh:3269-3924)
 * with Program = bfs (Algorithms/BFS/bfs.h:28-298) followed by
 * CsrProblem::ExtractResults (csr_problem.cuh:433-458). */
int mg_bfs(mg_graph *g, int32_t src, int32_t *depths, mg_stats *stats,
           const mg_options *opts);
/* mg_bfs plus predecessors, replacing pred_extract
 * (Algorithms/BFS/predextract.cuh:246-375): preds[v] = the largest in-neighbour u
 * with depths[v] - depths[u] == 1, else -1 (gather_edge :143-154, max reduce
 * :211-218). preds has nodes entries, host or device like depths. */
int mg_bfs_pred(mg_graph *g, int32_t src, int32_t *depths, int32_t *preds,
                mg_stats *stats, const mg_options *opts);
/* One BFS seeded with several roots at depth 0 (bfs::Initialize with num_srcs > 1,
 * bfs.h:62-79): depth = distance to the nearest root. */
int mg_bfs_roots(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depths,
                 mg_stats *stats, const mg_options *opts);
/* nsrc <= 64 independent BFS runs in one pass with a 64-bit per-vertex mask frontier.
 * depths is [nsrc][nodes], row s equal to mg_bfs(srcs[s]). The reference runs
 * them one after the other (Algorithms/BFS/bfs.cu:865-881). */
int mg_bfs_multi(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depths,
                 mg_stats *stats, const mg_options *opts);
/* One BFS per graph of a batch made with mg_graph_create_batch, all in the same
 * launches. srcs[i] is a vertex id local to graph i; depths is [nodes] (global ids). */
int mg_bfs_batch(mg_graph *g, const int32_t *srcs, int32_t *depths, mg_stats *stats,
                 const mg_options *opts);

/* SSSP distances with int32 edge weights, 100000000 = unreachable
 * (Program = sssp, Algorithms/SSSP/sssp.h:34-393). */
int mg_sssp(mg_graph *g, int32_t src, int32_t *dists, mg_stats *stats,
            const mg_options *opts);
/* nsrc <= 64 SSSP runs in one pass; dists is [nsrc][nodes]. */
int mg_sssp_multi(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dists,
                  mg_stats *stats, const mg_options *opts);

/* Connected components by min-label propagation (Program = cc,
 * Algorithms/CC/cc.h:32-349): labels[v] = smallest vertex id reachable from v
 * along edges (for a symmetric graph: the component's minimum id). */
int mg_cc(mg_graph *g, int32_t *labels, mg_stats *stats, const mg_options *opts);

/* Normalised PageRank: r' = (1-d)/N + d*(A^T D^-1 r + dangling(r)/N), FP32 ranks
 * and accumulation, FP64 global norms; stops at L1(r'-r) <= tolerance or iter_num.
 * Pull SpMV over the CSC replacing gather_mgpu + ReduceByKey
 * (enactor_vertex_centric.cuh:2104-2725, mgpukernel/kernel.cuh:300-404). */
int mg_pagerank(mg_graph *g, float *ranks, mg_stats *stats, const mg_options *opts);
/* The reference's own PageRank program (Algorithms/PageRank/PageRank.h:33-409):
 * unnormalised r = 0.15 + 0.85*sum(r[u]/outdeg[u]) over in-edges, frontier of
 * vertices whose |delta| >= tolerance (reference default 0.01), run on the
 * generic GAS engine. */
int mg_pagerank_gas(mg_graph *g, float *ranks, mg_stats *stats, const mg_options *opts);

/* Personalised PageRank with nvec teleport columns (device pointers, row-major
 * [nodes][nvec]): R = (1-d) T + d P^T R, P[u,v] = edge_weight[e(u,v)] (weights given
 * per CSR edge, already row-normalised by the caller). No reference counterpart.
 * Both solves iterate until the L1 change over all entries is <= tolerance times
 * the L1 norm of their right-hand side (T here, dL/dR for the adjoint). */
int mg_ppr_forward(mg_graph *g, const float *edge_weights, const float *teleport,
                   int32_t nvec, float *ranks, mg_stats *stats, const mg_options *opts);
/* Adjoint of mg_ppr_forward: given the converged ranks and dL/dR, solves
 * lambda = dL/dR + d P lambda by power iteration over the out-edges and returns
 * dL/dT = (1-d) lambda and dL/dP[e(u,v)] = d <lambda[v,:], R[u,:]>. */
int mg_ppr_backward(mg_graph *g, const float *edge_weights, const float *ranks,
                    const float *grad_ranks, int32_t nvec, float *grad_edge_weights,
                    float *grad_teleport, mg_stats *stats, const mg_options *opts);

/* BFS for callers that cannot allocate device memory (no counterpart in the
 * reference). The graph (CSR row offsets and column indices, well formed) and
 * the depths output are device pointers the caller owns; every working buffer
 * lives in one static device array of about 14 MiB per GPU, so the call itself
 * allocates nothing. Limits: nodes <= 2^20, edges <= 2^24 (MG_ERR_ARG beyond).
 * Runs push levels only; results equal mg_bfs. The first call on a device looks
 * up the array's device address, so make it before any stream capture; under
 * CUDA's lazy module loading that first call may also be when the driver loads
 * the module and backs the array, so a caller about to reserve nearly all
 * device memory for its own pool should make one call before reserving. Calls
 * share the array: calls that overlap on the GPU race and must be serialised.
 * stats (may be NULL): iterations, vertices_reached and edges_traversed as
 * mg_bfs reports them; device_ms is 0 (no timing events are created).
 * stream may be NULL (legacy default stream). */
int mg_bfs_noalloc(const int32_t *d_row_offsets, const int32_t *d_column_indices, int64_t nodes,
                   int64_t edges, int32_t src, int32_t *d_depths, void *stream, mg_stats *stats);

/* ------------------------------------------------------------- autotuner -- */
enum { MG_TUNE_BFS = 0, MG_TUNE_BFS_MULTI = 1, MG_TUNE_SSSP = 2, MG_TUNE_CC = 3, MG_TUNE_PAGERANK = 4,
       MG_TUNE_PPR = 5 };
/* Chooses the launch parameters the reference fixes at compile time
 * (KernelPolicy and the CTA/warp gather thresholds,
 * GASengine/enactor_vertex_centric.cuh:3934-3970) by timing candidates on this
 * graph and these sources: expand tile (tile_items 1024/2048) x ctas_per_sm
 * (2..5), then alpha (or alpha_multi) and beta for the direction switch.
 * MG_TUNE_PAGERANK (mg_pagerank) and MG_TUNE_PPR (mg_ppr_forward) search
 * ctas_per_sm of their SpMV (2..8), timing a fixed number of iterations; PPR
 * solves nsrc teleport columns, one-hot at srcs, over row-normalised uniform
 * weights (the launch shape does not depend on the values).
 * *inout is the starting point and receives the best options; report (may be
 * NULL) receives a JSON record of every trial. srcs: 1..64 sources (unused for
 * MG_TUNE_CC and MG_TUNE_PAGERANK). */
int mg_autotune(mg_graph *g, int32_t kind, const int32_t *srcs, int32_t nsrc, mg_options *inout,
                char *report, int64_t report_len);

/* -------------------------------------------------------------- builders -- */
/* Seeded R-MAT generator (replaces the unseeded BuildRmatGraph,
 * b40c/graph/builder/rmat.cuh:145-224): edgefactor * 2^scale edges by recursive
 * quadrant choice with probabilities a, b, c, 1-a-b-c. symmetrize: store each
 * edge both ways. clean: drop self-loops and duplicate edges. */
int mg_build_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c,
                  uint64_t seed, int32_t symmetrize, int32_t clean, mg_host_csr *out);
/* width x width 4-neighbour grid (cf. BuildGrid2dGraph, b40c/graph/builder/grid2d.cuh:46-107,
 * without its self-loops), each undirected lattice edge dropped with probability
 * drop_frac, plus round(shortcut_frac * kept) random undirected long edges. */
int mg_build_road_grid(int32_t width, double drop_frac, double shortcut_frac, uint64_t seed,
                       mg_host_csr *out);
/* Symmetric uint32 weights in [lo, hi]: w(u,v) = w(v,u) from a hash of
 * (min(u,v), max(u,v), seed). Fills out->edge_values. */
int mg_build_weights(mg_host_csr *csr, uint32_t lo, uint32_t hi, uint64_t seed);
/* Matrix Market reader with the reference's semantics (ReadMarketStream,
 * b40c/graph/builder/market.cuh:42-141, then CsrGraph::FromCoo,
 * b40c/graph/csr_graph.cuh:120-210): 1-based ids, values read as int, undirected
 * inserts the reverse of every edge, rows stably sorted by (row, col), self-loops
 * and duplicates kept. A "pattern" file gets value 1 on every edge. */
int mg_read_market(const char *path, int32_t undirected, mg_host_csr *out);
/* CSV graph (GASengine/csv_graph_reader.cuh): format 0 = rows "src,dst:val,...",
 * format 1 = rows "src,dst,val"; ids renumbered densely in sorted order;
 * undirected != 0 adds the reversed edges. Edge values are int32. */
int mg_read_csv(const char *path, int32_t format, int32_t undirected, mg_host_csr *out);
/* Transpose (CSC) of a host CSR: column offsets and row indices, stable by row. */
int mg_host_csr_transpose(const mg_host_csr *in, mg_host_csr *out);
/* Frees the arrays of a host CSR filled by the builders and readers above. */
void mg_host_csr_free(mg_host_csr *csr);

#ifdef __cplusplus
}
#endif
#endif /* MAPGRAPH_B200_H */
