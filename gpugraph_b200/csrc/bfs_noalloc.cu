// mg_bfs_noalloc: BFS for callers that cannot allocate device memory.
//
// Some callers are not allowed to call cudaMalloc: applications that carve all
// GPU memory out of their own pool up front and forbid any further allocation,
// and latency-critical loops that must not hit cudaMalloc's implicit device
// synchronisation. For them this entry point runs the same push-level kernels
// as mg_bfs on a graph the caller already holds in device memory, with every
// working buffer (frontier queues, degree scan, tile partitions, look-back
// status words, bitmaps, control block) carved from one file-scope static
// device array of fixed size. Nothing here calls cudaMalloc, cudaFree,
// cudaMallocHost or any other allocating routine.
//
// Limits: nodes <= kNaMaxNodes (2^20) and edges <= kNaMaxEdges (2^24); the
// array takes about 14 MiB on every GPU that loads the library, until exit.
// Only push levels are run, because the in-edges a pull level reads would need
// a transpose the caller may not have.
//
// Under CUDA's lazy module loading (the default) the first call on a device
// may be the moment the driver loads this module and backs the array, so a
// caller that reserves nearly all device memory for its own pool should make
// one call (any small graph) before reserving.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the bitmaps that must start cleared are cleared by each call, and
// the look-back epoch carried in the control block keeps stale status words
// from matching. Calls whose work overlaps on the GPU (e.g. from two streams
// at once) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/mapgraph_b200.h"
#include "gas/driver.cuh"
#include "gas/engine.cuh"
#include "gas/programs.cuh"
#include "host_util.h"

namespace mg {

constexpr int64_t kNaMaxNodes = 1 << 20;
constexpr int64_t kNaMaxEdges = 1 << 24;
constexpr size_t kNaAlign = 256;
constexpr size_t na_round(size_t b) { return (b + kNaAlign - 1) & ~(kNaAlign - 1); }
constexpr size_t kNaWords = (size_t)kNaMaxNodes / 32 + 4;
constexpr size_t kNaPart = (size_t)(kNaMaxNodes + kNaMaxEdges) / 1024 + 8;
constexpr size_t kNaStatus = (size_t)(kNaMaxNodes + kNaMaxEdges) / 1024 + 64;
constexpr size_t kNaOffQueue0 = 0;
constexpr size_t kNaOffQueue1 = kNaOffQueue0 + na_round((size_t)kNaMaxNodes * 4);
constexpr size_t kNaOffScan = kNaOffQueue1 + na_round((size_t)kNaMaxNodes * 4);
constexpr size_t kNaOffPart = kNaOffScan + na_round(((size_t)kNaMaxNodes + 1 + 64) * 4);
constexpr size_t kNaOffStatus = kNaOffPart + na_round(kNaPart * 4);
constexpr size_t kNaOffBm0 = kNaOffStatus + na_round(kNaStatus * 8);
constexpr size_t kNaOffBm1 = kNaOffBm0 + na_round(kNaWords * 4);
constexpr size_t kNaOffVisited = kNaOffBm1 + na_round(kNaWords * 4);
constexpr size_t kNaOffChanged = kNaOffVisited + na_round(kNaWords * 4);
constexpr size_t kNaOffCtl = kNaOffChanged + na_round((size_t)kNaMaxNodes);
constexpr size_t kNaBytes = kNaOffCtl + na_round(sizeof(Ctl));

// The scratch array. In host code this name is only a host-side stand-in:
// kernels get the device address obtained with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

using NaP = programs::bfs;

// Kernels defined with the rest of the BFS path (bfs.cu).
__global__ void k_bfs_level_end(Ctl *ctl, int32_t V, int64_t E, cudaGraphConditionalHandle h, int use_handle);
__global__ void k_bfs_init(Ctl *ctl, int32_t *queue0, int queue0_ready, int32_t root, int32_t nsrc, int32_t *labels,
                           uint32_t *visited, uint32_t *bm0, const int32_t *ro, uint32_t dir_policy, float alpha,
                           float beta);

namespace {
constexpr int kNaMaxDevices = 64;
// Per-device device address of the array, filled by the first call on that
// device (with that device current).
unsigned char *g_na_base[kNaMaxDevices] = {nullptr};
uint64_t g_na_epochs[kNaMaxDevices] = {0};
}  // namespace

}  // namespace mg

using namespace mg;

extern "C" int mg_bfs_noalloc(const int32_t *d_row_offsets, const int32_t *d_column_indices, int64_t nodes,
                              int64_t edges, int32_t src, int32_t *d_depths, void *stream, mg_stats *stats) {
  clear_error();
  if (!d_row_offsets || !d_depths || (edges > 0 && !d_column_indices))
    return set_error(MG_ERR_ARG, "mg_bfs_noalloc: null device pointer");
  if (nodes < 1 || nodes > kNaMaxNodes)
    return set_error(MG_ERR_ARG, "mg_bfs_noalloc: nodes must be in [1, " + std::to_string(kNaMaxNodes) +
                                     "] (fixed scratch size)");
  if (edges < 0 || edges > kNaMaxEdges)
    return set_error(MG_ERR_ARG, "mg_bfs_noalloc: edges must be in [0, " + std::to_string(kNaMaxEdges) +
                                     "] (fixed scratch size)");
  if (src < 0 || (int64_t)src >= nodes) return set_error(MG_ERR_ARG, "mg_bfs_noalloc: source out of range");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kNaMaxDevices) return set_error(MG_ERR_UNSUPPORTED, "mg_bfs_noalloc: device ordinal too large");
  // Set-up, once per device, with that device current.
  if (!g_na_base[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                   "mg_bfs_noalloc: cudaGetSymbolAddress");
    g_na_base[dev] = static_cast<unsigned char *>(p);
  }
  unsigned char *base = g_na_base[dev];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t *q0 = reinterpret_cast<int32_t *>(base + kNaOffQueue0);
  int32_t *q1 = reinterpret_cast<int32_t *>(base + kNaOffQueue1);
  uint32_t *scan = reinterpret_cast<uint32_t *>(base + kNaOffScan);
  int32_t *part = reinterpret_cast<int32_t *>(base + kNaOffPart);
  unsigned long long *status = reinterpret_cast<unsigned long long *>(base + kNaOffStatus);
  uint32_t *bm0 = reinterpret_cast<uint32_t *>(base + kNaOffBm0);
  uint32_t *bm1 = reinterpret_cast<uint32_t *>(base + kNaOffBm1);
  uint32_t *visited = reinterpret_cast<uint32_t *>(base + kNaOffVisited);
  uint8_t *changed = reinterpret_cast<uint8_t *>(base + kNaOffChanged);
  Ctl *ctl = reinterpret_cast<Ctl *>(base + kNaOffCtl);
  const size_t words = (size_t)(nodes + 31) / 32 + 4;

  // Look-back epochs grow across calls; clear the status words and the control
  // block long before the 30-bit epoch field could wrap.
  if (g_na_epochs[dev] > (1ull << 27)) {
    e = cudaMemsetAsync(status, 0, kNaStatus * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctl, 0, sizeof(Ctl), s);
    if (e != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: status reset");
    g_na_epochs[dev] = 0;
  }
  e = cudaMemsetAsync(visited, 0, words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bm0, 0, words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bm1, 0, words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(changed, 0, (size_t)nodes, s);
  if (e != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: init");

  GasArgs<NaP> a;
  memset(&a, 0, sizeof(a));
  a.g.row_offsets = const_cast<int32_t *>(d_row_offsets);
  a.g.col = const_cast<int32_t *>(d_column_indices);
  a.g.csc_offsets = a.g.row_offsets;
  a.g.csc_rows = a.g.col;
  a.g.pull_rows = a.g.col;
  a.g.V = (int32_t)nodes;
  a.g.E = (int32_t)edges;
  a.vl.d_labels = d_depths;
  a.vl.d_visited = visited;
  a.vl.nodes = (int)nodes;
  a.vl.edges = (int)edges;
  a.el.nodes = (int)nodes;
  a.el.edges = (int)edges;
  a.queue0 = q0;
  a.queue1 = q1;
  a.scan = scan;
  a.part = part;
  a.status = status;
  a.bm0 = bm0;
  a.bm1 = bm1;
  a.changed = changed;
  a.ctl = ctl;
  a.gather_dir = NO_GATHER_EDGES;

  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = sms * 4;
  const uint32_t max_iter = (uint32_t)nodes + 2;
  k_fill_i32<<<sms * 4, 256, 0, s>>>(d_depths, NaP::INIT_VALUE, nodes);
  k_ctl_init<<<1, 32, 0, s>>>(ctl, 1u, max_iter, 1ull << 22, MODE_QUEUE, 0u);
  k_bfs_init<<<1, 256, 0, s>>>(ctl, q0, 0, src, 1, d_depths, visited, bm0, d_row_offsets, (uint32_t)MG_DIR_PUSH, 15.f,
                               18.f);
  count_launch(3);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: init kernels");
  Ctl hc;
  for (;;) {
    // a few push levels per check of the control block (levels after the last
    // one return at once because ctl->active is 0)
    for (int k = 0; k < 4; ++k) {
      k_frontier_scan<NaP, 4, 8><<<grid, kNT, 0, s>>>(a);
      k_expand<NaP, 8><<<grid, kNT, 0, s>>>(a);
      k_bfs_level_end<<<1, 32, 0, s>>>(ctl, (int32_t)nodes, edges, 0, 0);
      count_launch(3);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: level kernels");
    e = cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "mg_bfs_noalloc: control block read");
    if (!hc.active) break;
  }
  g_na_epochs[dev] += 4ull * ((uint64_t)hc.level + 2);
  if (hc.error) return set_error(hc.error, std::string("mg_bfs_noalloc: device reported ") + mg_status_string(hc.error));
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->iterations = (int32_t)hc.level;
    stats->push_iterations = (int32_t)hc.push_levels;
    stats->converged = hc.frontier_size == 0 ? 1 : 0;
    stats->vertices_reached = (int64_t)hc.visited_count;
    // out-degrees of the reached vertices, summed level by level on the device
    // (the same count mg_bfs reports); device_ms stays 0: timing events are
    // driver resources this entry point does not create
    stats->edges_traversed = (int64_t)hc.visited_edges;
  }
  return MG_OK;
}
