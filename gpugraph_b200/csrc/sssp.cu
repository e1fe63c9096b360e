// Single-source SSSP as one fused relaxation kernel per level. The reference's
// sssp program (Algorithms/SSSP/sssp.h:34-393) runs each Bellman-Ford level as
// expand (candidate src_dist + w, :334-343), contract (atomicMin into a
// temporary, :383), apply (min with the distance, :240-255) and post_apply
// (copy/reset, :265-266); the distances it converges to are the unique
// shortest-path distances, so relaxing straight into the distance array with
// atomicMin, and queueing each improved vertex once per level, reaches the same
// fixpoint (the same int32 output, 100000000 = unreachable) in one kernel per
// level. The bundled Program still runs through the generic engine with
// mg_options.generic_engine = 1.
//
// Per level: the frontier scan (degree prefix and merge-path partition of the
// frontier's out-edges, shared with the engine) and k_sssp_relax, whose
// threads take their VT items through independent batches of memory
// operations: column and weight loads, then the heads' distances, then the
// atomicMin of every improving candidate, then the next-level dedup bit.
#include <cuda_runtime.h>

#include <climits>

#include "algo_util.cuh"
#include "gas/run_gas.cuh"

namespace mg {

namespace {

// Frontier-scan Program for the fused kernel: every frontier vertex expands its out-edges.
struct sssp_relax {
  typedef int DataType;
  typedef int MiscType;
  typedef int GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = 100000000;  // sssp::INIT_VALUE (Algorithms/SSSP/sssp.h:43)
  struct VertexType {
    int32_t *dist;
  };
  struct EdgeType {
    int nodes;
  };
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
};

constexpr int kSsVTS = 4;
constexpr int kSsVT = 8;

template <int VT>
__global__ void __launch_bounds__(kNT, 5) k_sssp_relax(GasArgs<sssp_relax> a) {
  constexpr int NV = kNT * VT;
  __shared__ int32_t s_v[NV + 1];
  __shared__ int32_t s_base[NV + 1];
  __shared__ int32_t s_rs[NV + 1];
  __shared__ int32_t s_own[NV];
  __shared__ int32_t s_du[NV + 1];
  __shared__ uint32_t s_cnt[VT * kNW + 1];
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ int s_fail;
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t level = ctl->level, n = ctl->frontier_size, total = ctl->edge_total;
  const uint32_t ntiles = ctl->exp_tiles, epoch = ctl->epoch + 1;
  const unsigned long long spin_limit = ctl->spin_limit;
  const bool ordered = ctl->ordered != 0;
  const unsigned long long items = (unsigned long long)n + total;
  const int32_t *F = cur_queue(a, level);
  int32_t *Fout = nxt_queue(a, level);
  uint32_t *dedup = nxt_bm(a, level);
  int32_t *dist = a.vl.dist;
  const int32_t *ro = a.g.row_offsets, *col = a.g.col, *wgt = a.g.wgt;
  const int32_t V = a.g.V;
  unsigned long long my_bytes = 0;
  if (threadIdx.x == 0) s_fail = 0;
  // tiles through the atomic counter: their relaxations vary in cost (a static
  // deal measured 2 % slower at R-MAT 22)
  for (;;) {
    const uint32_t tile = next_tile(&ctl->tile_ctr[1], &s_tile);
    if (tile >= ntiles || s_fail) break;
    int cnt;
    // each frontier vertex's distance is read once per tile, with its offsets
    if (!decode_tile<VT>(tile, ntiles, n, items, a.part, a.scan, F, ro, s_v, s_base, s_rs, s_own, &cnt,
                         [&](int j, int v) { s_du[j] = __ldcg(&dist[v]); })) {
      if (threadIdx.x == 0) {
        raise_error(ctl, MG_ERR_OVERFLOW);
        s_fail = 1;
      }
      __syncthreads();
      break;
    }
    int32_t head[VT], cand[VT] = {};
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int k = r * kNT + threadIdx.x;
      head[r] = -1;
      if (k < cnt) {
        const int j = s_own[k];
        const int el = k - s_base[j] - 1;
        my_bytes += el >= 0 ? 12ull : 16ull;  // column + weight + head distance; a vertex's own item
        if (el >= 0) {
          const int eid = s_rs[j] + el;
          if ((unsigned)eid < (unsigned)a.g.E) {
            head[r] = col[eid];
            cand[r] = s_du[j] + wgt[eid];
          } else {
            raise_error(ctl, MG_ERR_OVERFLOW);
          }
        }
      }
    }
    int32_t dv[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) dv[r] = ((unsigned)head[r] < (unsigned)V) ? __ldcg(&dist[head[r]]) : INT_MIN;
    // An improving candidate lowers the distance with a reduction (nothing waits
    // for the old value); its improvement is read from the loaded distance. If
    // another relaxation lowered the head further in between, the head is queued
    // by that relaxation too, so the next frontier is the same set.
    bool better[VT];
    uint32_t probe[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      better[r] = head[r] >= 0 && cand[r] < dv[r];
      probe[r] = ~0u;
      if (better[r]) {
        atomicMin(&dist[head[r]], cand[r]);
        probe[r] = ld_volatile(dedup + (head[r] >> 5));
        my_bytes += 4;  // the improved distance
      }
    }
    // the test-and-sets of all VT items in flight together, then the ballots
    bool surv[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      surv[r] = false;
      if (better[r]) {
        const uint32_t bit = 1u << (head[r] & 31);
        if (!(probe[r] & bit)) surv[r] = !(atomicOr(dedup + (head[r] >> 5), bit) & bit);
      }
    }
    uint32_t bal[VT];
    int32_t outv[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      if (surv[r]) my_bytes += 8;  // queue entry + dedup word
      bal[r] = __ballot_sync(0xffffffffu, surv[r]);
      outv[r] = head[r];
    }
    if (!tile_enqueue<VT>(bal, outv, s_cnt, &s_prefix, &s_fail, ordered, a.status, tile, ntiles, epoch, spin_limit,
                          Fout, (uint32_t)V, ctl))
      break;
  }
  add_bytes(ctl, KID_EXPAND, my_bytes);
}

__global__ void k_sssp_seed(int32_t *dist, int32_t *queue0, int32_t src) {
  dist[src] = 0;
  queue0[0] = src;
}

}  // namespace

// Fused single-source SSSP (called by mg_sssp).
int sssp_fused(mg_graph *g, int32_t src, int32_t *dists, mg_stats *stats, const mg_options *o) {
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK) return st;
  using P = sssp_relax;
  GasArgs<P> a = base_args<P>(g);
  a.vl.dist = g->ws.vbuf[0];
  a.el.nodes = (int)g->nodes;
  const int32_t V = g->csr.V;
  const int grid = persistent_grid(g, o, 4);
  // 5 CTAs per SM fit the relax kernel (at most 48 registers, 37 KB of shared memory)
  const int relax_grid = std::max(grid, g->num_sms * 5);
  const uint32_t max_iter = (uint32_t)std::min<int64_t>(o->iter_num > 0 ? o->iter_num : 0, g->nodes + 2);
  cudaError_t e = cudaMemsetAsync(g->ws.bm[0], 0, g->ws.words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.bm[1], 0, g->ws.words * 4, s);
  if ((st = cuda_status(e, "sssp init")) != MG_OK) return st;
  // sssp::Initialize (sssp.h:73-166): every distance unreachable but the source's, frontier = {src}
  k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(a.vl.dist, P::INIT_VALUE, V);
  k_sssp_seed<<<1, 1, 0, s>>>(a.vl.dist, a.queue0, src);
  k_ctl_init<<<1, 32, 0, s>>>(a.ctl, 1u, max_iter, (unsigned long long)o->spin_limit, MODE_QUEUE, ctl_flags(o));
  count_launch(3);
  if ((st = launch_check("sssp init")) != MG_OK) return st;
  const bool small_tiles = o->tile_items > 0 && o->tile_items <= 1024;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    if (small_tiles) {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kSsVTS, 4><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_sssp_relax<4><<<relax_grid, kNT, 0, ss>>>(a)));
    } else {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<P, kSsVTS, kSsVT><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_sssp_relax<kSsVT><<<relax_grid, kNT, 0, ss>>>(a)));
    }
    MG_LAUNCH(KID_OTHER, ss, k_level_end<<<1, 32, 0, ss>>>(a.ctl, h, use_h));
  };
  LoopResult res;
  st = run_level_loop(g, s, "sssp_fused/" + std::to_string(grid) + (small_tiles ? "/t1024" : "/t2048"), 3, body,
                      o->use_cuda_graph != 0, &res);
  if (st != MG_OK) return st;
  finish_run(g, res.ctl.level);
  if (res.ctl.error) return set_error(res.ctl.error, std::string("sssp: device reported ") + mg_status_string(res.ctl.error));
  if (stats) {
    stats->iterations = (int32_t)res.ctl.level;
    stats->push_iterations = (int32_t)res.ctl.level;
    stats->pull_iterations = 0;
    stats->converged = (res.ctl.frontier_size == 0) ? 1 : 0;
    stats->device_ms = res.ms;
    stats->vertices_reached = 0;
    stats->edges_traversed = 0;
    if (want_stats(o) && (st = reach_stats(g, s, a.vl.dist, P::INIT_VALUE, 1, 1, &stats->vertices_reached,
                                           &stats->edges_traversed)) != MG_OK)
      return st;
  }
  return copy_out(s, dists, a.vl.dist, (size_t)V * 4, o->outputs_on_device != 0);
}

}  // namespace mg
