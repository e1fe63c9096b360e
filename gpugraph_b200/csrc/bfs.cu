// Direction-optimising BFS (push/pull switching): push levels run the bfs Program's
// expand + contract (Algorithms/BFS/bfs.h:28-298) fused into k_bfs_push over a
// vertex queue; pull levels run a bottom-up sweep in which every unvisited
// vertex scans its in-edges (hubs first) for a parent in the frontier bitmap
// and stops at the first hit.
// The switch follows Beamer's rule: push -> pull when the next frontier's
// out-edges exceed (unvisited edges)/alpha while the frontier grows, pull ->
// push when the frontier shrinks below nodes/beta. Depths are unique, so every
// schedule gives the same labels as the reference's CPUBFS
// (Algorithms/BFS/bfs.cu:57-111).
#include <cuda_runtime.h>

#include <algorithm>

#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"
#include "gas/programs.cuh"

namespace mg {

using BfsP = programs::bfs;
constexpr int kVTS = 4;  // frontier entries per thread in the scan
constexpr int kVT = 8;   // items per thread in the expand (NV = 2048)

// Bottom-up level: a warp takes kPullWords consecutive 32-vertex bitmap words
// per ticket (lane = vertex within a word). For every unvisited vertex the
// first four in-edges of all the warp's words are probed at once (their row
// indices, then their frontier-bitmap words), so one round trip serves
// kPullWords x 32 vertices; the in-lists are ordered hubs first, so most
// vertices with a parent find it there. Vertices still searching continue four
// in-edges per step and stop at the first parent.
constexpr int kPullWords = 4;
__global__ void __launch_bounds__(kNT, 6) k_bfs_pull(GasArgs<BfsP> a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_BITMAP) return;
  const uint32_t level = ctl->level;
  const uint32_t *cur = cur_bm(a, level);
  uint32_t *nxt = nxt_bm(a, level);
  uint32_t *visited = a.vl.d_visited;
  const int32_t V = a.g.V;
  const uint32_t words = ((uint32_t)V + 31) / 32;
  const uint32_t tickets = (words + kPullWords - 1) / kPullWords;
  const int32_t *coff = a.g.csc_offsets, *crow = a.g.pull_rows, *ro = a.g.row_offsets;
  const int lane = lane_id();
  unsigned long long my_cnt = 0, my_edges = 0, my_bytes = 0;
  __shared__ unsigned long long s_tot[2];
  if (threadIdx.x < 2) s_tot[threadIdx.x] = 0;
  __syncthreads();
  // Tickets (kPullWords words each) are dealt round-robin over the grid's
  // warps: one atomic per ticket on a shared counter costs more than the
  // imbalance it would remove (measured on R-MAT 22: 317 vs 342 us per BFS).
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tickets; t += nwarps) {
    uint32_t vis[kPullWords];
    int beg[kPullWords], end[kPullWords];
#pragma unroll
    for (int q = 0; q < kPullWords; ++q) {
      const uint32_t w = t * kPullWords + q;
      const int v = (int)(w * 32 + lane);
      vis[q] = w < words ? visited[w] : ~0u;
      beg[q] = v < V ? coff[v] : 0;
      end[q] = v < V ? coff[v + 1] : 0;
    }
    // first step for every word at once: up to four in-edges per searching vertex
    int u[kPullWords][4];
    bool search[kPullWords];
#pragma unroll
    for (int q = 0; q < kPullWords; ++q) {
      const int v = (int)((t * kPullWords + q) * 32 + lane);
      search[q] = v < V && !((vis[q] >> lane) & 1u);
      if (!search[q]) end[q] = beg[q];  // nothing to scan
#pragma unroll
      for (int k = 0; k < 4; ++k) u[q][k] = beg[q] + k < end[q] ? __ldcs(crow + beg[q] + k) : -1;
    }
    bool found[kPullWords];
#pragma unroll
    for (int q = 0; q < kPullWords; ++q) {
      uint32_t hit = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (u[q][k] >= 0) hit |= __ldg(&cur[u[q][k] >> 5]) >> (u[q][k] & 31);
      found[q] = hit & 1u;
    }
#pragma unroll
    for (int q = 0; q < kPullWords; ++q) {
      const uint32_t w = t * kPullWords + q;
      const int v = (int)(w * 32 + lane);
      int e = min(beg[q] + 4, end[q]);
      int probed = e - beg[q];
      if (!found[q]) {
        // continue four in-edges per step (independent loads in flight)
        while (e < end[q]) {
          const int c = min(4, end[q] - e);
          const int u0 = __ldcs(crow + e);
          const int u1 = c > 1 ? __ldcs(crow + e + 1) : u0;
          const int u2 = c > 2 ? __ldcs(crow + e + 2) : u0;
          const int u3 = c > 3 ? __ldcs(crow + e + 3) : u0;
          const uint32_t hit = ((__ldg(&cur[u0 >> 5]) >> (u0 & 31)) | (__ldg(&cur[u1 >> 5]) >> (u1 & 31)) |
                                (__ldg(&cur[u2 >> 5]) >> (u2 & 31)) | (__ldg(&cur[u3 >> 5]) >> (u3 & 31))) &
                               1u;
          e += c;
          probed += c;
          if (hit) {
            found[q] = true;
            break;
          }
        }
      }
      // offsets + per inspected edge: row index and frontier-bitmap word
      if (search[q]) my_bytes += 8 + 8ull * (unsigned long long)probed;
      const uint32_t bal = __ballot_sync(0xffffffffu, found[q]);
      if (lane == 0 && w < words) {
        nxt[w] = bal;
        if (bal) visited[w] = vis[q] | bal;
        my_cnt += __popc(bal);
        my_bytes += 8;  // visited word + next-frontier word
      }
      if (found[q]) {
        my_bytes += 4;
        a.vl.d_labels[v] = (int)level + 1;
        my_edges += (unsigned long long)(ro[v + 1] - ro[v]);
      }
    }
  }
  add_bytes(ctl, KID_BFS_PULL, my_bytes);
  // totals per CTA, then one atomic per CTA and counter on the control block
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_cnt) atomicAdd(&s_tot[0], my_cnt);
  if (lane == 0 && my_edges) atomicAdd(&s_tot[1], my_edges);
  __syncthreads();
  if (threadIdx.x == 0 && s_tot[0]) atomicAdd((unsigned long long *)&ctl->acc[0], s_tot[0]);
  if (threadIdx.x == 0 && s_tot[1]) atomicAdd(&ctl->next_edges, s_tot[1]);
}

// Top-down level of the bfs program (the engine's expand + contract with the
// bfs functors, Algorithms/BFS/bfs.h:233-286, fused and specialised): tiles of
// NV = kNT*VT items (frontier vertices and their out-edges) from the frontier
// scan's merge-path partition. Every thread takes its VT items through three
// batches of independent memory operations instead of VT dependent chains:
// all column loads, then all visited-word loads, then the test-and-set
// atomics of the unvisited ones; a winner writes its depth and its bit in the
// next frontier bitmap (which a following bottom-up level reads) and is
// compacted into the next queue.
template <int VT>
__global__ void __launch_bounds__(kNT, 6) k_bfs_push(GasArgs<BfsP> a) {
  constexpr int NV = kNT * VT;
  __shared__ int32_t s_v[NV + 1];
  __shared__ int32_t s_base[NV + 1];
  __shared__ int32_t s_rs[NV + 1];
  __shared__ int32_t s_own[NV];
  __shared__ uint32_t s_cnt[VT * kNW + 1];
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ int s_fail;
  __shared__ unsigned long long s_edges;
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_QUEUE) return;
  const uint32_t level = ctl->level, n = ctl->frontier_size, total = ctl->edge_total;
  const uint32_t ntiles = ctl->exp_tiles, epoch = ctl->epoch + 1;
  const unsigned long long spin_limit = ctl->spin_limit;
  const bool ordered = ctl->ordered != 0;
  const unsigned long long items = (unsigned long long)n + total;
  const int32_t *F = cur_queue(a, level);
  int32_t *Fout = nxt_queue(a, level);
  uint32_t *next_bm = nxt_bm(a, level);
  uint32_t *visited = a.vl.d_visited;
  int32_t *labels = a.vl.d_labels;
  const int32_t *ro = a.g.row_offsets, *col = a.g.col;
  const int32_t V = a.g.V;
  const int lane = lane_id();
  unsigned long long my_edges = 0, my_bytes = 0;
  if (threadIdx.x == 0) {
    s_fail = 0;
    s_edges = 0;
  }
  for (uint32_t k = 0;; ++k) {
    const uint32_t tile = take_tile(&ctl->tile_ctr[1], &s_tile, ordered, k);
    if (tile >= ntiles || s_fail) break;
    int cnt;
    if (!decode_tile<VT>(tile, ntiles, n, items, a.part, a.scan, F, ro, s_v, s_base, s_rs, s_own, &cnt,
                         [](int, int) {})) {
      if (threadIdx.x == 0) {
        raise_error(ctl, MG_ERR_OVERFLOW);
        s_fail = 1;
      }
      __syncthreads();
      break;
    }
    int32_t nbr[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int k = r * kNT + threadIdx.x;
      nbr[r] = -1;
      if (k < cnt) {
        const int j = s_own[k];
        const int el = k - s_base[j] - 1;
        my_bytes += el >= 0 ? 8ull : 12ull;  // column + visited probe; a vertex's own item: its offsets + queue entry
        if (el >= 0) {
          const int eid = s_rs[j] + el;
          if ((unsigned)eid < (unsigned)a.g.E) nbr[r] = __ldcs(col + eid);
          else raise_error(ctl, MG_ERR_OVERFLOW);
        }
      }
    }
    uint32_t word[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) word[r] = ((unsigned)nbr[r] < (unsigned)V) ? ld_volatile(&visited[nbr[r] >> 5]) : ~0u;
    // the test-and-sets of all VT items in flight together, then the winners'
    // out-degrees, then their writes and ballots (each step waits only once)
    uint32_t surv = 0;  // bit r: item r won its test-and-set
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int u = nbr[r];
      if ((unsigned)u < (unsigned)V) {
        const uint32_t bit = 1u << (u & 31);
        if (!(word[r] & bit) && !(atomicOr(&visited[u >> 5], bit) & bit)) surv |= 1u << r;
      }
    }
    int d0[VT], d1[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      d0[r] = d1[r] = 0;
      if ((surv >> r) & 1u) {
        d0[r] = ro[nbr[r]];
        d1[r] = ro[nbr[r] + 1];
      }
    }
    uint32_t bal[VT];
    int32_t outv[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int u = nbr[r];
      const bool won = (surv >> r) & 1u;
      if (won) {
        labels[u] = (int)level + 1;
        atomicOr(&next_bm[u >> 5], 1u << (u & 31));
        my_edges += (unsigned long long)(d1[r] - d0[r]);
        my_bytes += 8;  // queue entry + depth
      }
      bal[r] = __ballot_sync(0xffffffffu, won);
      outv[r] = u;
    }
    if (!tile_enqueue<VT>(bal, outv, s_cnt, &s_prefix, &s_fail, ordered, a.status, tile, ntiles, epoch, spin_limit,
                          Fout, (uint32_t)V, ctl))
      break;
  }
  add_bytes(ctl, KID_EXPAND, my_bytes);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_edges) atomicAdd(&s_edges, my_edges);
  __syncthreads();
  if (threadIdx.x == 0 && s_edges) atomicAdd(&ctl->next_edges, s_edges);
}

// Predecessors after a BFS, the rule of the reference's pred_extract
// (Algorithms/BFS/predextract.cuh:143-154 gather_edge, :211-218 max reduce,
// :236 empty in-lists): pred[v] = max(-1, max over in-neighbours u with
// depth[v] - depth[u] == 1 of u). Depth arithmetic is kept as it is there, so a
// root of a directed graph takes an unreached (-1) in-neighbour as its
// predecessor. Warp per 32-vertex group: lists of up to 32 in-edges are scanned
// by their own lane, longer ones by the whole warp (32 edges per step, then a
// warp max). Unreached vertices (depth -1) cannot match and are not scanned.
__global__ void __launch_bounds__(kNT) k_bfs_pred(const int32_t *coff, const int32_t *crow, const int32_t *depth,
                                                  int32_t *pred, int32_t V) {
  const int lane = lane_id();
  const uint32_t groups = ((uint32_t)V + 31) / 32;
  for (uint32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) / 32; grp < groups;
       grp += (gridDim.x * blockDim.x) / 32) {
    const int v = (int)(grp * 32) + lane;
    const bool valid = v < V;
    const int dv = valid ? depth[v] : -1;
    const int b = valid ? coff[v] : 0, e = valid ? coff[v + 1] : 0;
    const bool scan = dv >= 0 && e > b;
    int best = -1;
    if (scan && e - b <= 32) {
      for (int k = b; k < e; ++k) {
        const int u = crow[k];
        if (dv - depth[u] == 1) best = max(best, u);
      }
    }
    uint32_t hv = __ballot_sync(0xffffffffu, scan && e - b > 32);
    while (hv) {
      const int h = __ffs(hv) - 1;
      hv &= hv - 1;
      const int hb = __shfl_sync(0xffffffffu, b, h), he = __shfl_sync(0xffffffffu, e, h);
      const int hd = __shfl_sync(0xffffffffu, dv, h);
      int m = -1;
      for (int k = hb + lane; k < he; k += 32) {
        const int u = crow[k];
        if (hd - depth[u] == 1) m = max(m, u);
      }
      m = __reduce_max_sync(0xffffffffu, m);
      if (lane == h) best = m;
    }
    if (valid) pred[v] = best;
  }
}

// Pull -> push conversion at the start of a level: ordered compaction of the
// frontier bitmap into the queue (decoupled look-back), and clearing of the
// bitmap the coming push level will fill.
__global__ void __launch_bounds__(kNT) k_bm_to_queue(GasArgs<BfsP> a) {
  constexpr int WPT = 4;
  constexpr uint32_t TW = kNT * WPT;
  __shared__ uint32_t s_red[kNW + 1];
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ int s_fail;
  Ctl *ctl = a.ctl;
  if (!ctl->active || !ctl->convert) return;
  const uint32_t level = ctl->level, epoch = ctl->epoch + 2;
  const unsigned long long spin_limit = ctl->spin_limit;
  const uint32_t *src = cur_bm(a, level);
  uint32_t *clr = nxt_bm(a, level);
  int32_t *Q = cur_queue(a, level);
  const uint32_t words = ((uint32_t)a.g.V + 31) / 32;
  const uint32_t ntiles = (words + TW - 1) / TW;
  if (threadIdx.x == 0) s_fail = 0;
  for (;;) {
    const uint32_t tile = next_tile(&ctl->tile_ctr[3], &s_tile);
    if (tile >= ntiles || s_fail) break;
    const uint32_t wb = tile * TW + threadIdx.x * WPT;
    uint32_t wv[WPT], c = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
      wv[k] = (wb + k < words) ? src[wb + k] : 0u;
      if (wb + k < words) clr[wb + k] = 0u;
      c += __popc(wv[k]);
    }
    uint32_t tot;
    const uint32_t ex = cta_exclusive_sum(c, s_red, &tot);
    if (warp_id() == 0) {
      bool failed = false;
      const uint32_t pre = lookback(a.status, tile, tot, epoch, spin_limit, &failed);
      if (lane_id() == 0) {
        s_prefix = pre;
        if (failed) {
          s_fail = 1;
          raise_error(ctl, MG_ERR_TIMEOUT);
        } else if (tile == ntiles - 1) {
          ctl->frontier_size = pre + tot;
        }
      }
    }
    __syncthreads();
    if (s_fail) break;
    uint32_t pos = s_prefix + ex;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
      uint32_t x = wv[k];
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        if (pos < (uint32_t)a.g.V) Q[pos] = (int32_t)((wb + k) * 32 + b);
        ++pos;
      }
    }
  }
}

__global__ void k_bfs_level_end(Ctl *ctl, int32_t V, int64_t E, cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x != 0) return;
  if (ctl->active) {
    const uint32_t mode = ctl->mode;
    uint32_t n_next;
    if (mode == MODE_BITMAP) {
      unsigned long long *cnt = (unsigned long long *)&ctl->acc[0];
      n_next = (uint32_t)*cnt;
      *cnt = 0;
      ctl->pull_levels += 1;
    } else {
      n_next = ctl->next_size;
      ctl->push_levels += 1;
    }
    const unsigned long long m_next = ctl->next_edges;
    ctl->visited_edges += m_next;
    ctl->visited_count += n_next;
    uint32_t new_mode = mode;
    if (ctl->dir_policy == MG_DIR_PUSH) {
      new_mode = MODE_QUEUE;
    } else if (ctl->dir_policy == MG_DIR_PULL) {
      new_mode = MODE_BITMAP;
    } else if (mode == MODE_QUEUE) {
      const double unvisited_edges = (double)E - (double)ctl->visited_edges;
      // only while the frontier grows: near the end of a search the unvisited
      // edges are few, and a sweep over every vertex costs more than the push
      if ((double)m_next > unvisited_edges / (double)ctl->alpha && n_next > ctl->frontier_size)
        new_mode = MODE_BITMAP;
    } else {
      if ((double)n_next < (double)V / (double)ctl->beta && n_next < ctl->frontier_size) new_mode = MODE_QUEUE;
    }
    ctl->convert = (mode == MODE_BITMAP && new_mode == MODE_QUEUE) ? 1u : 0u;
    ctl->mode = new_mode;
    ctl->level += 1;
    ctl->frontier_size = n_next;
    ctl->next_size = 0;
    ctl->edge_total = 0;
    ctl->exp_tiles = 0;
    ctl->next_edges = 0;
    ctl->epoch += 4;
    for (int i = 0; i < 4; ++i) ctl->tile_ctr[i] = 0;
    ctl->active = (n_next > 0 && ctl->level < ctl->max_iter && ctl->error == 0) ? 1u : 0u;
  }
  if (use_handle) cudaGraphSetConditional(h, ctl->active);
}

// Level-0 state. The roots are already in queue0, or (queue0_ready == 0, one
// root) passed by value and written there here.
__global__ void k_bfs_init(Ctl *ctl, int32_t *queue0, int queue0_ready, int32_t root, int32_t nsrc, int32_t *labels,
                           uint32_t *visited, uint32_t *bm0, const int32_t *ro, uint32_t dir_policy, float alpha,
                           float beta) {
  __shared__ unsigned long long s_edges;
  if (threadIdx.x == 0) {
    s_edges = 0;
    if (!queue0_ready) queue0[0] = root;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
    const int v = queue0_ready ? queue0[i] : root;
    labels[v] = 0;
    atomicOr(&visited[v >> 5], 1u << (v & 31));
    atomicOr(&bm0[v >> 5], 1u << (v & 31));
    atomicAdd(&s_edges, (unsigned long long)(ro[v + 1] - ro[v]));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ctl->visited_edges = s_edges;
    ctl->visited_count = (unsigned long long)nsrc;
    ctl->dir_policy = dir_policy;
    ctl->alpha = alpha;
    ctl->beta = beta;
    ctl->mode = (dir_policy == MG_DIR_PULL) ? MODE_BITMAP : MODE_QUEUE;
    ctl->convert = 0;
  }
}

// Level-0 state of a single-root BFS in one launch (instead of clearing the
// three bitmaps, filling the depths, and initialising the control block and
// the root separately): every depth and bitmap word is written once, the
// root's with its level-0 value.
__global__ void k_bfs_start(Ctl *ctl, int32_t *queue0, int32_t root, int32_t *labels, uint32_t *visited, uint32_t *bm0,
                            uint32_t *bm1, int32_t V, const int32_t *ro, uint32_t max_iter,
                            unsigned long long spin_limit, uint32_t flags, uint32_t dir_policy, float alpha,
                            float beta) {
  const int64_t words = ((int64_t)V + 31) / 32;
  const int64_t rw = root >> 5;
  const uint32_t rb = 1u << (root & 31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    labels[i] = (i == root) ? 0 : BfsP::INIT_VALUE;
    if (i < words) {
      const uint32_t x = (i == rw) ? rb : 0u;
      visited[i] = x;
      bm0[i] = x;
      bm1[i] = 0u;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl_init_body(ctl, 1u, max_iter, spin_limit, MODE_QUEUE, flags);
    queue0[0] = root;
    ctl->visited_edges = (unsigned long long)(ro[root + 1] - ro[root]);
    ctl->visited_count = 1;
    ctl->dir_policy = dir_policy;
    ctl->alpha = alpha;
    ctl->beta = beta;
    ctl->mode = (dir_policy == MG_DIR_PULL) ? MODE_BITMAP : MODE_QUEUE;
    ctl->convert = 0;
  }
}

// Shared by mg_bfs, mg_bfs_roots and mg_bfs_batch.
// `preds` (optional): predecessors by the pred_extract rule (k_bfs_pred).
int bfs_run(mg_graph *g, const std::vector<int32_t> &roots, int32_t *depths, mg_stats *stats, const mg_options *o,
            int32_t *preds = nullptr) {
  mg_options dflt;
  if (!o) {
    mg_options_init(&dflt);
    o = &dflt;
  }
  // (pull needs in-edges; every graph has them: its CSC or the symmetric CSR)
  if (o->direction != MG_DIR_PULL && o->direction != MG_DIR_AUTO && o->direction != MG_DIR_PUSH)
    return set_error(MG_ERR_ARG, "unknown direction policy");
  cudaStream_t s = run_stream(g, o);
  int st = ensure_workspace(g);
  if (st != MG_OK) return st;
  if ((st = prepare_run(g, s)) != MG_OK) return st;
  Workspace &w = g->ws;
  GasArgs<BfsP> a;
  a.g = g->csr;
  a.vl.d_labels = w.vbuf[0];
  a.vl.d_visited = w.visited;
  a.vl.nodes = (int)g->nodes;
  a.vl.edges = (int)g->edges;
  a.el.nodes = (int)g->nodes;
  a.el.edges = (int)g->edges;
  a.queue0 = w.queue[0];
  a.queue1 = w.queue[1];
  a.scan = w.scan;
  a.part = w.part;
  a.status = w.status;
  a.bm0 = w.bm[0];
  a.bm1 = w.bm[1];
  a.changed = w.changed;
  a.gather_tmp = w.gather_tmp;
  a.gather_res = w.gather_tmp;
  a.ctl = w.ctl;
  a.expand_in = 0;
  a.gather_dir = NO_GATHER_EDGES;
  const int V = (int)g->nodes;
  const uint32_t nsrc = (uint32_t)roots.size();
  // Every level of a traversal settles at least one vertex, so V + 2 levels bound
  // the device loop even if a Program never empties its frontier.
  const uint32_t max_iter = (uint32_t)std::min<int64_t>(o->iter_num > 0 ? o->iter_num : 0, g->nodes + 2);
  // one root goes to the start kernel by value; several are copied to the queue
  const int queue0_ready = nsrc > 1 ? 1 : 0;
  if (queue0_ready) {
    cudaError_t e = cudaMemcpyAsync(w.queue[0], roots.data(), nsrc * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.visited, 0, w.words * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.bm[0], 0, w.words * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.bm[1], 0, w.words * 4, s);
    if ((st = cuda_status(e, "bfs init")) != MG_OK) return st;
  }
  const int grid = persistent_grid(g, o, 4);
  // the pull kernel holds no shared memory and at most 40 registers: 48 warps per SM
  const int pull_grid = g->num_sms * 6;
  // the push kernel: at most 40 registers and 25 KB of shared memory, 6 CTAs per SM
  const int push_grid = std::max(grid, g->num_sms * 6);
  if (queue0_ready) {
    k_fill_i32<<<g->num_sms * 4, 256, 0, s>>>(w.vbuf[0], BfsP::INIT_VALUE, V);
    k_ctl_init<<<1, 32, 0, s>>>(w.ctl, nsrc, max_iter, (unsigned long long)o->spin_limit, MODE_QUEUE, ctl_flags(o));
    k_bfs_init<<<1, 256, 0, s>>>(w.ctl, w.queue[0], queue0_ready, roots[0], (int32_t)nsrc, w.vbuf[0], w.visited,
                                 w.bm[0], g->csr.row_offsets, (uint32_t)o->direction, (float)o->alpha, (float)o->beta);
    count_launch(3);
  } else {
    k_bfs_start<<<g->num_sms * 4, 256, 0, s>>>(w.ctl, w.queue[0], roots[0], w.vbuf[0], w.visited, w.bm[0], w.bm[1], V,
                                               g->csr.row_offsets, max_iter, (unsigned long long)o->spin_limit,
                                               ctl_flags(o), (uint32_t)o->direction, (float)o->alpha,
                                               (float)o->beta);
    count_launch(1);
  }
  if ((st = launch_check("bfs init kernels")) != MG_OK) return st;
  const int32_t Vv = g->csr.V;
  const int64_t E = g->edges;
  // expand tile: 1024 or 2048 items (mg_options.tile_items; 0 = 2048)
  const bool small_tiles = o->tile_items > 0 && o->tile_items <= 1024;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    MG_LAUNCH(KID_CONVERT, ss, k_bm_to_queue<<<grid, kNT, 0, ss>>>(a));
    if (small_tiles) {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<BfsP, kVTS, 4><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_bfs_push<4><<<push_grid, kNT, 0, ss>>>(a)));
    } else {
      MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<BfsP, kVTS, kVT><<<grid, kNT, 0, ss>>>(a)));
      MG_LAUNCH(KID_EXPAND, ss, (k_bfs_push<kVT><<<push_grid, kNT, 0, ss>>>(a)));
    }
    MG_LAUNCH(KID_BFS_PULL, ss, k_bfs_pull<<<pull_grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_OTHER, ss, k_bfs_level_end<<<1, 32, 0, ss>>>(a.ctl, Vv, E, h, use_h));
  };
  LoopResult res;
  // device output without predecessors: the depths are copied before the
  // control block is read back (one host synchronisation)
  const bool early_copy = o->outputs_on_device != 0 && !preds && depths;
  int32_t *labels = w.vbuf[0];
  const std::function<void(cudaStream_t)> epi = [=](cudaStream_t ss) {
    cudaMemcpyAsync(depths, labels, (size_t)V * 4, cudaMemcpyDeviceToDevice, ss);
  };
  st = run_level_loop(g, s, "bfs/" + std::to_string(grid) + (small_tiles ? "/t1024" : "/t2048"), 5, body,
                      o->use_cuda_graph != 0, &res, early_copy ? &epi : nullptr);
  if (st != MG_OK) return st;
  finish_run(g, res.ctl.level);
  if (res.ctl.error) return set_error(res.ctl.error, "bfs: device reported " + std::string(mg_status_string(res.ctl.error)));
  if (stats) {
    stats->iterations = (int32_t)res.ctl.level;
    stats->push_iterations = (int32_t)res.ctl.push_levels;
    stats->pull_iterations = (int32_t)res.ctl.pull_levels;
    stats->converged = (res.ctl.frontier_size == 0) ? 1 : 0;
    stats->device_ms = res.ms;
    stats->vertices_reached = (int64_t)res.ctl.visited_count;
    stats->edges_traversed = 0;
    if (want_stats(o)) {
      int64_t r = 0, ed = 0;
      if ((st = reach_stats(g, s, w.vbuf[0], -1, 1, 1, &r, &ed)) != MG_OK) return st;
      stats->vertices_reached = r;
      stats->edges_traversed = ed;
    }
  }
  if (preds) {
    k_bfs_pred<<<g->num_sms * 8, kNT, 0, s>>>(g->csr.csc_offsets, g->csr.csc_rows, w.vbuf[0], w.vbuf[1], V);
    count_launch();
    if ((st = launch_check("bfs predecessors")) != MG_OK) return st;
    if ((st = copy_out(s, preds, w.vbuf[1], (size_t)V * 4, o->outputs_on_device != 0)) != MG_OK) return st;
  }
  if (early_copy) return MG_OK;
  return copy_out(s, depths, w.vbuf[0], (size_t)V * 4, o->outputs_on_device != 0);
}

}  // namespace mg

using namespace mg;

extern "C" {

int mg_bfs(mg_graph *g, int32_t src, int32_t *depths, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  std::vector<int32_t> roots;
  int st = check_sources(g, &src, 1, &roots);
  if (st != MG_OK) return st;
  return bfs_run(g, roots, depths, stats, opts);
}

int mg_bfs_pred(mg_graph *g, int32_t src, int32_t *depths, int32_t *preds, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (!preds) return set_error(MG_ERR_ARG, "preds is NULL");
  std::vector<int32_t> roots;
  int st = check_sources(g, &src, 1, &roots);
  if (st != MG_OK) return st;
  return bfs_run(g, roots, depths, stats, opts, preds);
}

int mg_bfs_roots(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depths, mg_stats *stats,
                 const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  std::vector<int32_t> roots;
  int st = check_sources(g, srcs, nsrc, &roots);
  if (st != MG_OK) return st;
  return bfs_run(g, roots, depths, stats, opts);
}

int mg_bfs_batch(mg_graph *g, const int32_t *srcs, int32_t *depths, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (g->graph_offsets.empty()) return set_error(MG_ERR_UNSUPPORTED, "graph was not created with mg_graph_create_batch");
  if (!srcs) return set_error(MG_ERR_ARG, "srcs is NULL");
  const int ng = (int)g->graph_offsets.size() - 1;
  std::vector<int32_t> roots((size_t)ng);
  for (int i = 0; i < ng; ++i) {
    const int64_t n_i = g->graph_offsets[i + 1] - g->graph_offsets[i];
    if (srcs[i] < 0 || srcs[i] >= n_i) return set_error(MG_ERR_ARG, "batch source out of range in graph " + std::to_string(i));
    roots[i] = (int32_t)(g->graph_offsets[i] + srcs[i]);
  }
  return bfs_run(g, roots, depths, stats, opts);
}

}  // extern "C"
