// Batched traversal: up to 64 BFS or SSSP sources in one pass, carried as a
// 64-bit mask per vertex. The reference runs sources
// one after the other (Algorithms/BFS/bfs.cu:865-881, Algorithms/SSSP/sssp.cu:389-404);
// here one sweep over an edge serves every source whose frontier contains its
// tail, so the column indices are read once per level instead of once per
// source and level.
//
// HBM layout (per graph, allocated on first use):
//   mask[0]      visit[V]   u64: bit s set once source s has reached v (BFS)
//   mask[1..2]   F[2][V]    u64: level-parity frontier masks
//   multi_out    [V][64]    per-source results: int32 SSSP distances (256 bytes
//                           per vertex); a batched BFS splits it into the level
//                           stack and 16-bit depth rows (below)
// Results are transposed to the caller's int32 [nsrc][V] layout at the end.
//
// Batched BFS depths. The frontier masks of levels 0..15 are kept, one [V] u64
// array per level (the level stack, first half of multi_out): a pull level
// writes its next masks there for every vertex (a coalesced 32 MB stream at
// R-MAT scale 22, which the level writes anyway) instead of scattering 2-byte
// depths into per-vertex rows, and the end-of-run transpose reads the depth of
// (v, s) as the level whose mask holds bit s. A push level's next masks are
// ORed into the parity arrays (they need a zeroed target) and copied to the
// stack for the queued vertices only, with a per-level bitmap of the valid
// entries. Depths of levels 16 and deeper go to [V][64] uint16 rows (the second
// half of multi_out); a run that would pass level 65534 stops there and is rerun
// with int32 depth rows (all of multi_out, no stack).
//
// BFS levels switch between push (the GAS engine's load-balanced expand with
// an OR-into-mask Program, next frontier as a vertex queue) and pull (every
// vertex still missing sources ORs its in-neighbours' frontier masks, stopping
// as soon as every missing source is found). SSSP relaxes warp-per-edge:
// lane l owns sources l and l+32, so one edge reads the two 256-byte distance
// rows with coalesced loads and atomicMin's only improved entries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"
#include "gas/programs.cuh"

namespace mg {

typedef unsigned long long u64;
constexpr int kMVTS = 4;
constexpr int kMVT = 8;
// Batched SSSP relaxes four edges per warp step (each 512 bytes of distance
// rows), so its expand tiles are the smallest the workspace allows (1024
// items): more CTAs share a level's edges.
constexpr int kMSVT = 4;
constexpr int kMssSparse = 24; // active sources per edge up to which a lane relaxes a whole edge alone

// Push step of the batched BFS as a GAS Program: expand_edge emits the
// sources that reach the neighbour for the first time, contract ORs them into
// the neighbour's next-level mask; the engine's bitmap puts each neighbour in
// the next queue once.
struct msbfs_push {
  typedef int DataType;
  typedef u64 MiscType;
  typedef int GatherType;
  typedef int VertexId;
  typedef int SizeT;
  static const int INIT_VALUE = -1;
  static const bool allow_duplicates = false;
  static const bool track_next_edges = true;
  static const int probe_bytes = 8;  // the neighbour's visit mask
  struct VertexType {
    u64 *visit;
    u64 *F0;
    u64 *F1;
    const u64 *stk;  // level stack ([kMsStackLevels][V]), or null
  };
  struct EdgeType {
    int nodes;
  };
  static SrcVertex srcVertex() { return SINGLE; }
  static GatherEdges gatherOverEdges() { return NO_GATHER_EDGES; }
  static ApplyVertices applyOverEdges() { return NO_APPLY_VERTICES; }
  static PostApplyVertices postApplyOverEdges() { return NO_POST_APPLY_VERTICES; }
  static ExpandEdges expandOverEdges() { return EXPAND_OUT_EDGES; }
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
  struct expand_edge {
    __device__ void operator()(const bool, const int iteration, const int u, const int v, const int, VertexType &vl,
                               EdgeType &, int &frontier, u64 &misc) {
      const u64 f = (iteration & 1) ? vl.F1[u] : vl.F0[u];
      const u64 m = f & ~vl.visit[v];
      if (m) {
        frontier = v;
        misc = m;
      }
    }
  };
  struct contract {
    __device__ void operator()(const int iteration, int &v, VertexType &vl, EdgeType &, int *, u64 &misc) {
      u64 *nx = (iteration & 1) ? vl.F0 : vl.F1;
      if ((nx[v] | misc) != nx[v]) atomicOr(&nx[v], misc);
    }
  };
};

struct MultiArgs {
  DevCsr g;
  u64 *visit, *F0, *F1;
  int32_t *out;       // [V][64] int32 rows (SSSP)
  void *rows;         // depth rows of a batched BFS: int32, or uint16 after the level stack
  u64 *stk;           // level stack [kMsStackLevels][V], or null
  uint32_t *stk_bm;   // [kMsStackLevels][stk_words] valid entries of push-made stack levels
  uint32_t stk_words;
  const int32_t *heavy;  // in-lists longer than kMsHeavyList, longest first
  int32_t nheavy;
  int32_t *q0, *q1;
  uint32_t *bm0, *bm1;
  unsigned long long *status;
  Ctl *ctl;
  u64 all;  // mask of the sources in use
};

MG_DEVINL u64 *cur_F(const MultiArgs &a, uint32_t L) { return (L & 1) ? a.F1 : a.F0; }
// The [V][64] depth rows seen as DT (uint16_t or int32_t depths).
template <typename DT>
MG_DEVINL DT *depth_rows(const MultiArgs &a) { return reinterpret_cast<DT *>(a.rows); }
// Level L's array of the level stack.
MG_DEVINL u64 *stk_level(const MultiArgs &a, uint32_t L) { return a.stk + (size_t)L * (uint32_t)a.g.V; }
// The frontier masks of level L: the stack array when a pull level wrote it
// for every vertex, otherwise the parity array (levels made by a push, whose
// parity entries are exact, or levels past the stack).
MG_DEVINL const u64 *front_masks(const MultiArgs &a, const Ctl *ctl, uint32_t L) {
  if (L < ctl->stk_levels && ((ctl->stk_pull >> L) & 1u)) return stk_level(a, L);
  return cur_F(a, L);
}
// Levels a uint16 depth row can hold (depth 65535 is never written).
constexpr uint32_t kMsDepth16Levels = 65534;
MG_DEVINL u64 *nxt_F(const MultiArgs &a, uint32_t L) { return (L & 1) ? a.F0 : a.F1; }
MG_DEVINL int32_t *cur_Q(const MultiArgs &a, uint32_t L) { return (L & 1) ? a.q1 : a.q0; }
MG_DEVINL int32_t *nxt_Q(const MultiArgs &a, uint32_t L) { return (L & 1) ? a.q0 : a.q1; }

// A batched run's sources, passed by value to the init kernels (no host
// staging copy): source s of the run is src[s]; the level-0 queue is the
// sorted distinct list; dir/alpha/beta are the direction policy.
struct SrcList {
  int32_t src[64];
  int32_t distinct[64];
  int32_t nsrc, ndistinct;
  uint32_t dir;
  float alpha, beta;
};

// Level-0 state of a batched run (one CTA of 64 threads).
// bfs: 0 = SSSP (int32 rows), 1 = BFS with int32 depth rows, 2 = BFS with the
// level stack and uint16 rows.
__global__ void k_ms_init(MultiArgs a, SrcList L, int bfs) {
  const int t = threadIdx.x;
  if (t < L.nsrc) {
    const int v = L.src[t];
    atomicOr(&a.F0[v], 1ull << t);
    if (bfs) atomicOr(&a.visit[v], 1ull << t);
    if (bfs == 0) a.out[(int64_t)v * 64 + t] = 0;
    else if (bfs == 1) depth_rows<int32_t>(a)[(int64_t)v * 64 + t] = 0;
  }
  if (t < L.ndistinct) {
    const int v = L.distinct[t];
    a.q0[t] = v;
    if (bfs == 2) {  // level 0 of the stack: each distinct source vertex with its sources
      u64 m = 0;
      for (int s = 0; s < L.nsrc; ++s)
        if (L.src[s] == v) m |= 1ull << s;
      stk_level(a, 0)[v] = m;
      atomicOr(&a.stk_bm[v >> 5], 1u << (v & 31));
    }
  }
  if (t == 0 && bfs) {
    a.ctl->srcmask[0] = a.all;
    a.ctl->srcmask[1] = 0;
    a.ctl->dir_policy = L.dir;
    a.ctl->alpha = L.alpha;
    a.ctl->beta = L.beta;
    a.ctl->stk_levels = bfs == 2 ? kMsStackLevels : 0u;
    a.ctl->stk_pull = 0;
    a.ctl->clear_pending = 0;
  }
}

// Start of a level. After a push level (apply_pending) the queued vertices
// keep only their new sources (depth = level), recorded in the level stack
// (mask and valid bit) or, past it, in the depth rows. A large queue is walked
// in vertex order through the level's dedup bitmap, whose bits are exactly the
// queued vertices (a warp per 32-vertex word: coalesced mask, visit and stack
// accesses, the word itself copied as the stack level's valid bits); a small
// one through the queue. When the previous level's frontier came from a push
// (clear_pending), its parity masks are cleared at its queue entries (through
// its dedup bitmap when that level ran as a pull), so the parity array is all
// zero again before this level's push ORs into it.
template <typename DT>
MG_DEVINL void ms_apply_vertex(const MultiArgs &a, int v, u64 *Fc, u64 *Sk, uint32_t L, u64 &nb, u64 &act,
                               unsigned long long &my_bytes) {
  const u64 vis = a.visit[v];
  nb = Fc[v] & ~vis;
  Fc[v] = nb;
  act |= nb;
  my_bytes += 24;  // visit and mask read, mask write
  if (nb) {
    a.visit[v] = vis | nb;
    my_bytes += 8 + (Sk ? 8ull : sizeof(DT) * (unsigned long long)__popcll(nb));
  }
  if (Sk) Sk[v] = nb;
}

// the depth rows of the warp's vertices with new sources (lane l: sources l and l+32)
template <typename DT>
MG_DEVINL void ms_write_rows(const MultiArgs &a, int v, u64 nb, uint32_t L, int lane) {
  uint32_t wv = __ballot_sync(0xffffffffu, nb != 0);
  while (wv) {
    const int j = __ffs(wv) - 1;
    wv &= wv - 1;
    const u64 m = __shfl_sync(0xffffffffu, nb, j);
    DT *row = depth_rows<DT>(a) + (int64_t)__shfl_sync(0xffffffffu, v, j) * 64;
    if ((m >> lane) & 1ull) row[lane] = (DT)L;
    if ((m >> (lane + 32)) & 1ull) row[lane + 32] = (DT)L;
  }
}

template <typename DT>
__global__ void __launch_bounds__(kNT) k_ms_apply(MultiArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || !(ctl->apply_pending | ctl->clear_pending)) return;
  const uint32_t L = ctl->level, pn = ctl->prev_size;
  const uint32_t n = ctl->apply_pending ? ctl->frontier_size : 0u;
  const bool to_stk = L < ctl->stk_levels;
  u64 *Fc = cur_F(a, L), *Fp = nxt_F(a, L);
  const int32_t *Q = cur_Q(a, L), *Qp = nxt_Q(a, L);
  u64 *Sk = to_stk ? stk_level(a, L) : nullptr;
  uint32_t *Sb = to_stk ? a.stk_bm + (size_t)L * a.stk_words : nullptr;
  const uint32_t V = (uint32_t)a.g.V, words = (V + 31) / 32;
  u64 act = 0;
  unsigned long long my_bytes = 0;
  const int lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  if (n >= words / 8) {
    const uint32_t *B = (L & 1) ? a.bm1 : a.bm0;  // the dedup bitmap the previous push filled
    for (uint32_t c = gwarp; c * 32 < words; c += nwarps) {
      const uint32_t w = c * 32 + lane;
      const uint32_t bits = w < words ? B[w] : 0u;
      my_bytes += w < words ? 4 : 0;
      if (Sb && bits) Sb[w] = bits;
      uint32_t nz = __ballot_sync(0xffffffffu, bits != 0u);
      // four non-zero words per step: their visit and mask loads in flight together
      while (nz) {
        constexpr int W = 4;
        int v[W];
        bool has[W];
        u64 vis[W], fc[W];
#pragma unroll
        for (int q = 0; q < W; ++q) {
          const int j = nz ? __ffs(nz) - 1 : 0;
          const uint32_t wb = __shfl_sync(0xffffffffu, bits, j);
          has[q] = nz != 0u && ((wb >> lane) & 1u);
          nz &= nz - 1;
          v[q] = (int)((c * 32 + j) * 32 + lane);
          if (has[q]) {
            vis[q] = a.visit[v[q]];
            fc[q] = Fc[v[q]];
          }
        }
#pragma unroll
        for (int q = 0; q < W; ++q) {
          u64 nb = 0;
          if (has[q]) {
            nb = fc[q] & ~vis[q];
            Fc[v[q]] = nb;
            act |= nb;
            my_bytes += 24;  // visit and mask read, mask write
            if (nb) {
              a.visit[v[q]] = vis[q] | nb;
              my_bytes += 8 + (Sk ? 8ull : sizeof(DT) * (unsigned long long)__popcll(nb));
            }
            if (Sk) Sk[v[q]] = nb;
          }
          if (!to_stk) ms_write_rows<DT>(a, v[q], nb, L, lane);
        }
      }
    }
  } else {
    // whole warps walk the queue, so the depth rows can be written by the warp
    const uint32_t n_pad = (n + 31) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += gridDim.x * blockDim.x) {
      int v = -1;
      u64 nb = 0;
      if (i < n) {
        v = Q[i];
        my_bytes += 4;
        ms_apply_vertex<DT>(a, v, Fc, Sk, L, nb, act, my_bytes);
        if (Sb) atomicOr(&Sb[v >> 5], 1u << (v & 31));
      }
      if (!to_stk) ms_write_rows<DT>(a, v, nb, L, lane);
    }
  }
  if (ctl->clear_pending) {
    if (!ctl->apply_pending && L >= 2 && pn >= words / 8) {
      // the previous level ran as a pull, so its dedup bitmap (set by the push
      // before it; level 0's sources have none) still holds its queue: cleared
      // in vertex order, a warp per non-zero word writing the word's 32 entries
      const uint32_t *B = (L & 1) ? a.bm0 : a.bm1;
      for (uint32_t c = gwarp; c * 32 < words; c += nwarps) {
        const uint32_t w = c * 32 + lane;
        my_bytes += w < words ? 4 : 0;
        uint32_t nz = __ballot_sync(0xffffffffu, w < words && B[w] != 0u);
        while (nz) {
          const int j = __ffs(nz) - 1;
          nz &= nz - 1;
          const uint32_t v = (c * 32 + j) * 32 + lane;
          if (v < V) Fp[v] = 0;
          my_bytes += 8;
        }
      }
    } else {
      for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pn; i += gridDim.x * blockDim.x) {
        Fp[Qp[i]] = 0;
        my_bytes += 12;
      }
    }
  }
  add_bytes(ctl, KID_MS_APPLY, my_bytes);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) act |= __shfl_xor_sync(0xffffffffu, act, o);
  if (lane_id() == 0 && act) atomicOr(&ctl->srcmask[L & 1], act);
}

// Push level of the batched BFS, fused (the msbfs_push Program's expand_edge
// and contract with the engine's dedup and compaction): tiles of NV = kNT*VT
// items from the frontier scan's merge-path partition; every thread takes its
// VT items through batches of independent memory operations -- all column
// loads, then all tail-mask and head-visit loads, then the OR of the new
// sources into the heads' next masks (reductions, nothing to wait for) with
// the dedup-bitmap probes, then the test-and-sets -- instead of one dependent
// chain per item; heads that win their dedup bit are compacted into the next
// queue with one reservation per tile.
template <int VT>
__global__ void __launch_bounds__(kNT, 4) k_ms_push(GasArgs<msbfs_push> a) {
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
  uint32_t *dedup = nxt_bm(a, level);
  const int32_t V = a.g.V;
  // the tails' masks: the stack array of a level a pull wrote, else the parity array
  const u64 *Fc = (level < ctl->stk_levels && ((ctl->stk_pull >> level) & 1u)) ? a.vl.stk + (size_t)level * (uint32_t)V
                                                                               : ((level & 1) ? a.vl.F1 : a.vl.F0);
  u64 *Fn = (level & 1) ? a.vl.F0 : a.vl.F1;
  const u64 *visit = a.vl.visit;
  const int32_t *ro = a.g.row_offsets, *col = a.g.col;
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
    int32_t head[VT], tail[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int k = r * kNT + threadIdx.x;
      head[r] = -1;
      tail[r] = 0;
      if (k < cnt) {
        const int j = s_own[k];
        const int el = k - s_base[j] - 1;
        my_bytes += 12;  // column + head visit mask, or a vertex's own item: offsets + queue entry
        if (el >= 0) {
          const int eid = s_rs[j] + el;
          tail[r] = s_v[j];
          if ((unsigned)eid < (unsigned)a.g.E) head[r] = __ldcs(col + eid);
          else raise_error(ctl, MG_ERR_OVERFLOW);
        }
      }
    }
    u64 m[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      m[r] = 0;
      if ((unsigned)head[r] < (unsigned)V) m[r] = __ldg(Fc + tail[r]) & ~__ldg(visit + head[r]);
    }
    uint32_t probe[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      probe[r] = ~0u;
      if (m[r]) {
        atomicOr(&Fn[head[r]], m[r]);  // result unused: a reduction
        probe[r] = ld_volatile(&dedup[head[r] >> 5]);
        my_bytes += 8;
      }
    }
    // the test-and-sets of all VT items in flight together, then the winners'
    // out-degrees, then the ballots (each step waits only once)
    uint32_t old[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const uint32_t bit = 1u << (head[r] & 31);
      old[r] = (m[r] && !(probe[r] & bit)) ? atomicOr(&dedup[head[r] >> 5], bit) : bit;
    }
    int d0[VT], d1[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      d0[r] = d1[r] = 0;
      if (!(old[r] & (1u << (head[r] & 31)))) {
        d0[r] = ro[head[r]];
        d1[r] = ro[head[r] + 1];
      }
    }
    uint32_t bal[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const bool surv = !(old[r] & (1u << (head[r] & 31)));
      if (surv) {
        my_edges += (unsigned long long)(d1[r] - d0[r]);
        my_bytes += 8;  // queue entry + next-mask word
      }
      bal[r] = __ballot_sync(0xffffffffu, surv);
    }
    if (!tile_enqueue<VT>(bal, head, s_cnt, &s_prefix, &s_fail, ordered, a.status, tile, ntiles, epoch, spin_limit,
                          Fout, (uint32_t)V, ctl))
      break;
  }
  add_bytes(ctl, KID_EXPAND, my_bytes);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_edges) atomicAdd(&s_edges, my_edges);
  __syncthreads();
  if (threadIdx.x == 0 && s_edges) atomicAdd(&ctl->next_edges, s_edges);
}

// OR of a 64-bit value over the warp.
MG_DEVINL u64 warp_or(u64 x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// in-edges each pulling list probes lane by lane before the warp sweeps it
// (probing lists of up to 4, 6 or 8 in-edges whole instead was no faster per run
// at R-MAT 22: 5 to 11 us slower on one machine, within 5 us on another)
constexpr int kMsProbe = 2;
constexpr int kMsHeavyK = 4;  // loads per lane and round of a long in-list
constexpr int kMsSub = 4;     // 32-edge sub-chunks whose loads are in flight together

// One 32-edge sub-chunk [ck, ck+32) of a group sweep: lane i holds the
// frontier mask of edge ck+i's tail (0 when not loaded). A segmented inclusive
// OR scan with a head at every non-empty list start in the sub-chunk (and at
// lane 0) leaves the OR of each list's part at its last lane, which the list's
// owner takes when it is still pulling. A step of offset d ORs lane i-d into
// lane i when no head lies in (i-d, i], i.e. when i minus the last head at or
// before i (le = lanes [0, i]) is at least d.
MG_DEVINL void ms_segment(u64 x, int ck, int b, int e, bool starts, bool take, uint32_t le, u64 &acc) {
  const int p = b - ck;
  const uint32_t head = __reduce_or_sync(0xffffffffu, (starts && p >= 0 && p < 32) ? 1u << p : 0u) | 1u;
  if (head == 1u) {
    // no list starts inside the sub-chunk: one list holds all of it (positions
    // past the pulling lists carry 0), so a plain warp OR is its part
    const u64 all = ((u64)__reduce_or_sync(0xffffffffu, (uint32_t)(x >> 32)) << 32) |
                    __reduce_or_sync(0xffffffffu, (uint32_t)x);
    if (take && max(b, ck) < min(e, ck + 32)) acc |= all;
    return;
  }
  // distance from this lane back to the head of its segment: a step of offset
  // d ORs lane i-d in while that lane is still in the segment
  const int run = (31 - __clz(le)) - (31 - __clz(head & le));
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const u64 t = __shfl_up_sync(0xffffffffu, x, d);
    if (run >= d) x |= t;
  }
  const int q = min(e, ck + 32) - 1 - ck;
  const u64 t = __shfl_sync(0xffffffffu, x, q < 0 ? 0 : (q > 31 ? 31 : q));
  if (take && max(b, ck) < min(e, ck + 32)) acc |= t;
}

// Pull level over warp groups of 32 consecutive vertices (lane j owns vertex
// v0+j). A vertex pulls when an active source (ctl->srcmask: a source whose
// frontier is not empty) has not reached it yet. First every pulling lane
// probes the first two in-edges of its own list in one step (the lists are
// hub-first, so after the densest levels the first in-neighbour usually
// carries every missing source); a list that found them all or ended drops
// out. If lists remain, the warp sweeps their contiguous in-edge range in
// rounds of kMsSub x 32 edges from the first unprobed edge (coalesced
// row-index loads, independent mask gathers, a segmented OR scan per
// sub-chunk; an edge probed before may be ORed again, which changes nothing);
// after each round it drops the lists that found every missing source or
// ended, and resumes at the first list still pulling, so the early exit of the
// bottom-up step is kept at round granularity while the loads stay coalesced
// and balanced across lanes. The next masks go to the level stack; past it,
// the new depths of a vertex are written by the whole warp (lane l: sources l
// and l+32 of its row).
template <typename DT>
__global__ void __launch_bounds__(kNT, 6) k_ms_pull(MultiArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_BITMAP) return;
  const uint32_t L = ctl->level;
  const u64 active_src = ctl->srcmask[L & 1] & a.all;
  const u64 *Fc = front_masks(a, ctl, L);
  // next masks: written for every vertex, into the level stack while it has
  // room (the depths are read from it at the end), else into the parity array
  // with the new depths written to the rows
  const bool to_stk = L + 1 < ctl->stk_levels;
  u64 *Fn = to_stk ? stk_level(a, L + 1) : nxt_F(a, L);
  const int32_t V = a.g.V;
  const int32_t *coff = a.g.csc_offsets, *crow = a.g.pull_rows, *ro = a.g.row_offsets;
  const int lane = lane_id();
  const uint32_t le = 0xffffffffu >> (31 - lane);  // lanes [0, lane]
  unsigned long long my_cnt = 0, my_edges = 0, my_bytes = 0;
  u64 act = 0;
  const uint32_t groups = ((uint32_t)V + 31) / 32;
  __shared__ unsigned long long s_tot[3];
  if (threadIdx.x < 3) s_tot[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5, gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  // Long in-lists first, dealt back and forth over the warps in order of length
  // (the groups below skip them). Lane k of a warp takes the warp's k-th list:
  // its visit mask and, when it needs a source, its first kMsProbe in-edges
  // (hub-first lists: usually enough once the densest level is past); the lists
  // still open are then swept by the whole warp, one at a time, in rounds of
  // 32 x kMsHeavyK edges (lane-local ORs, one warp OR per round for the early
  // exit). Every long list's next mask is written here.
  for (uint32_t k0 = 0; k0 * nwarps < (uint32_t)a.nheavy; k0 += 32) {
    const uint32_t k = k0 + lane;
    const uint32_t pos = k * nwarps + ((k & 1) ? nwarps - 1 - gw : gw);
    int hv = -1, hb = 0, he = 0;
    u64 hvis = 0, hneed = 0, hacc = 0;
    if (k * nwarps < (uint32_t)a.nheavy && pos < (uint32_t)a.nheavy) {
      hv = a.heavy[pos];
      hvis = a.visit[hv];
      hneed = active_src & ~hvis;
      hb = coff[hv];
      he = coff[hv + 1];
      my_bytes += 24;  // visit, offsets, next mask
    }
    if (hneed) {
      int u[kMsProbe];
#pragma unroll
      for (int q = 0; q < kMsProbe; ++q) u[q] = __ldcs(crow + hb + q);  // a long list has more than kMsProbe
#pragma unroll
      for (int q = 0; q < kMsProbe; ++q) hacc |= __ldg(&Fc[u[q]]);
      my_bytes += 12ull * kMsProbe;
    }
    bool open = hneed != 0ull && (hacc & hneed) != hneed;
    for (uint32_t todo = __ballot_sync(0xffffffffu, open); todo; todo &= todo - 1) {
      const int j = __ffs(todo) - 1;
      const u64 need = __shfl_sync(0xffffffffu, hneed, j);
      const int e = __shfl_sync(0xffffffffu, he, j);
      u64 all = __shfl_sync(0xffffffffu, hacc, j);
      unsigned long long probes = 0;
      for (int c = __shfl_sync(0xffffffffu, hb, j) + kMsProbe; c < e; c += 32 * kMsHeavyK) {
        int uu[kMsHeavyK];
#pragma unroll
        for (int q = 0; q < kMsHeavyK; ++q) {
          const int i = c + 32 * q + lane;
          uu[q] = i < e ? __ldcs(crow + i) : -1;
        }
        u64 x = 0;
#pragma unroll
        for (int q = 0; q < kMsHeavyK; ++q)
          if (uu[q] >= 0) {
            x |= __ldg(&Fc[uu[q]]);
            ++probes;
          }
        all |= ((u64)__reduce_or_sync(0xffffffffu, (uint32_t)(x >> 32)) << 32) |
               __reduce_or_sync(0xffffffffu, (uint32_t)x);
        if ((all & need) == need) break;
      }
      my_bytes += 12ull * probes;
      if (lane == j) hacc = all;
    }
    const u64 hfound = hacc & hneed;
    if (hv >= 0) {
      Fn[hv] = hfound;
      if (hfound) {
        my_bytes += 8 + (to_stk ? 0ull : sizeof(DT) * (unsigned long long)__popcll(hfound));
        a.visit[hv] = hvis | hfound;
        my_cnt += 1;
        my_edges += (unsigned long long)(ro[hv + 1] - ro[hv]);
        act |= hfound;
      }
    }
    if (!to_stk) ms_write_rows<DT>(a, hv, hfound, L + 1, lane);
  }
  // 32-vertex groups, dealt round-robin over the grid's warps: an atomic ticket
  // per group on one shared counter cost more than the imbalance it removed
  // (batched step 2.16 vs 2.08 ms on R-MAT 22, 4.69 vs 4.42 ms on the road grid)
  for (uint32_t grp = gw; grp < groups; grp += nwarps) {
    const int v0 = (int)(grp * 32);
    const int v = v0 + lane;
    const bool valid = v < V;
    const u64 vis = valid ? a.visit[v] : ~0ull;
    const u64 need = active_src & ~vis;
    const int b = valid ? coff[v] : 0, e = valid ? coff[v + 1] : 0;
    const bool own = valid && e - b <= kMsHeavyList;  // a long list is pulled above
    my_bytes += own ? 16 : 0;  // visit read + next-mask write
    const bool pulls = own && need != 0 && e > b;
    u64 acc = 0;
    unsigned long long probes = 0;
    bool open = pulls;
    int bs = b;  // first in-edge of the list not probed yet
    // one probe step: the first kMsProbe in-edges of every list that takes
    // part, the loads in flight together
    if (__any_sync(0xffffffffu, open)) {
      const int lim = min(e, b + kMsProbe);
      int u[kMsProbe];
#pragma unroll
      for (int k = 0; k < kMsProbe; ++k) u[k] = (open && bs + k < lim) ? __ldcs(crow + bs + k) : -1;
#pragma unroll
      for (int k = 0; k < kMsProbe; ++k)
        if (u[k] >= 0) acc |= __ldg(&Fc[u[k]]);
      if (open) {
        probes += (unsigned long long)(lim - bs);
        bs = lim;
        open = (acc & need) != need && bs < e;
      }
    }
    uint32_t pending = __ballot_sync(0xffffffffu, open);
    if (pending) {
      const bool starts = valid && e > b;
      int c = __shfl_sync(0xffffffffu, bs, __ffs(pending) - 1);
      for (;;) {
        // one round from c; nothing past the last pulling list is loaded
        const int lim = __shfl_sync(0xffffffffu, e, 31 - __clz(pending));
        u64 x[kMsSub];
#pragma unroll
        for (int k = 0; k < kMsSub; ++k) {
          const int i = c + 32 * k + lane;
          x[k] = 0;
          if (i < lim) {
            x[k] = __ldg(&Fc[__ldcs(crow + i)]);
            ++probes;
          }
        }
#pragma unroll
        for (int k = 0; k < kMsSub; ++k)
          if (c + 32 * k < lim) ms_segment(x[k], c + 32 * k, b, e, starts, (pending >> lane) & 1u, le, acc);
        c += kMsSub * 32;
        // keep the lists that still miss a source and have edges left
        pending = __ballot_sync(0xffffffffu, ((pending >> lane) & 1u) && (acc & need) != need && e > c);
        if (!pending) break;
        c = max(c, __shfl_sync(0xffffffffu, bs, __ffs(pending) - 1));
      }
    }
    my_bytes += pulls ? 8 + 12ull * probes : 0;  // offsets; row index + mask per probe
    acc &= need;
    if (own) Fn[v] = acc;
    if (acc) {
      my_bytes += 8 + (to_stk ? 0ull : sizeof(DT) * (unsigned long long)__popcll(acc));  // visit write (+ depths)
      a.visit[v] = vis | acc;
      my_cnt += 1;
      my_edges += (unsigned long long)(ro[v + 1] - ro[v]);
      act |= acc;
    }
    if (to_stk) continue;
    uint32_t wv = __ballot_sync(0xffffffffu, acc != 0);
    while (wv) {
      const int j = __ffs(wv) - 1;
      wv &= wv - 1;
      const u64 m = __shfl_sync(0xffffffffu, acc, j);
      DT *row = depth_rows<DT>(a) + (int64_t)(v0 + j) * 64;
      if ((m >> lane) & 1ull) row[lane] = (DT)(L + 1);
      if ((m >> (lane + 32)) & 1ull) row[lane + 32] = (DT)(L + 1);
    }
  }
  add_bytes(ctl, KID_MS_PULL, my_bytes);
  // totals per CTA, then one atomic per CTA and counter on the control block
  act = warp_or(act);
  my_cnt = warp_sum(my_cnt);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && act) atomicOr(&s_tot[0], act);
  if (lane == 0 && my_cnt) atomicAdd(&s_tot[1], my_cnt);
  if (lane == 0 && my_edges) atomicAdd(&s_tot[2], my_edges);
  __syncthreads();
  if (threadIdx.x == 0 && s_tot[0]) atomicOr(&ctl->srcmask[(L + 1) & 1], s_tot[0]);
  if (threadIdx.x == 0 && s_tot[1]) atomicAdd((unsigned long long *)&ctl->acc[0], s_tot[1]);
  if (threadIdx.x == 0 && s_tot[2]) atomicAdd(&ctl->next_edges, s_tot[2]);
}

// Pull -> push: compaction of the vertices with a non-empty mask into
// the queue; clears both dedup bitmaps and, when the previous level's masks
// went to the parity array for every vertex (past the level stack), that array,
// which the push writes into next. Within the stack the parity arrays are
// already zero: push-made entries are cleared after use (k_ms_apply).
// A CTA takes tiles of 4096 vertices: warp w covers 512 consecutive vertices
// with 16 coalesced mask loads in flight per lane; within a tile the queue
// follows vertex order (ballots within the warp, a scan over the CTA's warps),
// and each tile reserves its range with one atomic (an ordered look-back over
// the tiles cost 12 us more per batched BFS at R-MAT 22). The last CTA to
// finish publishes the queue length.
constexpr int kCvK = 16;  // vertices per lane and tile
__global__ void __launch_bounds__(kNT) k_ms_convert(MultiArgs a) {
  constexpr uint32_t TV = kNT * kCvK;
  __shared__ uint32_t s_w[kNW];
  __shared__ uint32_t s_tile, s_last;
  Ctl *ctl = a.ctl;
  if (!ctl->active || !ctl->convert) return;
  const uint32_t L = ctl->level;
  const uint32_t V = (uint32_t)a.g.V;
  const u64 *Fc = front_masks(a, ctl, L);
  u64 *Fo = (L - 1 >= ctl->stk_levels) ? nxt_F(a, L) : nullptr;
  int32_t *Q = cur_Q(a, L);
  const uint32_t words = (V + 31) / 32;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    a.bm0[w] = 0;
    a.bm1[w] = 0;
  }
  const uint32_t ntiles = (V + TV - 1) / TV;
  const int lane = lane_id(), warp = warp_id();
  for (;;) {
    const uint32_t tile = next_tile(&ctl->tile_ctr[3], &s_tile);
    if (tile >= ntiles) break;
    const uint32_t wb = tile * TV + (uint32_t)warp * (32u * kCvK);  // the warp's first vertex
    u64 f[kCvK];
#pragma unroll
    for (int k = 0; k < kCvK; ++k) {
      const uint32_t v = wb + 32u * k + lane;
      f[k] = v < V ? Fc[v] : 0ull;
    }
    uint32_t bal[kCvK], wtot = 0;
#pragma unroll
    for (int k = 0; k < kCvK; ++k) {
      bal[k] = __ballot_sync(0xffffffffu, f[k] != 0ull);
      wtot += __popc(bal[k]);
      const uint32_t v = wb + 32u * k + lane;
      if (Fo && v < V) Fo[v] = 0;
    }
    if (lane == 0) s_w[warp] = wtot;
    __syncthreads();
    if (warp == 0) {
      const uint32_t x = lane < kNW ? s_w[lane] : 0u;
      const uint32_t inc = warp_inclusive_sum(x);
      const uint32_t tot = __shfl_sync(0xffffffffu, inc, kNW - 1);
      uint32_t pre = 0;
      if (lane == 0 && tot) pre = atomicAdd(&ctl->next_size, tot);
      pre = __shfl_sync(0xffffffffu, pre, 0);
      if (lane < kNW) s_w[lane] = pre + inc - x;  // queue position of each warp's first vertex
    }
    __syncthreads();
    uint32_t pos = s_w[warp];
#pragma unroll
    for (int k = 0; k < kCvK; ++k) {
      if ((bal[k] >> lane) & 1u) {
        const uint32_t q = pos + __popc(bal[k] & lanemask_lt());
        if (q < V) Q[q] = (int32_t)(wb + 32u * k + lane);
      }
      pos += __popc(bal[k]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ctl->done_ctas[3], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    ctl->frontier_size = *(volatile uint32_t *)&ctl->next_size;
    ctl->next_size = 0;
    ctl->done_ctas[3] = 0;
  }
}

__global__ void k_ms_level_end(Ctl *ctl, int32_t V, int64_t E, cudaGraphConditionalHandle h, int use_handle) {
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
    uint32_t new_mode = mode;
    if (ctl->dir_policy == MG_DIR_PUSH) {
      new_mode = MODE_QUEUE;
    } else if (ctl->dir_policy == MG_DIR_PULL) {
      new_mode = MODE_BITMAP;
    } else if (mode == MODE_QUEUE) {
      if ((double)m_next > (double)E / (double)ctl->alpha) new_mode = MODE_BITMAP;
    } else {
      if ((double)n_next < (double)V / (double)ctl->beta && n_next < ctl->frontier_size) new_mode = MODE_QUEUE;
    }
    ctl->srcmask[ctl->level & 1] = 0;  // consumed; the level after next accumulates it afresh
    // this level's parity masks, when a push (or the sources, at level 0) made
    // them, are cleared at its queue entries at the start of the next level
    ctl->clear_pending = (mode == MODE_QUEUE || ctl->apply_pending || ctl->level == 0) ? 1u : 0u;
    if (mode == MODE_BITMAP && ctl->level + 1 < ctl->stk_levels) ctl->stk_pull |= 1u << (ctl->level + 1);
    ctl->apply_pending = (mode == MODE_QUEUE) ? 1u : 0u;
    ctl->convert = (mode == MODE_BITMAP && new_mode == MODE_QUEUE) ? 1u : 0u;
    ctl->mode = new_mode;
    ctl->prev_size = ctl->frontier_size;
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

// [V][64] -> [ns][V] for sources s_begin .. s_begin+ns-1, widening uint16
// depth rows to int32. A CTA walks tiles of kTrV vertices (grid-stride):
// 16-byte loads of the rows into shared memory, then each source's kTrV results
// leave as 128-byte coalesced stores; the next tile's loads are in flight while
// the current tile is written out. With `visit` given (batched BFS), an entry
// whose visit bit is clear is unreached: it comes out as -1, and its slot,
// which the traversal never wrote, is not read (a 16-byte piece with no bits
// set is not read at all).
template <typename T>
struct TrShape {
  static constexpr int kV = sizeof(T) == 2 ? 128 : 64;  // vertices per tile (4 KB of each row type in flight)
  static constexpr int kPer = 16 / (int)sizeof(T);     // entries per 16-byte piece
  static constexpr int kPieces = 64 / kPer;            // pieces per row
  static constexpr int kQ = kV * kPieces / 256;        // pieces per thread per tile
};

template <typename T>
MG_DEVINL void tr_load(const T *in, const u64 *visit, int32_t V, int64_t v0, int4 (&q)[TrShape<T>::kQ],
                       uint32_t (&qb)[TrShape<T>::kQ]) {
  constexpr int PER = TrShape<T>::kPer, PIECES = TrShape<T>::kPieces;
  constexpr uint32_t FULL = (1u << PER) - 1u;
#pragma unroll
  for (int k = 0; k < TrShape<T>::kQ; ++k) {
    const int idx = threadIdx.x + 256 * k, r = idx / PIECES, c = idx % PIECES;
    const int64_t v = v0 + r;
    uint32_t bits = 0;
    if (v < V) bits = visit ? (uint32_t)(visit[v] >> (PER * c)) & FULL : FULL;
    qb[k] = bits;
    q[k] = bits ? *reinterpret_cast<const int4 *>(in + v * 64 + PER * c) : make_int4(0, 0, 0, 0);
  }
}

// entry i (< 16 / sizeof(T)) of a 16-byte piece, widened to int32
template <typename T>
MG_DEVINL int32_t tr_entry(const int4 &q, int i) {
  const uint32_t w[4] = {(uint32_t)q.x, (uint32_t)q.y, (uint32_t)q.z, (uint32_t)q.w};
  if (sizeof(T) == 4) return (int32_t)w[i];
  return (int32_t)((w[i >> 1] >> (16 * (i & 1))) & 0xffffu);
}

template <typename T>
__global__ void __launch_bounds__(256, 6) k_ms_transpose(const T *in, const u64 *visit, int32_t *out, int32_t V,
                                                      int32_t s_begin, int32_t ns) {
  constexpr int PER = TrShape<T>::kPer, PIECES = TrShape<T>::kPieces, Q = TrShape<T>::kQ, kTrV = TrShape<T>::kV;
  __shared__ int32_t t[kTrV][65];
  const int64_t ntiles = ((int64_t)V + kTrV - 1) / kTrV;
  const int lane = lane_id(), warp = warp_id();
  int4 q[Q];
  uint32_t qb[Q];
  int64_t tile = blockIdx.x;
  if (tile < ntiles) tr_load<T>(in, visit, V, tile * kTrV, q, qb);
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t v0 = tile * kTrV;
    __syncthreads();  // the previous tile has been written out of t
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int idx = threadIdx.x + 256 * k, r = idx / PIECES, c = PER * (idx % PIECES);
#pragma unroll
      for (int i = 0; i < PER; ++i) t[r][c + i] = ((qb[k] >> i) & 1u) ? tr_entry<T>(q[k], i) : -1;
    }
    __syncthreads();
    if (tile + gridDim.x < ntiles) tr_load<T>(in, visit, V, (tile + gridDim.x) * kTrV, q, qb);
    for (int seg = warp; seg < ns * (kTrV / 32); seg += kNW) {
      const int s = seg / (kTrV / 32), r = (seg % (kTrV / 32)) * 32 + lane;
      if (v0 + r < V) __stcs(out + (int64_t)s * V + v0 + r, t[r][s_begin + s]);
    }
  }
}

// Batched BFS depths from the level stack to the caller's int32 [ns][V]
// layout: the depth of (v, s) is the level L whose stack mask at v holds bit s
// (a level a pull wrote is valid for every vertex; a push-made level only where
// its bitmap says so), else, for levels past the stack, the uint16 depth row;
// -1 where the visit mask lacks bit s. The stack's extent comes from the
// control block, so the kernel can run as the level loop's epilogue.
//
// A warp takes 32 consecutive vertices, one per lane. It loads the valid-entry
// words and then the masks of up to eight levels at once and folds them into
// four bit planes of the depth (plane b holds source s when bit b of its level
// is set) and the found mask. Each lane then turns the planes into depth bytes,
// four sources at a time (a 4-bit piece of a plane times 0x00204081 puts its
// bits 8 apart, as the four partial products do not overlap; sources not found
// get 0xff), and stores them into the warp's [64][32] byte tile in shared
// memory; the tile leaves as 16-byte stores of four vertices of one source,
// each byte sign-extended (0xff -> -1), a 128-byte row segment per source,
// marked evict-first (the 1 GiB output is not read again here: 20 us less per
// run at R-MAT 22 than plain stores).
// Sources reached past the stack are rewritten from the depth rows afterwards.
constexpr int kTsBatch = 8;  // stack levels whose loads are in flight together
static_assert(kMsStackLevels == 2 * kTsBatch, "two load batches cover the stack");

template <int B>
MG_DEVINL void ts_fold(const u64 *stk, const uint32_t *stk_bm, uint32_t words, uint32_t nst, uint32_t full, int32_t V,
                       uint32_t grp, int64_t v, bool in, int lane, u64 (&p)[4], u64 &found) {
  uint32_t bw[kTsBatch];
#pragma unroll
  for (int k = 0; k < kTsBatch; ++k) {
    const uint32_t L = B * kTsBatch + k;
    bw[k] = 0;
    if (L < nst) bw[k] = ((full >> L) & 1u) ? ~0u : __ldg(&stk_bm[(size_t)L * words + grp]);
  }
  u64 m[kTsBatch];
#pragma unroll
  for (int k = 0; k < kTsBatch; ++k) {
    const uint32_t L = B * kTsBatch + k;
    m[k] = (in && ((bw[k] >> lane) & 1u)) ? __ldcs(&stk[(size_t)L * (uint32_t)V + v]) : 0ull;
  }
#pragma unroll
  for (int k = 0; k < kTsBatch; ++k) {
    const int L = B * kTsBatch + k;
    found |= m[k];
    if (L & 1) p[0] |= m[k];
    if (L & 2) p[1] |= m[k];
    if (L & 4) p[2] |= m[k];
    if (L & 8) p[3] |= m[k];
  }
}

// bits 0..3 of x moved to bits 0, 8, 16, 24
MG_DEVINL uint32_t spread4(uint32_t x) { return ((x & 0xfu) * 0x00204081u) & 0x01010101u; }
// byte k of x as a signed value
MG_DEVINL int32_t sbyte(uint32_t x, int k) { return (int32_t)(int8_t)(uint8_t)(x >> (8 * k)); }

__global__ void __launch_bounds__(256) k_ms_transpose_stk(const u64 *stk, const uint32_t *stk_bm, uint32_t words,
                                                       const uint16_t *rows, const u64 *visit, const Ctl *ctl,
                                                       int32_t *out, int32_t V, int32_t ns) {
  __shared__ uint32_t tile[kNW][64][8];  // per warp: [source][32 vertices as 8 words of 4 depth bytes]
  const uint32_t nst = min(ctl->level + 1, ctl->stk_levels);  // stack levels this run produced
  const uint32_t full = ctl->stk_pull;
  const uint32_t groups = ((uint32_t)V + 31) / 32;
  const int lane = lane_id(), warp = warp_id();
  const bool vec = (V & 3) == 0;  // every source row starts 16-byte aligned
  uint8_t *tb = reinterpret_cast<uint8_t *>(tile[warp]);
  // The CTA takes 8 consecutive groups at a time and its warps start each step
  // together, so the grid's stores move through every source row as one narrow
  // front (with the warps on their own, 6 to 11 us slower per run at R-MAT 22
  // and 17 us slower in a cold capture; four consecutive groups per warp, a
  // wider front, 35 us slower).
  for (uint32_t base = blockIdx.x * kNW; base < groups; base += gridDim.x * kNW) {
    __syncthreads();  // every warp of the CTA runs the same steps
    const uint32_t grp = base + warp;
    if (grp >= groups) continue;
    const int64_t v = (int64_t)grp * 32 + lane;
    const bool in = v < V;
    const u64 vis = in ? __ldcs(&visit[v]) : 0ull;
    u64 p[4] = {0, 0, 0, 0}, found = 0;
    ts_fold<0>(stk, stk_bm, words, nst, full, V, grp, v, in, lane, p, found);
    if (nst > kTsBatch) ts_fold<1>(stk, stk_bm, words, nst, full, V, grp, v, in, lane, p, found);
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      const uint32_t q0 = (uint32_t)(p[0] >> (32 * hf)), q1 = (uint32_t)(p[1] >> (32 * hf));
      const uint32_t q2 = (uint32_t)(p[2] >> (32 * hf)), q3 = (uint32_t)(p[3] >> (32 * hf));
      const uint32_t nf = ~(uint32_t)(found >> (32 * hf));
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        const int sh = 4 * w;
        const uint32_t b = spread4(q0 >> sh) | (spread4(q1 >> sh) << 1) | (spread4(q2 >> sh) << 2) |
                           (spread4(q3 >> sh) << 3) | (spread4(nf >> sh) * 0xffu);
        const int s0 = 32 * hf + sh;
#pragma unroll
        for (int k = 0; k < 4; ++k) tb[(s0 + k) * 32 + lane] = (uint8_t)(b >> (8 * k));
      }
    }
    __syncwarp();
    // lane l writes vertices 4(l%8) .. 4(l%8)+3 of sources l/8, l/8+4, ...
    const int64_t vb = (int64_t)grp * 32 + 4 * (lane & 7);
#pragma unroll 4
    for (int s = lane >> 3; s < ns; s += 4) {
      const uint32_t x = tile[warp][s][lane & 7];
      int32_t *o = out + (int64_t)s * V + vb;
      if (vec && vb + 3 < V) {
        __stcs(reinterpret_cast<int4 *>(o), make_int4(sbyte(x, 0), sbyte(x, 1), sbyte(x, 2), sbyte(x, 3)));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (vb + k < V) __stcs(o + k, sbyte(x, k));
      }
    }
    // sources reached past the stack: their depths from the rows, over the -1
    // just written (ordered after it by the warp barrier)
    const u64 deep = vis & ~found;
    if (__any_sync(0xffffffffu, deep != 0ull)) {
      __syncwarp();
      for (u64 x = deep; x; x &= x - 1) {
        const int s = __ffsll((long long)x) - 1;
        if (s < ns) out[(int64_t)s * V + v] = (int32_t)rows[v * 64 + s];
      }
    }
    __syncwarp();  // the tile is rewritten by the next group
  }
}

// The level stack and the uint16 depth rows of a batched BFS inside multi_out.
static u64 *stack_of(mg_graph *g) { return reinterpret_cast<u64 *>(g->multi_out); }
static uint16_t *rows16_of(mg_graph *g) {
  return reinterpret_cast<uint16_t *>(stack_of(g) + (size_t)kMsStackLevels * (size_t)g->csr.V);
}

// Transposes a run's results to the caller's [nsrc][V] int32 layout on stream
// s: from the level stack and uint16 rows (stack), else from int32 rows.
static void launch_transpose(mg_graph *g, bool stack, const u64 *visit, int32_t *out, int32_t nsrc, cudaStream_t s) {
  const int32_t V = g->csr.V;
  // vertices per CTA and resident CTAs per SM (the stack variant: 8 warps of 32
  // vertices, 64 registers, 4 CTAs per SM: 2 leave too few loads in flight, 60 us
  // more per run at R-MAT 22, and 3 were no faster; the row variant: 6 CTAs fit)
  const int kv = stack ? 256 : TrShape<int32_t>::kV, per_sm = stack ? 4 : 6;
  const unsigned nblk = (unsigned)std::min<int64_t>((int64_t)g->num_sms * per_sm, ((int64_t)V + kv - 1) / kv);
  if (stack)
    k_ms_transpose_stk<<<nblk, 256, 0, s>>>(stack_of(g), g->multi_stk_bm, (uint32_t)((V + 31) / 32), rows16_of(g),
                                            visit, g->ws.ctl, out, V, nsrc);
  else
    k_ms_transpose<int32_t><<<nblk, 256, 0, s>>>(g->multi_out, visit, out, V, 0, nsrc);
  count_launch();
}

// Reached (vertex, source) pairs and the out-edges of their vertices, from the
// visit masks of a batched BFS.
__global__ void k_ms_mask_stats(const u64 *visit, u64 all, const int32_t *ro, int32_t V, unsigned long long *out) {
  unsigned long long cnt = 0, edg = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long c = (unsigned long long)__popcll(visit[v] & all);
    cnt += c;
    edg += c * (unsigned long long)(ro[v + 1] - ro[v]);
  }
  cnt = warp_sum(cnt);
  edg = warp_sum(edg);
  if (lane_id() == 0) {
    atomicAdd(&out[0], cnt);
    atomicAdd(&out[1], edg);
  }
}

// ------------------------------------------------------------ batched SSSP --
struct mssp_scan {
  typedef int DataType;
  typedef int MiscType;
  typedef int GatherType;
  typedef int VertexId;
  typedef int SizeT;
  struct VertexType {
    int nodes;
  };
  struct EdgeType {
    int nodes;
  };
  struct expand_vertex {
    __device__ bool operator()(const int, const char, VertexType &, EdgeType &) { return true; }
  };
};

// Clears the previous level's masks (they were read by the previous expand).
__global__ void __launch_bounds__(kNT) k_mss_clear(MultiArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level, pn = ctl->prev_size;
  u64 *Fp = nxt_F(a, L);
  const int32_t *Qp = nxt_Q(a, L);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pn; i += gridDim.x * blockDim.x) Fp[Qp[i]] = 0;
}

// Lowers a distance entry to c (a fire-and-forget reduction: nothing waits for
// the old value) and marks source t improved. The caller saw c below the entry
// it loaded: if another relaxation lowered the entry further in between, the
// mark is spurious and costs one extra expansion of (v, t) next level, but every
// reduction that does lower an entry is marked by its own thread, so the
// fixpoint is unchanged.
MG_DEVINL void relax_min(int32_t *p, int32_t c, u64 &imp, int t) {
  atomicMin(p, c);
  imp |= 1ull << t;
}

template <int VT>
__global__ void __launch_bounds__(kNT) k_mss_expand(MultiArgs a, const uint32_t *scan, const int32_t *part) {
  constexpr int NV = kNT * VT;
  constexpr int PER_WARP = NV / kNW;
  __shared__ int32_t s_v[NV + 1];
  __shared__ int32_t s_base[NV + 1];
  __shared__ int32_t s_rs[NV + 1];
  __shared__ int32_t s_own[NV];
  __shared__ int32_t s_q[NV];  // per warp: its queued vertices of the current tile
  __shared__ uint32_t s_tile;
  __shared__ int s_fail;
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level, n = ctl->frontier_size, total = ctl->edge_total, ntiles = ctl->exp_tiles;
  const unsigned long long items = (unsigned long long)n + total;
  const int32_t *Q = cur_Q(a, L);
  int32_t *Qn = nxt_Q(a, L);
  const u64 *Fc = cur_F(a, L);
  u64 *Fn = nxt_F(a, L);
  uint32_t *dedup = (L & 1) ? a.bm0 : a.bm1;
  const int32_t *ro = a.g.row_offsets, *col = a.g.col, *wgt = a.g.wgt;
  const int32_t V = a.g.V;
  const int lane = lane_id(), warp = warp_id();
  unsigned long long my_bytes = 0;
  if (threadIdx.x == 0) s_fail = 0;
  for (;;) {
    const uint32_t tile = next_tile(&ctl->tile_ctr[1], &s_tile);
    if (tile >= ntiles || s_fail) break;
    int cnt;
    if (!decode_tile<VT>(tile, ntiles, n, items, part, scan, Q, ro, s_v, s_base, s_rs, s_own, &cnt,
                         [](int, int) {})) {
      if (threadIdx.x == 0) {
        raise_error(ctl, MG_ERR_OVERFLOW);
        s_fail = 1;
      }
      __syncthreads();
      break;
    }
    // The warp takes its items 32 at a time; lane i loads item k+i's edge (tail,
    // head, weight, tail's source mask), the next batch while the current one
    // is relaxed. If every edge of the batch carries at most kMssSparse active
    // sources, each lane relaxes its own edge source by source (scalar loads
    // from the two 256-byte rows); otherwise the batch goes four edges per
    // step, the 8 lanes of group g owning sources 8*sub .. 8*sub+7 of edge
    // 4q+g, read with two 16-byte loads from each row.
    const int k0 = warp * PER_WARP;
    const int k1 = min(cnt, k0 + PER_WARP);
    const int grp = lane >> 3, sub = lane & 7;
    auto fetch = [&](int k, int &u, int &v, int &w, u64 &am) {
      u = -1;
      if (k >= k1) return;
      const int j = s_own[k];
      const int el = k - s_base[j] - 1;
      if (el < 0) return;
      const int eid = s_rs[j] + el;
      if ((unsigned)eid >= (unsigned)a.g.E) {
        raise_error(ctl, MG_ERR_OVERFLOW);
        return;
      }
      u = s_v[j];
      v = __ldcs(col + eid);
      w = __ldcs(wgt + eid);
      am = Fc[u];
    };
    // next-level mask and dedup bit of the vertices that improved; the ones
    // that won the dedup bit are staged in the warp's part of s_q (an item
    // queues at most one vertex, so PER_WARP slots suffice) and reserved in the
    // queue once per warp and tile (a reservation per step was a same-address
    // atomic for every 32 or 4 edges)
    int32_t *wq = s_q + warp * PER_WARP;
    int qn = 0;  // warp-uniform
    auto enqueue = [&](bool has, int v, u64 mask) {
      bool enq = false;
      if (has) {
        my_bytes += 8 + 4ull * (unsigned long long)__popcll(mask);
        atomicOr(&Fn[v], mask);
        const uint32_t bit = 1u << (v & 31);
        enq = !(ld_volatile(&dedup[v >> 5]) & bit) && !(atomicOr(&dedup[v >> 5], bit) & bit);
      }
      const uint32_t eb = __ballot_sync(0xffffffffu, enq);
      if (enq) {
        const int pos = qn + __popc(eb & lanemask_lt());
        if (pos < PER_WARP) wq[pos] = v;
        else raise_error(ctl, MG_ERR_OVERFLOW);
      }
      qn = min(qn + __popc(eb), PER_WARP);
    };
    int nu = -1, nv = 0, nw = 0;
    u64 nam = 0;
    fetch(k0 + lane, nu, nv, nw, nam);
    for (int kb = k0; kb < k1; kb += 32) {
      const int bu = nu, bv = nv, bw = nw;
      const u64 bam = nam;
      fetch(kb + 32 + lane, nu, nv, nw, nam);
      if (bu >= 0) my_bytes += 16 + 8ull * (unsigned long long)__popcll(bam);
      if (__all_sync(0xffffffffu, bu < 0 || __popcll(bam) <= kMssSparse)) {
        u64 imp = 0;
        if (bu >= 0) {
          const int32_t *du = a.out + (int64_t)bu * 64;
          int32_t *dv = a.out + (int64_t)bv * 64;
          // four active sources per step, their row entries loaded together
          for (u64 m = bam; m;) {
            int t[4], du4[4], dv4[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              t[q] = m ? __ffsll((long long)m) - 1 : -1;
              m &= m - 1;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (t[q] >= 0) {
                du4[q] = __ldcg(du + t[q]);
                dv4[q] = __ldcg(dv + t[q]);
              }
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (t[q] >= 0 && du4[q] + bw < dv4[q]) relax_min(dv + t[q], du4[q] + bw, imp, t[q]);
          }
        }
        enqueue(imp != 0, bv, imp);
        continue;
      }
#pragma unroll 1
      for (int q = 0; q < 8; ++q) {
        const int src = 4 * q + grp;
        const int u = __shfl_sync(0xffffffffu, bu, src), v = __shfl_sync(0xffffffffu, bv, src);
        const int w = __shfl_sync(0xffffffffu, bw, src);
        const u64 am = __shfl_sync(0xffffffffu, bam, src);
        uint32_t imp = 0;
        const uint32_t bits = u >= 0 ? (uint32_t)(am >> (8 * sub)) & 0xffu : 0u;
        if (bits) {
          const int4 *pu = reinterpret_cast<const int4 *>(a.out + (int64_t)u * 64 + 8 * sub);
          int32_t *dvp = a.out + (int64_t)v * 64 + 8 * sub;
          const int4 *pv = reinterpret_cast<const int4 *>(dvp);
          const int4 u0 = __ldcg(pu), u1 = __ldcg(pu + 1), v0 = __ldcg(pv), v1 = __ldcg(pv + 1);
          const int du[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
          const int dv[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            if (((bits >> t) & 1u) && du[t] + w < dv[t]) {
              atomicMin(&dvp[t], du[t] + w);  // result unused: a reduction (see relax_min)
              imp |= 1u << t;
            }
          }
        }
        // improved sources of the group's edge: OR of the 8 lanes' byte masks
        u64 mask = (u64)imp << (8 * sub);
        mask |= __shfl_xor_sync(0xffffffffu, mask, 1);
        mask |= __shfl_xor_sync(0xffffffffu, mask, 2);
        mask |= __shfl_xor_sync(0xffffffffu, mask, 4);
        enqueue(sub == 0 && mask != 0, v, mask);
      }
    }
    __syncwarp();
    if (qn) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&ctl->next_size, (uint32_t)qn);
      base = __shfl_sync(0xffffffffu, base, 0);
      for (int i = lane; i < qn; i += 32) {
        if (base + (uint32_t)i < (uint32_t)V) Qn[base + i] = wq[i];
        else raise_error(ctl, MG_ERR_OVERFLOW);
      }
    }
  }
  add_bytes(ctl, KID_MSS_EXPAND, my_bytes);
}

__global__ void k_mss_level_end(Ctl *ctl, cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x != 0) return;
  if (ctl->active) {
    ctl->prev_size = ctl->frontier_size;
    ctl->level += 1;
    ctl->push_levels += 1;
    ctl->frontier_size = ctl->next_size;
    ctl->next_size = 0;
    ctl->edge_total = 0;
    ctl->exp_tiles = 0;
    ctl->epoch += 4;
    for (int i = 0; i < 4; ++i) ctl->tile_ctr[i] = 0;
    ctl->active = (ctl->frontier_size > 0 && ctl->level < ctl->max_iter && ctl->error == 0) ? 1u : 0u;
  }
  if (use_handle) cudaGraphSetConditional(h, ctl->active);
}

static MultiArgs multi_args(mg_graph *g) {
  MultiArgs a;
  a.g = g->csr;
  a.visit = g->mask[0];
  a.F0 = g->mask[1];
  a.F1 = g->mask[2];
  a.out = g->multi_out;
  a.rows = g->multi_out;
  a.stk = nullptr;
  a.stk_bm = g->multi_stk_bm;
  a.stk_words = (uint32_t)((g->csr.V + 31) / 32);
  a.heavy = g->ms_heavy;
  a.nheavy = std::max(g->ms_nheavy, 0);
  a.q0 = g->ws.queue[0];
  a.q1 = g->ws.queue[1];
  a.bm0 = g->ws.bm[0];
  a.bm1 = g->ws.bm[1];
  a.status = g->ws.status;
  a.ctl = g->ws.ctl;
  a.all = 0;
  return a;
}

static int multi_prepare(mg_graph *g, const int32_t *srcs, int32_t nsrc, const mg_options *o, cudaStream_t s,
                         SrcList *list, int32_t fill, bool stack = false) {
  if (nsrc < 1 || nsrc > 64) return set_error(MG_ERR_ARG, "nsrc must be in [1, 64]");
  std::vector<int32_t> distinct;
  int st = check_sources(g, srcs, nsrc, &distinct);
  if (st != MG_OK) return st;
  memset(list, 0, sizeof(*list));
  std::copy(srcs, srcs + nsrc, list->src);
  std::copy(distinct.begin(), distinct.end(), list->distinct);
  list->nsrc = nsrc;
  list->ndistinct = (int32_t)distinct.size();
  if ((st = ensure_workspace(g)) != MG_OK) return st;
  if ((st = ensure_multi(g)) != MG_OK) return st;
  if ((st = prepare_run(g, s)) != MG_OK) return st;
  const size_t V = (size_t)g->nodes;
  cudaError_t e = cudaMemsetAsync(g->mask[0], 0, V * 8, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->mask[1], 0, V * 8, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->mask[2], 0, V * 8, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.bm[0], 0, g->ws.words * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->ws.bm[1], 0, g->ws.words * 4, s);
  // valid-entry bitmaps of the stack levels a push makes
  if (e == cudaSuccess && stack)
    e = cudaMemsetAsync(g->multi_stk_bm, 0, (size_t)kMsStackLevels * ((V + 31) / 32) * 4, s);
  if ((st = cuda_status(e, "batched init")) != MG_OK) return st;
  // batched BFS leaves the depth rows unset: the visit masks say which entries
  // were written; batched SSSP relaxes with atomicMin from `fill`
  if (fill != -1) {
    k_fill_i32<<<g->num_sms * 8, 256, 0, s>>>(g->multi_out, fill, (int64_t)V * 64);
    count_launch();
  }
  (void)o;
  return MG_OK;
}

// Device output: the transpose runs as the level loop's epilogue, before the
// control block is read back.
static std::function<void(cudaStream_t)> transpose_epilogue(mg_graph *g, int32_t nsrc, int32_t *out, bool bfs,
                                                            bool stack) {
  const u64 *visit = bfs ? g->mask[0] : nullptr;
  return [=](cudaStream_t ss) { launch_transpose(g, stack, visit, out, nsrc, ss); };
}

static int multi_finish(mg_graph *g, cudaStream_t s, int32_t nsrc, int32_t *out, int32_t unreached, mg_stats *stats,
                        const mg_options *o, const LoopResult &res, bool stack) {
  finish_run(g, res.ctl.level);
  if (res.ctl.error) return set_error(res.ctl.error, std::string("batched traversal: device reported ") +
                                                         mg_status_string(res.ctl.error));
  // batched BFS (unreached == -1) reads reachability from the visit masks
  const u64 *visit = unreached == -1 ? g->mask[0] : nullptr;
  const u64 all = nsrc == 64 ? ~0ull : ((1ull << nsrc) - 1);
  const int32_t V = g->csr.V;
  int st;
  if (stats) {
    stats->iterations = (int32_t)res.ctl.level;
    stats->push_iterations = (int32_t)res.ctl.push_levels;
    stats->pull_iterations = (int32_t)res.ctl.pull_levels;
    stats->converged = res.ctl.frontier_size == 0 ? 1 : 0;
    stats->device_ms = res.ms;
    stats->vertices_reached = 0;
    stats->edges_traversed = 0;
    if (want_stats(o)) {
      if (visit) {
        unsigned long long *acc = reinterpret_cast<unsigned long long *>(g->ws.ctl->acc);
        unsigned long long h[2] = {0, 0};
        cudaError_t e = cudaMemsetAsync(acc, 0, 16, s);
        if (e == cudaSuccess) {
          k_ms_mask_stats<<<g->num_sms * 4, 256, 0, s>>>(visit, all, g->csr.row_offsets, V, acc);
          count_launch();
          e = cudaMemcpyAsync(h, acc, 16, cudaMemcpyDeviceToHost, s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if ((st = cuda_status(e, "batched stats")) != MG_OK) return st;
        stats->vertices_reached = (int64_t)h[0];
        stats->edges_traversed = (int64_t)h[1];
      } else if ((st = reach_stats(g, s, g->multi_out, unreached, nsrc, 64, &stats->vertices_reached,
                                   &stats->edges_traversed)) != MG_OK) {
        return st;
      }
    }
  }
  if (o->outputs_on_device) return MG_OK;  // transposed by the loop's epilogue
  // Host output: transpose every source into a device staging buffer (kept for
  // later runs), then one copy to the caller.
  if (!g->multi_stage && (st = device_alloc(g, (void **)&g->multi_stage, (size_t)V * 64 * 4)) != MG_OK) return st;
  launch_transpose(g, stack, visit, g->multi_stage, nsrc, s);
  cudaError_t e = cudaMemcpyAsync(out, g->multi_stage, (size_t)nsrc * V * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_status(e, "batched result copy");
}

}  // namespace mg

using namespace mg;

static const mg_options *opts_or_default(const mg_options *o, mg_options *d) {
  if (o) return o;
  mg_options_init(d);
  return d;
}

// One batched BFS: with DT = uint16_t the level stack plus uint16 depth rows
// past it, with DT = int32_t int32 depth rows only. A uint16 run stops after
// level kMsDepth16Levels; *depth_overflow then tells the caller to rerun with
// int32.
template <typename DT>
static int bfs_multi_run(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depths, mg_stats *stats,
                         const mg_options *o, bool *depth_overflow) {
  constexpr bool d16 = sizeof(DT) == 2;
  *depth_overflow = false;
  cudaStream_t s = run_stream(g, o);
  SrcList list;
  int st = multi_prepare(g, srcs, nsrc, o, s, &list, -1, d16);
  if (st != MG_OK) return st;
  MultiArgs a = multi_args(g);
  a.all = (nsrc == 64) ? ~0ull : ((1ull << nsrc) - 1);
  if (d16) {
    a.stk = stack_of(g);
    a.rows = rows16_of(g);
  }
  GasArgs<msbfs_push> ga;
  ga.g = g->csr;
  ga.vl.visit = a.visit;
  ga.vl.F0 = a.F0;
  ga.vl.F1 = a.F1;
  ga.vl.stk = a.stk;
  ga.el.nodes = (int)g->nodes;
  ga.queue0 = g->ws.queue[0];
  ga.queue1 = g->ws.queue[1];
  ga.scan = g->ws.scan;
  ga.part = g->ws.part;
  ga.status = g->ws.status;
  ga.bm0 = g->ws.bm[0];
  ga.bm1 = g->ws.bm[1];
  ga.changed = g->ws.changed;
  ga.gather_tmp = g->ws.gather_tmp;
  ga.gather_res = g->ws.gather_tmp;
  ga.ctl = g->ws.ctl;
  ga.expand_in = 0;
  ga.gather_dir = NO_GATHER_EDGES;
  const uint32_t max_iter_asked = (uint32_t)std::min<int64_t>(o->iter_num > 0 ? o->iter_num : 0, g->nodes + 2);
  const uint32_t max_iter = d16 ? std::min(max_iter_asked, kMsDepth16Levels) : max_iter_asked;
  const int dir = o->direction;
  // direction policy and switch factors go to the control block with the sources
  list.dir = (uint32_t)dir;
  list.alpha = (float)(o->alpha_multi > 0 ? o->alpha_multi : 5.0);
  list.beta = (float)o->beta;
  k_ctl_init<<<1, 32, 0, s>>>(g->ws.ctl, (uint32_t)list.ndistinct, max_iter, (unsigned long long)o->spin_limit,
                              dir == MG_DIR_PULL ? MODE_BITMAP : MODE_QUEUE, ctl_flags(o));
  k_ms_init<<<1, 64, 0, s>>>(a, list, d16 ? 2 : 1);
  count_launch(2);
  if ((st = launch_check("batched bfs init")) != MG_OK) return st;
  const int grid = persistent_grid(g, o, 4);
  // the pull kernel holds no shared memory and at most 40 registers: 48 warps per
  // SM (a few bytes spill; 10 us faster per run at R-MAT 22 than 40 warps at 48)
  const int pull_grid = g->num_sms * 6;
  const int32_t V = g->csr.V;
  const int64_t E = g->edges;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    MG_LAUNCH(KID_MS_APPLY, ss, k_ms_apply<DT><<<grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_CONVERT, ss, k_ms_convert<<<grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<msbfs_push, kMVTS, kMVT><<<grid, kNT, 0, ss>>>(ga)));
    MG_LAUNCH(KID_EXPAND, ss, (k_ms_push<kMVT><<<grid, kNT, 0, ss>>>(ga)));
    MG_LAUNCH(KID_MS_PULL, ss, k_ms_pull<DT><<<pull_grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_OTHER, ss, k_ms_level_end<<<1, 32, 0, ss>>>(a.ctl, V, E, h, use_h));
  };
  LoopResult res;
  const auto epi = transpose_epilogue(g, nsrc, depths, true, d16);
  st = run_level_loop(g, s, std::string(d16 ? "bfs_multi16/" : "bfs_multi/") + std::to_string(grid), 6, body,
                      o->use_cuda_graph != 0, &res, o->outputs_on_device ? &epi : nullptr);
  if (st != MG_OK) return st;
  if (d16 && res.ctl.frontier_size > 0 && res.ctl.level >= kMsDepth16Levels && max_iter_asked > kMsDepth16Levels) {
    finish_run(g, res.ctl.level);
    *depth_overflow = true;  // deeper than a uint16 depth row holds
    return MG_OK;
  }
  return multi_finish(g, s, nsrc, depths, -1, stats, o, res, d16);
}

extern "C" {

int mg_bfs_multi(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *depths, mg_stats *stats,
                 const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (!depths) return set_error(MG_ERR_ARG, "depths is NULL");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  bool overflow = false;
  int st = bfs_multi_run<uint16_t>(g, srcs, nsrc, depths, stats, o, &overflow);
  if (st != MG_OK || !overflow) return st;
  return bfs_multi_run<int32_t>(g, srcs, nsrc, depths, stats, o, &overflow);
}

int mg_sssp_multi(mg_graph *g, const int32_t *srcs, int32_t nsrc, int32_t *dists, mg_stats *stats,
                  const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (!dists) return set_error(MG_ERR_ARG, "dists is NULL");
  if (!g->csr.wgt) return set_error(MG_ERR_UNSUPPORTED, "SSSP needs int32 edge weights (value_type MG_VAL_I32)");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  cudaStream_t s = run_stream(g, o);
  SrcList list;
  int st = multi_prepare(g, srcs, nsrc, o, s, &list, programs::sssp::INIT_VALUE);
  if (st != MG_OK) return st;
  MultiArgs a = multi_args(g);
  a.all = (nsrc == 64) ? ~0ull : ((1ull << nsrc) - 1);
  GasArgs<mssp_scan> ga;
  ga.g = g->csr;
  ga.queue0 = g->ws.queue[0];
  ga.queue1 = g->ws.queue[1];
  ga.scan = g->ws.scan + 0;
  ga.part = g->ws.part;
  ga.status = g->ws.status;
  ga.bm0 = g->ws.bm[0];
  ga.bm1 = g->ws.bm[1];
  ga.changed = g->ws.changed;
  ga.gather_tmp = g->ws.gather_tmp;
  ga.gather_res = g->ws.gather_tmp;
  ga.ctl = g->ws.ctl;
  ga.expand_in = 0;
  ga.gather_dir = NO_GATHER_EDGES;
  const uint32_t max_iter = (uint32_t)std::min<int64_t>(o->iter_num > 0 ? o->iter_num : 0, g->nodes + 2);
  k_ctl_init<<<1, 32, 0, s>>>(g->ws.ctl, (uint32_t)list.ndistinct, max_iter, (unsigned long long)o->spin_limit,
                              MODE_QUEUE, ctl_flags(o));
  k_ms_init<<<1, 64, 0, s>>>(a, list, 0);
  count_launch(2);
  if ((st = launch_check("batched sssp init")) != MG_OK) return st;
  const int grid = persistent_grid(g, o, 4);
  uint32_t *scan = g->ws.scan;
  int32_t *part = g->ws.part;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    MG_LAUNCH(KID_MS_APPLY, ss, k_mss_clear<<<grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_SCAN, ss, (k_frontier_scan<mssp_scan, kMVTS, kMSVT><<<grid, kNT, 0, ss>>>(ga)));
    MG_LAUNCH(KID_MSS_EXPAND, ss, k_mss_expand<kMSVT><<<grid, kNT, 0, ss>>>(a, scan, part));
    MG_LAUNCH(KID_OTHER, ss, k_mss_level_end<<<1, 32, 0, ss>>>(a.ctl, h, use_h));
  };
  LoopResult res;
  const auto epi = transpose_epilogue(g, nsrc, dists, false, false);
  st = run_level_loop(g, s, "sssp_multi/" + std::to_string(grid), 4, body, o->use_cuda_graph != 0, &res,
                      o->outputs_on_device ? &epi : nullptr);
  if (st != MG_OK) return st;
  return multi_finish(g, s, nsrc, dists, programs::sssp::INIT_VALUE, stats, o, res, false);
}

}  // extern "C"
