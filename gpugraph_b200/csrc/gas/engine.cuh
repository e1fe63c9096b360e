// Generic Gather-Apply-Scatter engine for sm_100a, templated on a Program
// functor struct with the reference's contract (Algorithms/SSSP/sssp.h:34-393):
// typedefs DataType/MiscType/GatherType/VertexId/SizeT, INIT_VALUE,
// allow_duplicates, policy selectors srcVertex/gatherOverEdges/applyOverEdges/
// postApplyOverEdges/expandOverEdges (GASengine/Enums.h:2-25) and the device
// functors gather_edge, gather_sum, apply, post_apply, expand_vertex,
// expand_edge, contract with their upstream MapGraph signatures.
//
// One GAS iteration (reference loop: enactor_vertex_centric.cuh:3386-3630) is
//   [gather] -> [apply] -> [post_apply] -> frontier scan -> expand+contract -> level end
// Every kernel is persistent (grid = SMs x CTAs/SM), reads the frontier size
// and level from the device control block, and never returns to the host, so
// the whole level loop is captured once in a CUDA graph (WHILE conditional node
// driven by the level-end kernel) instead of the reference's per-level
// cudaDeviceSynchronize + D->H size copy (enactor_vertex_centric.cuh:3801-3845).
//
// Expand (replaces expand_atomic::Kernel, expand_atomic/cta.cuh:633-755, and the
// two-phase kernel_scatter_mgpu, mgpukernel/kernel.cuh:63-180): the frontier scan
// computes the exclusive degree prefix of the frontier with a decoupled
// look-back and writes merge-path tile partitions over the item space
// (one item per frontier vertex + one per edge). Each expand tile then holds
// exactly NV items, whatever the degrees: a hub's adjacency is split over many
// CTAs (grid-cooperative), a mid-degree list is swept by consecutive lanes of
// one warp or CTA (warp/CTA-cooperative), and low-degree lists are packed
// together, with consecutive lanes reading consecutive column indices.
//
// Contract (replaces contract_atomic::Kernel, contract_atomic/cta.cuh:529-629):
// the Program's contract functor runs inline on every emitted edge, then a
// next-frontier bitmap test-and-set removes duplicates exactly, and survivors
// are compacted with warp ballots, a CTA scan and a decoupled look-back over
// tiles, so the next frontier keeps a deterministic order and needs no global
// atomics per element.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "../common.cuh"
#include "../graph.cuh"
#include "driver.cuh"
#include "enums.h"

namespace mg {

// Optional Program traits (detected; the reference programs need none).
template <class P, class = void>
struct skip_unchanged_trait : std::false_type {};
template <class P>
struct skip_unchanged_trait<P, std::void_t<decltype(P::skip_unchanged_vertices)>>
    : std::integral_constant<bool, P::skip_unchanged_vertices> {};

// Bytes the Program reads per expanded edge besides the column index (its
// status probe of the neighbour), for the algorithmic byte count; default 4.
template <class P, class = void>
struct probe_bytes_trait : std::integral_constant<int, 4> {};
template <class P>
struct probe_bytes_trait<P, std::void_t<decltype(P::probe_bytes)>> : std::integral_constant<int, P::probe_bytes> {};

template <class P, class = void>
struct track_next_edges_trait : std::false_type {};
template <class P>
struct track_next_edges_trait<P, std::void_t<decltype(P::track_next_edges)>>
    : std::integral_constant<bool, P::track_next_edges> {};

template <class P>
struct GasArgs {
  DevCsr g;
  typename P::VertexType vl;
  typename P::EdgeType el;
  int32_t *queue0, *queue1;
  uint32_t *scan;
  int32_t *part;
  unsigned long long *status;
  uint32_t *bm0, *bm1;
  uint8_t *changed;
  typename P::GatherType *gather_tmp;  // contract scratch / apply input
  typename P::GatherType *gather_res;  // gather phase output
  Ctl *ctl;
  // 0: expand over the out-edges (EXPAND_OUT_EDGES), 1: over the in-edges of the
  // transpose (EXPAND_IN_EDGES), 2: over both (EXPAND_ALL_EDGES; a vertex's items
  // are its out-edges, then its in-edges)
  int32_t expand_in;
  int32_t gather_dir; // GatherEdges value
};

template <class P>
MG_DEVINL int32_t *cur_queue(const GasArgs<P> &a, uint32_t level) { return (level & 1) ? a.queue1 : a.queue0; }
template <class P>
MG_DEVINL int32_t *nxt_queue(const GasArgs<P> &a, uint32_t level) { return (level & 1) ? a.queue0 : a.queue1; }
template <class P>
MG_DEVINL uint32_t *cur_bm(const GasArgs<P> &a, uint32_t level) { return (level & 1) ? a.bm1 : a.bm0; }
template <class P>
MG_DEVINL uint32_t *nxt_bm(const GasArgs<P> &a, uint32_t level) { return (level & 1) ? a.bm0 : a.bm1; }

// ---------------------------------------------------------------- gather ----
// Warp per frontier vertex; lanes sweep the adjacency with stride 32 and the
// partial results are combined with the Program's gather_sum in a fixed
// butterfly order (deterministic). Replaces gather_mgpu (enactor:2104-2725).
template <class P>
__global__ void __launch_bounds__(kNT) k_gather(GasArgs<P> a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_QUEUE) return;
  const uint32_t level = ctl->level, n = ctl->frontier_size;
  const int32_t *F = cur_queue(a, level);
  typename P::gather_edge gedge;
  typename P::gather_sum gsum;
  typedef typename P::GatherType G;
  const int lane = lane_id();
  const uint32_t wstride = gridDim.x * kNW;
  for (uint32_t i = blockIdx.x * kNW + warp_id(); i < n; i += wstride) {
    const int v = F[i];
    G acc = G();
    bool has = false;
    for (int pass = 0; pass < 2; ++pass) {
      const bool in = (pass == 0);
      if (in && !(a.gather_dir == GATHER_IN_EDGES || a.gather_dir == GATHER_ALL_EDGES)) continue;
      if (!in && !(a.gather_dir == GATHER_OUT_EDGES || a.gather_dir == GATHER_ALL_EDGES)) continue;
      const int32_t *off = in ? a.g.csc_offsets : a.g.row_offsets;
      const int32_t *nb = in ? a.g.csc_rows : a.g.col;
      const int beg = off[v], end = off[v + 1];
      for (int e = beg + lane; e < end; e += 32) {
        const int u = nb[e];
        const int eid = (in && a.g.csc_eid) ? a.g.csc_eid[e] : e;
        G val;
        gedge(v, eid, u, a.vl, a.el, val);
        acc = has ? gsum(acc, val) : val;
        has = true;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      G oacc = __shfl_xor_sync(0xffffffffu, acc, o);
      bool ohas = __shfl_xor_sync(0xffffffffu, (int)has, o) != 0;
      if (ohas) acc = has ? ((lane & o) ? gsum(oacc, acc) : gsum(acc, oacc)) : oacc;
      has = has || ohas;
    }
    if (lane == 0) a.gather_res[v] = has ? acc : G();
  }
}

// ------------------------------------------------------- apply/post-apply ---
// kernel_apply / reset_gather_result (mgpukernel/kernel.cuh:182-198, 572-607).
template <class P>
__global__ void __launch_bounds__(kNT) k_apply(GasArgs<P> a, int all_vertices, int has_gather) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_QUEUE) return;
  const uint32_t level = ctl->level;
  const uint32_t n = all_vertices ? (uint32_t)a.g.V : ctl->frontier_size;
  const int32_t *F = cur_queue(a, level);
  typename P::apply ap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = all_vertices ? (int)i : F[i];
    typename P::GatherType gv = has_gather ? a.gather_res[v] : a.gather_tmp[v];
    char ch = (char)a.changed[v];
    ap(v, (int)level, gv, a.vl, a.el, ch);
    a.changed[v] = (uint8_t)ch;
  }
}

template <class P>
__global__ void __launch_bounds__(kNT) k_post_apply(GasArgs<P> a, int all_vertices) {
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_QUEUE) return;
  const uint32_t level = ctl->level;
  const uint32_t n = all_vertices ? (uint32_t)a.g.V : ctl->frontier_size;
  const int32_t *F = cur_queue(a, level);
  typename P::post_apply pa;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = all_vertices ? (int)i : F[i];
    pa(v, a.vl, a.el, a.gather_tmp);
  }
}

// ---------------------------------------------------------- frontier scan ---
// Exclusive prefix of expanded degrees over the frontier + merge-path tile
// partitions of the item space. Also clears the current frontier's bits in the
// parity bitmap so it is clean when reused two levels later.
template <class P, int VTS, int VT>
__global__ void __launch_bounds__(kNT) k_frontier_scan(GasArgs<P> a) {
  constexpr uint32_t TV = kNT * VTS;
  constexpr uint32_t NV = kNT * VT;
  __shared__ uint32_t s_red[kNW + 1];
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ int s_fail;
  Ctl *ctl = a.ctl;
  if (!ctl->active || ctl->mode != MODE_QUEUE) return;
  const uint32_t level = ctl->level, n = ctl->frontier_size, epoch = ctl->epoch;
  const unsigned long long spin_limit = ctl->spin_limit;
  const int32_t *F = cur_queue(a, level);
  uint32_t *clear_bm = cur_bm(a, level);
  const int32_t *ro = a.expand_in == 1 ? a.g.csc_offsets : a.g.row_offsets;
  const bool both = a.expand_in == 2;
  const uint32_t ntiles = (n + TV - 1) / TV;
  typename P::expand_vertex ev;
  unsigned long long my_bytes = 0;
  if (threadIdx.x == 0) s_fail = 0;
  for (;;) {
    const uint32_t tile = next_tile(&ctl->tile_ctr[0], &s_tile);
    if (tile >= ntiles || s_fail) break;
    const uint32_t ib = tile * TV + threadIdx.x * VTS;
    uint32_t deg[VTS];
    uint32_t tsum = 0;
#pragma unroll
    for (int k = 0; k < VTS; ++k) {
      const uint32_t i = ib + k;
      uint32_t d = 0;
      if (i < n) {
        const int v = F[i];
        atomicAnd(&clear_bm[v >> 5], ~(1u << (v & 31)));
        bool expand = true;
        if (skip_unchanged_trait<P>::value) expand = ev(v, (char)a.changed[v], a.vl, a.el);
        d = expand ? (uint32_t)(ro[v + 1] - ro[v]) : 0u;
        if (expand && both) d += (uint32_t)(a.g.csc_offsets[v + 1] - a.g.csc_offsets[v]);
      }
      deg[k] = d;
      tsum += d;
    }
    uint32_t tile_total;
    const uint32_t excl = cta_exclusive_sum(tsum, s_red, &tile_total);
    if (warp_id() == 0) {
      bool failed = false;
      const uint32_t pre = lookback(a.status, tile, tile_total, epoch, spin_limit, &failed);
      if (lane_id() == 0) {
        s_prefix = pre;
        if (failed) {
          s_fail = 1;
          raise_error(ctl, MG_ERR_TIMEOUT);
        } else if (tile == ntiles - 1) {
          const uint32_t total = pre + tile_total;
          ctl->edge_total = total;
          ctl->exp_tiles = (uint32_t)(((unsigned long long)n + total + NV - 1) / NV);
        }
      }
    }
    __syncthreads();
    if (s_fail) break;
    uint32_t run = s_prefix + excl;
#pragma unroll
    for (int k = 0; k < VTS; ++k) {
      const uint32_t i = ib + k;
      if (i < n) {
        a.scan[i] = run;
        const unsigned long long base = (unsigned long long)i + run;
        const uint32_t t0 = (uint32_t)((base + NV - 1) / NV);
        const uint32_t t1 = (uint32_t)((base + deg[k]) / NV);
        for (uint32_t t = t0; t <= t1; ++t) a.part[t] = (int32_t)i;
        run += deg[k];
        my_bytes += 20;  // frontier id, two row offsets, scan entry, bitmap word
      }
    }
  }
  add_bytes(ctl, KID_SCAN, my_bytes);
}

// ------------------------------------------------------------ tile decode --
// Loads the frontier blocks of expand tile `tile` into shared memory and finds
// the owner block of every item (the last block starting at or before it), so
// item k of the tile is edge (k - s_base[s_own[k]] - 1) of vertex
// s_v[s_own[k]] (negative: the vertex's own item). per_block(j, v) runs once per
// loaded block. Returns false (nothing decoded) on an inconsistent partition.
// Must be called by all kNT threads; ends with __syncthreads().
template <int VT, class PerBlock>
MG_DEVINL bool decode_tile(uint32_t tile, uint32_t ntiles, uint32_t n, unsigned long long items, const int32_t *part,
                           const uint32_t *scan, const int32_t *F, const int32_t *ro, int32_t *s_v, int32_t *s_base,
                           int32_t *s_rs, int32_t *s_own, int *cnt_out, PerBlock per_block) {
  constexpr int NV = kNT * VT;
  const unsigned long long d0 = (unsigned long long)tile * NV;
  const int cnt = (int)((items - d0) < (unsigned long long)NV ? (items - d0) : (unsigned long long)NV);
  const int i0 = part[tile];
  int i1 = (tile + 1 < ntiles) ? part[tile + 1] : (int)n - 1;
  if (i1 > (int)n - 1) i1 = (int)n - 1;
  const int nblk = i1 - i0 + 1;
  *cnt_out = cnt;
  if (nblk < 1 || nblk > NV + 1 || i0 < 0) return false;
  for (int j = threadIdx.x; j < nblk; j += kNT) {
    const int i = i0 + j;
    const int v = F[i];
    s_v[j] = v;
    s_base[j] = (int32_t)((long long)i + (long long)scan[i] - (long long)d0);
    s_rs[j] = ro[v];
    per_block(j, v);
  }
  __syncthreads();
  // Owners: thread t covers items [t*VT, t*VT+VT). Block starts (s_base) are
  // increasing and block 0 starts at or before the tile, so the owner of the
  // first item is the last block starting at or before it (binary search); the
  // next VT-1 items walk forward.
  const int k0 = threadIdx.x * VT;
  if (k0 < cnt) {
    int lo = 0, hi = nblk - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_base[mid] <= k0) lo = mid;
      else hi = mid - 1;
    }
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int k = k0 + r;
      if (k < cnt) {
        while (lo + 1 < nblk && s_base[lo + 1] <= k) ++lo;
        s_own[k] = lo;
      }
    }
  }
  __syncthreads();
  return true;
}

// ------------------------------------------------------ tile compaction ---
// Appends a tile's surviving items to the next queue. bal[r]/outv[r]: each
// warp's round-r survivor ballot and item. The (round, warp) counts are
// scanned by warp 0, then either one atomic reservation per tile places the
// tile (no tile waits for another) or, with `ordered`, a decoupled look-back
// over tiles keeps the queue in tile order. Called by all kNT threads; returns
// false when the look-back gave up (the error is raised).
template <int VT>
MG_DEVINL bool tile_enqueue(const uint32_t (&bal)[VT], const int32_t (&outv)[VT], uint32_t *s_cnt,
                            uint32_t *s_prefix, int *s_fail, bool ordered, unsigned long long *status, uint32_t tile,
                            uint32_t ntiles, uint32_t epoch, unsigned long long spin_limit, int32_t *Fout, uint32_t V,
                            Ctl *ctl) {
  const int lane = lane_id(), warp = warp_id();
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < VT; ++r) s_cnt[r * kNW + warp] = __popc(bal[r]);
  }
  __syncthreads();
  if (warp == 0) {
    // Exclusive scan over the VT*kNW (round, warp) counts; 2 per lane for VT*kNW <= 64.
    constexpr int C = VT * kNW;
    constexpr int PER = (C + 31) / 32;
    uint32_t x[PER];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int idx = lane * PER + q;
      x[q] = idx < C ? s_cnt[idx] : 0u;
      s += x[q];
    }
    const uint32_t inc = warp_inclusive_sum(s);
    uint32_t run = inc - s;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int idx = lane * PER + q;
      if (idx < C) s_cnt[idx] = run;
      run += x[q];
    }
    const uint32_t tile_total = __shfl_sync(0xffffffffu, inc, 31);
    if (ordered) {
      bool failed = false;
      const uint32_t pre = lookback(status, tile, tile_total, epoch, spin_limit, &failed);
      if (lane == 0) {
        *s_prefix = pre;
        if (failed) {
          *s_fail = 1;
          raise_error(ctl, MG_ERR_TIMEOUT);
        } else if (tile == ntiles - 1) {
          ctl->next_size = pre + tile_total;
        }
      }
    } else if (lane == 0) {
      *s_prefix = tile_total ? atomicAdd(&ctl->next_size, tile_total) : 0u;
    }
  }
  __syncthreads();
  if (*s_fail) return false;
#pragma unroll
  for (int r = 0; r < VT; ++r) {
    if ((bal[r] >> lane) & 1u) {
      const uint32_t pos = *s_prefix + s_cnt[r * kNW + warp] + __popc(bal[r] & lanemask_lt());
      if (pos < V) Fout[pos] = outv[r];
    }
  }
  return true;
}

// ------------------------------------------------------ expand + contract ---
template <class P, int VT>
__global__ void __launch_bounds__(kNT) k_expand(GasArgs<P> a) {
  constexpr int NV = kNT * VT;
  __shared__ int32_t s_v[NV + 1];
  __shared__ int32_t s_base[NV + 1];
  __shared__ int32_t s_rs[NV + 1];
  __shared__ int32_t s_own[NV];
  __shared__ uint8_t s_ch[NV + 1];
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
  const int32_t *ro = a.expand_in == 1 ? a.g.csc_offsets : a.g.row_offsets;
  const int32_t *nb = a.expand_in == 1 ? a.g.csc_rows : a.g.col;
  const bool both = a.expand_in == 2;
  const int32_t V = a.g.V;
  typename P::expand_vertex ev;
  typename P::expand_edge ee;
  typename P::contract ct;
  const int lane = lane_id(), warp = warp_id();
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
                         [&](int j, int v) { s_ch[j] = (uint8_t)ev(v, (char)a.changed[v], a.vl, a.el); })) {
      // Inconsistent partition (cannot happen for a well-formed scan): record
      // it and stop instead of indexing out of bounds.
      if (threadIdx.x == 0) {
        raise_error(ctl, MG_ERR_OVERFLOW);
        s_fail = 1;
      }
      __syncthreads();
      break;
    }
    __syncthreads();
    // The thread's VT items go through the Program in phases, so the memory
    // operations of one phase are independent and in flight together: the
    // neighbour ids, then every expand_edge, then every contract (as the
    // reference engine runs expand over the whole edge frontier before
    // contract), then the dedup probes, then the test-and-sets.
    int nbr[VT], vv[VT], eidv[VT], jj[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      const int k = r * kNT + threadIdx.x;
      nbr[r] = -1;
      if (k < cnt) {
        const int j = s_own[k];
        const int el = k - s_base[j] - 1;
        my_bytes += (el >= 0) ? (unsigned long long)(4 + probe_bytes_trait<P>::value) : 12ull;
        if (el >= 0) {
          const int v = s_v[j];
          int eid = s_rs[j] + el;
          const int32_t *nbp = nb;
          bool in_edge = a.expand_in == 1;
          if (both) {  // past the out-edges: the in-edges of v
            const int od = ro[v + 1] - s_rs[j];
            if (el >= od) {
              eid = a.g.csc_offsets[v] + (el - od);
              nbp = a.g.csc_rows;
              in_edge = true;
            }
          }
          if ((unsigned)eid < (unsigned)a.g.E) {
            nbr[r] = __ldcs(nbp + eid);
            vv[r] = v;
            jj[r] = j;
            eidv[r] = (in_edge && a.g.csc_eid) ? a.g.csc_eid[eid] : eid;
          } else {
            raise_error(ctl, MG_ERR_OVERFLOW);
          }
        }
      }
    }
    int fo[VT];
    typename P::MiscType misc[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      fo[r] = -1;
      misc[r] = typename P::MiscType();
      if (nbr[r] >= 0) {
        ee(s_ch[jj[r]] != 0, (int)level, vv[r], nbr[r], eidv[r], a.vl, a.el, fo[r], misc[r]);
        if (fo[r] >= V) {
          raise_error(ctl, MG_ERR_OVERFLOW);
          fo[r] = -1;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      if (fo[r] >= 0) {
        ct((int)level, fo[r], a.vl, a.el, a.gather_tmp, misc[r]);
        if (fo[r] >= V) {
          raise_error(ctl, MG_ERR_OVERFLOW);
          fo[r] = -1;
        }
      }
    }
    uint32_t probe[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) probe[r] = fo[r] >= 0 ? ld_volatile(dedup + (fo[r] >> 5)) : ~0u;
    // the test-and-sets of all VT items in flight together, then the winners'
    // degrees, then the ballots (each step waits only once)
    bool surv[VT];
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      surv[r] = false;
      if (fo[r] >= 0) {
        const uint32_t bit = 1u << (fo[r] & 31);
        if (!(probe[r] & bit)) surv[r] = !(atomicOr(dedup + (fo[r] >> 5), bit) & bit);
      }
    }
    uint32_t bal[VT];
    int32_t outv[VT];
    if (track_next_edges_trait<P>::value) {
      int32_t dg[VT];
#pragma unroll
      for (int r = 0; r < VT; ++r) {
        dg[r] = 0;
        if (surv[r]) {
          dg[r] = ro[fo[r] + 1] - ro[fo[r]];
          if (both) dg[r] += a.g.csc_offsets[fo[r] + 1] - a.g.csc_offsets[fo[r]];
        }
      }
#pragma unroll
      for (int r = 0; r < VT; ++r) my_edges += (unsigned long long)dg[r];
    }
#pragma unroll
    for (int r = 0; r < VT; ++r) {
      bal[r] = __ballot_sync(0xffffffffu, surv[r]);
      outv[r] = fo[r];
      if (surv[r]) my_bytes += 8;  // queue entry + the Program's per-vertex write
    }
    if (!tile_enqueue<VT>(bal, outv, s_cnt, &s_prefix, &s_fail, ordered, a.status, tile, ntiles, epoch, spin_limit,
                          Fout, (uint32_t)V, ctl))
      break;
  }
  add_bytes(ctl, KID_EXPAND, my_bytes);
  if (track_next_edges_trait<P>::value) {
    my_edges = warp_sum(my_edges);
    if (lane == 0 && my_edges) atomicAdd(&s_edges, my_edges);
    __syncthreads();
    if (threadIdx.x == 0 && s_edges) atomicAdd(&ctl->next_edges, s_edges);
  }
}

// The small kernels every level loop launches are defined here with internal
// linkage, so each translation unit that launches them (the library's and a
// separately built Program's alike) registers and launches its own copy.

// ---------------------------------------------------------------- level end -
// Advances the level and decides whether the loop continues; inside a CUDA
// graph it drives the WHILE node's condition.
static __global__ void k_level_end(Ctl *ctl, cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x != 0) return;
  if (ctl->active) {
    ctl->level += 1;
    ctl->push_levels += 1;
    ctl->frontier_size = ctl->next_size;
    ctl->next_size = 0;
    ctl->edge_total = 0;
    ctl->exp_tiles = 0;
    ctl->next_edges = 0;
    ctl->epoch += 4;
    for (int i = 0; i < 4; ++i) ctl->tile_ctr[i] = 0;
    ctl->active = (ctl->frontier_size > 0 && ctl->level < ctl->max_iter && ctl->error == 0) ? 1u : 0u;
  }
  if (use_handle) cudaGraphSetConditional(h, ctl->active);
}

static __global__ void k_fill_i32(int32_t *p, int32_t v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

static __global__ void k_sequence_i32(int32_t *p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int32_t)i;
}

// flags: bit 0 = ordered frontier compaction (mg_options.ordered_frontier),
// bit 1 = count algorithmic bytes (profiling)
MG_DEVINL void ctl_init_body(Ctl *ctl, uint32_t frontier_size, uint32_t max_iter, unsigned long long spin_limit,
                             uint32_t mode, uint32_t flags) {
  // The epoch keeps growing across runs so stale look-back words never match;
  // the host zeroes the status words and the control block before the 30-bit
  // field could wrap (see prepare_run).
  const uint32_t epoch = ctl->epoch + 4;
  Ctl c;
  memset(&c, 0, sizeof(c));
  c.epoch = epoch;
  c.frontier_size = frontier_size;
  c.max_iter = max_iter;
  c.spin_limit = spin_limit;
  c.mode = mode;
  c.next_mode = mode;
  c.active = (frontier_size > 0 && max_iter > 0) ? 1u : 0u;
  c.ordered = flags & 1u;
  c.count_bytes = (flags >> 1) & 1u;
  *ctl = c;
}

static __global__ void k_ctl_init(Ctl *ctl, uint32_t frontier_size, uint32_t max_iter, unsigned long long spin_limit,
                                  uint32_t mode, uint32_t flags) {
  if (threadIdx.x == 0) ctl_init_body(ctl, frontier_size, max_iter, spin_limit, mode, flags);
}

inline uint32_t ctl_flags(const mg_options *o) {
  return ((o && o->ordered_frontier) ? 1u : 0u) | (prof_on() ? 2u : 0u);
}

}  // namespace mg
