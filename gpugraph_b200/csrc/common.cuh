// Device-side building blocks shared by every kernel of the library: the
// per-run control block, acquire/release accessors, bounded spin waits, warp and
// CTA scans, and the decoupled look-back used for order-preserving compaction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mapgraph_b200.h"

#define MG_DEVINL __device__ __forceinline__

namespace mg {

constexpr int kWarp = 32;
constexpr int kNT = 256;  // threads per CTA of the level-loop kernels
constexpr int kNW = kNT / kWarp;

// Frontier representation of the current level.
enum : uint32_t { MODE_QUEUE = 0, MODE_BITMAP = 1 };

// Device control block of one traversal. Lives in device memory; every
// level-loop kernel reads the fields it needs at entry, so the kernels can be
// captured once in a CUDA graph and replayed without host round trips.
struct Ctl {
  uint32_t level;           // current GAS iteration
  uint32_t frontier_size;   // |F| of the current level (queue mode)
  uint32_t next_size;       // |F| produced by the current level
  uint32_t edge_total;      // sum of expanded degrees of the current frontier
  uint32_t exp_tiles;       // expand tiles of the current level
  uint32_t tile_ctr[4];     // dynamic tile counters (scan, expand, pull, convert)
  uint32_t done_ctas[4];    // CTA completion counters ("last CTA" finalisers)
  uint32_t epoch;           // look-back epoch base; never reset between runs
  uint32_t mode;            // MODE_QUEUE / MODE_BITMAP of the current level
  uint32_t next_mode;       // decided at the end of a level
  uint32_t active;          // 1 while the loop must continue
  uint32_t max_iter;        // iteration cap
  int32_t error;            // MG_OK or MG_ERR_TIMEOUT/MG_ERR_OVERFLOW
  uint32_t push_levels;
  uint32_t pull_levels;
  uint32_t dir_policy;      // MG_DIR_* (BFS)
  uint32_t convert;         // 1: rebuild the queue from the bitmap at level start
  uint32_t ordered;         // 1: compact the next frontier in tile order (look-back)
  uint32_t prev_size;       // |F| of the previous level (batched traversals)
  uint32_t apply_pending;   // 1: the previous push level left bits to apply
  uint32_t count_bytes;     // 1: kernels add their algorithmic bytes to kbytes (profiling)
  // Batched BFS level stack: the frontier masks of levels below stk_levels are
  // kept, one [V] array per level (bit L of stk_pull: level L's array was written
  // for every vertex by a pull level; otherwise only the queued vertices' entries
  // are valid, marked in that level's bitmap). clear_pending: the previous
  // level's parity masks are cleared at its queue entries before this level's
  // push writes into them.
  uint32_t stk_levels;
  uint32_t stk_pull;
  uint32_t clear_pending;
  // Batched BFS: OR of the frontier masks of level parity p (the sources that
  // can still reach new vertices); accumulated while the level's masks are
  // produced, cleared once consumed.
  unsigned long long srcmask[2];
  float alpha, beta;        // direction-switch factors (BFS)
  unsigned long long next_edges;     // sum of degrees of the next frontier
  unsigned long long visited_edges;  // sum of degrees of visited vertices (BFS)
  unsigned long long visited_count;
  unsigned long long spin_limit;
  double residual;          // PageRank L1 residual of the last iteration
  double dangling;          // PageRank dangling mass of the current ranks
  double acc[4];            // FP64 reduction slots
  // Algorithmic bytes moved by each kernel kind over the run (element-granular
  // reads and writes the algorithm needs; see KernelId).
  unsigned long long kbytes[13];
};

// Kernel kinds for per-kernel byte accounting and profiling.
enum KernelId : int {
  KID_SCAN = 0,
  KID_EXPAND = 1,
  KID_BFS_PULL = 2,
  KID_MS_PULL = 3,
  KID_MS_APPLY = 4,
  KID_CONVERT = 5,
  KID_MSS_EXPAND = 6,
  KID_PR_PULL = 7,
  KID_GATHER = 8,
  KID_APPLY = 9,
  KID_PPR = 10,
  KID_CC = 11,
  KID_OTHER = 12
};
constexpr int kNumKernelKinds = 13;

// Adds a warp's byte count to the run's counter for kernel kind `kid` (one
// atomic per warp; call from every thread with its own count). Only while
// profiling: otherwise the counters are not read and the atomics, all on one
// cache line, would be contended work at the end of every launch.
MG_DEVINL void add_bytes(Ctl *ctl, int kid, unsigned long long mine) {
  if (!ctl->count_bytes) return;
  mine += __shfl_xor_sync(0xffffffffu, mine, 16);
  mine += __shfl_xor_sync(0xffffffffu, mine, 8);
  mine += __shfl_xor_sync(0xffffffffu, mine, 4);
  mine += __shfl_xor_sync(0xffffffffu, mine, 2);
  mine += __shfl_xor_sync(0xffffffffu, mine, 1);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&ctl->kbytes[kid], mine);
}

MG_DEVINL uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
MG_DEVINL unsigned long long ld_acquire(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
MG_DEVINL void st_release(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
MG_DEVINL void st_release(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
MG_DEVINL uint32_t ld_volatile(const uint32_t *p) { return *(volatile const uint32_t *)p; }

MG_DEVINL uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
MG_DEVINL int lane_id() { return threadIdx.x & 31; }
MG_DEVINL int warp_id() { return threadIdx.x >> 5; }

template <typename T>
MG_DEVINL T warp_inclusive_sum(T x) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane_id() >= o) x += y;
  }
  return x;
}
template <typename T>
MG_DEVINL T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Exclusive CTA-wide scan of one value per thread (blockDim.x == kNT).
// Returns the exclusive prefix; *total receives the CTA sum. Uses smem[kNW+1].
template <typename T>
MG_DEVINL T cta_exclusive_sum(T x, T *smem, T *total) {
  T inc = warp_inclusive_sum(x);
  if (lane_id() == 31) smem[warp_id()] = inc;
  __syncthreads();
  if (warp_id() == 0) {
    T w = lane_id() < kNW ? smem[lane_id()] : T(0);
    T wi = warp_inclusive_sum(w);
    if (lane_id() < kNW) smem[lane_id()] = wi - w;
    if (lane_id() == kNW - 1) smem[kNW] = wi;
  }
  __syncthreads();
  T r = smem[warp_id()] + inc - x;
  *total = smem[kNW];
  __syncthreads();
  return r;
}

// Sum of one double per thread over the CTA (every thread calls it): the total
// in thread 0, 0 elsewhere. Lets a kernel add a CTA's total to a control-block
// counter with one atomic instead of one per warp (same-line atomics from
// every warp of a full grid are a measurable tail on short launches).
MG_DEVINL double cta_sum_f64(double x) {
  __shared__ double s_part[32];
  x = warp_sum(x);
  __syncthreads();  // the previous call's reads of s_part are done
  if (lane_id() == 0) s_part[warp_id()] = x;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s_part[i];
  return t;
}

// Records a device-side failure without faulting: the first error wins.
MG_DEVINL void raise_error(Ctl *ctl, int code) { atomicCAS(&ctl->error, 0, code); }

// ---------------------------------------------------------------------------
// Decoupled look-back (single-pass prefix over tiles processed in tile order).
// Status word: [epoch:30][flag:2][value:32]; a word from another epoch reads as
// "not yet published", so the status array is never cleared between launches.
// Tiles are handed out by an atomic counter, so every predecessor of a tile is
// already running or done: a wait only ends by publication or by the bounded
// spin limit, after which the tile reports MG_ERR_TIMEOUT.
enum : uint32_t { LB_AGG = 1, LB_INC = 2 };

MG_DEVINL unsigned long long lb_pack(uint32_t epoch, uint32_t flag, uint32_t v) {
  return ((unsigned long long)((epoch << 2) | flag) << 32) | v;
}

// Called by warp 0 of the tile. Publishes the tile aggregate and returns the
// exclusive prefix of all earlier tiles (valid in every lane of warp 0). On a
// timeout returns 0 and sets *failed.
MG_DEVINL uint32_t lookback(unsigned long long *status, uint32_t tile, uint32_t agg, uint32_t epoch,
                            unsigned long long spin_limit, bool *failed) {
  const int lane = lane_id();
  const uint32_t ep = epoch & 0x3fffffffu;
  if (tile == 0) {
    if (lane == 0) st_release(&status[0], lb_pack(ep, LB_INC, agg));
    return 0;
  }
  if (lane == 0) st_release(&status[tile], lb_pack(ep, LB_AGG, agg));
  uint32_t prefix = 0;
  int64_t p = (int64_t)tile - 1;
  unsigned long long spins = 0;
  while (true) {
    int64_t idx = p - lane;
    uint32_t flag = LB_INC, val = 0;
    if (idx >= 0) {
      unsigned long long s = ld_acquire(&status[idx]);
      uint32_t hi = (uint32_t)(s >> 32);
      flag = ((hi >> 2) == ep) ? (hi & 3u) : 0u;
      val = (uint32_t)s;
    }
    uint32_t not_ready = __ballot_sync(0xffffffffu, flag == 0);
    uint32_t inc_mask = __ballot_sync(0xffffffffu, flag == LB_INC);
    // Lanes up to (and including) the nearest inclusive predecessor must be ready.
    uint32_t need = inc_mask ? ((inc_mask & (0u - inc_mask)) << 1) - 1u : 0xffffffffu;
    if (not_ready & need) {
      if (++spins >= spin_limit) {
        *failed = true;
        return 0;
      }
      if (spins > 64) __nanosleep(64);
      continue;
    }
    uint32_t contrib = (need >> lane) & 1u ? val : 0u;
    prefix += warp_sum(contrib);
    if (inc_mask) break;
    p -= 32;
  }
  if (lane == 0) st_release(&status[tile], lb_pack(ep, LB_INC, prefix + agg));
  return prefix;
}

// Grabs the next tile index for the whole CTA (thread 0 increments, broadcast via smem).
MG_DEVINL uint32_t next_tile(uint32_t *ctr, uint32_t *smem_slot) {
  __syncthreads();
  if (threadIdx.x == 0) *smem_slot = atomicAdd(ctr, 1u);
  __syncthreads();
  return *smem_slot;
}

// The CTA's k-th tile of an expand level: through the atomic counter when the
// next queue is ordered (the look-back needs every earlier tile running or
// done), otherwise dealt statically (merge-path tiles all hold the same number
// of items). Call from all threads with k = 0, 1, ...; begins with a barrier,
// so the previous tile's shared state has been read.
MG_DEVINL uint32_t take_tile(uint32_t *ctr, uint32_t *smem_slot, bool ordered, uint32_t k) {
  if (ordered) return next_tile(ctr, smem_slot);
  __syncthreads();
  return blockIdx.x + k * gridDim.x;
}

}  // namespace mg
