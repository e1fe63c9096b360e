// Normalised PageRank as a pull SpMV over the transposed graph (north_star (e)),
// replacing the reference's gather_mgpu + ReduceByKey pipeline
// (GASengine/enactor_vertex_centric.cuh:2104-2725, mgpukernel/kernel.cuh:300-404),
// which writes and re-reads (dst, value) pairs for every edge.
//
//   r'[v] = base + d * sum_{u->v} contrib[u],  contrib[u] = r[u] / outdeg[u] (0 if dangling)
//   base  = (1-d)/N + d * (sum of r over dangling vertices)/N
// stop after the iteration whose L1(r' - r) <= tolerance, or after iter_num.
//
// Precision: ranks, contributions and every per-vertex sum are FP32; each thread
// accumulates its |r' - r| and its dangling mass with Kahan compensation; only
// the grid-wide residual and dangling reductions are FP64.
//
// Work split (deterministic sums): vertices with in-degree <= kPrHeavy are summed
// by their own thread in CSC order; a CTA takes 256 consecutive vertices and
// stages their 257 column offsets in shared memory with one TMA bulk copy.
// Heavier in-lists are cut into kPrChunk-edge chunks, each summed by one warp
// (lanes stride the chunk, then a fixed butterfly), and a fix-up pass adds a
// vertex's chunk partials in chunk order. The next iteration's contributions
// are written in the same pass that produces the ranks, so an iteration reads
// the CSC once (4 bytes per edge) plus 4 bytes per edge of L2-resident
// contribution gathers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"
#include "tma.cuh"

namespace mg {

constexpr int kPrHeavy = 32;
constexpr int kPrChunk = 1024;
constexpr int kPrTileV = kNT;  // vertices per light tile (one thread each)

struct PrArgs {
  const int32_t *coff, *crow;
  const float *inv;
  float *r0, *r1, *c0, *c1, *partial;
  const int32_t *chunk_v, *chunk_b, *chunk_e, *heavy_v, *heavy_first;
  int32_t V, nchunks, nheavy, coff_len;
  float damping;
  Ctl *ctl;
};

MG_DEVINL void kahan_add(float &sum, float &comp, float x) {
  const float y = x - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

MG_DEVINL void pr_finalize(const PrArgs &a, int v, float s, float base, const float *rold, float *rnew, float *cnew,
                           float &rs, float &rc, float &ds, float &dc) {
  const float nr = fmaf(a.damping, s, base);
  kahan_add(rs, rc, fabsf(nr - rold[v]));
  const float iv = a.inv[v];
  if (iv == 0.f) kahan_add(ds, dc, nr);
  rnew[v] = nr;
  cnew[v] = nr * iv;
}

// Reduces the per-thread compensated accumulators in FP64 into ctl->acc[1..2].
MG_DEVINL void pr_flush(Ctl *ctl, float rs, float rc, float ds, float dc) {
  double r = (double)rs - (double)rc, d = (double)ds - (double)dc;
  r = warp_sum(r);
  d = warp_sum(d);
  if (lane_id() == 0) {
    if (r != 0.0) atomicAdd(&ctl->acc[1], r);
    if (d != 0.0) atomicAdd(&ctl->acc[2], d);
  }
}

// Issues the bulk copy of tile `tile`'s column offsets into buffer `buf`.
MG_DEVINL void pr_stage_offsets(const PrArgs &a, uint32_t tile, int32_t *buf, uint64_t *bar) {
  const int v0 = (int)tile * kPrTileV;
  // offsets v0 .. v0+259, clamped to the padded array (both ends multiples of 4 entries)
  const int n_off = min(kPrTileV + 4, a.coff_len - v0);
  const uint32_t bytes = (uint32_t)n_off * 4u;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(bar, bytes);
  bulk_copy_g2s(buf, a.coff + v0, bytes, bar);
}

constexpr int kPrTileEdges = kPrTileV * kPrHeavy;  // upper bound on a tile's light in-edges

__global__ void __launch_bounds__(kNT) k_pr_iter(PrArgs a) {
  __shared__ alignas(16) int32_t s_off[2][kPrTileV + 4];
  __shared__ float s_val[kPrTileEdges];
  __shared__ uint64_t s_bar[2];
  __shared__ int s_ok;
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float base = (float)ctl->dangling;
  const unsigned long long spin_limit = ctl->spin_limit;
  const float *cold = (L & 1) ? a.c1 : a.c0;
  const float *rold = (L & 1) ? a.r1 : a.r0;
  float *rnew = (L & 1) ? a.r0 : a.r1;
  float *cnew = (L & 1) ? a.c0 : a.c1;
  float rs = 0.f, rc = 0.f, ds = 0.f, dc = 0.f;
  unsigned long long my_bytes = 0;
  const uint32_t ntiles = ((uint32_t)a.V + kPrTileV - 1) / kPrTileV;
  // Tiles are taken round-robin (every tile's work is bounded: a small tile
  // holds <= kPrTileEdges edges, an oversized one only in-lists <= kPrHeavy),
  // so the next tile is known without an atomic and its offsets are in flight
  // while the current tile is summed.
  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    if (blockIdx.x < ntiles) pr_stage_offsets(a, blockIdx.x, s_off[0], &s_bar[0]);
  }
  __syncthreads();
  uint32_t tile = blockIdx.x;
  uint32_t parity[2] = {0u, 0u};
  int cur = 0;
  while (tile < ntiles) {
    __syncthreads();  // everyone has finished with the other buffer
    const uint32_t par = parity[cur];
    const uint32_t next = tile + gridDim.x;
    if (threadIdx.x == 0) {
      s_ok = mbar_wait_bounded(&s_bar[cur], par, spin_limit) ? 1 : 0;
      if (!s_ok) {
        // give the copy in flight one more bounded wait before leaving
        mbar_wait_bounded(&s_bar[cur], par, spin_limit);
      } else if (next < ntiles) {
        // prefetch the next tile's offsets into the other buffer while this one is processed
        pr_stage_offsets(a, next, s_off[cur ^ 1], &s_bar[cur ^ 1]);
      }
    }
    parity[cur] ^= 1u;
    __syncthreads();
    if (!s_ok) {
      if (threadIdx.x == 0) raise_error(ctl, MG_ERR_TIMEOUT);
      break;
    }
    // every thread observes the completed phase itself (acquire of the copy's writes)
    if (!mbar_wait_bounded(&s_bar[cur], par, 1024)) raise_error(ctl, MG_ERR_TIMEOUT);
    const int32_t *off = s_off[cur];
    const int v0 = (int)tile * kPrTileV;
    const int nv = min(kPrTileV, a.V - v0);
    const int e_lo = off[0], e_hi = off[nv];
    const bool small_tile = (e_hi - e_lo) <= kPrTileEdges;
    if (small_tile) {
      // phase 1: every thread strides the tile's whole edge range (coalesced
      // row-index loads, eight independent gathers per step) into s_val
      // rounds of 8 x kNT edges with predicated loads, so the tail of the
      // range is not walked as a chain of dependent single loads
      for (int k = e_lo + (int)threadIdx.x; k < e_hi; k += 8 * kNT) {
        int u[8];
        float x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) u[j] = (k + j * kNT < e_hi) ? a.crow[k + j * kNT] : -1;
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = (u[j] >= 0) ? __ldg(&cold[u[j]]) : 0.f;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (u[j] >= 0) s_val[k + j * kNT - e_lo] = x[j];
      }
    }
    __syncthreads();
    // phase 2: thread per vertex, sum in CSC order (deterministic). In a small
    // tile, in-lists longer than kPrHeavy are summed by the whole warp from
    // s_val (lanes stride the list, fixed butterfly); in an oversized tile they
    // are left to the chunk pass.
    const bool valid_v = (int)threadIdx.x < nv;
    const int beg = valid_v ? off[threadIdx.x] : 0, end = valid_v ? off[threadIdx.x + 1] : 0;
    if (small_tile) {
      const int lane = lane_id();
      uint32_t hv = __ballot_sync(0xffffffffu, valid_v && end - beg > kPrHeavy);
      float hsum = 0.f;
      while (hv) {
        const int h = __ffs(hv) - 1;
        hv &= hv - 1;
        const int hb = __shfl_sync(0xffffffffu, beg, h) - e_lo, he = __shfl_sync(0xffffffffu, end, h) - e_lo;
        float acc = 0.f;
        for (int k = hb + lane; k < he; k += 32) acc += s_val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == h) hsum = acc;
      }
      if (valid_v) {
        float s = 0.f;
        if (end - beg > kPrHeavy) {
          s = hsum;
        } else {
          for (int e = beg; e < end; ++e) s += s_val[e - e_lo];
        }
        pr_finalize(a, v0 + (int)threadIdx.x, s, base, rold, rnew, cnew, rs, rc, ds, dc);
        my_bytes += 20 + 8ull * (unsigned long long)(end - beg);
      }
    } else if (valid_v) {
      const int v = v0 + (int)threadIdx.x;
      if (end - beg <= kPrHeavy) {
        float s = 0.f;
        {
          int e = beg;
          for (; e + 4 <= end; e += 4) {
            const int u0 = a.crow[e], u1 = a.crow[e + 1], u2 = a.crow[e + 2], u3 = a.crow[e + 3];
            const float x0 = __ldg(&cold[u0]), x1 = __ldg(&cold[u1]), x2 = __ldg(&cold[u2]), x3 = __ldg(&cold[u3]);
            s += x0;
            s += x1;
            s += x2;
            s += x3;
          }
          for (; e < end; ++e) s += __ldg(&cold[a.crow[e]]);
        }
        pr_finalize(a, v, s, base, rold, rnew, cnew, rs, rc, ds, dc);
        my_bytes += 20 + 8ull * (unsigned long long)(end - beg);
      }
    }
    tile = next;
    cur ^= 1;
  }
  // heavy chunks: warp per chunk, round-robin over the grid's warps (a chunk is
  // at most kPrChunk edges, and a shared atomic work counter would serialise
  // tens of thousands of warps on one address)
  const int lane = lane_id();
  const uint32_t nwarps = gridDim.x * kNW;
  for (uint32_t c = blockIdx.x * kNW + warp_id(); c < (uint32_t)a.nchunks; c += nwarps) {
    const int b = a.chunk_b[c], e = a.chunk_e[c];
    float acc = 0.f;
    int k = b + lane;
    // eight independent row-index loads, then eight independent gathers, per step
    for (; k + 7 * 32 < e; k += 8 * 32) {
      int u[8];
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) u[j] = a.crow[k + 32 * j];
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = __ldg(&cold[u[j]]);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc += x[j];
    }
    for (; k < e; k += 32) acc += __ldg(&cold[a.crow[k]]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      a.partial[c] = acc;
      my_bytes += 4 + 8ull * (unsigned long long)(e - b);
    }
  }
  add_bytes(ctl->kbytes, KID_PR_PULL, my_bytes);
  pr_flush(ctl, rs, rc, ds, dc);
}

// Heavy vertices: chunk partials added in chunk order.
__global__ void __launch_bounds__(kNT) k_pr_fixup(PrArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float base = (float)ctl->dangling;
  const float *rold = (L & 1) ? a.r1 : a.r0;
  float *rnew = (L & 1) ? a.r0 : a.r1;
  float *cnew = (L & 1) ? a.c0 : a.c1;
  float rs = 0.f, rc = 0.f, ds = 0.f, dc = 0.f;
  unsigned long long my_bytes = 0;
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < a.nheavy; h += gridDim.x * blockDim.x) {
    const int v = a.heavy_v[h];
    float s = 0.f;
    for (int c = a.heavy_first[h]; c < a.heavy_first[h + 1]; ++c) s += a.partial[c];
    pr_finalize(a, v, s, base, rold, rnew, cnew, rs, rc, ds, dc);
    my_bytes += 28 + 4ull * (unsigned long long)(a.heavy_first[h + 1] - a.heavy_first[h]);
  }
  add_bytes(ctl->kbytes, KID_PR_PULL, my_bytes);
  pr_flush(ctl, rs, rc, ds, dc);
}

__global__ void k_pr_level_end(Ctl *ctl, double damping, double inv_n, double tol, cudaGraphConditionalHandle h,
                               int use_handle) {
  if (threadIdx.x != 0) return;
  if (ctl->active) {
    const double res = ctl->acc[1], dang = ctl->acc[2];
    ctl->acc[1] = 0.0;
    ctl->acc[2] = 0.0;
    ctl->residual = res;
    ctl->level += 1;
    ctl->push_levels += 1;
    ctl->dangling = (1.0 - damping) * inv_n + damping * dang * inv_n;  // base of the next iteration
    for (int i = 0; i < 4; ++i) ctl->tile_ctr[i] = 0;
    ctl->active = (res > tol && ctl->level < ctl->max_iter && ctl->error == 0) ? 1u : 0u;
  }
  if (use_handle) cudaGraphSetConditional(h, ctl->active);
}

__global__ void k_pr_init(const float *inv, float *r, float *c, int32_t V, float r0) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    r[v] = r0;
    c[v] = r0 * inv[v];
  }
}

// One-time plan: 1/outdeg, dangling count, heavy vertices and their chunks.
static int pr_plan(mg_graph *g, cudaStream_t s) {
  if (g->pr_rank[0]) return MG_OK;
  const int64_t V = g->nodes;
  const size_t ro_n = ((size_t)(V + 1 + 3) & ~(size_t)3) + 4;
  std::vector<int32_t> ro((size_t)V + 1), co((size_t)V + 1);
  cudaError_t e = cudaMemcpyAsync(ro.data(), g->csr.row_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(co.data(), g->csr.csc_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "pagerank plan read");
  std::vector<float> inv((size_t)V);
  int64_t ndang = 0;
  std::vector<int32_t> cv, cb, ce, hv, hf;
  for (int64_t v = 0; v < V; ++v) {
    const int32_t od = ro[v + 1] - ro[v];
    inv[v] = od > 0 ? 1.0f / (float)od : 0.0f;
    ndang += od == 0;
    const int32_t b = co[v], en = co[v + 1];
    // the same rule as k_pr_iter: a tile of kPrTileV vertices whose in-edges fit
    // in shared memory is summed whole; in a larger tile, in-lists longer than
    // kPrHeavy are chunked
    const int64_t t0 = (v / kPrTileV) * kPrTileV, t1 = std::min<int64_t>(V, t0 + kPrTileV);
    const bool small_tile = (int64_t)co[t1] - co[t0] <= kPrTileEdges;
    if (!small_tile && en - b > kPrHeavy) {
      hv.push_back((int32_t)v);
      hf.push_back((int32_t)cv.size());
      for (int32_t x = b; x < en; x += kPrChunk) {
        cv.push_back((int32_t)v);
        cb.push_back(x);
        ce.push_back(std::min(en, x + kPrChunk));
      }
    }
  }
  hf.push_back((int32_t)cv.size());
  int st;
  float *inv_d = nullptr;
  const size_t nc = std::max<size_t>(cv.size(), 1), nh = std::max<size_t>(hv.size(), 1);
  if ((st = device_alloc(g, (void **)&inv_d, (size_t)V * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_chunk_v, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_chunk_b, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_chunk_e, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_heavy_v, nh * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_heavy_first, (nh + 1) * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&g->pr_partial, nc * 4)) != MG_OK)
    return st;
  for (int i = 0; i < 2; ++i)
    if ((st = device_alloc(g, (void **)&g->pr_rank[i], (size_t)V * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&g->pr_contrib[i], (size_t)V * 4)) != MG_OK)
      return st;
  e = cudaMemcpyAsync(inv_d, inv.data(), (size_t)V * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !cv.empty()) {
    e = cudaMemcpyAsync(g->pr_chunk_v, cv.data(), cv.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->pr_chunk_b, cb.data(), cb.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->pr_chunk_e, ce.data(), ce.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->pr_heavy_v, hv.data(), hv.size() * 4, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->pr_heavy_first, hf.data(), hf.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "pagerank plan upload");
  g->inv_outdeg = inv_d;
  g->pr_nchunks = (int32_t)cv.size();
  g->pr_nheavy = (int32_t)hv.size();
  g->pr_ndangling = ndang;
  (void)ro_n;
  return MG_OK;
}

}  // namespace mg

using namespace mg;

extern "C" int mg_pagerank(mg_graph *g, float *ranks, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (!ranks) return set_error(MG_ERR_ARG, "ranks is NULL");
  mg_options dflt;
  const mg_options *o = opts;
  if (!o) {
    mg_options_init(&dflt);
    o = &dflt;
  }
  if (!(o->damping >= 0.0 && o->damping < 1.0)) return set_error(MG_ERR_ARG, "damping must be in [0, 1)");
  if (!(o->tolerance >= 0.0)) return set_error(MG_ERR_ARG, "tolerance must be >= 0");
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK) return st;
  if ((st = pr_plan(g, s)) != MG_OK) return st;
  const int32_t V = g->csr.V;
  const double d = o->damping, inv_n = 1.0 / (double)V;
  // the reference's iteration cap knob; the BASELINE specification stops at 100
  const uint32_t max_iter = (uint32_t)std::max<int32_t>(0, std::min<int32_t>(o->iter_num, 1 << 20));
  PrArgs a;
  a.coff = g->csr.csc_offsets;
  a.crow = g->csr.csc_rows;
  a.inv = g->inv_outdeg;
  a.r0 = g->pr_rank[0];
  a.r1 = g->pr_rank[1];
  a.c0 = g->pr_contrib[0];
  a.c1 = g->pr_contrib[1];
  a.partial = g->pr_partial;
  a.chunk_v = g->pr_chunk_v;
  a.chunk_b = g->pr_chunk_b;
  a.chunk_e = g->pr_chunk_e;
  a.heavy_v = g->pr_heavy_v;
  a.heavy_first = g->pr_heavy_first;
  a.V = V;
  a.nchunks = g->pr_nchunks;
  a.nheavy = g->pr_nheavy;
  a.coff_len = (int32_t)(((size_t)(V + 1 + 3) & ~(size_t)3) + 4);
  a.damping = (float)d;
  a.ctl = g->ws.ctl;
  k_pr_init<<<g->num_sms * 4, 256, 0, s>>>(a.inv, a.r0, a.c0, V, (float)inv_n);
  k_ctl_init<<<1, 32, 0, s>>>(a.ctl, 1u, max_iter, (unsigned long long)o->spin_limit, MODE_QUEUE, 0u);
  count_launch(2);
  const double base0 = (1.0 - d) * inv_n + d * ((double)g->pr_ndangling * inv_n) * inv_n;
  cudaError_t e = cudaMemcpyAsync(&a.ctl->dangling, &base0, sizeof(double), cudaMemcpyHostToDevice, s);
  if ((st = cuda_status(e, "pagerank init")) != MG_OK) return st;
  const int grid = persistent_grid(g, o, 6);  // 35 KB of shared memory per CTA: 6 fit on an SM
  const int fix_grid = std::max(1, std::min(g->num_sms * 4, (g->pr_nheavy + kNT - 1) / kNT));
  const double tol = o->tolerance;
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    MG_LAUNCH(KID_PR_PULL, ss, k_pr_iter<<<grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_GATHER, ss, k_pr_fixup<<<fix_grid, kNT, 0, ss>>>(a));
    MG_LAUNCH(KID_OTHER, ss, k_pr_level_end<<<1, 32, 0, ss>>>(a.ctl, d, inv_n, tol, h, use_h));
  };
  LoopResult res;
  // the body's kernel arguments carry d and tol: key the cached graph on them
  char key[96];
  snprintf(key, sizeof(key), "pagerank/%d/%.17g/%.17g", grid, d, tol);
  if ((st = run_level_loop(g, s, key, 3, body, o->use_cuda_graph != 0, &res)) != MG_OK) return st;
  finish_run(g, res.ctl.level);
  if (res.ctl.error) return set_error(res.ctl.error, std::string("pagerank: device reported ") +
                                                         mg_status_string(res.ctl.error));
  if (stats) {
    stats->iterations = (int32_t)res.ctl.level;
    stats->push_iterations = 0;
    stats->pull_iterations = (int32_t)res.ctl.level;
    stats->converged = (res.ctl.level > 0 && res.ctl.residual <= tol) ? 1 : 0;
    stats->device_ms = res.ms;
    stats->residual = res.ctl.residual;
    stats->vertices_reached = g->nodes;
    stats->edges_traversed = g->edges * (int64_t)res.ctl.level;
  }
  const float *final_r = (res.ctl.level & 1) ? a.r1 : a.r0;
  return copy_out(s, ranks, final_r, (size_t)V * 4, o->outputs_on_device != 0);
}
