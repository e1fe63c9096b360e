// Normalised PageRank as a pull SpMV over the transposed graph,
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
// Work split (deterministic sums: the order of every addition depends only on
// the graph): a warp takes 32 consecutive vertices and sweeps their contiguous
// in-edges 32 at a time with a segmented warp scan, so the edge loads are
// coalesced and balanced across the lanes whatever the in-degrees (a group of
// short lists is summed lane by lane). In-lists longer than kPrBig are cut into
// kPrChunk-edge chunks, each summed by one warp (lanes stride the chunk, then a
// fixed butterfly), and a fix-up pass adds a vertex's chunk partials in chunk
// order. The next iteration's contributions are written in the same pass that
// produces the ranks, so an iteration reads the CSC once (4 bytes per edge)
// plus 4 bytes per edge of L2-resident contribution gathers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"

namespace mg {

constexpr int kPrBig = 512;     // longer in-lists are summed by the chunk pass
constexpr int kPrChunk = 1024;  // edges per chunk of a long in-list
constexpr int kPrGroup = 32;    // vertices per warp group (one per lane)
constexpr int kPrSub = 4;       // 32-edge sub-chunks whose loads are in flight together
constexpr int kPrSerial = 8;    // a group whose lists are all this short is summed lane by lane
constexpr double kPrSkew = 64.0;  // renumber by out-degree when the largest is this many times the mean

struct PrArgs {
  const int32_t *coff, *crow;
  const float *inv;
  float *r0, *r1, *c0, *c1, *partial;
  const int32_t *chunk_v, *chunk_b, *chunk_e, *heavy_v, *heavy_first;
  int32_t V, nchunks, nheavy;
  float damping;
  Ctl *ctl;
};

MG_DEVINL void kahan_add(float &sum, float &comp, float x) {
  const float y = x - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// New rank of v from its in-edge sum s, given its old rank and 1/outdeg.
MG_DEVINL void pr_store(float damping, int v, float s, float base, float r_old, float iv, float *rnew, float *cnew,
                        float &rs, float &rc, float &ds, float &dc) {
  const float nr = fmaf(damping, s, base);
  kahan_add(rs, rc, fabsf(nr - r_old));
  if (iv == 0.f) kahan_add(ds, dc, nr);
  rnew[v] = nr;
  cnew[v] = nr * iv;
}

MG_DEVINL void pr_finalize(const PrArgs &a, int v, float s, float base, const float *rold, float *rnew, float *cnew,
                           float &rs, float &rc, float &ds, float &dc) {
  pr_store(a.damping, v, s, base, rold[v], a.inv[v], rnew, cnew, rs, rc, ds, dc);
}

// Reduces the per-thread compensated accumulators in FP64 into ctl->acc[1..2]
// (one atomic per CTA and slot); called by every thread of the CTA.
MG_DEVINL void pr_flush(Ctl *ctl, float rs, float rc, float ds, float dc) {
  const double r = cta_sum_f64((double)rs - (double)rc);
  const double d = cta_sum_f64((double)ds - (double)dc);
  if (threadIdx.x == 0) {
    if (r != 0.0) atomicAdd(&ctl->acc[1], r);
    if (d != 0.0) atomicAdd(&ctl->acc[2], d);
  }
}

// One 32-edge sub-chunk [ck, ck+32) of a group sweep: lane i holds the
// contribution of edge ck+i (0 outside the sweep). A segmented inclusive scan
// with a head at every list start in the sub-chunk (and at lane 0) leaves the
// sum of each list's part at its last lane; the list's owner lane adds it. A
// step of offset d adds lane i-d's value into lane i when no head lies in
// (i-d, i], a test on the head mask alone: with le = lanes [0, i], that window
// is le & ~(le >> d), and for i < d it takes in lane 0, which is always a head.
MG_DEVINL void pr_segment(float x, int ck, int b, int e, bool mine, uint32_t le, float &acc) {
  const int p = b - ck;
  const uint32_t head = __reduce_or_sync(0xffffffffu, (mine && p >= 0 && p < 32) ? 1u << p : 0u) | 1u;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const float t = __shfl_up_sync(0xffffffffu, x, d);
    if ((head & le & ~(le >> d)) == 0u) x += t;
  }
  const int q = min(e, ck + 32) - 1 - ck;
  const float t = __shfl_sync(0xffffffffu, x, q < 0 ? 0 : (q > 31 ? 31 : q));
  // the list has edges in this sub-chunk (an empty list has none anywhere)
  if (mine && max(b, ck) < min(e, ck + 32)) acc += t;
}

// Pull SpMV over warp groups of kPrGroup consecutive vertices (lane j owns
// vertex v0+j). The warp sweeps the group's contiguous in-edge range in rounds
// of kPrSub x 32 edges: coalesced row-index loads, then kPrSub independent
// contribution gathers per lane, then one segmented warp scan per sub-chunk.
// In-lists longer than kPrBig are skipped here (the chunk pass sums them), so
// a group's sweep is at most kPrGroup * kPrBig edges. A group whose lists are
// all at most kPrSerial long is summed lane by lane instead. Groups are dealt
// round-robin to the grid's warps, and each warp loads its next group's
// offsets while it sweeps the current one. No shared memory, no block
// barriers. (Staging the 33 offsets of a group with a bulk copy on an
// mbarrier measured slower than the two coalesced loads per lane.)
__global__ void __launch_bounds__(kNT, 6) k_pr_iter(PrArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float base = (float)ctl->dangling;
  const float *cold = (L & 1) ? a.c1 : a.c0;
  const float *rold = (L & 1) ? a.r1 : a.r0;
  float *rnew = (L & 1) ? a.r0 : a.r1;
  float *cnew = (L & 1) ? a.c0 : a.c1;
  float rs = 0.f, rc = 0.f, ds = 0.f, dc = 0.f;
  unsigned long long my_bytes = 0;
  const int lane = lane_id(), w = warp_id();
  const uint32_t le = 0xffffffffu >> (31 - lane);  // lanes [0, lane]
  const uint32_t ngroups = ((uint32_t)a.V + kPrGroup - 1) / kPrGroup;
  const uint32_t nwarps = gridDim.x * kNW;
  uint32_t grp = blockIdx.x * kNW + w;
  // offsets of the next group, loaded one group ahead (lanes past the last
  // vertex load nothing)
  int nb = 0, ne = 0;
  if (grp < ngroups && (int)(grp * kPrGroup) + lane < a.V) {
    nb = a.coff[grp * kPrGroup + lane];
    ne = a.coff[grp * kPrGroup + lane + 1];
  }
  for (; grp < ngroups; grp += nwarps) {
    const int v0 = (int)grp * kPrGroup;
    const int nv = min(kPrGroup, a.V - v0);
    const bool valid = lane < nv;
    const int b = nb, e = ne;
    const int g_end = __shfl_sync(0xffffffffu, e, nv - 1);
    int seg_b = __shfl_sync(0xffffffffu, b, 0);
    const uint32_t next = grp + nwarps;
    if (next < ngroups && (int)(next * kPrGroup) + lane < a.V) {
      nb = a.coff[next * kPrGroup + lane];
      ne = a.coff[next * kPrGroup + lane + 1];
    }
    const bool big = valid && e - b > kPrBig;
    const bool mine = valid && !big;
    // the finalize inputs are independent of the sweep: load them first
    const int v = v0 + lane;
    const float r_old = mine ? rold[v] : 0.f, iv = mine ? a.inv[v] : 0.f;
    float acc = 0.f;
    if (__ballot_sync(0xffffffffu, valid && e - b > kPrSerial) == 0u) {
      // every list of the group is short: each lane sums its own, all its
      // loads in flight at once (CSC order)
      int u[kPrSerial];
      float x[kPrSerial];
#pragma unroll
      for (int k = 0; k < kPrSerial; ++k) u[k] = b + k < e ? __ldcs(a.crow + b + k) : -1;
#pragma unroll
      for (int k = 0; k < kPrSerial; ++k) x[k] = u[k] >= 0 ? __ldg(&cold[u[k]]) : 0.f;
#pragma unroll
      for (int k = 0; k < kPrSerial; ++k) acc += x[k];
    } else {
    uint32_t pending = __ballot_sync(0xffffffffu, big);
    for (;;) {
      const int h = pending ? __ffs(pending) - 1 : -1;
      const int seg_e = h >= 0 ? __shfl_sync(0xffffffffu, b, h) : g_end;
      for (int c = seg_b; c < seg_e; c += kPrSub * 32) {
        int u[kPrSub];
        float x[kPrSub];
#pragma unroll
        for (int k = 0; k < kPrSub; ++k) {
          const int i = c + 32 * k + lane;
          u[k] = i < seg_e ? __ldcs(a.crow + i) : -1;
        }
#pragma unroll
        for (int k = 0; k < kPrSub; ++k) x[k] = u[k] >= 0 ? __ldg(&cold[u[k]]) : 0.f;
#pragma unroll
        for (int k = 0; k < kPrSub; ++k)
          if (c + 32 * k < seg_e) pr_segment(x[k], c + 32 * k, b, e, mine, le, acc);
      }
      if (h < 0) break;
      pending &= pending - 1;
      seg_b = __shfl_sync(0xffffffffu, e, h);
    }
    }
    if (mine) {
      pr_store(a.damping, v, acc, base, r_old, iv, rnew, cnew, rs, rc, ds, dc);
      my_bytes += 20 + 8ull * (unsigned long long)(e - b);
    }
  }
  // heavy chunks: warp per chunk, round-robin over the grid's warps (a chunk is
  // at most kPrChunk edges, and a shared atomic work counter would serialise
  // tens of thousands of warps on one address)
  for (uint32_t c = blockIdx.x * kNW + w; c < (uint32_t)a.nchunks; c += nwarps) {
    const int cb = a.chunk_b[c], ce = a.chunk_e[c];
    float acc = 0.f;
    int k = cb + lane;
    // eight independent row-index loads, then eight independent gathers, per step
    for (; k + 7 * 32 < ce; k += 8 * 32) {
      int u[8];
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) u[j] = __ldcs(a.crow + k + 32 * j);
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = __ldg(&cold[u[j]]);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc += x[j];
    }
    for (; k < ce; k += 32) acc += __ldg(&cold[__ldcs(a.crow + k)]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      a.partial[c] = acc;
      my_bytes += 4 + 8ull * (unsigned long long)(ce - cb);
    }
  }
  add_bytes(ctl, KID_PR_PULL, my_bytes);
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
  add_bytes(ctl, KID_PR_PULL, my_bytes);
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

// Control block of a PageRank run, with the base term of the first iteration
// (passed by value, so no host buffer has to outlive the launch).
__global__ void k_pr_ctl_init(Ctl *ctl, uint32_t max_iter, unsigned long long spin_limit, uint32_t flags,
                              double base0) {
  if (threadIdx.x == 0) {
    ctl_init_body(ctl, 1u, max_iter, spin_limit, MODE_QUEUE, flags);
    ctl->dangling = base0;
  }
}

__global__ void k_pr_init(const float *inv, float *r, float *c, int32_t V, float r0) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    r[v] = r0;
    c[v] = r0 * inv[v];
  }
}

// Renumbered in-lists: new vertex i is old vertex old_of[i]; its in-list is the
// old in-list with every neighbour renumbered (order kept). Warp per vertex.
__global__ void __launch_bounds__(kNT) k_pr_renumber(const int32_t *old_of, const int32_t *new_of,
                                                     const int32_t *co, const int32_t *crow, const int32_t *coff_new,
                                                     int32_t *crow_new, int32_t V) {
  const int lane = lane_id();
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < V; i += (gridDim.x * blockDim.x) / 32) {
    const int v = old_of[i];
    const int b = co[v], n = co[v + 1] - b, o = coff_new[i];
    for (int k = lane; k < n; k += 32) crow_new[o + k] = new_of[crow[b + k]];
  }
}

// ranks in the caller's numbering: out[v] = r[new_of[v]]
__global__ void k_pr_unrenumber(const float *r, const int32_t *new_of, float *out, int32_t V) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) out[v] = r[new_of[v]];
}

// One-time plan: the in-lists to read (renumbered by descending out-degree when
// the distribution is skewed, so the contributions of the most-gathered
// vertices share cache lines), 1/outdeg, dangling count, heavy vertices and
// their chunks.
static int pr_plan(mg_graph *g, cudaStream_t s) {
  if (g->pr_rank[0]) return MG_OK;
  const int64_t V = g->nodes;
  const size_t ro_n = ((size_t)(V + 1 + 3) & ~(size_t)3) + 4;
  std::vector<int32_t> ro((size_t)V + 1), co((size_t)V + 1);
  cudaError_t e = cudaMemcpyAsync(ro.data(), g->csr.row_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(co.data(), g->csr.csc_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "pagerank plan read");
  // Renumber when the out-degree distribution is skewed (a power law): the
  // largest out-degree is many times the mean. Grid-like graphs keep their own
  // numbering, whose locality is already good.
  int32_t max_od = 0;
  for (int64_t v = 0; v < V; ++v) max_od = std::max(max_od, ro[v + 1] - ro[v]);
  const double mean_od = V ? (double)ro[V] / (double)V : 0.0;
  const bool renumber = V > 0 && (double)max_od > kPrSkew * std::max(1.0, mean_od);
  std::vector<int32_t> old_of, new_of;
  if (renumber) {
    old_of.resize((size_t)V);
    new_of.resize((size_t)V);
    for (int64_t v = 0; v < V; ++v) old_of[v] = (int32_t)v;
    std::stable_sort(old_of.begin(), old_of.end(),
                     [&](int32_t x, int32_t y) { return ro[x + 1] - ro[x] > ro[y + 1] - ro[y]; });
    for (int64_t i = 0; i < V; ++i) new_of[old_of[i]] = (int32_t)i;
    // offsets of the renumbered in-lists
    std::vector<int32_t> cn((size_t)V + 1, 0);
    for (int64_t i = 0; i < V; ++i) cn[i + 1] = cn[i] + (co[old_of[i] + 1] - co[old_of[i]]);
    int st;
    int32_t *d_old = nullptr, *d_new = nullptr, *d_cn = nullptr, *d_crow = nullptr;
    if ((st = device_alloc(g, (void **)&d_old, (size_t)V * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&d_new, (size_t)V * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&d_cn, ((size_t)V + 1) * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&d_crow, (size_t)g->edges * 4 + 64)) != MG_OK)
      return st;
    cudaError_t e2 = cudaMemcpyAsync(d_old, old_of.data(), (size_t)V * 4, cudaMemcpyHostToDevice, s);
    if (e2 == cudaSuccess) e2 = cudaMemcpyAsync(d_new, new_of.data(), (size_t)V * 4, cudaMemcpyHostToDevice, s);
    if (e2 == cudaSuccess) e2 = cudaMemcpyAsync(d_cn, cn.data(), ((size_t)V + 1) * 4, cudaMemcpyHostToDevice, s);
    if (e2 != cudaSuccess) return cuda_status(e2, "pagerank renumbering upload");
    k_pr_renumber<<<g->num_sms * 8, kNT, 0, s>>>(d_old, d_new, g->csr.csc_offsets, g->csr.csc_rows, d_cn, d_crow,
                                                  (int32_t)V);
    count_launch();
    if ((st = launch_check("pagerank renumbering")) != MG_OK) return st;
    g->pr_coff = d_cn;
    g->pr_crow = d_crow;
    g->pr_new_of = d_new;
    co.swap(cn);  // the plan below is built on the renumbered in-lists
  } else {
    g->pr_coff = g->csr.csc_offsets;
    g->pr_crow = g->csr.csc_rows;
    g->pr_new_of = nullptr;
  }
  std::vector<float> inv((size_t)V);
  int64_t ndang = 0;
  std::vector<int32_t> cv, cb, ce, hv, hf;
  for (int64_t v = 0; v < V; ++v) {
    const int64_t ov = renumber ? old_of[v] : v;  // v in the numbering the kernels use
    const int32_t od = ro[ov + 1] - ro[ov];
    inv[v] = od > 0 ? 1.0f / (float)od : 0.0f;
    ndang += od == 0;
    const int32_t b = co[v], en = co[v + 1];
    // the same rule as k_pr_iter: in-lists longer than kPrBig are chunked
    if (en - b > kPrBig) {
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
  // the reference's iteration cap knob (iter_num), clamped to 2^20
  const uint32_t max_iter = (uint32_t)std::max<int32_t>(0, std::min<int32_t>(o->iter_num, 1 << 20));
  PrArgs a;
  a.coff = g->pr_coff;
  a.crow = g->pr_crow;
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
  a.damping = (float)d;
  a.ctl = g->ws.ctl;
  k_pr_init<<<g->num_sms * 4, 256, 0, s>>>(a.inv, a.r0, a.c0, V, (float)inv_n);
  const double base0 = (1.0 - d) * inv_n + d * ((double)g->pr_ndangling * inv_n) * inv_n;
  k_pr_ctl_init<<<1, 32, 0, s>>>(a.ctl, max_iter, (unsigned long long)o->spin_limit, ctl_flags(nullptr), base0);
  count_launch(2);
  if ((st = launch_check("pagerank init")) != MG_OK) return st;
  const int grid = persistent_grid(g, o, 6);  // 48 warps per SM (40 registers per thread)
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
  if (g->pr_new_of) {
    // back to the caller's numbering, through the other rank buffer
    float *out = (res.ctl.level & 1) ? a.r0 : a.r1;
    k_pr_unrenumber<<<g->num_sms * 4, 256, 0, s>>>(final_r, g->pr_new_of, out, V);
    count_launch();
    if ((st = launch_check("pagerank renumbering")) != MG_OK) return st;
    final_r = out;
  }
  return copy_out(s, ranks, final_r, (size_t)V * 4, o->outputs_on_device != 0);
}
