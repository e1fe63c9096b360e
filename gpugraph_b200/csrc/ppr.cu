// Personalised PageRank with its adjoint (no reference counterpart): the
// forward solve and the gradients of a loss with respect to the teleport
// vectors and the edge weights.
//
// Forward:  R = (1-d) T + d P^T R,  R, T in [V][nvec] (row-major), P[u,v] = w(e(u,v))
//           solved by power iteration pulled over the in-edges (CSC):
//           R'[v,:] = (1-d) T[v,:] + d * sum_{u->v} w(u,v) R[u,:]
// Adjoint:  for L with G = dL/dR, lambda = G + d P lambda, pulled over the
//           out-edges (CSR): lambda'[u,:] = G[u,:] + d * sum_{u->v} w(u,v) lambda[v,:]
//           dL/dT = (1-d) lambda,  dL/dw(u,v) = d * <lambda[v,:], R[u,:]>
// Both solves stop when the L1 change over all entries is <= tolerance times
// the L1 norm of their right-hand side (T or G; for teleport columns that are
// distributions that is tolerance * nvec), or after iter_num iterations.
//
// Layout and work split: a warp owns one chunk of one vertex's adjacency and
// lane c owns columns c and c+32, so every edge costs one coalesced read of a
// 128-byte row (nvec = 32) plus a broadcast index/weight load; eight edges
// (four for nvec > 32) are in flight per step. The forward solve reads the
// weights gathered into CSC order once per solve. In-lists longer than
// kPprChunk are cut into chunks whose partial rows are added in chunk order by
// a fix-up pass (deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"

namespace mg {

constexpr int kPprChunk = 256;
constexpr int kPprMaxVec = 64;

struct PprArgs {
  const int32_t *off, *idx, *eid;  // adjacency of the solve (CSC forward, CSR adjoint); eid may be null
  const float *w;                  // weights per CSR edge
  const float *rhs;                // T (forward) or G (adjoint), [V][nvec]
  float alpha, d;                  // X' = alpha*rhs + d*sum(...)
  float *x0, *x1, *partial;
  const int32_t *cv, *cb, *ce, *cslot, *mv, *mfirst;
  int32_t nchunks, nmulti, nvec, V;
  Ctl *ctl;
};

template <int NC>
MG_DEVINL void ppr_finalize_row(const PprArgs &a, int v, const float (&acc)[NC], const float *xold, float *xnew,
                                double &res) {
  const int lane = lane_id();
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const int c = lane + 32 * q;
    if (c < a.nvec) {
      const int64_t o = (int64_t)v * a.nvec + c;
      const float xn = fmaf(a.d, acc[q], a.alpha * a.rhs[o]);
      res += (double)fabsf(xn - xold[o]);
      xnew[o] = xn;
    }
  }
}

template <int NC>
__global__ void __launch_bounds__(kNT) k_ppr_iter(PprArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float *xold = (L & 1) ? a.x1 : a.x0;
  float *xnew = (L & 1) ? a.x0 : a.x1;
  const int lane = lane_id();
  double res = 0.0;
  unsigned long long my_bytes = 0;
  const uint32_t nwarps = gridDim.x * kNW;
  for (uint32_t c = blockIdx.x * kNW + warp_id(); c < (uint32_t)a.nchunks; c += nwarps) {
    const int v = a.cv[c], b = a.cb[c], e = a.ce[c], slot = a.cslot[c];
    float acc[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) acc[q] = 0.f;
    // EPS edges per step, all their loads in flight (predicated at the end of
    // the chunk): index and weight, then the EPS gathered rows
    constexpr int EPS = NC == 1 ? 8 : 4;
    for (int k = b; k < e; k += EPS) {
      int u[EPS];
      float wt[EPS];
#pragma unroll
      for (int j = 0; j < EPS; ++j) {
        const bool in = k + j < e;
        u[j] = in ? a.idx[k + j] : -1;
        wt[j] = in ? a.w[a.eid ? a.eid[k + j] : k + j] : 0.f;
      }
      float row[EPS][NC];
#pragma unroll
      for (int j = 0; j < EPS; ++j)
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          const int col = lane + 32 * q;
          row[j][q] = (u[j] >= 0 && col < a.nvec) ? __ldg(&xold[(int64_t)u[j] * a.nvec + col]) : 0.f;
        }
#pragma unroll
      for (int j = 0; j < EPS; ++j)
#pragma unroll
        for (int q = 0; q < NC; ++q) acc[q] = fmaf(wt[j], row[j][q], acc[q]);
    }
    if (lane == 0) my_bytes += (unsigned long long)(e - b) * (8ull + 4ull * a.nvec);
    if (slot < 0) {
      ppr_finalize_row<NC>(a, v, acc, xold, xnew, res);
      if (lane == 0) my_bytes += 12ull * a.nvec;
    } else {
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        const int col = lane + 32 * q;
        if (col < a.nvec) a.partial[(int64_t)slot * a.nvec + col] = acc[q];
      }
    }
  }
  add_bytes(ctl, KID_PPR, my_bytes);
  res = cta_sum_f64(res);
  if (threadIdx.x == 0 && res != 0.0) atomicAdd(&ctl->acc[1], res);
}

// Vector variant for nvec % 4 == 0 (rows 16-byte aligned): a group of G lanes
// owns one chunk and lane l of the group columns 4l..4l+3, one 16-byte load
// per gathered row, so a warp works on 32/G chunks at once (4 for nvec <= 32,
// 2 for nvec <= 64): that many chunks' index, weight and row loads are in
// flight per step instead of one. Per column the edges are added in the same
// order as in k_ppr_iter, so both give the same ranks.
template <int G>
__global__ void __launch_bounds__(kNT, 4) k_ppr_iter_v(PprArgs a) {
  constexpr int PER = 32 / G;
  constexpr int EPS = 8;
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float *xold = (L & 1) ? a.x1 : a.x0;
  float *xnew = (L & 1) ? a.x0 : a.x1;
  const int lane = lane_id();
  const int gl = lane & (G - 1);
  const int col = gl * 4;
  const bool cok = col < a.nvec;
  double res = 0.0;
  unsigned long long my_bytes = 0;
  const uint32_t nslots = gridDim.x * kNW * PER;
  for (uint32_t c = (blockIdx.x * kNW + warp_id()) * PER + lane / G; c < (uint32_t)a.nchunks; c += nslots) {
    const int v = a.cv[c], b = a.cb[c], e = a.ce[c], slot = a.cslot[c];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = b; k < e; k += EPS) {
      int u[EPS];
      float wt[EPS];
#pragma unroll
      for (int j = 0; j < EPS; ++j) {
        const bool in = k + j < e;
        u[j] = in ? a.idx[k + j] : -1;
        wt[j] = in ? a.w[a.eid ? a.eid[k + j] : k + j] : 0.f;
      }
      float4 row[EPS];
#pragma unroll
      for (int j = 0; j < EPS; ++j)
        row[j] = (u[j] >= 0 && cok) ? __ldg(reinterpret_cast<const float4 *>(xold + (int64_t)u[j] * a.nvec + col))
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int j = 0; j < EPS; ++j) {
        acc.x = fmaf(wt[j], row[j].x, acc.x);
        acc.y = fmaf(wt[j], row[j].y, acc.y);
        acc.z = fmaf(wt[j], row[j].z, acc.z);
        acc.w = fmaf(wt[j], row[j].w, acc.w);
      }
    }
    if (gl == 0) my_bytes += (unsigned long long)(e - b) * (8ull + 4ull * a.nvec);
    if (slot < 0) {
      if (cok) {
        const int64_t o = (int64_t)v * a.nvec + col;
        const float4 r = *reinterpret_cast<const float4 *>(a.rhs + o);
        const float4 xo = *reinterpret_cast<const float4 *>(xold + o);
        float4 xn;
        xn.x = fmaf(a.d, acc.x, a.alpha * r.x);
        xn.y = fmaf(a.d, acc.y, a.alpha * r.y);
        xn.z = fmaf(a.d, acc.z, a.alpha * r.z);
        xn.w = fmaf(a.d, acc.w, a.alpha * r.w);
        res += (double)fabsf(xn.x - xo.x) + (double)fabsf(xn.y - xo.y) + (double)fabsf(xn.z - xo.z) +
               (double)fabsf(xn.w - xo.w);
        *reinterpret_cast<float4 *>(xnew + o) = xn;
      }
      if (gl == 0) my_bytes += 12ull * a.nvec;
    } else if (cok) {
      *reinterpret_cast<float4 *>(a.partial + (int64_t)slot * a.nvec + col) = acc;
    }
  }
  add_bytes(ctl, KID_PPR, my_bytes);
  res = cta_sum_f64(res);
  if (threadIdx.x == 0 && res != 0.0) atomicAdd(&ctl->acc[1], res);
}

// Split vertices: partial rows added in chunk order.
template <int NC>
__global__ void __launch_bounds__(kNT) k_ppr_fixup(PprArgs a) {
  Ctl *ctl = a.ctl;
  if (!ctl->active) return;
  const uint32_t L = ctl->level;
  const float *xold = (L & 1) ? a.x1 : a.x0;
  float *xnew = (L & 1) ? a.x0 : a.x1;
  const int lane = lane_id();
  double res = 0.0;
  const uint32_t nwarps = gridDim.x * kNW;
  for (uint32_t m = blockIdx.x * kNW + warp_id(); m < (uint32_t)a.nmulti; m += nwarps) {
    const int v = a.mv[m];
    float acc[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) acc[q] = 0.f;
    // eight partial rows loaded at once, then added in chunk order (a hub has
    // hundreds of chunks; one dependent load per chunk made this the tail)
    int s = a.mfirst[m];
    const int se = a.mfirst[m + 1];
    for (; s + 8 <= se; s += 8) {
      float t[8][NC];
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          const int col = lane + 32 * q;
          t[j][q] = col < a.nvec ? a.partial[(int64_t)(s + j) * a.nvec + col] : 0.f;
        }
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int q = 0; q < NC; ++q) acc[q] += t[j][q];
    }
    for (; s < se; ++s)
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        const int col = lane + 32 * q;
        if (col < a.nvec) acc[q] += a.partial[(int64_t)s * a.nvec + col];
      }
    ppr_finalize_row<NC>(a, v, acc, xold, xnew, res);
  }
  res = cta_sum_f64(res);
  if (threadIdx.x == 0 && res != 0.0) atomicAdd(&ctl->acc[1], res);
}

// ctl->acc[2] holds the L1 norm of the right-hand side (k_ppr_rhs_norm).
__global__ void k_ppr_level_end(Ctl *ctl, double tol, cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x != 0) return;
  if (ctl->active) {
    const double res = ctl->acc[1];
    ctl->acc[1] = 0.0;
    ctl->residual = res;
    ctl->level += 1;
    ctl->push_levels += 1;
    ctl->active = (res > tol * ctl->acc[2] && ctl->level < ctl->max_iter && ctl->error == 0) ? 1u : 0u;
  }
  if (use_handle) cudaGraphSetConditional(h, ctl->active);
}

// dL/dw(u,v) = d <lambda[v,:], R[u,:]>: warp per out-edge chunk of the CSR
// chunk plan (a row, or at most kPprChunk edges of a long row, so a hub's row
// is spread over many warps), R[u,:] held in registers, EPS out-edges per step
// with all their row gathers in flight before the warp reductions.
template <int NC>
__global__ void __launch_bounds__(kNT) k_ppr_edge_grad(const int32_t *cv, const int32_t *cb, const int32_t *ce,
                                                       int32_t nchunks, const int32_t *col, int32_t nvec,
                                                       const float *lam, const float *R, float d, float *grad_w,
                                                       Ctl *ctl) {
  constexpr int EPS = NC == 1 ? 8 : 4;
  const int lane = lane_id();
  const uint32_t nwarps = gridDim.x * kNW;
  unsigned long long my_bytes = 0;
  for (uint32_t c = blockIdx.x * kNW + warp_id(); c < (uint32_t)nchunks; c += nwarps) {
    const int u = cv[c], b = cb[c], e = ce[c];
    if (b == e) continue;
    float ru[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const int cc = lane + 32 * q;
      ru[q] = (cc < nvec) ? R[(int64_t)u * nvec + cc] : 0.f;
    }
    for (int k = b; k < e; k += EPS) {
      int v[EPS];
#pragma unroll
      for (int j = 0; j < EPS; ++j) v[j] = (k + j < e) ? col[k + j] : -1;
      float dot[EPS];
#pragma unroll
      for (int j = 0; j < EPS; ++j) {
        dot[j] = 0.f;
        if (v[j] >= 0) {
#pragma unroll
          for (int q = 0; q < NC; ++q) {
            const int cc = lane + 32 * q;
            if (cc < nvec) dot[j] = fmaf(__ldg(&lam[(int64_t)v[j] * nvec + cc]), ru[q], dot[j]);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < EPS; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot[j] += __shfl_xor_sync(0xffffffffu, dot[j], o);
      }
      // lane j writes edge k + j
      float mine = dot[0];
#pragma unroll
      for (int j = 1; j < EPS; ++j)
        if (lane == j) mine = dot[j];
      if (lane < EPS && k + lane < e) grad_w[k + lane] = d * mine;
    }
    if (lane == 0) my_bytes += 4ull * nvec + (unsigned long long)(e - b) * (8ull + 4ull * nvec);
  }
  add_bytes(ctl, KID_PPR, my_bytes);
}

// L1 norm of the right-hand side into ctl->acc[2] (FP64 accumulation).
__global__ void k_ppr_rhs_norm(const float *rhs, int64_t n, Ctl *ctl) {
  double sum = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    sum += fabs((double)rhs[i]);
  sum = cta_sum_f64(sum);
  if (threadIdx.x == 0 && sum != 0.0) atomicAdd(&ctl->acc[2], sum);
}

__global__ void k_scale_copy(const float *src, float *dst, float s, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = s * src[i];
}

__global__ void k_copy_f32(const float *src, float *dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

__global__ void k_gather_f32(const int32_t *idx, const float *src, float *dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

// Chunk plan for the solve over `off` (host copy of the offsets).
static int build_plan(mg_graph *g, const std::vector<int32_t> &off, mg_graph::PprPlan *p, cudaStream_t s) {
  const int64_t V = g->nodes;
  std::vector<int32_t> cv, cb, ce, cs, mv, mf;
  int32_t slots = 0;
  for (int64_t v = 0; v < V; ++v) {
    const int32_t b = off[v], e = off[v + 1];
    if (e - b <= kPprChunk) {
      cv.push_back((int32_t)v);
      cb.push_back(b);
      ce.push_back(e);
      cs.push_back(-1);
    } else {
      mv.push_back((int32_t)v);
      mf.push_back(slots);
      for (int32_t x = b; x < e; x += kPprChunk) {
        cv.push_back((int32_t)v);
        cb.push_back(x);
        ce.push_back(std::min(e, x + kPprChunk));
        cs.push_back(slots++);
      }
    }
  }
  mf.push_back(slots);
  int st;
  const size_t nc = std::max<size_t>(cv.size(), 1), nm = std::max<size_t>(mv.size(), 1);
  if ((st = device_alloc(g, (void **)&p->cv, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&p->cb, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&p->ce, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&p->cslot, nc * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&p->mv, nm * 4)) != MG_OK ||
      (st = device_alloc(g, (void **)&p->mfirst, (nm + 1) * 4)) != MG_OK)
    return st;
  cudaError_t e = cudaSuccess;
  if (!cv.empty()) {
    e = cudaMemcpyAsync(p->cv, cv.data(), cv.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->cb, cb.data(), cb.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->ce, ce.data(), ce.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->cslot, cs.data(), cs.size() * 4, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess && !mv.empty()) e = cudaMemcpyAsync(p->mv, mv.data(), mv.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->mfirst, mf.data(), mf.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "ppr plan upload");
  p->nchunks = (int32_t)cv.size();
  p->nmulti = (int32_t)mv.size();
  p->nslots = slots;
  return MG_OK;
}

static int ppr_prepare(mg_graph *g, int32_t nvec, cudaStream_t s) {
  int st;
  if (!g->ppr_plan[0].cv) {
    const int64_t V = g->nodes;
    std::vector<int32_t> co((size_t)V + 1), ro((size_t)V + 1);
    cudaError_t e = cudaMemcpyAsync(co.data(), g->csr.csc_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ro.data(), g->csr.row_offsets, (V + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "ppr plan read");
    if ((st = build_plan(g, co, &g->ppr_plan[0], s)) != MG_OK) return st;
    if ((st = build_plan(g, ro, &g->ppr_plan[1], s)) != MG_OK) return st;
  }
  if (g->ppr_cap_nvec < nvec) {
    const size_t V = (size_t)g->nodes;
    const int32_t slots = std::max(std::max(g->ppr_plan[0].nslots, g->ppr_plan[1].nslots), 1);
    if ((st = device_alloc(g, (void **)&g->ppr_x[0], V * nvec * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&g->ppr_x[1], V * nvec * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&g->ppr_rhs, V * nvec * 4)) != MG_OK ||
        (st = device_alloc(g, (void **)&g->ppr_partial, (size_t)slots * nvec * 4)) != MG_OK)
      return st;
    g->ppr_cap_nvec = nvec;
  }
  if (!g->ppr_w && (st = device_alloc(g, (void **)&g->ppr_w, (size_t)g->edges * 4 + 64)) != MG_OK) return st;
  return MG_OK;
}

static bool is_device_ptr(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Runs one power-iteration solve; on return the solution is in *result.
static int ppr_solve(mg_graph *g, int dir, const float *w, const float *rhs, float alpha, int32_t nvec,
                     const mg_options *o, cudaStream_t s, const char *name, float **result, LoopResult *res) {
  const mg_graph::PprPlan &p = g->ppr_plan[dir];
  // The level loop is captured once and replayed: its kernels read the inputs
  // from the graph's own buffers, so callers may pass different pointers.
  const int64_t n = (int64_t)g->nodes * nvec;
  k_copy_f32<<<g->num_sms * 4, 256, 0, s>>>(rhs, g->ppr_rhs, n);
  // the weights in the order the solve reads its adjacency (CSC order for the
  // forward pull, so no edge-id indirection per edge and iteration)
  if (dir == 0) k_gather_f32<<<g->num_sms * 4, 256, 0, s>>>(g->csr.csc_eid, w, g->ppr_w, g->edges);
  else k_copy_f32<<<g->num_sms * 4, 256, 0, s>>>(w, g->ppr_w, g->edges);
  count_launch(2);
  w = g->ppr_w;
  rhs = g->ppr_rhs;
  PprArgs a;
  a.off = dir == 0 ? g->csr.csc_offsets : g->csr.row_offsets;
  a.idx = dir == 0 ? g->csr.csc_rows : g->csr.col;
  a.eid = nullptr;
  a.w = w;
  a.rhs = rhs;
  a.alpha = alpha;
  a.d = (float)o->damping;
  a.x0 = g->ppr_x[0];
  a.x1 = g->ppr_x[1];
  a.partial = g->ppr_partial;
  a.cv = p.cv;
  a.cb = p.cb;
  a.ce = p.ce;
  a.cslot = p.cslot;
  a.mv = p.mv;
  a.mfirst = p.mfirst;
  a.nchunks = p.nchunks;
  a.nmulti = p.nmulti;
  a.nvec = nvec;
  a.V = g->csr.V;
  a.ctl = g->ws.ctl;
  // start from the right-hand side
  k_copy_f32<<<g->num_sms * 4, 256, 0, s>>>(rhs, a.x0, n);
  const uint32_t max_iter = (uint32_t)std::max<int32_t>(0, std::min<int32_t>(o->iter_num, 100000));
  k_ctl_init<<<1, 32, 0, s>>>(a.ctl, 1u, max_iter, (unsigned long long)o->spin_limit, MODE_QUEUE, ctl_flags(nullptr));
  k_ppr_rhs_norm<<<g->num_sms * 4, 256, 0, s>>>(rhs, n, a.ctl);
  count_launch(3);
  const int grid = persistent_grid(g, o, 4);
  const double tol = o->tolerance;
  const bool two = nvec > 32;
  const bool vec = nvec % 4 == 0;  // 16-byte rows: the vector variant
  LevelBody body = [=](cudaStream_t ss, cudaGraphConditionalHandle h, int use_h) {
    if (two) {
      if (vec) MG_LAUNCH(KID_PPR, ss, k_ppr_iter_v<16><<<grid, kNT, 0, ss>>>(a));
      else MG_LAUNCH(KID_PPR, ss, k_ppr_iter<2><<<grid, kNT, 0, ss>>>(a));
      MG_LAUNCH(KID_PPR, ss, k_ppr_fixup<2><<<grid, kNT, 0, ss>>>(a));
    } else {
      if (vec) MG_LAUNCH(KID_PPR, ss, k_ppr_iter_v<8><<<grid, kNT, 0, ss>>>(a));
      else MG_LAUNCH(KID_PPR, ss, k_ppr_iter<1><<<grid, kNT, 0, ss>>>(a));
      MG_LAUNCH(KID_PPR, ss, k_ppr_fixup<1><<<grid, kNT, 0, ss>>>(a));
    }
    MG_LAUNCH(KID_OTHER, ss, k_ppr_level_end<<<1, 32, 0, ss>>>(a.ctl, tol, h, use_h));
  };
  char key[160];
  snprintf(key, sizeof(key), "%s/%d/%d/%.9g/%.17g/%.17g", name, grid, nvec, (double)alpha, o->damping, tol);
  int st = run_level_loop(g, s, key, 3, body, o->use_cuda_graph != 0, res);
  if (st != MG_OK) return st;
  finish_run(g, res->ctl.level);
  if (res->ctl.error)
    return set_error(res->ctl.error, std::string(name) + ": device reported " + mg_status_string(res->ctl.error));
  *result = (res->ctl.level & 1) ? a.x1 : a.x0;
  return MG_OK;
}

static void ppr_stats(mg_stats *stats, const LoopResult &res, double tol, mg_graph *g) {
  const double tol_total = tol * res.ctl.acc[2];
  if (!stats) return;
  stats->iterations = (int32_t)res.ctl.level;
  stats->push_iterations = 0;
  stats->pull_iterations = (int32_t)res.ctl.level;
  stats->converged = res.ctl.residual <= tol_total ? 1 : 0;
  stats->device_ms = res.ms;
  stats->residual = res.ctl.residual;
  stats->vertices_reached = g->nodes;
  stats->edges_traversed = g->edges * (int64_t)res.ctl.level;
}

static const mg_options *opts_or_default(const mg_options *o, mg_options *d) {
  if (o) return o;
  mg_options_init(d);
  d->tolerance = 1e-7;
  return d;
}

}  // namespace mg

using namespace mg;

extern "C" {

int mg_ppr_forward(mg_graph *g, const float *edge_weights, const float *teleport, int32_t nvec, float *ranks,
                   mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (nvec < 1 || nvec > kPprMaxVec) return set_error(MG_ERR_ARG, "nvec must be in [1, 64]");
  if (!g->directed)
    return set_error(MG_ERR_UNSUPPORTED, "personalised PageRank needs the transpose: create the graph with directed=1");
  if (!edge_weights || !teleport || !ranks) return set_error(MG_ERR_ARG, "NULL pointer");
  if (!is_device_ptr(edge_weights) || !is_device_ptr(teleport) || !is_device_ptr(ranks))
    return set_error(MG_ERR_ARG, "mg_ppr_forward takes device pointers");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  if (!(o->damping >= 0.0 && o->damping < 1.0)) return set_error(MG_ERR_ARG, "damping must be in [0, 1)");
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK || (st = ppr_prepare(g, nvec, s)) != MG_OK) return st;
  float *x = nullptr;
  LoopResult res;
  if ((st = ppr_solve(g, 0, edge_weights, teleport, (float)(1.0 - o->damping), nvec, o, s, "ppr_fwd", &x, &res)) !=
      MG_OK)
    return st;
  ppr_stats(stats, res, o->tolerance, g);
  return copy_out(s, ranks, x, (size_t)g->nodes * nvec * 4, true);
}

int mg_ppr_backward(mg_graph *g, const float *edge_weights, const float *ranks, const float *grad_ranks, int32_t nvec,
                    float *grad_edge_weights, float *grad_teleport, mg_stats *stats, const mg_options *opts) {
  clear_error();
  if (!g) return set_error(MG_ERR_ARG, "graph is NULL");
  if (nvec < 1 || nvec > kPprMaxVec) return set_error(MG_ERR_ARG, "nvec must be in [1, 64]");
  if (!g->directed)
    return set_error(MG_ERR_UNSUPPORTED, "personalised PageRank needs the transpose: create the graph with directed=1");
  if (!edge_weights || !ranks || !grad_ranks) return set_error(MG_ERR_ARG, "NULL pointer");
  if (!is_device_ptr(edge_weights) || !is_device_ptr(ranks) || !is_device_ptr(grad_ranks) ||
      (grad_edge_weights && !is_device_ptr(grad_edge_weights)) || (grad_teleport && !is_device_ptr(grad_teleport)))
    return set_error(MG_ERR_ARG, "mg_ppr_backward takes device pointers");
  mg_options d;
  const mg_options *o = opts_or_default(opts, &d);
  if (!(o->damping >= 0.0 && o->damping < 1.0)) return set_error(MG_ERR_ARG, "damping must be in [0, 1)");
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK || (st = ppr_prepare(g, nvec, s)) != MG_OK) return st;
  float *lam = nullptr;
  LoopResult res;
  if ((st = ppr_solve(g, 1, edge_weights, grad_ranks, 1.0f, nvec, o, s, "ppr_adj", &lam, &res)) != MG_OK) return st;
  const int grid = persistent_grid(g, o, 4);
  if (grad_edge_weights) {
    const mg_graph::PprPlan &pl = g->ppr_plan[1];  // chunks of the out-edge rows
    if (nvec > 32)
      k_ppr_edge_grad<2><<<grid, kNT, 0, s>>>(pl.cv, pl.cb, pl.ce, pl.nchunks, g->csr.col, nvec, lam, ranks,
                                              (float)o->damping, grad_edge_weights, g->ws.ctl);
    else
      k_ppr_edge_grad<1><<<grid, kNT, 0, s>>>(pl.cv, pl.cb, pl.ce, pl.nchunks, g->csr.col, nvec, lam, ranks,
                                              (float)o->damping, grad_edge_weights, g->ws.ctl);
    count_launch();
  }
  if (grad_teleport) {
    k_scale_copy<<<g->num_sms * 4, 256, 0, s>>>(lam, grad_teleport, (float)(1.0 - o->damping),
                                                (int64_t)g->nodes * nvec);
    count_launch();
  }
  ppr_stats(stats, res, o->tolerance, g);
  return cuda_status(cudaStreamSynchronize(s), "ppr backward");
}

}  // extern "C"
