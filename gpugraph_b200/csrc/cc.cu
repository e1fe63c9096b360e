// Connected components of a symmetric graph by concurrent union-find, giving
// the labels of the reference's cc program (Algorithms/CC/cc.h:32-349: every
// vertex starts with its own id and atomicMin-propagates it along out-edges
// to a fixpoint, so on a symmetric graph each vertex ends with the smallest
// id of its component). Links always put the larger root under the smaller,
// so a root is the smallest id of its tree and the final find() of a vertex is
// exactly that label. Directed graphs keep the GAS program (mg_cc in
// gas_algos.cu), whose semantics there are not components.
//
// Order of work (the sampling scheme of Sutton et al., "Optimizing Parallel
// Graph Connectivity Computation via Subgraph Sampling", IPDPS 2018):
//   1. every vertex links with its first kCcSample neighbours, compressing the
//      trees after each round;
//   2. the most frequent root among kCcProbe fixed sample vertices names the
//      large component;
//   3. every vertex not already under that root links the rest of its edges.
// An edge skipped in step 3 joins two vertices of the large component, or is
// linked from its other end, which is not in it; on power-law graphs step 3
// touches a small share of the edges.
#include <cuda_runtime.h>

#include <climits>

#include "algo_util.cuh"
#include "gas/driver.cuh"
#include "gas/engine.cuh"

namespace mg {

// Root of x with path halving. Parent ids only decrease along a path and a
// root only ever becomes a non-root, so the walk ends and every shortcut
// written points to an ancestor.
MG_DEVINL int32_t cc_find(int32_t *parent, int32_t x) {
  for (;;) {
    const int32_t p = __ldcg(&parent[x]);
    if (p == x) return x;
    const int32_t gp = __ldcg(&parent[p]);
    if (gp == p) return p;
    parent[x] = gp;
    x = gp;
  }
}

// Links the components of a and b: the larger root is hooked under the smaller
// with atomicMin, which always succeeds. If the larger one was no longer a
// root (another link hooked it to `old` first), its tree and the smaller root
// still have to be joined: link old with the smaller root next. Every round
// hooks something, parent values only decrease, and the retries are bounded
// all the same (a failure is reported, not looped on).
MG_DEVINL bool cc_unite(int32_t *parent, int32_t a, int32_t b, unsigned long long limit) {
  for (unsigned long long it = 0; it < limit; ++it) {
    a = cc_find(parent, a);
    b = cc_find(parent, b);
    if (a == b) return true;
    const int32_t hi = a > b ? a : b, lo = a > b ? b : a;
    const int32_t old = atomicMin(&parent[hi], lo);
    if (old == hi) return true;
    a = old;
    b = lo;
  }
  return false;
}

constexpr int kCcSample = 2;    // neighbours linked per vertex before the large component is picked
constexpr int kCcProbe = 1024;  // sample vertices voting for the large component (one CTA)

// Step 1, round r: vertex v links with its r-th neighbour.
__global__ void __launch_bounds__(kNT) k_cc_sample(const int32_t *ro, const int32_t *col, int32_t *parent, int32_t V,
                                                   int r, Ctl *ctl) {
  const unsigned long long limit = ctl->spin_limit;
  bool ok = true;
  unsigned long long my_bytes = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int e = ro[v] + r;
    my_bytes += 8;  // two offsets
    if (e < ro[v + 1]) {
      my_bytes += 12;  // the neighbour id, the two parents read by the link
      if (!cc_unite(parent, v, col[e], limit)) ok = false;
    }
  }
  if (!ok) raise_error(ctl, MG_ERR_TIMEOUT);
  add_bytes(ctl, KID_CC, my_bytes);
}

// Step 2: the root held by most of kCcProbe fixed sample vertices (ties: the
// smaller root); parent[] is flat here. Written to *giant.
__global__ void __launch_bounds__(kCcProbe) k_cc_giant(const int32_t *parent, int32_t V, int32_t *giant) {
  __shared__ int32_t s_lab[kCcProbe];
  __shared__ unsigned long long s_best[kCcProbe / 32];
  const int t = threadIdx.x;
  // fixed multiplicative-hash sample of the vertex ids
  const int v = (int)(((unsigned long long)(t + 1) * 2654435761ull) % (unsigned long long)V);
  s_lab[t] = parent[v];
  __syncthreads();
  const int mine = s_lab[t];
  int cnt = 0;
  for (int k = 0; k < kCcProbe; ++k) cnt += s_lab[k] == mine;
  // largest count, then smallest root: pack (count, ~root) and take the max
  unsigned long long key = ((unsigned long long)cnt << 32) | (uint32_t)(~(uint32_t)mine);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other > key ? other : key;
  }
  if (lane_id() == 0) s_best[warp_id()] = key;
  __syncthreads();
  if (t < 32) {
    key = s_best[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
      key = other > key ? other : key;
    }
    if (t == 0) *giant = (int32_t)(~(uint32_t)(key & 0xffffffffu));
  }
}

// Step 3: vertices outside the large component link their remaining edges. A
// warp takes 32 consecutive vertices; lists up to 32 edges are walked by their
// own lane, longer ones by the whole warp (32 edges per step).
__global__ void __launch_bounds__(kNT) k_cc_rest(const int32_t *ro, const int32_t *col, int32_t *parent, int32_t V,
                                                 const int32_t *giant, Ctl *ctl) {
  const unsigned long long limit = ctl->spin_limit;
  const int32_t big = *giant;
  const int lane = lane_id();
  bool ok = true;
  unsigned long long my_bytes = 0;
  const uint32_t groups = ((uint32_t)V + 31) / 32;
  for (uint32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) / 32; grp < groups;
       grp += (gridDim.x * blockDim.x) / 32) {
    const int v = (int)(grp * 32) + lane;
    bool work = false;
    int b = 0, e = 0;
    if (v < V) {
      my_bytes += 12;  // parent, two offsets
      b = ro[v] + kCcSample;
      e = ro[v + 1];
      work = b < e && __ldcg(&parent[v]) != big;
    }
    if (work && e - b <= 32) {
      for (int k = b; k < e; ++k) {
        my_bytes += 4;
        if (!cc_unite(parent, v, col[k], limit)) ok = false;
      }
    }
    uint32_t heavy = __ballot_sync(0xffffffffu, work && e - b > 32);
    while (heavy) {
      const int h = __ffs(heavy) - 1;
      heavy &= heavy - 1;
      const int hv = (int)(grp * 32) + h;
      const int hb = __shfl_sync(0xffffffffu, b, h), he = __shfl_sync(0xffffffffu, e, h);
      for (int k = hb + lane; k < he; k += 32) {
        my_bytes += 4;
        if (!cc_unite(parent, hv, col[k], limit)) ok = false;
      }
    }
  }
  if (!ok) raise_error(ctl, MG_ERR_TIMEOUT);
  add_bytes(ctl, KID_CC, my_bytes);
}

// Final labels: every vertex's root (the smallest id of its component).
__global__ void __launch_bounds__(kNT) k_cc_flatten(int32_t *parent, int32_t V, Ctl *ctl) {
  unsigned long long my_bytes = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int r = cc_find(parent, v);
    parent[v] = r;
    my_bytes += 12;  // the vertex's parent, its root's parent, the write
  }
  add_bytes(ctl, KID_CC, my_bytes);
}

// Union-find CC on a symmetric graph (called by mg_cc).
int cc_union_find(mg_graph *g, int32_t *labels, mg_stats *stats, const mg_options *o) {
  cudaStream_t s = run_stream(g, o);
  int st = prepare_run(g, s);
  if (st != MG_OK) return st;
  const int32_t V = g->csr.V;
  if (V < 1) return set_error(MG_ERR_ARG, "cc: empty graph");
  int32_t *parent = g->ws.vbuf[0];
  Ctl *ctl = g->ws.ctl;
  cudaError_t e = cudaEventRecord(g->ev0, s);
  if (e != cudaSuccess) return cuda_status(e, "event record");
  int32_t *giant = reinterpret_cast<int32_t *>(g->ws.scan);  // scratch word (the scan buffer is free here)
  const int vgrid = g->num_sms * 8;
  MG_LAUNCH(KID_CC, s, (k_sequence_i32<<<g->num_sms * 4, 256, 0, s>>>(parent, V)));
  k_ctl_init<<<1, 32, 0, s>>>(ctl, 1u, 1u, (unsigned long long)o->spin_limit, MODE_QUEUE, ctl_flags(nullptr));
  for (int r = 0; r < kCcSample; ++r) {
    MG_LAUNCH(KID_CC, s, (k_cc_sample<<<vgrid, kNT, 0, s>>>(g->csr.row_offsets, g->csr.col, parent, V, r, ctl)));
    MG_LAUNCH(KID_CC, s, (k_cc_flatten<<<vgrid, kNT, 0, s>>>(parent, V, ctl)));
  }
  MG_LAUNCH(KID_CC, s, (k_cc_giant<<<1, kCcProbe, 0, s>>>(parent, V, giant)));
  MG_LAUNCH(KID_CC, s, (k_cc_rest<<<vgrid, kNT, 0, s>>>(g->csr.row_offsets, g->csr.col, parent, V, giant, ctl)));
  MG_LAUNCH(KID_CC, s, (k_cc_flatten<<<vgrid, kNT, 0, s>>>(parent, V, ctl)));
  count_launch(5 + 2 * kCcSample);
  if ((st = launch_check("cc union-find")) != MG_OK) return st;
  e = cudaEventRecord(g->ev1, s);
  if (e != cudaSuccess) return cuda_status(e, "event record");
  Ctl c;
  if ((st = read_ctl(g, s, &c)) != MG_OK) return st;
  prof_flush(s, c.kbytes);
  if (c.error) return set_error(c.error, std::string("cc: device reported ") + mg_status_string(c.error));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, g->ev0, g->ev1);
  finish_run(g, 1);
  if (stats) {
    stats->iterations = 1;
    stats->push_iterations = 1;
    stats->pull_iterations = 0;
    stats->converged = 1;
    stats->device_ms = ms;
    stats->residual = 0.0;
    stats->vertices_reached = g->nodes;
    stats->edges_traversed = g->edges;
  }
  return copy_out(s, labels, parent, (size_t)V * 4, o->outputs_on_device != 0);
}

}  // namespace mg
