/*
 * ORACLE -- test infrastructure only, never part of the product path.
 *
 * Plain-C restatement of the reference's CPU algorithms for the GAS hot path,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to
 * check (and time) the CUDA library. Each function cites the reference code it
 * follows (paths relative to the reference project). Where the reference CPU
 * code is too slow at benchmark sizes (the O(V^2) CPUSSSP) or implements a
 * different specification (CPUPR vs the normalised PageRank), the restatement
 * says so; the reference functions themselves are compiled from their sources
 * into oracle/_ref/ by oracle/build_ref.sh and pin these restatements in the
 * tests.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SSSP_INF 100000000 /* sssp::INIT_VALUE, Algorithms/SSSP/sssp.h:43 */

/* CPUBFS (Algorithms/BFS/bfs.cu:57-111): FIFO BFS over out-edges, depth -1 when
 * unreachable. Several roots start at depth 0 together, as bfs::Initialize
 * (Algorithms/BFS/bfs.h:62-79) seeds every source with label 0. */
int oracle_bfs(int64_t n, const int32_t *ro, const int32_t *col, const int32_t *srcs, int32_t nsrc, int32_t *out) {
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  if (!q) return -1;
  for (int64_t i = 0; i < n; ++i) out[i] = -1;
  int64_t head = 0, tail = 0;
  for (int32_t i = 0; i < nsrc; ++i) {
    if (out[srcs[i]] == -1) {
      out[srcs[i]] = 0;
      q[tail++] = srcs[i];
    }
  }
  while (head < tail) {
    const int32_t u = q[head++];
    const int32_t nd = out[u] + 1;
    for (int32_t e = ro[u]; e < ro[u + 1]; ++e) {
      const int32_t v = col[e];
      if (out[v] == -1) {
        out[v] = nd;
        q[tail++] = v;
      }
    }
  }
  free(q);
  return 0;
}

/* CPUSSSP (Algorithms/SSSP/sssp.cu:126-183): Dijkstra selecting the unvisited
 * vertex of smallest distance by a linear scan (O(V^2)); a vertex at distance
 * >= SSSP_INF is never selected; relaxations compute in 64 bits. */
int oracle_sssp_array(int64_t n, const int32_t *ro, const int32_t *col, const int32_t *w, int32_t src, int32_t *dist) {
  char *visited = (char *)calloc((size_t)(n > 0 ? n : 1), 1);
  if (!visited) return -1;
  for (int64_t i = 0; i < n; ++i) dist[i] = SSSP_INF;
  dist[src] = 0;
  for (;;) {
    int64_t u = -1;
    int32_t sd = SSSP_INF;
    for (int64_t i = 0; i < n; ++i)
      if (!visited[i] && dist[i] < sd) {
        sd = dist[i];
        u = i;
      }
    if (u < 0) break;
    visited[u] = 1;
    for (int32_t j = ro[u]; j < ro[u + 1]; ++j) {
      const int32_t v = col[j];
      const long nl = (long)dist[u] + (long)w[j];
      if (nl < dist[v]) dist[v] = (int32_t)nl;
    }
  }
  free(visited);
  return 0;
}

/* Same output as CPUSSSP with a binary heap (O(E log V)): shortest distances are
 * unique, so the selection order does not change the result. Needed at scale 22,
 * where CPUSSSP "takes hours" (Makefile:151-163). */
typedef struct {
  int32_t d, v;
} hitem;
static void hpush(hitem *h, int64_t *sz, hitem x) {
  int64_t i = (*sz)++;
  while (i > 0) {
    int64_t p = (i - 1) >> 1;
    if (h[p].d <= x.d) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = x;
}
static hitem hpop(hitem *h, int64_t *sz) {
  hitem top = h[0], x = h[--(*sz)];
  int64_t i = 0, n = *sz;
  for (;;) {
    int64_t c = 2 * i + 1;
    if (c >= n) break;
    if (c + 1 < n && h[c + 1].d < h[c].d) ++c;
    if (h[c].d >= x.d) break;
    h[i] = h[c];
    i = c;
  }
  if (n > 0) h[i] = x;
  return top;
}
int oracle_sssp_heap(int64_t n, const int32_t *ro, const int32_t *col, const int32_t *w, int32_t src, int32_t *dist) {
  const int64_t m = ro[n];
  hitem *h = (hitem *)malloc(sizeof(hitem) * (size_t)(m + 2));
  if (!h) return -1;
  int64_t sz = 0;
  for (int64_t i = 0; i < n; ++i) dist[i] = SSSP_INF;
  dist[src] = 0;
  hitem s0 = {0, src};
  hpush(h, &sz, s0);
  while (sz > 0) {
    hitem t = hpop(h, &sz);
    if (t.d != dist[t.v]) continue;
    for (int32_t j = ro[t.v]; j < ro[t.v + 1]; ++j) {
      const int32_t v = col[j];
      const long nl = (long)t.d + (long)w[j];
      if (nl < dist[v]) {
        dist[v] = (int32_t)nl;
        hitem x = {(int32_t)nl, v};
        hpush(h, &sz, x);
      }
    }
  }
  free(h);
  return 0;
}

/* CPUCC (Algorithms/CC/cc.cu:127-169): labels start at the vertex id; sweeps in
 * id order set label[v] = min(label[v], min label of v's out-neighbours) until
 * no label changes. */
int oracle_cc_sweep(int64_t n, const int32_t *ro, const int32_t *col, int32_t *label) {
  for (int64_t i = 0; i < n; ++i) label[i] = (int32_t)i;
  int changed = 1;
  while (changed) {
    changed = 0;
    for (int64_t v = 0; v < n; ++v) {
      int32_t m = SSSP_INF;
      for (int32_t j = ro[v]; j < ro[v + 1]; ++j)
        if (label[col[j]] < m) m = label[col[j]];
      if (m < label[v]) {
        label[v] = m;
        changed = 1;
      }
    }
  }
  return 0;
}

/* The GAS cc program's fixpoint (Algorithms/CC/cc.h:262-342): labels pushed along
 * out-edges, label[v] = min id over the vertices with a path to v. Equal to
 * oracle_cc_sweep on symmetric graphs. Union-find for symmetric graphs would be
 * faster but would not state the directed semantics. */
int oracle_cc_push(int64_t n, const int32_t *ro, const int32_t *col, int32_t *label) {
  for (int64_t i = 0; i < n; ++i) label[i] = (int32_t)i;
  int changed = 1;
  while (changed) {
    changed = 0;
    for (int64_t u = 0; u < n; ++u) {
      const int32_t lu = label[u];
      for (int32_t j = ro[u]; j < ro[u + 1]; ++j)
        if (label[col[j]] > lu) {
          label[col[j]] = lu;
          changed = 1;
        }
    }
  }
  return 0;
}

/* The GAS pagerank program (Algorithms/PageRank/PageRank.h:33-409) restated
 * sequentially: ranks start at 0.15, the frontier starts with every vertex;
 * per iteration every frontier vertex gathers sum(rank[u]/outdeg[u]) over its
 * in-edges (all gathers before any apply), apply sets rank = 0.15 + 0.85*sum and
 * changed = |delta| >= tol; the next frontier is the out-neighbours of changed
 * vertices. outdeg is the reference's (row degree, plus column degree when
 * undirected). FP32 arithmetic, sequential sums. */
int oracle_pr_gas(int64_t n, const int32_t *ro, const int32_t *col, const int32_t *coff, const int32_t *crow,
                  const int32_t *outdeg, float tol, int32_t max_iter, float *rank, int32_t *iters) {
  char *inF = (char *)calloc((size_t)n, 1), *nxt = (char *)calloc((size_t)n, 1), *chg = (char *)calloc((size_t)n, 1);
  float *g = (float *)malloc(sizeof(float) * (size_t)n);
  if (!inF || !nxt || !chg || !g) return -1;
  for (int64_t v = 0; v < n; ++v) {
    rank[v] = 0.15f;
    inF[v] = 1;
  }
  int32_t it = 0;
  int64_t fsize = n;
  while (fsize > 0 && it < max_iter) {
    for (int64_t v = 0; v < n; ++v) {
      if (!inF[v]) continue;
      float s = 0.f;
      for (int32_t j = coff[v]; j < coff[v + 1]; ++j) s += rank[crow[j]] / (float)outdeg[crow[j]];
      g[v] = s;
    }
    for (int64_t v = 0; v < n; ++v) {
      if (!inF[v]) continue;
      const float nv = 0.15f + (1.0f - 0.15f) * g[v];
      chg[v] = fabsf(rank[v] - nv) < tol ? 0 : 1;
      rank[v] = nv;
    }
    memset(nxt, 0, (size_t)n);
    fsize = 0;
    for (int64_t u = 0; u < n; ++u) {
      if (!inF[u] || !chg[u]) continue;
      for (int32_t j = ro[u]; j < ro[u + 1]; ++j)
        if (!nxt[col[j]]) {
          nxt[col[j]] = 1;
          ++fsize;
        }
    }
    memcpy(inF, nxt, (size_t)n);
    ++it;
  }
  *iters = it;
  free(inF);
  free(nxt);
  free(chg);
  free(g);
  return 0;
}

/* Normalised PageRank in FP64 (the specification the CUDA mg_pagerank follows;
 * the reference's own PageRank is unnormalised, see oracle_pr_gas and CPUPR):
 *   r0 = 1/N;  r'[v] = (1-d)/N + d * (sum_{u->v} r[u]/outdeg[u] + dangling/N),
 *   dangling = sum of r over vertices with no out-edge;
 * stop after the iteration whose L1(r' - r) <= tol, or after max_iter. */
int oracle_pagerank_fp64(int64_t n, const int32_t *ro, const int32_t *coff, const int32_t *crow, double d, double tol,
                         int32_t max_iter, double *r, int32_t *iters, double *resid) {
  double *nr = (double *)malloc(sizeof(double) * (size_t)n);
  double *contrib = (double *)malloc(sizeof(double) * (size_t)n);
  if (!nr || !contrib) return -1;
  for (int64_t v = 0; v < n; ++v) r[v] = 1.0 / (double)n;
  int32_t it = 0;
  double l1 = 0.0;
  while (it < max_iter) {
    double dangling = 0.0;
    for (int64_t u = 0; u < n; ++u) {
      const int32_t od = ro[u + 1] - ro[u];
      if (od == 0) {
        dangling += r[u];
        contrib[u] = 0.0;
      } else {
        contrib[u] = r[u] / (double)od;
      }
    }
    const double base = (1.0 - d) / (double)n + d * dangling / (double)n;
    l1 = 0.0;
    for (int64_t v = 0; v < n; ++v) {
      double s = 0.0;
      for (int32_t j = coff[v]; j < coff[v + 1]; ++j) s += contrib[crow[j]];
      nr[v] = base + d * s;
      l1 += fabs(nr[v] - r[v]);
    }
    memcpy(r, nr, sizeof(double) * (size_t)n);
    ++it;
    if (l1 <= tol) break;
  }
  *iters = it;
  *resid = l1;
  free(nr);
  free(contrib);
  return 0;
}

/* pred_extract (Algorithms/BFS/predextract.cuh:246-375): for every vertex, the
 * in-edges' gather_edge values (:143-154: the in-neighbour u when
 * depth[v] - depth[u] == 1, else -1) reduced with max (ReduceFunctor :211-218)
 * from INIT_VALUE -1, so a vertex without such an in-neighbour (or without
 * in-edges, :236) gets -1. coff/crow: the in-lists (CSC). */
int oracle_bfs_pred(int64_t n, const int32_t *coff, const int32_t *crow, const int32_t *depth, int32_t *pred) {
  for (int64_t v = 0; v < n; ++v) {
    int32_t best = -1;
    for (int32_t j = coff[v]; j < coff[v + 1]; ++j) {
      const int32_t u = crow[j];
      const int32_t val = (depth[v] - depth[u]) == 1 ? u : -1;
      if (val > best) best = val;
    }
    pred[v] = best;
  }
  return 0;
}
