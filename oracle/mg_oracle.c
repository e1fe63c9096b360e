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

/* Seeded R-MAT input generator: a plain-C restatement of the product library's
 * host builder (mg_build_rmat: recursive quadrant choice as in the reference's
 * BuildRmatGraph, b40c/graph/builder/rmat.cuh:145-224, with counter-hash draws,
 * no per-level jitter and a seeded vertex relabelling; then a CSR with sorted
 * rows, optionally symmetrised, self-loops and duplicates dropped). It exists so
 * that the reference CPU baseline builds its input without loading the product
 * library; tests assert the two CSRs are byte-identical. Draw (seed, stream,
 * index) -> 64 bits: splitmix64 of splitmix64(seed ^ stream*K) ^ index. */
static uint64_t om_splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
static uint64_t om_hash3(uint64_t seed, uint64_t stream, uint64_t idx) {
  return om_splitmix(om_splitmix(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ idx);
}
/* ascending sort of ids: quicksort (median of three) down to runs of 16, then
 * insertion sort */
static void om_sort_ids(int32_t *p, int64_t d) {
  while (d > 16) {
    int32_t x = p[0], y = p[d / 2], z = p[d - 1], piv;
    piv = x < y ? (y < z ? y : (x < z ? z : x)) : (x < z ? x : (y < z ? z : y));
    int64_t i = 0, j = d - 1;
    for (;;) {
      while (p[i] < piv) ++i;
      while (p[j] > piv) --j;
      if (i >= j) break;
      const int32_t t = p[i];
      p[i++] = p[j];
      p[j--] = t;
    }
    /* recurse into the smaller side, loop on the larger */
    if (j + 1 < d - j - 1) {
      om_sort_ids(p, j + 1);
      p += j + 1;
      d -= j + 1;
    } else {
      om_sort_ids(p + j + 1, d - j - 1);
      d = j + 1;
    }
  }
  for (int64_t i = 1; i < d; ++i) {
    const int32_t x = p[i];
    int64_t k = i;
    while (k > 0 && p[k - 1] > x) {
      p[k] = p[k - 1];
      --k;
    }
    p[k] = x;
  }
}

/* On success *ro_out (n+1 entries) and *col_out (*edges_out entries) are
 * malloc'd; release them with oracle_free. */
int oracle_build_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c, uint64_t seed,
                      int32_t symmetrize, int32_t clean, int32_t **ro_out, int32_t **col_out, int64_t *edges_out) {
  if (scale < 1 || scale > 30 || edgefactor < 1) return -1;
  const int64_t n = (int64_t)1 << scale, m = (int64_t)edgefactor * n;
  const double s32 = 4294967296.0;
  const uint64_t tA = (uint64_t)(a * s32), tAB = (uint64_t)((a + b) * s32), tABC = (uint64_t)((a + b + c) * s32);
  int32_t *perm = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *src = (int32_t *)malloc(sizeof(int32_t) * (size_t)m), *dst = (int32_t *)malloc(sizeof(int32_t) * (size_t)m);
  int64_t *off = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  if (!perm || !src || !dst || !off) return -1;
  for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)i;
  for (int64_t i = n - 1; i > 0; --i) { /* Fisher-Yates over the counter hash */
    const uint64_t r = om_hash3(seed, 0x7065726dull, (uint64_t)i) % (uint64_t)(i + 1);
    const int32_t t = perm[i];
    perm[i] = perm[r];
    perm[r] = t;
  }
  for (int64_t k = 0; k < m; ++k) {
    uint32_t u = 0, v = 0;
    uint64_t h = 0;
    for (int lvl = 0; lvl < scale; ++lvl) {
      if ((lvl & 1) == 0) h = om_hash3(seed, 0x726d6174ull + (uint64_t)(lvl >> 1), (uint64_t)k);
      const uint64_t r = (lvl & 1) ? (h >> 32) : (h & 0xffffffffull);
      const uint32_t bu = r >= tAB, bv = (r >= tA && r < tAB) || r >= tABC;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    src[k] = perm[u];
    dst[k] = perm[v];
  }
  free(perm);
  for (int64_t k = 0; k < m; ++k) {
    if (clean && src[k] == dst[k]) continue;
    ++off[src[k] + 1];
    if (symmetrize) ++off[dst[k] + 1];
  }
  for (int64_t v = 0; v < n; ++v) off[v + 1] += off[v];
  int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(off[n] > 0 ? off[n] : 1));
  int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  if (!tmp || !cur) return -1;
  memcpy(cur, off, sizeof(int64_t) * (size_t)n);
  for (int64_t k = 0; k < m; ++k) {
    if (clean && src[k] == dst[k]) continue;
    tmp[cur[src[k]]++] = dst[k];
    if (symmetrize) tmp[cur[dst[k]]++] = src[k];
  }
  free(src);
  free(dst);
  /* sort every row, drop duplicates; cur[v] becomes the kept length */
  for (int64_t v = 0; v < n; ++v) {
    int32_t *p = tmp + off[v];
    const int64_t d = off[v + 1] - off[v];
    om_sort_ids(p, d);
    int64_t k = d;
    if (clean && d > 1) {
      k = 1;
      for (int64_t i = 1; i < d; ++i)
        if (p[i] != p[k - 1]) p[k++] = p[i];
    }
    cur[v] = k;
  }
  int32_t *ro = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int64_t total = 0;
  for (int64_t v = 0; v < n; ++v) total += cur[v];
  int32_t *col = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  if (!ro || !col) return -1;
  ro[0] = 0;
  for (int64_t v = 0; v < n; ++v) ro[v + 1] = ro[v] + (int32_t)cur[v];
  for (int64_t v = 0; v < n; ++v) memcpy(col + ro[v], tmp + off[v], sizeof(int32_t) * (size_t)cur[v]);
  free(tmp);
  free(cur);
  free(off);
  *ro_out = ro;
  *col_out = col;
  *edges_out = total;
  return 0;
}

void oracle_free(void *p) { free(p); }
