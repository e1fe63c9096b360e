// Host graph builders: seeded R-MAT, road-like grid, symmetric weights, Matrix
// Market reader and host transpose. These replace the reference's host builders
// (b40c/graph/builder/{rmat,grid2d,market}.cuh and CsrGraph::FromCoo,
// b40c/graph/csr_graph.cuh:120-210). They run once per input, off the timed path;
// they are multithreaded so that scale-22/23 graphs build in seconds.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <climits>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/mapgraph_b200.h"
#include "host_util.h"

namespace {

using mg::set_error;

inline uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Counter-based hash of (seed, stream, index): every draw is a pure function of
// its coordinates, so the output does not depend on the thread count.
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t idx) {
  return splitmix(splitmix(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ idx);
}

unsigned num_threads() {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 1;
  if (t > 64) t = 64;
  return t;
}

template <typename F>
void parallel_for(int64_t n, F f) {
  unsigned T = num_threads();
  if (n < 4096 || T == 1) {
    f(0, n, 0u);
    return;
  }
  std::vector<std::thread> th;
  int64_t chunk = (n + T - 1) / T;
  for (unsigned t = 0; t < T; ++t) {
    int64_t b = (int64_t)t * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([=, &f] { f(b, e, t); });
  }
  for (auto &x : th) x.join();
}

// Dynamic-chunk parallel loop for skewed work (row sorts of R-MAT hubs).
template <typename F>
void parallel_for_dynamic(int64_t n, int64_t chunk, F f) {
  unsigned T = num_threads();
  std::atomic<int64_t> next(0);
  auto worker = [&] {
    for (;;) {
      int64_t b = next.fetch_add(chunk);
      if (b >= n) break;
      f(b, std::min<int64_t>(n, b + chunk));
    }
  };
  if (T == 1 || n < chunk) {
    worker();
    return;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < T; ++t) th.emplace_back(worker);
  for (auto &x : th) x.join();
}

bool alloc_csr(mg_host_csr *out, int64_t nodes, int64_t edges, bool values) {
  out->nodes = nodes;
  out->edges = edges;
  out->row_offsets = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nodes + 1));
  out->column_indices = (int32_t *)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1));
  out->edge_values = values ? (int32_t *)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1)) : nullptr;
  if (!out->row_offsets || !out->column_indices || (values && !out->edge_values)) {
    mg_host_csr_free(out);
    return false;
  }
  return true;
}

// Build a CSR from an edge list (src[i] -> dst[i]). symmetrize stores each edge
// both ways; clean drops self-loops and duplicates. Rows come out sorted by
// column id. Result is independent of thread scheduling.
int csr_from_edges(int64_t nodes, const std::vector<int32_t> &src, const std::vector<int32_t> &dst,
                   bool symmetrize, bool clean, mg_host_csr *out) {
  const int64_t m = (int64_t)src.size();
  std::vector<uint32_t> deg((size_t)nodes + 1, 0);
  parallel_for(m, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t i = b; i < e; ++i) {
      int32_t u = src[i], v = dst[i];
      if (clean && u == v) continue;
      __atomic_fetch_add(&deg[u], 1u, __ATOMIC_RELAXED);
      if (symmetrize) __atomic_fetch_add(&deg[v], 1u, __ATOMIC_RELAXED);
    }
  });
  std::vector<int64_t> off((size_t)nodes + 1, 0);
  for (int64_t v = 0; v < nodes; ++v) off[v + 1] = off[v] + deg[v];
  const int64_t total = off[nodes];
  std::vector<int32_t> tmp((size_t)std::max<int64_t>(total, 1));
  std::vector<int64_t> cur(off.begin(), off.end() - 1);
  parallel_for(m, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t i = b; i < e; ++i) {
      int32_t u = src[i], v = dst[i];
      if (clean && u == v) continue;
      int64_t p = __atomic_fetch_add(&cur[u], (int64_t)1, __ATOMIC_RELAXED);
      tmp[p] = v;
      if (symmetrize) {
        int64_t q = __atomic_fetch_add(&cur[v], (int64_t)1, __ATOMIC_RELAXED);
        tmp[q] = u;
      }
    }
  });
  // Sort every row; drop duplicates if asked.
  std::vector<uint32_t> newdeg((size_t)nodes, 0);
  parallel_for_dynamic(nodes, 2048, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      int32_t *p = tmp.data() + off[v];
      int64_t d = off[v + 1] - off[v];
      std::sort(p, p + d);
      if (clean) d = std::unique(p, p + d) - p;
      newdeg[v] = (uint32_t)d;
    }
  });
  int64_t E = 0;
  for (int64_t v = 0; v < nodes; ++v) E += newdeg[v];
  if (nodes >= INT32_MAX || E >= INT32_MAX) return set_error(MG_ERR_ARG, "graph too large for int32 CSR");
  if (!alloc_csr(out, nodes, E, false)) return set_error(MG_ERR_OOM, "host allocation failed");
  out->row_offsets[0] = 0;
  for (int64_t v = 0; v < nodes; ++v) out->row_offsets[v + 1] = out->row_offsets[v] + (int32_t)newdeg[v];
  parallel_for(nodes, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t v = b; v < e; ++v)
      memcpy(out->column_indices + out->row_offsets[v], tmp.data() + off[v], sizeof(int32_t) * newdeg[v]);
  });
  out->directed = symmetrize ? 0 : 1;
  return MG_OK;
}

}  // namespace

extern "C" {

void mg_host_csr_free(mg_host_csr *csr) {
  if (!csr) return;
  free(csr->row_offsets);
  free(csr->column_indices);
  free(csr->edge_values);
  csr->row_offsets = nullptr;
  csr->column_indices = nullptr;
  csr->edge_values = nullptr;
  csr->nodes = csr->edges = 0;
}

// Recursive quadrant choice as in BuildRmatGraph (rmat.cuh:145-224, ChoosePartition
// rmat.cuh:71-97) but seeded and without the per-level +-5% parameter jitter,
// followed by a seeded vertex relabelling (Graph500 practice: hubs do not cluster
// at low ids).
int mg_build_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c, uint64_t seed,
                  int32_t symmetrize, int32_t clean, mg_host_csr *out) {
  if (!out) return set_error(MG_ERR_ARG, "out is NULL");
  memset(out, 0, sizeof(*out));
  if (scale < 1 || scale > 30 || edgefactor < 1) return set_error(MG_ERR_ARG, "bad scale/edgefactor");
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return set_error(MG_ERR_ARG, "bad R-MAT probabilities");
  const int64_t nodes = (int64_t)1 << scale;
  const int64_t m = (int64_t)edgefactor * nodes;
  if (m * (symmetrize ? 2 : 1) >= INT32_MAX) return set_error(MG_ERR_ARG, "too many edges for int32 CSR");
  const double s32 = 4294967296.0;
  const uint64_t tA = (uint64_t)(a * s32), tAB = (uint64_t)((a + b) * s32), tABC = (uint64_t)((a + b + c) * s32);
  // Seeded permutation of vertex ids (Fisher-Yates over a counter hash).
  std::vector<int32_t> perm((size_t)nodes);
  for (int64_t i = 0; i < nodes; ++i) perm[i] = (int32_t)i;
  for (int64_t i = nodes - 1; i > 0; --i) {
    uint64_t r = hash3(seed, 0x7065726dull, (uint64_t)i) % (uint64_t)(i + 1);
    std::swap(perm[i], perm[r]);
  }
  std::vector<int32_t> src((size_t)m), dst((size_t)m);
  parallel_for(m, [&](int64_t bgn, int64_t end, unsigned) {
    for (int64_t k = bgn; k < end; ++k) {
      uint32_t u = 0, v = 0;
      uint64_t h = 0;
      for (int lvl = 0; lvl < scale; ++lvl) {
        if ((lvl & 1) == 0) h = hash3(seed, 0x726d6174ull + (uint64_t)(lvl >> 1), (uint64_t)k);
        uint64_t r = (lvl & 1) ? (h >> 32) : (h & 0xffffffffull);
        uint32_t bu = 0, bv = 0;
        if (r < tA) {
        } else if (r < tAB) {
          bv = 1;
        } else if (r < tABC) {
          bu = 1;
        } else {
          bu = 1;
          bv = 1;
        }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      src[k] = perm[u];
      dst[k] = perm[v];
    }
  });
  return csr_from_edges(nodes, src, dst, symmetrize != 0, clean != 0, out);
}

int mg_build_road_grid(int32_t width, double drop_frac, double shortcut_frac, uint64_t seed, mg_host_csr *out) {
  if (!out) return set_error(MG_ERR_ARG, "out is NULL");
  memset(out, 0, sizeof(*out));
  if (width < 2 || width > 40000 || drop_frac < 0 || drop_frac >= 1 || shortcut_frac < 0)
    return set_error(MG_ERR_ARG, "bad grid parameters");
  const int64_t W = width, nodes = W * W;
  const uint64_t tdrop = (uint64_t)(drop_frac * 4294967296.0);
  std::vector<int32_t> src, dst;
  src.reserve((size_t)(2 * nodes));
  dst.reserve((size_t)(2 * nodes));
  // Lattice edges, indexed: horizontal (r,c)-(r,c+1) as r*(W-1)+c; vertical after them.
  for (int64_t r = 0; r < W; ++r)
    for (int64_t c = 0; c + 1 < W; ++c) {
      uint64_t idx = (uint64_t)(r * (W - 1) + c);
      if ((hash3(seed, 0x64726f70ull, idx) & 0xffffffffull) < tdrop) continue;
      src.push_back((int32_t)(r * W + c));
      dst.push_back((int32_t)(r * W + c + 1));
    }
  for (int64_t r = 0; r + 1 < W; ++r)
    for (int64_t c = 0; c < W; ++c) {
      uint64_t idx = (uint64_t)(W * (W - 1) + r * W + c);
      if ((hash3(seed, 0x64726f70ull, idx) & 0xffffffffull) < tdrop) continue;
      src.push_back((int32_t)(r * W + c));
      dst.push_back((int32_t)((r + 1) * W + c));
    }
  const int64_t kept = (int64_t)src.size();
  const int64_t nshort = (int64_t)std::llround(shortcut_frac * (double)kept);
  std::unordered_set<uint64_t> seen;
  seen.reserve((size_t)nshort * 2 + 16);
  auto key = [](int64_t u, int64_t v) {
    if (u > v) std::swap(u, v);
    return ((uint64_t)u << 32) | (uint64_t)v;
  };
  auto lattice_edge = [&](int64_t u, int64_t v) {
    if (u > v) std::swap(u, v);
    int64_t d = v - u;
    return (d == 1 && (v % W) != 0) || d == W;  // may or may not have been dropped
  };
  int64_t added = 0;
  for (uint64_t i = 0; added < nshort; ++i) {
    uint64_t h = hash3(seed, 0x73686f72ull, i);
    int64_t u = (int64_t)((h & 0xffffffffull) % (uint64_t)nodes);
    int64_t v = (int64_t)((h >> 32) % (uint64_t)nodes);
    if (u == v || lattice_edge(u, v)) continue;
    if (!seen.insert(key(u, v)).second) continue;
    src.push_back((int32_t)u);
    dst.push_back((int32_t)v);
    ++added;
  }
  return csr_from_edges(nodes, src, dst, true, true, out);
}

int mg_build_weights(mg_host_csr *csr, uint32_t lo, uint32_t hi, uint64_t seed) {
  if (!csr || !csr->row_offsets || !csr->column_indices) return set_error(MG_ERR_ARG, "csr is NULL");
  if (hi < lo || hi > (uint32_t)INT32_MAX) return set_error(MG_ERR_ARG, "bad weight range");
  if (!csr->edge_values) {
    csr->edge_values = (int32_t *)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(csr->edges, 1));
    if (!csr->edge_values) return set_error(MG_ERR_OOM, "host allocation failed");
  }
  const uint64_t span = (uint64_t)(hi - lo) + 1;
  parallel_for(csr->nodes, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t u = b; u < e; ++u)
      for (int32_t j = csr->row_offsets[u]; j < csr->row_offsets[u + 1]; ++j) {
        int64_t v = csr->column_indices[j];
        uint64_t x = (uint64_t)std::min<int64_t>(u, v), y = (uint64_t)std::max<int64_t>(u, v);
        uint64_t h = hash3(seed, 0x77656967ull, (x << 32) | y);
        csr->edge_values[j] = (int32_t)(lo + (uint32_t)(h % span));
      }
  });
  return MG_OK;
}

int mg_read_market(const char *path, int32_t undirected, mg_host_csr *out) {
  if (!path || !out) return set_error(MG_ERR_ARG, "path/out is NULL");
  memset(out, 0, sizeof(*out));
  FILE *f = fopen(path, "r");
  if (!f) return set_error(MG_ERR_IO, std::string("cannot open ") + path);
  struct Tup {
    int32_t row, col, val;
  };
  std::vector<Tup> coo;
  int64_t nodes = -1, declared = 0;
  bool pattern = false;
  char line[4096];
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '%') {
      if (strncmp(line, "%%MatrixMarket", 14) == 0 && strstr(line, "pattern")) pattern = true;
      continue;
    }
    if (line[0] == '\n' || line[0] == '\0') continue;
    if (nodes < 0) {
      long long nx, ny, ne;
      if (sscanf(line, "%lld %lld %lld", &nx, &ny, &ne) != 3 || nx != ny || nx < 0 || ne < 0) {
        fclose(f);
        return set_error(MG_ERR_IO, "bad Matrix Market size line");
      }
      nodes = nx;
      declared = ne;
      coo.reserve((size_t)(undirected ? 2 * ne : ne));
      continue;
    }
    long long r, c;
    double val = 1.0;
    int got = sscanf(line, "%lld %lld %lf", &r, &c, &val);
    if (got < 2 || (got == 2 && !pattern) || r < 1 || c < 1 || r > nodes || c > nodes) {
      fclose(f);
      return set_error(MG_ERR_IO, "badly formed edge line");
    }
    coo.push_back({(int32_t)(r - 1), (int32_t)(c - 1), (int32_t)val});
    if (undirected) coo.push_back({(int32_t)(c - 1), (int32_t)(r - 1), (int32_t)val});
  }
  fclose(f);
  if (nodes < 0) return set_error(MG_ERR_IO, "no graph found");
  if ((int64_t)coo.size() != (undirected ? 2 * declared : declared))
    return set_error(MG_ERR_IO, "edge count does not match the size line");
  std::stable_sort(coo.begin(), coo.end(), [](const Tup &x, const Tup &y) {
    return x.row < y.row || (x.row == y.row && x.col < y.col);
  });
  if (!alloc_csr(out, nodes, (int64_t)coo.size(), true)) return set_error(MG_ERR_OOM, "host allocation failed");
  std::fill(out->row_offsets, out->row_offsets + nodes + 1, 0);
  for (auto &t : coo) out->row_offsets[t.row + 1]++;
  for (int64_t v = 0; v < nodes; ++v) out->row_offsets[v + 1] += out->row_offsets[v];
  for (size_t i = 0; i < coo.size(); ++i) {
    out->column_indices[i] = coo[i].col;
    out->edge_values[i] = coo[i].val;
  }
  out->directed = undirected ? 0 : 1;
  return MG_OK;
}

// CSV graphs as csv_graph_reader reads them (GASengine/csv_graph_reader.cuh):
// format 0 (read(), :79-137) has one row per source, "src,dst:val,dst:val,...";
// format 1 (read2(), :147-205) one row per edge, "src,dst,val". Every id that
// appears (a lone "src" row included) becomes a vertex, numbered by sorted id
// (:98-111); `undirected` appends the reversed edges (:127-135); the CSR is
// ordered by (row, col) keeping duplicates (b40c CsrGraph::FromCoo with
// DimacsTupleCompare). A format-0 cell without ':' gives its own number as the
// value (the reference's substr(npos + 1) is the whole cell). Empty lines are
// skipped.
int mg_read_csv(const char *path, int32_t format, int32_t undirected, mg_host_csr *out) {
  if (!path || !out) return set_error(MG_ERR_ARG, "path/out is NULL");
  if (format != 0 && format != 1) return set_error(MG_ERR_ARG, "format must be 0 (adjacency rows) or 1 (edge rows)");
  memset(out, 0, sizeof(*out));
  FILE *f = fopen(path, "r");
  if (!f) return set_error(MG_ERR_IO, std::string("cannot open ") + path);
  struct Tup {
    int32_t row, col, val;
  };
  std::vector<Tup> coo;
  std::vector<int32_t> ids;
  std::string line;
  std::vector<std::string> cells;
  char buf[1 << 16];
  bool bad = false;
  while (!bad && fgets(buf, sizeof(buf), f)) {
    line.assign(buf);
    // a line longer than the buffer continues in the next reads
    while (!line.empty() && line.back() != '\n' && fgets(buf, sizeof(buf), f)) line.append(buf);
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
    if (line.empty()) continue;
    cells.clear();
    size_t b = 0;
    for (;;) {
      const size_t e = line.find(',', b);
      cells.push_back(line.substr(b, e == std::string::npos ? std::string::npos : e - b));
      if (e == std::string::npos) break;
      b = e + 1;
    }
    const int32_t src = (int32_t)atoi(cells[0].c_str());
    ids.push_back(src);
    if (format == 1) {
      if (cells.size() < 3) {
        bad = true;
        break;
      }
      const int32_t dst = (int32_t)atoi(cells[1].c_str());
      ids.push_back(dst);
      coo.push_back({src, dst, (int32_t)atoi(cells[2].c_str())});
      continue;
    }
    for (size_t i = 1; i < cells.size(); ++i) {
      const size_t pos = cells[i].find(':');
      const int32_t dst = (int32_t)atoi(cells[i].substr(0, pos).c_str());
      const int32_t val = (int32_t)atoi(pos == std::string::npos ? cells[i].c_str() : cells[i].c_str() + pos + 1);
      ids.push_back(dst);
      coo.push_back({src, dst, val});
    }
  }
  fclose(f);
  if (bad) return set_error(MG_ERR_IO, "an edge row needs src,dst,val");
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  const int64_t nodes = (int64_t)ids.size();
  auto dense = [&](int32_t id) { return (int32_t)(std::lower_bound(ids.begin(), ids.end(), id) - ids.begin()); };
  for (auto &t : coo) {
    t.row = dense(t.row);
    t.col = dense(t.col);
  }
  if (undirected) {
    const size_t m = coo.size();
    for (size_t i = 0; i < m; ++i) coo.push_back({coo[i].col, coo[i].row, coo[i].val});
  }
  if ((int64_t)coo.size() > INT32_MAX) return set_error(MG_ERR_OVERFLOW, "more than 2^31-1 edges");
  std::stable_sort(coo.begin(), coo.end(), [](const Tup &x, const Tup &y) {
    return x.row < y.row || (x.row == y.row && x.col < y.col);
  });
  if (!alloc_csr(out, nodes, (int64_t)coo.size(), true)) return set_error(MG_ERR_OOM, "host allocation failed");
  std::fill(out->row_offsets, out->row_offsets + nodes + 1, 0);
  for (auto &t : coo) out->row_offsets[t.row + 1]++;
  for (int64_t v = 0; v < nodes; ++v) out->row_offsets[v + 1] += out->row_offsets[v];
  for (size_t i = 0; i < coo.size(); ++i) {
    out->column_indices[i] = coo[i].col;
    out->edge_values[i] = coo[i].val;
  }
  out->directed = undirected ? 0 : 1;
  return MG_OK;
}

int mg_host_csr_transpose(const mg_host_csr *in, mg_host_csr *out) {
  if (!in || !out || !in->row_offsets) return set_error(MG_ERR_ARG, "NULL argument");
  memset(out, 0, sizeof(*out));
  const int64_t n = in->nodes, m = in->edges;
  if (!alloc_csr(out, n, m, in->edge_values != nullptr)) return set_error(MG_ERR_OOM, "host allocation failed");
  std::vector<int32_t> eid(in->edge_values ? (size_t)std::max<int64_t>(m, 1) : 0);
  mg::host_transpose(n, m, in->row_offsets, in->column_indices, out->row_offsets, out->column_indices,
                     in->edge_values ? eid.data() : nullptr);
  if (in->edge_values)
    for (int64_t p = 0; p < m; ++p) out->edge_values[p] = in->edge_values[eid[p]];
  out->directed = in->directed;
  return MG_OK;
}

}  // extern "C"
