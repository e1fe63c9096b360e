#include "host_util.h"

#include <cstring>

#include "../../include/mapgraph_b200.h"

namespace mg {

namespace {
thread_local std::string g_last_error;
thread_local int64_t g_launches = 0;
}  // namespace

int set_error(int status, const std::string &msg) {
  if (status != MG_OK) g_last_error = msg;
  return status;
}
void clear_error() { g_last_error.clear(); }
void count_launch(int64_t n) { g_launches += n; }

void host_transpose(int64_t nodes, int64_t edges, const int32_t *row_offsets, const int32_t *col, int32_t *t_offsets,
                    int32_t *t_rows, int32_t *t_eid) {
  std::vector<uint32_t> indeg((size_t)nodes, 0);
  host_parallel_for(edges, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t j = b; j < e; ++j) __atomic_fetch_add(&indeg[col[j]], 1u, __ATOMIC_RELAXED);
  });
  t_offsets[0] = 0;
  for (int64_t v = 0; v < nodes; ++v) t_offsets[v + 1] = t_offsets[v] + (int32_t)indeg[v];
  // Each thread owns a contiguous range of columns and sweeps the CSR in row
  // order, so entries land in row order within every column.
  // Every owner sweeps the whole CSR, so a few owners are enough.
  const unsigned T = (edges < 65536) ? 1u : std::min(8u, host_threads());
  std::vector<std::thread> th;
  auto work = [&](int64_t c0, int64_t c1) {
    std::vector<int32_t> cur(t_offsets + c0, t_offsets + c1);
    for (int64_t u = 0; u < nodes; ++u)
      for (int32_t j = row_offsets[u]; j < row_offsets[u + 1]; ++j) {
        const int32_t c = col[j];
        if (c < c0 || c >= c1) continue;
        const int32_t p = cur[c - c0]++;
        t_rows[p] = (int32_t)u;
        if (t_eid) t_eid[p] = j;
      }
  };
  if (T == 1) {
    work(0, nodes);
    return;
  }
  // Balance the column ranges by entry count.
  int64_t per = (edges + T - 1) / T;
  int64_t c0 = 0;
  for (unsigned t = 0; t < T && c0 < nodes; ++t) {
    int64_t target = std::min<int64_t>(edges, (int64_t)(t + 1) * per);
    int64_t c1 = (int64_t)(std::lower_bound(t_offsets, t_offsets + nodes + 1, (int32_t)target) - t_offsets);
    if (t == T - 1 || c1 > nodes) c1 = nodes;
    if (c1 <= c0) c1 = std::min<int64_t>(nodes, c0 + 1);
    th.emplace_back(work, c0, c1);
    c0 = c1;
  }
  if (c0 < nodes) th.emplace_back(work, c0, nodes);
  for (auto &x : th) x.join();
}

std::string validate_csr(int64_t nodes, int64_t edges, const int32_t *row_offsets, const int32_t *col) {
  if (nodes <= 0 || nodes >= INT32_MAX) return "nodes must be in [1, 2^31-1)";
  if (edges < 0 || edges >= INT32_MAX) return "edges must be in [0, 2^31-1)";
  if (!row_offsets) return "row_offsets is NULL";
  if (edges > 0 && !col) return "column_indices is NULL";
  if (row_offsets[0] != 0) return "row_offsets[0] must be 0";
  if ((int64_t)row_offsets[nodes] != edges) return "row_offsets[nodes] must equal edges";
  std::atomic<int64_t> bad_row(-1), bad_col(-1);
  host_parallel_for(nodes, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t v = b; v < e; ++v)
      if (row_offsets[v + 1] < row_offsets[v]) bad_row.store(v);
  });
  if (bad_row.load() >= 0) return "row_offsets not monotone at row " + std::to_string(bad_row.load());
  host_parallel_for(edges, [&](int64_t b, int64_t e, unsigned) {
    for (int64_t j = b; j < e; ++j)
      if (col[j] < 0 || (int64_t)col[j] >= nodes) bad_col.store(j);
  });
  if (bad_col.load() >= 0) return "column index out of range at edge " + std::to_string(bad_col.load());
  return std::string();
}

}  // namespace mg

extern "C" {

const char *mg_last_error(void) { return mg::g_last_error.c_str(); }

const char *mg_status_string(int status) {
  switch (status) {
    case MG_OK: return "MG_OK";
    case MG_ERR_ARG: return "MG_ERR_ARG";
    case MG_ERR_OOM: return "MG_ERR_OOM";
    case MG_ERR_OVERFLOW: return "MG_ERR_OVERFLOW";
    case MG_ERR_TIMEOUT: return "MG_ERR_TIMEOUT";
    case MG_ERR_CUDA: return "MG_ERR_CUDA";
    case MG_ERR_UNSUPPORTED: return "MG_ERR_UNSUPPORTED";
    case MG_ERR_IO: return "MG_ERR_IO";
    default: return "MG_ERR_UNKNOWN";
  }
}

int mg_abi_version(void) { return MG_ABI_VERSION; }

int64_t mg_kernel_launches(int reset) {
  int64_t v = mg::g_launches;
  if (reset) mg::g_launches = 0;
  return v;
}

void mg_options_init(mg_options *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(mg_options);
  o->outputs_on_device = 0;
  o->stream = nullptr;
  o->iter_num = 1 << 30;
  o->direction = MG_DIR_AUTO;
  o->alpha = 15.0;
  o->beta = 18.0;
  o->use_cuda_graph = 1;
  o->threshold = 0;
  o->damping = 0.85;
  o->tolerance = 1e-6;
  o->spin_limit = (int64_t)1 << 22;
  o->tile_items = 0;
  o->ctas_per_sm = 0;
  o->compute_stats = 1;
  o->alpha_multi = 5.0;
}

}  // extern "C"
