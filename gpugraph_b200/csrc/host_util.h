// Host-side helpers shared by every translation unit of the library: the
// thread-local last-error message, the kernel-launch counter and small
// parallel loops for host preprocessing.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

namespace mg {

// Records msg as this thread's last error and returns status unchanged, so a
// failing path can be written `return set_error(MG_ERR_ARG, "...")`.
int set_error(int status, const std::string &msg);
void clear_error();
// Counts launches of this library's own kernels (reported by the bench as gpu_launches).
void count_launch(int64_t n = 1);

inline unsigned host_threads() {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 1;
  if (t > 64) t = 64;
  return t;
}

// Static partition of [0, n) over the host threads; f(begin, end, thread_index).
template <typename F>
void host_parallel_for(int64_t n, F f) {
  unsigned T = host_threads();
  if (n < 65536 || T == 1) {
    f((int64_t)0, n, 0u);
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

// Transpose of a CSR (column offsets, row indices, CSR edge id of each entry),
// stable by row: the result is the same for any thread count.
void host_transpose(int64_t nodes, int64_t edges, const int32_t *row_offsets, const int32_t *col,
                    int32_t *t_offsets, int32_t *t_rows, int32_t *t_eid);

// Checks that a CSR is well formed (offsets monotone from 0 to edges, every
// column id in [0, nodes)). Returns an empty string when valid.
std::string validate_csr(int64_t nodes, int64_t edges, const int32_t *row_offsets, const int32_t *col);

}  // namespace mg
