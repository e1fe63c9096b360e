// Self-test of the bounded device-side waits: a tile looks back at a
// predecessor whose status word nothing ever publishes, so the wait must end
// at its spin limit with MG_ERR_TIMEOUT while the context stays usable. No
// fault, trap or unbounded loop is involved.
#include <cuda_runtime.h>

#include "common.cuh"
#include "graph.cuh"
#include "host_util.h"

namespace mg {

__global__ void k_selftest_wait(unsigned long long *status, unsigned long long spin_limit, int *out) {
  bool failed = false;
  // tile 1 waits for tile 0, which never publishes (its word stays 0)
  lookback(status, 1u, 1u, 7u, spin_limit, &failed);
  if (threadIdx.x == 0) *out = failed ? MG_ERR_TIMEOUT : MG_OK;
}

}  // namespace mg

extern "C" int mg_selftest_wait_timeout(int64_t spin_limit, double *elapsed_ms) {
  mg::clear_error();
  if (spin_limit < 1 || spin_limit > (int64_t)1 << 24) return mg::set_error(MG_ERR_ARG, "spin_limit out of range");
  unsigned long long *status = nullptr;
  int *out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&status, 64 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(status, 0, 64 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int result = MG_ERR_CUDA;
  if (e == cudaSuccess) {
    cudaEventRecord(e0, 0);
    mg::k_selftest_wait<<<1, 32>>>(status, (unsigned long long)spin_limit, out);
    mg::count_launch();
    cudaEventRecord(e1, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&result, out, sizeof(int), cudaMemcpyDeviceToHost);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (elapsed_ms) *elapsed_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (status) cudaFree(status);
  if (out) cudaFree(out);
  if (e != cudaSuccess) return mg::cuda_status(e, "selftest");
  if (result == MG_ERR_TIMEOUT) mg::set_error(MG_ERR_TIMEOUT, "bounded wait ran out (expected)");
  return result;
}
