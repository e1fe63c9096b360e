#include <algorithm>

#include "algo_util.cuh"

namespace mg {

int copy_out(cudaStream_t s, void *dst, const void *src, size_t bytes, bool dst_on_device) {
  if (!dst) return set_error(MG_ERR_ARG, "output pointer is NULL");
  cudaError_t e =
      cudaMemcpyAsync(dst, src, bytes, dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_status(e, "result copy");
}

__global__ void k_reach_stats(const int32_t *vals, int32_t unreached, int nsrc, int stride, const int32_t *ro, int32_t V,
                              unsigned long long *out) {
  unsigned long long cnt = 0, edg = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long d = (unsigned long long)(ro[v + 1] - ro[v]);
    for (int s = 0; s < nsrc; ++s) {
      if (vals[v * (int64_t)stride + s] != unreached) {
        cnt += 1;
        edg += d;
      }
    }
  }
  cnt = warp_sum(cnt);
  edg = warp_sum(edg);
  if (lane_id() == 0) {
    atomicAdd(&out[0], cnt);
    atomicAdd(&out[1], edg);
  }
}

int reach_stats(mg_graph *g, cudaStream_t s, const int32_t *vals, int32_t unreached, int nsrc, int stride_src,
                int64_t *reached, int64_t *edges) {
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(g->ws.ctl->acc);
  cudaError_t e = cudaMemsetAsync(acc, 0, 16, s);
  if (e != cudaSuccess) return cuda_status(e, "stats memset");
  k_reach_stats<<<g->num_sms * 4, 256, 0, s>>>(vals, unreached, nsrc, stride_src, g->csr.row_offsets, g->csr.V, acc);
  count_launch();
  unsigned long long h[2] = {0, 0};
  e = cudaMemcpyAsync(h, acc, 16, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "stats read");
  *reached = (int64_t)h[0];
  *edges = (int64_t)h[1];
  return MG_OK;
}

int check_sources(mg_graph *g, const int32_t *srcs, int32_t nsrc, std::vector<int32_t> *out) {
  if (!srcs || nsrc < 1) return set_error(MG_ERR_ARG, "no source vertices");
  out->clear();
  for (int i = 0; i < nsrc; ++i) {
    if (srcs[i] < 0 || (int64_t)srcs[i] >= g->nodes)
      return set_error(MG_ERR_ARG, "source vertex " + std::to_string(srcs[i]) + " out of range");
    out->push_back(srcs[i]);
  }
  std::sort(out->begin(), out->end());
  out->erase(std::unique(out->begin(), out->end()), out->end());
  return MG_OK;
}

}  // namespace mg
