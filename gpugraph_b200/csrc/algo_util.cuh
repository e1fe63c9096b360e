// Small helpers shared by the algorithm entry points: result extraction
// (CsrProblem::ExtractResults, csr_problem.cuh:433-458), reach statistics and
// argument checks.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "gas/driver.cuh"
#include "graph.cuh"
#include "host_util.h"

namespace mg {

// Copies a device result to the caller's buffer (host or device) on stream s
// and waits for it.
int copy_out(cudaStream_t s, void *dst, const void *src, size_t bytes, bool dst_on_device);

// vertices_reached / edges_traversed: vertices whose value differs from
// `unreached`, and the sum of their out-degrees (MapGraph "visited edges").
// vals is [V] or, with stride_src > 1, [V][stride_src] interleaved values of
// nsrc sources (counts summed over sources).
int reach_stats(mg_graph *g, cudaStream_t s, const int32_t *vals, int32_t unreached, int nsrc, int stride_src,
                int64_t *reached, int64_t *edges);

// Validates and de-duplicates a host array of source vertices.
int check_sources(mg_graph *g, const int32_t *srcs, int32_t nsrc, std::vector<int32_t> *out);

inline bool want_stats(const mg_options *o) { return !o || o->compute_stats; }

}  // namespace mg
