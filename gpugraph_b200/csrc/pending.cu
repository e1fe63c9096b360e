// Entry points whose kernels live in translation units that are not built yet.
#include "graph.cuh"
#include "host_util.h"

extern "C" {

int mg_ppr_forward(mg_graph *, const float *, const float *, int32_t, float *, mg_stats *, const mg_options *) {
  return mg::set_error(MG_ERR_UNSUPPORTED, "mg_ppr_forward not built");
}
int mg_ppr_backward(mg_graph *, const float *, const float *, const float *, int32_t, float *, float *, mg_stats *,
                    const mg_options *) {
  return mg::set_error(MG_ERR_UNSUPPORTED, "mg_ppr_backward not built");
}
}
