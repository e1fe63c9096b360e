// Host-side level-loop driver shared by every traversal: runs a level body
// (a fixed sequence of persistent kernels ending in a level-end kernel) until
// the device control block says stop. The body is captured once into a CUDA
// graph whose WHILE conditional node is driven from the device, so a run costs
// one cudaGraphLaunch and one small D->H read of the control block at the end
// (the reference synchronises and copies the frontier size back every level,
// enactor_vertex_centric.cuh:3801-3845).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>

#include "../graph.cuh"

namespace mg {

// Launches one level. h/use_handle are forwarded to the level-end kernel.
using LevelBody = std::function<void(cudaStream_t, cudaGraphConditionalHandle, int)>;

struct LoopResult {
  Ctl ctl;          // control block after the loop
  double ms = 0.0;  // CUDA-event time of the loop
  bool used_graph = false;
};

// Runs the loop on stream s. kernels_per_level is used for launch accounting.
// Events are recorded on s before the first and after the last level.
// `epilogue`, when given, enqueues work that follows the loop on the same
// stream before the control block is read back (one host synchronisation for
// both); it is not part of the loop's measured time.
int run_level_loop(mg_graph *g, cudaStream_t s, const std::string &key, int kernels_per_level,
                   const LevelBody &body, bool use_graph, LoopResult *res,
                   const std::function<void(cudaStream_t)> *epilogue = nullptr);

// Persistent grid for the level-loop kernels.
inline int persistent_grid(mg_graph *g, const mg_options *o, int default_per_sm) {
  int per = (o && o->ctas_per_sm > 0) ? o->ctas_per_sm : default_per_sm;
  return g->num_sms * per;
}

// Reads the control block back (synchronises s).
int read_ctl(mg_graph *g, cudaStream_t s, Ctl *out);

// Called before a run: clears the look-back status words and the control block
// once the epochs consumed approach the 30-bit epoch field's range.
int prepare_run(mg_graph *g, cudaStream_t s);
// Called after a run with the number of levels it executed.
void finish_run(mg_graph *g, uint32_t levels);

// Per-kernel profiling (mg_profile_enable): while on, level loops run
// host-driven and every kernel launch is bracketed by CUDA events on its
// stream. prof_mark(s, kid) is called right before launching a kernel of kind kid.
bool prof_on();
void prof_mark(cudaStream_t s, int kid);
// Closes the open interval on s, attributes the elapsed times, and adds the
// run's device byte counters.
void prof_flush(cudaStream_t s, const unsigned long long *kbytes);

#define MG_LAUNCH(kid, stream, ...) \
  do {                              \
    ::mg::prof_mark(stream, kid);   \
    __VA_ARGS__;                    \
  } while (0)

}  // namespace mg
