#!/bin/sh
# Builds oracle/_ref/libref_cpu.so: the reference's own CPU implementations
# (CPUBFS, CPUSSSP, CPUCC, CPUPR) compiled with g++ from their sources where
# they lie in the reference tree, plus oracle/ref_harness.inc (C wrappers).
# Test infrastructure only. The generated translation unit and the library stay
# in oracle/_ref/ (git-ignored); nothing from the reference is committed.
#
# The four functions sit in the CUDA drivers, which also pull in MPI and the
# GPU engine, so the recipe takes their exact line ranges:
#   Algorithms/BFS/bfs.cu:57-111            CPUBFS
#   Algorithms/SSSP/sssp.cu:126-183         CPUSSSP
#   Algorithms/CC/cc.cu:127-169             CPUCC
#   Algorithms/PageRank/PageRank.cu:108-161 CPUPR
# and compiles them against b40c/graph/csr_graph.cuh.
set -e
REF=${MG_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
CUDA_INC=${CUDA_HOME:-/usr/local/cuda}/include
if [ ! -f "$REF/Algorithms/BFS/bfs.cu" ]; then
  echo "reference tree not found at $REF; oracle/_ref not rebuilt" >&2
  exit 0
fi
mkdir -p "$OUT"
TU="$OUT/ref_cpu.cpp"
{
  printf '%s\n' '#include <cuda_runtime_api.h>' '#include <omp.h>' '#include <cmath>' '#include <deque>' \
    '#include <iostream>' '#include <numeric>' '#include <vector>' '#include <b40c/graph/csr_graph.cuh>' \
    'using namespace b40c;' 'using namespace b40c::graph;' 'using namespace std;'
  sed -n '57,111p' "$REF/Algorithms/BFS/bfs.cu"
  sed -n '126,183p' "$REF/Algorithms/SSSP/sssp.cu"
  sed -n '127,169p' "$REF/Algorithms/CC/cc.cu"
  sed -n '108,161p' "$REF/Algorithms/PageRank/PageRank.cu"
  cat "$HERE/ref_harness.inc"
} > "$TU"
# b40c/util/error_utils.cuh calls cudaGetLastError in inline helpers: link the static runtime.
CUDA_LIB=${CUDA_HOME:-/usr/local/cuda}/lib64
g++ -O2 -fopenmp -fPIC -shared -w -I"$REF" -I"$CUDA_INC" "$TU" -o "$OUT/libref_cpu.so" \
  -L"$CUDA_LIB" -lcudart_static -ldl -lrt -lpthread
echo "$OUT/libref_cpu.so"
