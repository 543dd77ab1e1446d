#!/usr/bin/env bash
# Builds the reference-side checkers into oracle/_ref/ (git-ignored), from the
# reference's own sources where they lie:
#   ref_cpulp  -- the OpenMP CPU path (tutorial/CPUlp.cuh + header/graph.h +
#                 header/myutil.h), with g++ and the include shims of
#                 oracle/ref_shim/;
#   ref_gpu_lp -- the GPU propagation kernels (header/kernel.cuh, copied
#                 here truncated before its non-compiling user-defined stub
#                 area at line 6071, + method/hashtable.cuh) and the SLPA
#                 speaker memory of tutorial/Base5prop.cuh, driven by
#                 oracle/ref_gpu_harness.cu, with nvcc for sm_100a and the
#                 include shims of oracle/ref_shim_gpu/.
# Needs the reference tree: $GLP_REFERENCE, else a `reference` directory
# beside the repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${GLP_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/tutorial/CPUlp.cuh" ]; then
  echo "reference tree not found at $REF; keeping any prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
g++ -O3 -std=c++17 -fopenmp -w -x c++ \
  -include "$HERE/ref_shim/host_cuda_compat.h" \
  -I "$HERE/ref_shim/inc" -I "$HERE/ref_shim" -I "$REF" \
  "$HERE/ref_cpulp_harness.cpp" -o "$OUT/ref_cpulp"
echo "built $OUT/ref_cpulp"
NVCC="${NVCC:-$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)}"
if [ -x "$NVCC" ] && [ -f "$REF/header/kernel.cuh" ]; then
  mkdir -p "$OUT/kshim/header"
  head -n 6070 "$REF/header/kernel.cuh" > "$OUT/kshim/header/kernel.cuh"
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -w \
    -I "$HERE/ref_shim_gpu" -I "$HERE/ref_shim_gpu/inc" -I "$OUT/kshim" -I "$REF" \
    "$HERE/ref_gpu_harness.cu" -o "$OUT/ref_gpu_lp"
  echo "built $OUT/ref_gpu_lp"
fi
