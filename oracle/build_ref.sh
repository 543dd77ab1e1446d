#!/usr/bin/env bash
# Builds oracle/_ref/ref_cpulp from the reference's own sources, where they lie
# (tutorial/CPUlp.cuh + header/graph.h + header/myutil.h), with g++ and the
# include shims of oracle/ref_shim/.  Outputs only into oracle/_ref/.
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
