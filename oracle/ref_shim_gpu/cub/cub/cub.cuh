// Include shim for oracle/ref_gpu_harness.cu: the reference's kernels include
// "cub/cub/cub.cuh" (its vendored CUB 1.8, which does not build against
// CUDA 12.9); this forwards to the CUB that ships with the CUDA toolkit.
#pragma once
#include <cub/cub.cuh>
