// smem_attr.h -- the per-process dynamic shared memory limit of a kernel.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace glp {

// Raises `kernel`'s dynamic shared memory limit on the current device to at
// least `bytes` and never lowers it.  The limit belongs to the process, not
// to a launch: graph handles or batches used from several host threads would
// otherwise undo one another's setting between its set and their launch.
inline cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limits[{dev, kernel}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

}  // namespace glp
