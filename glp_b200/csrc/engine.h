// engine.h -- internal host-side types of the label-propagation engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/glp.h"
#include "kernels.cuh"

namespace glp {

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
#define GLP_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Degree-tier parameters after defaults and limits are applied.
struct TierParams {
  int32_t tiny_max = 8;    // <= 8 (register tier width)
  int32_t mid_max = 256;   // <= 256 (per-warp table of 512 slots)
  int32_t big_max = 4096;  // <= 8192
  int32_t hub_chunk = 4096;
  bool operator==(const TierParams& o) const {
    return tiny_max == o.tiny_max && mid_max == o.mid_max && big_max == o.big_max && hub_chunk == o.hub_chunk;
  }
};
int resolve_tiers(const glp_params* p, TierParams* t);

// Host-side plan (pure function of the offsets and the tier parameters).
struct HostPlan {
  std::vector<int32_t> tiny, g16, g32, mid, big;  // vertex lists (ascending ids)
  int64_t isolated = 0;
  // hubs
  std::vector<int32_t> hub_v, hub_nchunks;
  std::vector<int64_t> hub_tbase, hub_ubase;
  std::vector<uint32_t> hub_tmask;
  std::vector<int32_t> chunk_hub, chunk_begin, chunk_end;
  int64_t table_slots = 0, used_slots = 0;
};
void build_host_plan(const int32_t* off, int32_t n, const TierParams& t, HostPlan* hp);

struct DevicePlan {
  TierParams tiers;
  bool valid = false;
  int32_t n_tiny = 0, n_g16 = 0, n_g32 = 0, n_mid = 0, n_big = 0, n_hubs = 0, n_chunks = 0;
  int64_t isolated = 0;
  int32_t *tiny = nullptr, *g16 = nullptr, *g32 = nullptr, *mid = nullptr, *big = nullptr;
  HubPlan hub{};
  std::vector<void*> allocs;
  uint32_t big_cap = 0, hub_cap = 0;
};

// Launch configuration of one synchronous step.
struct StepLaunch {
  const DevicePlan* plan;
  cudaStream_t stream;
  cudaEvent_t* ev;  // nullable: 7 pairs of (start, stop) for per-tier timing
};

template <bool W, class S>
int launch_step(const StepLaunch& L, const StepArgs& a, const S& score, int64_t* launches);

}  // namespace glp

struct glp_graph {
  int device = 0;
  int32_t n = 0;
  int64_t m = 0;
  int32_t max_degree = 0;
  int32_t* d_off = nullptr;
  int32_t* d_cols = nullptr;
  int32_t* d_w = nullptr;
  std::vector<int32_t> h_off;
  cudaStream_t stream = nullptr;
  glp::DevicePlan plan;
  // work buffers (grown on demand)
  int32_t* d_lab[2] = {nullptr, nullptr};
  int32_t* d_vol[2] = {nullptr, nullptr};
  int32_t* d_spoken = nullptr;
  int32_t* d_mem = nullptr;
  int64_t mem_elems = 0;
  unsigned long long* d_changed = nullptr;
  int32_t changed_cap = 0;
  uint32_t* d_err = nullptr;
  // method-4 spill tables (2 slots per CSR entry), allocated on first use
  uint32_t* d_hook_keys = nullptr;
  double* d_hook_vals = nullptr;
};
