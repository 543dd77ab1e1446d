// engine.h -- internal host-side types of the label-propagation engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/glp.h"
#include "backends.cuh"
#include "kernels.cuh"

namespace glp {

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
// Streaming multiprocessors of the current device (queried once per device).
int device_sms();
#define GLP_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Degree-tier parameters after defaults and limits are applied.
// Exact-count tier limits: a mid warp's table holds kMidCap slots, a big
// block's 32-bit table at most kBigCap slots (at most half full up to
// degree 8192, three quarters at 12288).
constexpr int kMidCap = 512, kBigCap = 16384;
// In full mode the big tier runs as one launch per degree range: range r
// holds degrees up to kBigPartMax[r] (and above the previous range), counted
// by kBigPartThreads[r]-thread blocks whose tables hold 2*kBigPartMax[r]
// slots, so that a range's table fits as many blocks per SM as it can.
// The last range counts unweighted graphs with 16-bit counts (k_big<...,
// C16>) up to 24576; weighted graphs count it with 32-bit counts in a
// kBigCap-slot table (128 KB) and so cap big_max at kBigMaxWeighted.
constexpr int kBigParts = 5;
constexpr int kBigPartMax[kBigParts] = {1024, 2048, 4096, 8192, 24576};
constexpr int kBigPartThreads[kBigParts] = {256, 256, 512, 1024, 1024};
constexpr int kBigMaxWeighted = 12288, kBigMaxUnweighted = 24576;
static_assert(kBigCap == (int)kBig32Slots, "the engine sizes 32-bit big tables as k_big caps them");

struct TierParams {
  int32_t tiny_max = 8;       // <= 8
  int32_t mid_max = 256;      // <= kMidCap / 2
  int32_t big_max = kBigMaxWeighted;  // <= kBigMaxUnweighted (unweighted graphs), <= kBigMaxWeighted (weighted)
  bool big_auto = true;               // big_max not given: the largest the graph's counts allow
  int32_t hub_chunk = 16384;  // edges per hub streaming block
  bool operator==(const TierParams& o) const {
    return tiny_max == o.tiny_max && mid_max == o.mid_max && big_max == o.big_max && hub_chunk == o.hub_chunk;
  }
};
int resolve_tiers(const glp_params* p, TierParams* t);
// resolve_tiers, then big_max for a graph with (weighted) or without weights.
int tiers_for_graph(const glp_params* p, bool weighted, TierParams* t);

// Host-side plan (pure function of the offsets and the tier parameters).
struct HostPlan {
  std::vector<int32_t> tiny, g16, g32, mid, big, mb;  // vertex lists (ascending ids); mb = mid + big
  std::vector<int32_t> big_part[kBigParts];            // the big tier by kBigPartMax range
  int64_t isolated = 0;
  int64_t edges[7] = {0, 0, 0, 0, 0, 0, 0};  // per tier, as the vertex counts of glp_graph_plan
  // hubs
  std::vector<int32_t> hub_v, hub_nb, hub_item0;
  int32_t max_nb = 0;
  std::vector<int64_t> hub_lbase;
  std::vector<int32_t> chunk_hub, chunk_begin, chunk_end;
  std::vector<int32_t> item_hub, item_bucket;
  int64_t hub_labels = 0;
};
void build_host_plan(const int32_t* off, int32_t n, const TierParams& t, HostPlan* hp);

struct DevicePlan {
  cudaStream_t setup = nullptr;  // stream of the set-up copies (the handle's)
  TierParams tiers;
  bool valid = false;
  Verts tiny{}, g16{}, g32{}, mid{}, big{}, mb{}, big_part[kBigParts]{};
  FailList fmid{}, fbig{};
  FailList fscreen{};  // big-tier vertices a summary screen left to the exact kernel
  // list counters: [majority mid, majority big, frontier tiny, g16, g32, mid,
  // big] are zeroed at the start of every step; [7 + s] counts the changed
  // list chg[s] that steps of parity s append to; [9] counts fscreen
  uint32_t* counts = nullptr;
  int32_t* chg[2] = {nullptr, nullptr};
  Frontier front{};
  int32_t* d_mode = nullptr;
  // two-step cycle detection (classic, symmetric): labels before the last
  // change, their step tags, and a mismatch word
  int32_t* cyc_old = nullptr;
  uint32_t* cyc_stamp = nullptr;
  uint32_t* cyc_mism = nullptr;
  bool mid_c16 = true;  // mid counts fit 16 bits (unweighted, or small weight sums)
  int32_t n_hubs = 0, n_chunks = 0;
  int64_t isolated = 0;
  HubPlan hub{};
  BigBound bb{};  // count bounds of a contiguous big tier (n = 0: the tier is an id list)
  std::vector<void*> allocs;
};

// Launch configuration of one synchronous step.
// The step forks onto two auxiliary streams (hubs; small tiers) and joins
// back before it returns: the tier kernels write disjoint vertices.
struct StepLaunch {
  const DevicePlan* plan;
  cudaStream_t stream;
  cudaEvent_t* ev;  // nullable: (start, stop) pairs for per-tier timing
  cudaStream_t aux[2];
  cudaEvent_t fork, join[2];
  // step-mode inputs (k_step_mode): previous step's changed count (nullptr
  // in the first step) and which shortcuts the method admits
  const unsigned long long* prev_changed = nullptr;
  int allow_majority = 0, allow_frontier = 0;
  Frontier front{};  // this step's frontier inputs (front.chg_in set from the second step)
  int32_t backend = GLP_BACKEND_EXACT;  // GLP_BACKEND_CM / _FA: summary screen on the big tier
  bool serial = false;  // every kernel on `stream` (per-tier timing without overlap)
  uint32_t majority_pm = 500, frontier_pm = 50;  // step-mode thresholds (changes per 1000 vertices)
  bool mid_prefetch = true;  // k_mid loads the next vertex's first batch while counting
  bool big_staged = false;   // k_big_staged for the first big range of full-count steps
  // k_hub_bound may decide hubs from their earlier counts: classic steps,
  // whose gathered labels are the current labels (not SLPA's spoken ones)
  bool hub_bound = false;
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
  std::vector<int32_t> h_off;  // host copy of the offsets, made on first need
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
  // method 5: seed flags (glp_graph_set_seeds) and integer spill tables
  uint8_t* d_seeds = nullptr;
  uint32_t* d_seed_keys = nullptr;
  uint32_t* d_seed_vals = nullptr;
  int symmetric = -1;    // -1 unknown, 0 no, 1 yes (every edge stored both ways)
  int rows_sorted = -1;  // -1 unknown, 0 no, 1 every row strictly ascending
  int deg_sorted = 0;    // 1: degrees never increase along the vertex ids
  uint32_t mid_wsum = 0;  // weighted: largest weight sum of a vertex of degree <= kMidCap / 2
  uint32_t max_wsum = 0;  // largest weight sum of a row (unweighted: the largest degree)
  int2* d_lv = nullptr;   // layered: (label, volume of the label) per vertex
  int64_t lv_elems = 0;
  cudaStream_t last_stream = nullptr;  // the stream of the latest run
  const volatile int32_t* cancel = nullptr;  // glp_graph_set_cancel_flag: non-zero stops a run
  uint32_t epoch = 0;  // frontier mark of the last step
  // two-step cycle detection: host-mapped verdict words (a ring of 4 steps),
  // their device alias, per-step events and the step tag
  uint32_t* h_cycle = nullptr;
  uint32_t* d_cycle = nullptr;
  cudaEvent_t cyc_ev[3] = {nullptr, nullptr, nullptr};
  uint32_t cyc_tag = 0;
  // auxiliary streams and fork/join events of a step
  cudaStream_t aux[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};
