// engine.cu -- graph handle, degree-tier planner, propagation drivers and the
// C ABI of include/glp.h.
//
// Reference correspondence:
//   glp_graph_create      <- CSRGraph + XProp::preprocess (header/graph.h:61-198,
//                            prop/classicLprop.cuh:65-78)
//   build_host_plan       <- degree binning + hub block plan + tiny packing
//                            (prop/classicLprop.cuh:196-308, kernel.cuh:6011-6046)
//   run_classic           <- classicLprop::perform_lp loop (prop/classicLprop.cuh:361-443)
//   run_layered           <- MultiLprop::perform_lp loop (prop/MultiLprop.cuh:308-374)
//   run_slpa              <- SLPA loop (tutorial/Base5prop.cuh:264-293)
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "engine.h"
#include "hooks_engine.cuh"
#include "seeded.cuh"
#include "smem_attr.h"

namespace glp {

int validate_csr_device(glp_graph* g);
static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_fail(cudaError_t e, const char* what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? GLP_ENOMEM : GLP_ECUDA;
}

// Streaming multiprocessors of the current device, queried once per device.
// Grid sizes are multiples of it (a failed query gives 1: the launch that
// follows reports the device error itself).
int device_sms() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (dev >= 0 && dev < 64) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 1;
  if (dev >= 0 && dev < 64) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

// Device memory of graph handles comes from the device's stream-ordered pool,
// set once per device to keep freed memory in this process (release
// threshold at its maximum): handles created and destroyed in a loop reuse
// memory instead of mapping and unmapping gigabytes every time.  An
// allocation is complete when dev_alloc returns (its stream is synchronised),
// so any stream may use it; dev_free is called only once no stream uses the
// memory any more.
static std::once_flag g_pool_once[64];
static cudaError_t dev_alloc_raw(void** p, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 64)
    std::call_once(g_pool_once[dev], [dev] {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    });
  e = cudaMallocAsync(p, std::max<size_t>(bytes, 1), cudaStreamPerThread);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  return e;
}
template <class T>
static cudaError_t dev_alloc(T** p, size_t bytes) {
  return dev_alloc_raw(reinterpret_cast<void**>(p), bytes);
}
static void dev_free(void* p) {
  if (p) cudaFreeAsync(p, cudaStreamPerThread);
}

// Waits for every stream a handle's work may be on.
static int quiesce(glp_graph* g) {
  for (cudaStream_t st : {g->stream, g->aux[0], g->aux[1], g->last_stream})
    if (st) GLP_CUDA(cudaStreamSynchronize(st));
  return GLP_OK;
}

static int require_device() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    set_error("no usable CUDA device (%s)", e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    return GLP_ENODEV;
  }
  return GLP_OK;
}


int resolve_tiers(const glp_params* p, TierParams* t) {
  TierParams d;
  if (p) {
    if (p->tiny_max > 0) d.tiny_max = p->tiny_max;
    if (p->tiny_max < 0) d.tiny_max = 0;
    if (p->mid_max > 0) d.mid_max = p->mid_max;
    if (p->big_max > 0) {
      d.big_max = p->big_max;
      d.big_auto = false;
    }
    if (p->hub_chunk > 0) d.hub_chunk = p->hub_chunk;
  }
  if (d.tiny_max > 8) {
    set_error("tiny_max %d > 8", d.tiny_max);
    return GLP_EINVAL;
  }
  if (d.mid_max < 32 || d.mid_max > kMidCap / 2) {
    set_error("mid_max %d outside [32, %d]", d.mid_max, kMidCap / 2);
    return GLP_EINVAL;
  }
  if (d.big_max < d.mid_max || d.big_max > kBigMaxUnweighted) {
    set_error("big_max %d outside [mid_max, %d]", d.big_max, kBigMaxUnweighted);
    return GLP_EINVAL;
  }
  if (d.hub_chunk < 256 || d.hub_chunk > 65536) {
    set_error("hub_chunk %d outside [256, 65536]", d.hub_chunk);
    return GLP_EINVAL;
  }
  *t = d;
  return GLP_OK;
}

int tiers_for_graph(const glp_params* p, bool weighted, TierParams* t) {
  int rc = resolve_tiers(p, t);
  if (rc) return rc;
  if (t->big_auto) {
    t->big_max = weighted ? kBigMaxWeighted : kBigMaxUnweighted;
  } else if (weighted && t->big_max > kBigMaxWeighted) {
    set_error("big_max %d above %d needs an unweighted graph (16-bit counts)", t->big_max, kBigMaxWeighted);
    return GLP_EINVAL;
  }
  static_assert(4 * kBigMaxWeighted <= 3 * kBigCap, "a weighted big table is at most three quarters full");
  return GLP_OK;
}

// Degree tiers; hubs get ceil(3*deg / kHubTable) hash buckets (one work item
// each) and streaming chunks of hub_chunk edges.
void build_host_plan(const int32_t* off, int32_t n, const TierParams& t, HostPlan* hp) {
  *hp = HostPlan{};
  for (int32_t v = 0; v < n; ++v) {
    const int32_t d = off[v + 1] - off[v];
    int tier;
    if (d == 0) {
      hp->isolated++;
      tier = 0;
    } else if (d <= t.tiny_max) {
      hp->tiny.push_back(v);
      tier = 1;
    } else if (d <= 16) {
      hp->g16.push_back(v);
      tier = 2;
    } else if (d <= 32) {
      hp->g32.push_back(v);
      tier = 3;
    } else if (d <= t.mid_max) {
      hp->mid.push_back(v);
      hp->mb.push_back(v);
      tier = 4;
    } else if (d <= t.big_max) {
      hp->big.push_back(v);
      hp->mb.push_back(v);
      int r = 0;
      while (r + 1 < kBigParts && d > kBigPartMax[r]) ++r;
      hp->big_part[r].push_back(v);
      tier = 5;
    } else {
      tier = 6;
      const int32_t h = (int32_t)hp->hub_v.size();
      const int32_t nb = (int32_t)((3ll * d + kHubTable - 1) / kHubTable);
      hp->hub_v.push_back(v);
      hp->hub_nb.push_back(nb);
      hp->hub_item0.push_back((int32_t)hp->item_hub.size());
      hp->max_nb = std::max(hp->max_nb, nb);
      hp->hub_lbase.push_back(hp->hub_labels);
      hp->hub_labels += d;
      for (int32_t b = 0; b < nb; ++b) {
        hp->item_hub.push_back(h);
        hp->item_bucket.push_back(b);
      }
      for (int64_t c = off[v]; c < off[v + 1]; c += t.hub_chunk) {
        hp->chunk_hub.push_back(h);
        hp->chunk_begin.push_back((int32_t)c);
        hp->chunk_end.push_back((int32_t)std::min<int64_t>(off[v + 1], c + t.hub_chunk));
      }
    }
    hp->edges[tier] += d;
  }
}

static void free_plan(DevicePlan* p) {
  for (void* a : p->allocs) dev_free(a);
  *p = DevicePlan{};
}

// Plan set-up copies and clears go on the handle's stream (a pageable
// source is staged before the call returns); ensure_plan synchronises that
// stream before any step kernel, on whatever stream, can read the plan.
template <class T>
static int upload(DevicePlan* p, const std::vector<T>& v, T** out) {
  *out = nullptr;
  if (v.empty()) return GLP_OK;
  void* d = nullptr;
  GLP_CUDA(dev_alloc(&d, v.size() * sizeof(T)));
  p->allocs.push_back(d);
  GLP_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, p->setup));
  *out = static_cast<T*>(d);
  return GLP_OK;
}

// A tier whose vertex ids are consecutive becomes a range (no id list).
static int upload_verts(DevicePlan* p, const std::vector<int32_t>& v, Verts* out) {
  *out = Verts{nullptr, 0, (int32_t)v.size()};
  if (v.empty()) return GLP_OK;
  bool range = true;
  for (size_t i = 1; i < v.size() && range; ++i) range = v[i] == v[0] + (int32_t)i;
  if (range) {
    out->base = v[0];
    return GLP_OK;
  }
  int32_t* d = nullptr;
  int rc = upload(p, v, &d);
  out->ids = d;
  return rc;
}

template <class T>
static int zeroed(DevicePlan* p, size_t count, T** out) {
  *out = nullptr;
  if (count == 0) return GLP_OK;
  void* d = nullptr;
  GLP_CUDA(dev_alloc(&d, count * sizeof(T)));
  p->allocs.push_back(d);
  GLP_CUDA(cudaMemsetAsync(d, 0, count * sizeof(T), p->setup));
  *out = static_cast<T*>(d);
  return GLP_OK;
}

static int ensure_host_offsets(glp_graph* g);
static int device_bounds(glp_graph* g, const int32_t* thr, int k, int32_t* out);

// Range-mode tier of a degree-sorted graph.
static Verts range_verts(int32_t lo, int32_t hi) { return Verts{nullptr, lo, hi > lo ? hi - lo : 0}; }

static int ensure_plan(glp_graph* g, const TierParams& t) {
  if (g->plan.valid && g->plan.tiers == t) return GLP_OK;
  free_plan(&g->plan);
  HostPlan hp;
  DevicePlan& p = g->plan;
  p.tiers = t;
  p.setup = g->stream;
  // weighted mid counts fit 16 bits when no mid vertex's weights sum past it
  p.mid_c16 = g->d_w == nullptr || g->mid_wsum < 65536u;
  int rc;
  int64_t n_mid = 0, n_big = 0, ntier[5] = {0, 0, 0, 0, 0};
  if (g->deg_sorted == 1) {
    // every tier is a contiguous range: its bounds come from binary searches
    // over the non-increasing degrees; only the hubs' offsets reach the host
    // thresholds, descending: big_max, the part bounds below it, mid_max, 32,
    // 16, tiny_max, 0; b[i] = vertices of degree > thr[i]
    constexpr int kT = kBigParts + 5;
    int32_t thr[kT];
    thr[0] = t.big_max;
    for (int r = kBigParts - 2, i = 1; r >= 0; --r, ++i) thr[i] = std::min<int32_t>(kBigPartMax[r], t.big_max);
    thr[kBigParts] = t.mid_max;
    thr[kBigParts + 1] = 32;
    thr[kBigParts + 2] = 16;
    thr[kBigParts + 3] = t.tiny_max;
    thr[kBigParts + 4] = 0;
    int32_t b[kT];
    if ((rc = device_bounds(g, thr, kT, b))) return rc;
    for (int i = 1; i < kBigParts; ++i) b[i] = std::min(std::max(b[i], b[i - 1]), b[kBigParts]);
    std::vector<int32_t> hub_off((size_t)b[0] + 1);
    GLP_CUDA(cudaMemcpy(hub_off.data(), g->d_off, sizeof(int32_t) * hub_off.size(), cudaMemcpyDeviceToHost));
    build_host_plan(hub_off.data(), b[0], t, &hp);  // all of them are hubs
    for (int r = 0; r < kBigParts; ++r) p.big_part[r] = range_verts(b[kBigParts - 1 - r], b[kBigParts - r]);
    p.big = range_verts(b[0], b[kBigParts]);
    p.mid = range_verts(b[kBigParts], b[kBigParts + 1]);
    p.mb = range_verts(b[0], b[kBigParts + 1]);
    p.g32 = range_verts(b[kBigParts + 1], b[kBigParts + 2]);
    p.g16 = range_verts(b[kBigParts + 2], b[kBigParts + 3]);
    p.tiny = range_verts(b[kBigParts + 3], b[kBigParts + 4]);
    p.isolated = g->n - b[kBigParts + 4];
  } else {
    if ((rc = ensure_host_offsets(g))) return rc;
    build_host_plan(g->h_off.data(), g->n, t, &hp);
    p.isolated = hp.isolated;
    if ((rc = upload_verts(&p, hp.tiny, &p.tiny)) || (rc = upload_verts(&p, hp.g16, &p.g16)) ||
        (rc = upload_verts(&p, hp.g32, &p.g32)) || (rc = upload_verts(&p, hp.mid, &p.mid)) ||
        (rc = upload_verts(&p, hp.big, &p.big)) || (rc = upload_verts(&p, hp.mb, &p.mb))) {
      free_plan(&p);
      return rc;
    }
    for (int r = 0; r < kBigParts; ++r)
      if ((rc = upload_verts(&p, hp.big_part[r], &p.big_part[r]))) {
        free_plan(&p);
        return rc;
      }
  }
  n_mid = p.mid.n;
  n_big = p.big.n;
  ntier[0] = p.tiny.n;
  ntier[1] = p.g16.n;
  ntier[2] = p.g32.n;
  ntier[3] = p.mid.n;
  ntier[4] = p.big.n;
  if ((rc = zeroed(&p, 10, &p.counts)) || (rc = zeroed(&p, std::max<size_t>((size_t)n_mid, 1), &p.fmid.ids)) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)n_big, 1), &p.fbig.ids)) || (rc = zeroed(&p, 2, &p.d_mode)) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)n_big, 1), &p.fscreen.ids)) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)g->n, 1), &p.front.act)) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)g->n, 1), &p.chg[0])) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)g->n, 1), &p.chg[1])) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)g->n, 1), &p.cyc_old)) ||
      (rc = zeroed(&p, std::max<size_t>((size_t)g->n, 1), &p.cyc_stamp)) || (rc = zeroed(&p, 1, &p.cyc_mism))) {
    free_plan(&p);
    return rc;
  }
  if (p.big.n && !p.big.ids) {  // a contiguous big tier: count bounds for its frontier steps
    if ((rc = zeroed(&p, (size_t)p.big.n, &p.bb.lbl)) || (rc = zeroed(&p, (size_t)p.big.n, &p.bb.lb)) ||
        (rc = zeroed(&p, (size_t)p.big.n, &p.bb.nchg))) {
      free_plan(&p);
      return rc;
    }
    p.bb.base = p.big.base;
    p.bb.n = p.big.n;
  }
  g->epoch = 0;  // fresh marks
  g->cyc_tag = 0;
  p.fmid.count = p.counts;
  p.fbig.count = p.counts + 1;
  p.fscreen.count = p.counts + 9;
  p.front.tiny_max = t.tiny_max;
  p.front.mid_max = t.mid_max;
  p.front.big_max = t.big_max;
  for (int k = 0; k < 5; ++k) {
    if ((rc = zeroed(&p, std::max<size_t>((size_t)ntier[k], 1), &p.front.tier[k].ids))) {
      free_plan(&p);
      return rc;
    }
    p.front.tier[k].count = p.counts + 2 + k;
  }
  p.n_hubs = (int32_t)hp.hub_v.size();
  p.n_chunks = (int32_t)hp.chunk_hub.size();
  if (p.n_hubs) {
    HubPlan& h = p.hub;
    if ((rc = upload(&p, hp.chunk_hub, (int32_t**)&h.chunk_hub)) ||
        (rc = upload(&p, hp.chunk_begin, (int32_t**)&h.chunk_begin)) ||
        (rc = upload(&p, hp.chunk_end, (int32_t**)&h.chunk_end)) || (rc = upload(&p, hp.hub_v, (int32_t**)&h.hub_v)) ||
        (rc = upload(&p, hp.hub_lbase, (int64_t**)&h.hub_lbase)) ||
        (rc = upload(&p, hp.hub_nb, (int32_t**)&h.hub_nb)) ||
        (rc = upload(&p, hp.item_hub, (int32_t**)&h.item_hub)) ||
        (rc = upload(&p, hp.item_bucket, (int32_t**)&h.item_bucket)) ||
        (rc = upload(&p, hp.hub_item0, (int32_t**)&h.hub_item0)) ||
        (rc = zeroed(&p, (size_t)hp.hub_labels, &h.hlab)) || (rc = zeroed(&p, (size_t)hp.hub_labels, &h.hsort)) ||
        (rc = zeroed(&p, hp.item_hub.size(), &h.bcnt)) || (rc = zeroed(&p, hp.item_hub.size(), &h.bstart)) ||
        (rc = zeroed(&p, hp.item_hub.size(), &h.bcur)) ||
        (g->d_w && ((rc = zeroed(&p, (size_t)hp.hub_labels, &h.hw)) ||
                    (rc = zeroed(&p, (size_t)hp.hub_labels, &h.hsw)))) ||
        (rc = zeroed(&p, (size_t)p.n_hubs, &h.hub_best)) ||
        (rc = zeroed(&p, (size_t)p.n_hubs, &h.hub_cand)) || (rc = zeroed(&p, (size_t)p.n_hubs, &h.hub_state)) ||
        (rc = zeroed(&p, (size_t)p.n_hubs, &h.hub_lbl)) || (rc = zeroed(&p, (size_t)p.n_hubs, &h.hub_lb))) {
      free_plan(&p);
      return rc;
    }
    h.nhubs = p.n_hubs;
    h.nitems = (int32_t)hp.item_hub.size();
    h.max_nb = hp.max_nb;
    if (hp.max_nb > 25600) {
      free_plan(&p);
      set_error("a vertex of degree above %d is not supported", 25600 / 3 * kHubTable);
      return GLP_ENOTSUP;
    }
  }
  const cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    free_plan(&p);
    return cuda_fail(e, "plan upload");
  }
  p.valid = true;
  return GLP_OK;
}

// --------------------------------------------------------------- launches
template <class K>
static int allow_smem(K kernel, size_t bytes) {
  // static + dynamic shared memory above 48 KB needs the opt-in
  GLP_CUDA(raise_smem_limit((const void*)kernel, bytes));
  return GLP_OK;
}

static inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }


// One launch over a device-built list of big-tier vertices (majority
// failures, frontier members, screen fallbacks): 512-thread blocks with a
// table for the tier's largest degree, with 16-bit counts on unweighted
// graphs when the tier reaches its last range (past 8192) or the score packs
// (classic, 32-bit layered): smaller tables, more blocks per SM.
template <bool W, class S>
static int launch_big_list(const DevicePlan& p, const StepArgs& a, const TierWork& tw, const S& score,
                           cudaStream_t s, int64_t* launches) {
  const unsigned grid = (unsigned)std::min<int64_t>(p.big.n, device_sms() * 4);
  ++*launches;
  if constexpr (!W) {
    const bool top = p.big_part[kBigParts - 1].n > 0;
    if (top || S::kPacked) {
      const size_t sm16 = (size_t)(top ? kBig16Slots : 2 * kBigPartMax[kBigParts - 2]) * 6;
      GLP_CUDA(raise_smem_limit((const void*)k_big<512, false, S, true>, sm16));
      k_big<512, false, S, true><<<grid, 512, sm16, s>>>(a, tw, score);
      return GLP_OK;
    }
  }
  const size_t sm = 2ull * kBigCap * sizeof(uint32_t);
  GLP_CUDA(raise_smem_limit((const void*)k_big<512, W, S>, sm));
  k_big<512, W, S><<<grid, 512, sm, s>>>(a, tw, score);
  return GLP_OK;
}

template <bool W, class S>
int launch_step(const StepLaunch& Lin, const StepArgs& a, const S& score, int64_t* launches) {
  StepLaunch L = Lin;
  if (L.serial) L.aux[0] = L.aux[1] = L.stream;
  const DevicePlan& p = *L.plan;
  cudaStream_t s = L.stream;
  auto mark_on = [&](cudaStream_t st, int i, int which) -> int {
    if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[2 * i + which], st));
    return GLP_OK;
  };
  int rc;
  const unsigned kMaxGrid = device_sms() * 32;
  if ((rc = mark_on(s, 8, 0))) return rc;  // whole-step start
  const bool modal = a.mode != nullptr;
  if (modal) {
    GLP_CUDA(cudaMemsetAsync(p.counts, 0, 7 * sizeof(uint32_t), s));
    k_step_mode<<<1, 1, 0, s>>>(L.prev_changed, a.n, a.n - (int32_t)p.isolated, L.allow_majority,
                                L.allow_frontier, L.majority_pm, L.frontier_pm, p.d_mode);
    ++*launches;
    if (L.allow_frontier && L.front.chg_in) {
      const unsigned fgrid = device_sms() * 16;
      k_frontier_push<<<fgrid, 256, 0, s>>>(a, L.front);
      k_frontier_copy<<<fgrid, 256, 0, s>>>(a, L.front);
      *launches += 2;
      if (p.n_hubs) {
        k_frontier_hubs<<<(unsigned)cdiv(p.n_hubs, 256), 256, 0, s>>>(a, L.front, p.hub);
        ++*launches;
      }
    }
  }
  auto work = [&](const Verts& all, int k, const FailList* major) {
    TierWork tw{all, major ? *major : FailList{nullptr, nullptr}, p.front.tier[k], 0};
    return tw;
  };
  // fork: hubs on aux[0], the small tiers on aux[1], the rest here
  GLP_CUDA(cudaEventRecord(L.fork, s));
  GLP_CUDA(cudaStreamWaitEvent(L.aux[0], L.fork, 0));
  GLP_CUDA(cudaStreamWaitEvent(L.aux[1], L.fork, 0));
  constexpr int kMidNT = 256, kBigNT = 256, kHubNT = 512, kBucketNT = 512;
  if (p.n_hubs) {
    const size_t sm = 2ull * kHubTable * sizeof(uint32_t);
    const size_t sm_hist = (size_t)p.hub.max_nb * sizeof(uint32_t);
    if ((rc = allow_smem(k_hub_bucket<kBucketNT, W, S>, sm)) || (rc = allow_smem(k_hub_gather<kHubNT, W>, sm_hist)) ||
        (rc = allow_smem(k_hub_scatter<kHubNT, W>, 2 * sm_hist)))
      return rc;
    if ((rc = mark_on(L.aux[0], 5, 0))) return rc;
    const unsigned grid = (unsigned)std::min<int64_t>(p.n_chunks, kMaxGrid);
    const unsigned hgrid = (unsigned)cdiv(p.n_hubs, 256);
    if (L.allow_majority && modal) {
      k_hub_bound<W><<<hgrid, 256, 0, L.aux[0]>>>(a, p.hub, L.prev_changed, L.hub_bound ? 1 : 0);
      k_hub_majority<kHubNT, W><<<grid, kHubNT, 0, L.aux[0]>>>(a, p.hub, p.n_chunks);
      *launches += 2;
    }
    k_hub_decide<<<hgrid, 256, 0, L.aux[0]>>>(a, p.hub);
    GLP_CUDA(cudaMemsetAsync(p.hub.bcnt, 0, sizeof(uint32_t) * p.hub.nitems, L.aux[0]));
    k_hub_gather<kHubNT, W><<<grid, kHubNT, sm_hist, L.aux[0]>>>(a, p.hub, p.n_chunks);
    k_hub_offsets<<<hgrid, 256, 0, L.aux[0]>>>(p.hub);
    k_hub_scatter<kHubNT, W><<<grid, kHubNT, 2 * sm_hist, L.aux[0]>>>(a, p.hub, p.n_chunks);
    k_hub_bucket<kBucketNT, W, S><<<(unsigned)std::min<int64_t>(p.hub.nitems, device_sms() * 8), kBucketNT, sm, L.aux[0]>>>(
        a, p.hub, score);
    k_hub_finalize<<<hgrid, 256, 0, L.aux[0]>>>(a, p.hub);
    *launches += 6;
    if ((rc = mark_on(L.aux[0], 5, 1))) return rc;
  }
  if (L.allow_majority && modal && p.mb.n) {
    if ((rc = mark_on(s, 7, 0))) return rc;  // slot 7: the majority pre-pass
    k_major_warp<W><<<(unsigned)std::min<int64_t>(cdiv((int64_t)p.mb.n * 32, 256), kMaxGrid), 256, 0, s>>>(
        a, p.mb, p.tiers.mid_max, p.fmid, p.fbig);
    if ((rc = mark_on(s, 7, 1))) return rc;
    ++*launches;
  }
  if (p.big.n && L.backend != GLP_BACKEND_EXACT) {
    // a summary screen decides what it can over the whole tier (its work
    // lists included); the exact kernel takes the vertices it lists
    if ((rc = mark_on(s, 4, 0))) return rc;
    GLP_CUDA(cudaMemsetAsync(p.fscreen.count, 0, sizeof(uint32_t), s));
    TierWork all = work(p.big, 4, &p.fbig);
    if (L.backend == GLP_BACKEND_CM) {
      k_big_cm<kBigNT, W, S><<<(unsigned)std::min<int64_t>(p.big.n, kMaxGrid), kBigNT, 0, s>>>(a, all, score,
                                                                                              p.fscreen);
    } else {
      constexpr int kFaNT = 128;
      k_big_fa<kFaNT, W, S><<<(unsigned)std::min<int64_t>(cdiv(p.big.n, kFaNT / 32), kMaxGrid), kFaNT, 0, s>>>(
          a, all, score, p.fscreen);
    }
    TierWork rest{Verts{nullptr, 0, 0}, p.fscreen, FailList{nullptr, nullptr}, 0, 1};
    if ((rc = launch_big_list<W, S>(p, a, rest, score, s, launches))) return rc;
    ++*launches;
    if ((rc = mark_on(s, 4, 1))) return rc;
  } else if (p.big.n) {
    // full mode: one launch per degree range, each with the table and block
    // size it needs; outside full mode the tier's majority / frontier list
    // goes to one launch with a table for any degree of the tier
    if ((rc = mark_on(s, 4, 0))) return rc;
    const FailList none{nullptr, nullptr};
    static_assert(kBigParts == 5 && kBigPartThreads[0] == 256 && kBigPartThreads[1] == 256 &&
                      kBigPartThreads[2] == 512 && kBigPartThreads[3] == 1024 && kBigPartThreads[4] == 1024,
                  "the launches below follow kBigPartThreads");
    // unweighted counts fit 16 bits: the claim-first 16-bit tables (and
    // S::kSMThreads threads per SM) fit more blocks, and with 32-register
    // scores the 2049..4096 range runs 1024-thread blocks (measured 9 %
    // faster than 512: one batch of four entries a thread covers its rows)
    constexpr bool k16 = !W && S::kPacked;
    for (int r = 0; r < kBigParts; ++r) {
      const Verts& vs = p.big_part[r];
      if (!vs.n) continue;
      const TierWork tw{vs, none, none, 1};
      const size_t smr = 4ull * kBigPartMax[r] * sizeof(uint32_t);
      const unsigned grid = (unsigned)std::min<int64_t>(vs.n, kMaxGrid);
      if (k16 && r < kBigParts - 1) {
        const size_t sm16 = 12ull * kBigPartMax[r];  // 2*max slots of 4 + 2 bytes
        bool staged = false;
        if constexpr (S::kPacked) {
          if (r == 0 && L.big_staged && kBigPartMax[0] <= kStagedRow) {
            // rows staged in shared memory by bulk copies, one vertex ahead
            k_big_staged<256, S><<<grid, 256, sm16, s>>>(a, tw, score);
            staged = true;
          }
        }
        if (staged) {
        } else if (r <= 1) {
          k_big<256, false, S, true><<<grid, 256, sm16, s>>>(a, tw, score);
        } else if (r == 2 && S::kSMThreads < 2048) {  // 40-register scores: 512 threads, three blocks per SM
          if ((rc = allow_smem(k_big<512, false, S, true>, sm16))) return rc;
          k_big<512, false, S, true><<<grid, 512, sm16, s>>>(a, tw, score);
        } else {  // 2049..8192: 1024 threads cover a row in one batch (48 / 96 KB tables, two blocks per SM)
          if ((rc = allow_smem(k_big<1024, false, S, true>, sm16))) return rc;
          k_big<1024, false, S, true><<<grid, 1024, sm16, s>>>(a, tw, score);
        }
      } else if (r < 2) {
        k_big<256, W, S><<<grid, 256, smr, s>>>(a, tw, score);
      } else if (r == 2) {
        if ((rc = allow_smem(k_big<512, W, S>, smr))) return rc;
        k_big<512, W, S><<<grid, 512, smr, s>>>(a, tw, score);
      } else if (r == 3) {
        if ((rc = allow_smem(k_big<1024, W, S>, smr))) return rc;
        k_big<1024, W, S><<<grid, 1024, smr, s>>>(a, tw, score);
      } else if constexpr (!W) {  // the 16-bit range of unweighted graphs, load-first
        const size_t sm16 = (size_t)kBig16Slots * 6;
        if ((rc = allow_smem(k_big<1024, false, S, true, false>, sm16))) return rc;
        k_big<1024, false, S, true, false><<<grid, 1024, sm16, s>>>(a, tw, score);
      } else {  // weighted 8193..kBigMaxWeighted: 32-bit counts, kBigCap slots (128 KB)
        const size_t smw = 2ull * kBigCap * sizeof(uint32_t);
        if ((rc = allow_smem(k_big<1024, W, S>, smw))) return rc;
        k_big<1024, W, S><<<grid, 1024, smw, s>>>(a, tw, score);
      }
      ++*launches;
    }
    if (modal) {
      if ((rc = launch_big_list<W, S>(p, a, work(Verts{nullptr, 0, 0}, 4, &p.fbig), score, s, launches))) return rc;
    }
    if ((rc = mark_on(s, 4, 1))) return rc;
  }
  if (p.mid.n) {
    if ((rc = mark_on(s, 3, 0))) return rc;
    const unsigned grid = (unsigned)std::min<int64_t>(cdiv(p.mid.n, kMidNT / 32), kMaxGrid);
    bool c16w = false;  // weighted classic with small weight sums: 16-bit counts
    const TierWork mw = work(p.mid, 3, &p.fmid);
    if constexpr (W && S::kPacked) {
      c16w = p.mid_c16;
      if (c16w) k_mid<kMidCap, kMidNT, W, S, true><<<grid, kMidNT, 0, s>>>(a, mw, score);
    }
    if (!c16w) {
      // the next vertex's first batch in flight while counting: unweighted
      // classic only (the other instantiations would spill at their register caps)
      if constexpr (S::kMajority && !W) {
        if (L.mid_prefetch) k_mid<kMidCap, kMidNT, W, S, true, true><<<grid, kMidNT, 0, s>>>(a, mw, score);
        else k_mid<kMidCap, kMidNT, W, S><<<grid, kMidNT, 0, s>>>(a, mw, score);
      } else {
        k_mid<kMidCap, kMidNT, W, S><<<grid, kMidNT, 0, s>>>(a, mw, score);
      }
    }
    if ((rc = mark_on(s, 3, 1))) return rc;
    ++*launches;
  }
  if (p.g32.n) {
    if ((rc = mark_on(L.aux[1], 2, 0))) return rc;
    k_tiny<32, W, S><<<(unsigned)std::min<int64_t>(cdiv(p.g32.n, 256), kMaxGrid), 256, 0, L.aux[1]>>>(
        a, work(p.g32, 2, nullptr), score);
    if ((rc = mark_on(L.aux[1], 2, 1))) return rc;
    ++*launches;
  }
  if (p.g16.n) {
    if ((rc = mark_on(L.aux[1], 1, 0))) return rc;
    k_tiny<16, W, S><<<(unsigned)std::min<int64_t>(cdiv(p.g16.n, 256), kMaxGrid), 256, 0, L.aux[1]>>>(
        a, work(p.g16, 1, nullptr), score);
    if ((rc = mark_on(L.aux[1], 1, 1))) return rc;
    ++*launches;
  }
  if (p.tiny.n) {
    if ((rc = mark_on(L.aux[1], 0, 0))) return rc;
    k_tiny<8, W, S><<<(unsigned)std::min<int64_t>(cdiv(p.tiny.n, 256), kMaxGrid), 256, 0, L.aux[1]>>>(
        a, work(p.tiny, 0, nullptr), score);
    if ((rc = mark_on(L.aux[1], 0, 1))) return rc;
    ++*launches;
  }
  // join
  GLP_CUDA(cudaEventRecord(L.join[0], L.aux[0]));
  GLP_CUDA(cudaEventRecord(L.join[1], L.aux[1]));
  GLP_CUDA(cudaStreamWaitEvent(s, L.join[0], 0));
  GLP_CUDA(cudaStreamWaitEvent(s, L.join[1], 0));
  if ((rc = mark_on(s, 8, 1))) return rc;  // whole-step stop
  GLP_CUDA(cudaGetLastError());
  return GLP_OK;
}

// ------------------------------------------------------------ run context
// Per-tier device timing: every step gets its own 16 events (start/stop for 8
// tiers), recorded on the run's stream around each kernel and read once after
// the run, so timing adds no host synchronisation inside the loop.
struct RunCtx {
  glp_graph* g = nullptr;
  cudaStream_t s = nullptr;
  glp_iter_cb cb = nullptr;
  void* user = nullptr;
  std::vector<int32_t> hbuf;
  bool timing = false;
  std::vector<std::vector<cudaEvent_t>> evs;
  std::vector<std::vector<bool>> ran;
  size_t used = 0;
  float tier_ms[8] = {};
  std::vector<float> step_ms, step_tier;
  int64_t launches = 0;
  int iter_base = 0;
  int32_t backend = GLP_BACKEND_EXACT;  // counting back-end of the big tier
  bool serial = false;                  // glp_params.serial_step: one stream per step
  uint32_t majority_pm = 500, frontier_pm = 50;  // glp_params step-mode thresholds
  bool l2_window = false;               // glp_params.l2_window
  bool mid_prefetch = true;             // glp_params.mid_prefetch
  bool big_staged = false;              // glp_params.big_staged
  bool cycle = false;                   // stop a classic run once it ends in a two-step cycle
  int32_t cycle_from = -1;              // first iteration not run (the labels repeat from there)

  ~RunCtx() {
    for (auto& v : evs)
      for (cudaEvent_t e : v)
        if (e) cudaEventDestroy(e);
  }
  // Events for the next step (nullptr when not timing).
  static constexpr int kSlots = 9;  // tiers 0-5, aux 6, majority 7, whole step 8
  cudaEvent_t* step_events() {
    if (!timing) return nullptr;
    if (used == evs.size()) {
      std::vector<cudaEvent_t> v(2 * kSlots, nullptr);
      for (auto& e : v)
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      evs.push_back(v);
    }
    ran.emplace_back(kSlots, false);
    return evs[used++].data();
  }
  void mark_ran(int tier) {
    if (timing && !ran.empty()) ran.back()[tier] = true;
  }
  StepLaunch launch() {
    cudaEvent_t* ev = step_events();
    if (ev) {
      const DevicePlan& p = g->plan;
      ran.back()[0] = p.tiny.n > 0;
      ran.back()[1] = p.g16.n > 0;
      ran.back()[2] = p.g32.n > 0;
      ran.back()[3] = p.mid.n > 0;
      ran.back()[4] = p.big.n > 0;
      ran.back()[5] = p.n_hubs > 0;
      ran.back()[7] = p.mb.n > 0;
      ran.back()[8] = true;
    }
    StepLaunch L{&g->plan, s, ev, {g->aux[0], g->aux[1]}, g->fork, {g->join[0], g->join[1]}};
    L.backend = backend;
    L.serial = serial;
    L.majority_pm = majority_pm;
    L.frontier_pm = frontier_pm;
    L.mid_prefetch = mid_prefetch;
    L.big_staged = big_staged;
    return L;
  }
  cudaEvent_t* current() { return timing && used ? evs[used - 1].data() : nullptr; }
  int harvest() {
    if (!timing) return GLP_OK;
    GLP_CUDA(cudaStreamSynchronize(s));
    step_ms.assign(used, 0.f);
    step_tier.assign(used * 8, 0.f);
    for (size_t i = 0; i < used; ++i)
      for (int t = 0; t < kSlots; ++t) {
        if (!ran[i][t]) continue;
        float ms = 0;
        // a majority slot whose pre-pass was not launched this step has no events
        if (cudaEventElapsedTime(&ms, evs[i][2 * t], evs[i][2 * t + 1]) != cudaSuccess) {
          (void)cudaGetLastError();
          continue;
        }
        if (t == 8) {
          step_ms[i] = ms;
        } else {
          tier_ms[t] += ms;
          step_tier[i * 8 + t] = ms;
        }
      }
    return GLP_OK;
  }
  // Record the aux-kernel events (tier 6) of the current step.
  int aux_mark(int which) {
    cudaEvent_t* ev = current();
    if (!ev) return GLP_OK;
    GLP_CUDA(cudaEventRecord(ev[12 + which], s));
    if (which == 1) mark_ran(6);
    return GLP_OK;
  }
};

static int check_err(glp_graph* g, cudaStream_t s) {
  uint32_t err = 0;
  GLP_CUDA(cudaMemcpyAsync(&err, g->d_err, sizeof err, cudaMemcpyDeviceToHost, s));
  GLP_CUDA(cudaStreamSynchronize(s));
  if (err) {
    GLP_CUDA(cudaMemsetAsync(g->d_err, 0, sizeof(uint32_t), s));
    GLP_CUDA(cudaStreamSynchronize(s));
    set_error("kernel error flags 0x%x (probe overflow=1, score range=2, hub plan=4, table past shared memory=8, bulk-copy wait ran out=16)",
              err);
    return GLP_EKERNEL;
  }
  return GLP_OK;
}

static int after_iter(RunCtx& c, int32_t iter, const int32_t* d_labels) {
  int rc;
  if (c.g->cancel && *c.g->cancel) {
    // stop enqueuing; the work already on the stream finishes first, so the
    // handle has nothing in flight when the call returns
    GLP_CUDA(cudaStreamSynchronize(c.s));
    set_error("run cancelled after iteration %d", iter);
    return GLP_ECANCELED;
  }
  if (!c.cb) return GLP_OK;
  c.hbuf.resize(c.g->n);
  GLP_CUDA(cudaMemcpyAsync(c.hbuf.data(), d_labels, sizeof(int32_t) * c.g->n, cudaMemcpyDeviceToHost, c.s));
  if ((rc = check_err(c.g, c.s))) return rc;
  if (c.cb(iter, c.hbuf.data(), c.g->n, c.user)) {
    set_error("run stopped by the iteration callback at iteration %d", iter);
    return GLP_ECANCELED;
  }
  return GLP_OK;
}

static int grow(int32_t** p, int64_t* have, int64_t need) {
  if (*have >= need && *p) return GLP_OK;
  if (*p) dev_free(*p);
  *p = nullptr;
  GLP_CUDA(dev_alloc(p, std::max<int64_t>(need, 1) * sizeof(int32_t)));
  *have = need;
  return GLP_OK;
}

static int ensure_work(glp_graph* g, int32_t total_iters) {
  if (!g->d_lab[0]) {
    GLP_CUDA(dev_alloc(&g->d_lab[0], sizeof(int32_t) * std::max(g->n, 1)));
    GLP_CUDA(dev_alloc(&g->d_lab[1], sizeof(int32_t) * std::max(g->n, 1)));
  }
  if (!g->d_err) {
    GLP_CUDA(dev_alloc(&g->d_err, sizeof(uint32_t)));
    GLP_CUDA(cudaMemsetAsync(g->d_err, 0, sizeof(uint32_t), g->stream));
    GLP_CUDA(cudaStreamSynchronize(g->stream));
  }
  if (g->changed_cap < total_iters + 1) {
    if (g->d_changed) dev_free(g->d_changed);
    g->d_changed = nullptr;
    GLP_CUDA(dev_alloc(&g->d_changed, sizeof(unsigned long long) * (total_iters + 1)));
    g->changed_cap = total_iters + 1;
  }
  return GLP_OK;
}

static int init_labels(RunCtx& c) {
  glp_graph* g = c.g;
  if (g->n == 0) return GLP_OK;
  k_iota<<<(unsigned)cdiv(g->n, 256), 256, 0, c.s>>>(g->d_lab[0], g->d_lab[1], g->n);
  ++c.launches;
  GLP_CUDA(cudaGetLastError());
  return GLP_OK;
}

// Decides (once per handle) whether every row is strictly ascending.
static int ensure_sorted(glp_graph* g) {
  if (g->rows_sorted >= 0) return GLP_OK;
  if (g->m == 0) {
    g->rows_sorted = 1;
    return GLP_OK;
  }
  uint32_t* d_bad = nullptr;
  GLP_CUDA(dev_alloc(&d_bad, sizeof(uint32_t)));
  GLP_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), g->stream));
  k_check_sorted<<<device_sms() * 32, 256, 0, g->stream>>>(g->d_off, g->d_cols, g->n, d_bad);
  uint32_t bad = 1;
  GLP_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  dev_free(d_bad);
  g->rows_sorted = bad == 0 ? 1 : 0;
  return GLP_OK;
}

// Exact first step when the labels are the vertex ids and rows are strictly
// ascending: unweighted, the row's last column (k_first_step); weighted, the
// row's largest (weight, label), per tier: a thread per vertex up to degree
// 32, a warp per mid vertex, a block per big vertex and hub.
// Per tier, the neighbour of largest key: a thread per vertex up to degree
// 32 (eight loads in flight), a warp per mid vertex, a block per big vertex
// and hub.
template <class K>
static int launch_first_keyed(const DevicePlan& p, const StepArgs& a, const K& key, cudaStream_t s,
                              int64_t* launches) {
  const unsigned kMaxGrid = device_sms() * 32;
  for (const Verts* vs : {&p.tiny, &p.g16, &p.g32})
    if (vs->n) {
      k_first_step_w<1, K><<<(unsigned)std::min<int64_t>(cdiv(vs->n, 256), kMaxGrid), 256, 0, s>>>(a, *vs, key);
      ++*launches;
    }
  if (p.mid.n) {
    k_first_step_w<32, K><<<(unsigned)std::min<int64_t>(cdiv((int64_t)p.mid.n * 32, 256), kMaxGrid), 256, 0, s>>>(
        a, p.mid, key);
    ++*launches;
  }
  if (p.big.n) {
    k_first_step_w_block<256, K><<<(unsigned)std::min<int64_t>(p.big.n, kMaxGrid), 256, 0, s>>>(a, p.big, key);
    ++*launches;
  }
  if (p.n_hubs) {
    k_first_step_w_block<1024, K><<<(unsigned)p.n_hubs, 1024, 0, s>>>(a, Verts{p.hub.hub_v, 0, p.n_hubs}, key);
    ++*launches;
  }
  GLP_CUDA(cudaGetLastError());
  return GLP_OK;
}

template <bool W>
static int launch_first_step(const DevicePlan& p, const StepArgs& a, cudaStream_t s, int64_t* launches) {
  if constexpr (!W) {
    const unsigned kMaxGrid = device_sms() * 32;
    k_first_step<<<(unsigned)std::min<int64_t>(cdiv(a.n, 256), kMaxGrid), 256, 0, s>>>(a);
    ++*launches;
    GLP_CUDA(cudaGetLastError());
    return GLP_OK;
  } else {
    return launch_first_keyed(p, a, FirstKeyW{}, s, launches);
  }
}

// The first step as its own timed step.
template <bool W>
static int first_step(RunCtx& c, const StepArgs& a) {
  StepLaunch L = c.launch();
  if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[16], c.s));
  int rc = launch_first_step<W>(c.g->plan, a, c.s, &c.launches);
  if (rc) return rc;
  if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[17], c.s));
  return GLP_OK;
}

// Decides (once per handle) whether the CSR stores every edge both ways.
static int ensure_symmetric(glp_graph* g) {
  if (g->symmetric >= 0) return GLP_OK;
  g->symmetric = 0;
  if (g->m == 0) {
    g->symmetric = 1;
    return GLP_OK;
  }
  uint32_t* d_bad = nullptr;
  GLP_CUDA(dev_alloc(&d_bad, sizeof(uint32_t)));
  GLP_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), g->stream));
  k_check_symmetric<<<device_sms() * 16, 256, 0, g->stream>>>(g->d_off, g->d_cols, g->n, g->m, d_bad);
  uint32_t bad = 1;
  GLP_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  dev_free(d_bad);
  g->symmetric = bad == 0 ? 1 : 0;
  return GLP_OK;
}

// glp_params.l2_window: the label array a step gathers from is kept in L2
// through a persisting access-policy window on the run's three streams (the
// persisting set-aside is a limit of this process's context; it is released
// when the run ends).  lab = nullptr clears the window.
static void set_l2_window(RunCtx& c, const int32_t* lab) {
  if (!c.l2_window) return;
  glp_graph* g = c.g;
  int max_win = 0, max_persist = 0;
  if (cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, g->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, g->device) != cudaSuccess ||
      max_win <= 0 || max_persist <= 0) {
    cudaGetLastError();
    return;
  }
  cudaStreamAttrValue v{};
  if (lab) {
    const size_t bytes = std::min<size_t>((size_t)g->n * sizeof(int32_t), (size_t)max_win);
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist);
    v.accessPolicyWindow.base_ptr = const_cast<int32_t*>(lab);
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = std::min(1.0f, (float)max_persist / (float)std::max<size_t>(bytes, 1));
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  } else {
    v.accessPolicyWindow.num_bytes = 0;
  }
  for (cudaStream_t st : {c.s, g->aux[0], g->aux[1]}) cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v);
  if (!lab) cudaCtxResetPersistingL2Cache();
  cudaGetLastError();
}

// Host-mapped verdict words and events of the two-step cycle detection.
static int ensure_cycle_state(glp_graph* g) {
  if (g->h_cycle) return GLP_OK;
  GLP_CUDA(cudaHostAlloc(&g->h_cycle, 4 * sizeof(uint32_t), cudaHostAllocMapped));
  GLP_CUDA(cudaHostGetDevicePointer(&g->d_cycle, g->h_cycle, 0));
  for (cudaEvent_t& e : g->cyc_ev) GLP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return GLP_OK;
}

template <bool W>
static int run_classic(RunCtx& c, int32_t niter) {
  glp_graph* g = c.g;
  int rc = init_labels(c);
  if (rc) return rc;
  // two-step cycle detection: symmetric graphs (their change lists are kept),
  // synchronous runs (the host reads the verdicts)
  const bool track = c.cycle && g->symmetric == 1 && niter > 2;
  if (track) {
    if ((rc = ensure_cycle_state(g))) return rc;
    for (int k = 0; k < 4; ++k) g->h_cycle[k] = 0u;
  }
  const uint32_t cyc_cap = (uint32_t)std::max<int64_t>(1024, g->n / 8);
  const unsigned cyc_grid = (unsigned)device_sms() * 4;
  // hub and big-tier count bounds belong to this run's labels (an earlier
  // run, SLPA's spoken labels among them, may have left its own); the big
  // tier's bounds serve unweighted exact-count runs
  if (g->plan.n_hubs) GLP_CUDA(cudaMemsetAsync(g->plan.hub.hub_lbl, 0xff, sizeof(int32_t) * g->plan.n_hubs, c.s));
  BigBound bb{};
  if (!W && c.backend == GLP_BACKEND_EXACT && g->plan.bb.n) {
    bb = g->plan.bb;
    GLP_CUDA(cudaMemsetAsync(bb.lbl, 0xff, sizeof(int32_t) * bb.n, c.s));
    GLP_CUDA(cudaMemsetAsync(bb.nchg, 0, sizeof(uint32_t) * bb.n, c.s));
  }
  for (int32_t it = 0; it < niter; ++it) {
    set_l2_window(c, g->d_lab[it & 1]);
    const bool fr = g->symmetric == 1;
    DevicePlan& p = g->plan;
    StepArgs a{g->d_off, g->d_cols, g->d_w, g->d_lab[it & 1], g->d_lab[it & 1], g->d_lab[(it + 1) & 1],
               g->d_changed + it, g->d_err, p.d_mode, g->n, fr ? p.chg[it & 1] : nullptr,
               fr ? p.counts + 7 + (it & 1) : nullptr};
    a.bb = bb;
    if (fr) GLP_CUDA(cudaMemsetAsync(p.counts + 7 + (it & 1), 0, sizeof(uint32_t), c.s));
    StepLaunch L = c.launch();
    L.prev_changed = it > 0 ? g->d_changed + it - 1 : nullptr;
    L.allow_majority = 1;
    L.allow_frontier = fr;
    L.hub_bound = true;
    if (fr && it > 0) {
      L.front = p.front;
      L.front.epoch = ++g->epoch;
      L.front.chg_in = p.chg[(it - 1) & 1];
      L.front.chg_in_n = p.counts + 7 + ((it - 1) & 1);
    }
    const uint32_t tag = ++g->cyc_tag;
    if (track && it >= 1) {
      // before the step overwrites them: L_{it-1} of the vertices step it-1 changed
      GLP_CUDA(cudaMemsetAsync(p.cyc_mism, 0, sizeof(uint32_t), c.s));
      k_cycle_save<<<cyc_grid, 256, 0, c.s>>>(p.chg[(it - 1) & 1], p.counts + 7 + ((it - 1) & 1), cyc_cap,
                                             g->d_lab[(it + 1) & 1], p.cyc_old, p.cyc_stamp, tag, p.cyc_mism);
      ++c.launches;
    }
    if (it == 0 && g->rows_sorted == 1) {
      if (c.timing) {  // first_step takes the step's events itself
        c.used--;
        c.ran.pop_back();
      }
      if ((rc = first_step<W>(c, a))) return rc;
    } else if ((rc = launch_step<W>(L, a, ScoreClassic{}, &c.launches))) {
      return rc;
    }
    if (track && it >= 1) {
      k_cycle_check<<<cyc_grid, 256, 0, c.s>>>(p.chg[it & 1], p.counts + 7 + (it & 1), p.counts + 7 + ((it - 1) & 1),
                                              cyc_cap, g->d_lab[(it + 1) & 1], p.cyc_old, p.cyc_stamp, tag,
                                              p.cyc_mism);
      k_cycle_verdict<<<1, 1, 0, c.s>>>(p.cyc_mism, g->d_cycle + (it & 3));
      c.launches += 2;
      GLP_CUDA(cudaGetLastError());
      GLP_CUDA(cudaEventRecord(g->cyc_ev[it % 3], c.s));
    }
    if ((rc = after_iter(c, it, g->d_lab[(it + 1) & 1]))) return rc;
    // the host stays at most two steps ahead: step it-1's verdict is read
    // while step it runs; once a step ended in the cycle, the steps already
    // enqueued are correct and the rest repeat the last two labelings
    if (track && it >= 2) {
      GLP_CUDA(cudaEventSynchronize(g->cyc_ev[(it - 1) % 3]));
      if (*(volatile uint32_t*)(g->h_cycle + ((it - 1) & 3))) {
        c.cycle_from = it + 1;
        break;
      }
    }
  }
  if (c.cycle_from > 0) {
    // L_t = L_{t-2} from here on, and L_t sits in buffer t & 1 already: the
    // final labels need no copy; per-iteration observers see both buffers in turn
    for (int32_t t = c.cycle_from; t < niter; ++t)
      if ((rc = after_iter(c, t, g->d_lab[(t + 1) & 1]))) return rc;
  }
  return GLP_OK;
}

template <bool W>
static int run_layered(RunCtx& c, const glp_params& p, int32_t niter) {
  glp_graph* g = c.g;
  int64_t have0 = 0, have1 = 0;
  int rc;
  if (!g->d_vol[0]) {
    if ((rc = grow(&g->d_vol[0], &have0, g->n)) || (rc = grow(&g->d_vol[1], &have1, g->n))) return rc;
  }
  int32_t* vol_r = g->d_vol[0];
  int32_t* vol_w = g->d_vol[1];
  GLP_CUDA(cudaMemsetAsync(vol_r, 0, sizeof(int32_t) * g->n, c.s));
  GLP_CUDA(cudaMemsetAsync(vol_w, 0, sizeof(int32_t) * g->n, c.s));
  // 32-bit layers gather (label, volume) pairs, rebuilt after every step
  bool any_narrow = false;
  for (int32_t layer = 0; layer < p.nlayers; ++layer)
    any_narrow = any_narrow || (int64_t)p.dstar[layer] * g->max_wsum + g->n < 2147483648LL;
  if (any_narrow && (g->lv_elems < g->n || !g->d_lv)) {
    dev_free(g->d_lv);
    g->d_lv = nullptr;
    GLP_CUDA(dev_alloc(&g->d_lv, sizeof(int2) * std::max(g->n, 1)));
    g->lv_elems = g->n;
  }
  const unsigned lv_grid = (unsigned)std::min<int64_t>(cdiv(std::max(g->n, 1), 256), device_sms() * 16);
  int32_t step = 0;
  int32_t* final_lab = g->d_lab[0];
  for (int32_t layer = 0; layer < p.nlayers; ++layer) {
    // 32-bit scores when every score of the layer fits them: a count is at
    // most a row's weight sum, a volume at most n
    const bool narrow = (int64_t)p.dstar[layer] * g->max_wsum + g->n < 2147483648LL;
    if ((rc = init_labels(c))) return rc;
    bool lv_fresh = false;  // d_lv holds (labels, vol_r) of this step's input
    for (int32_t it = 0; it < niter; ++it, ++step) {
      if (step > 0) {
        std::swap(vol_r, vol_w);
        GLP_CUDA(cudaMemsetAsync(vol_w, 0, sizeof(int32_t) * g->n, c.s));
      }
      const bool first = it == 0 && narrow && g->rows_sorted == 1;
      int32_t* lin = g->d_lab[it & 1];
      int32_t* lout = g->d_lab[(it + 1) & 1];
      set_l2_window(c, lin);
      // full counting every step; the step mode only chooses how the volume
      // term is looked up (from the previous step's changes within the layer)
      StepArgs a{g->d_off, g->d_cols, g->d_w, lin,     lin,   lout, g->d_changed + step, g->d_err,
                 g->plan.d_mode, g->n, nullptr, nullptr};
        StepLaunch L = c.launch();
      L.prev_changed = it > 0 ? g->d_changed + step - 1 : nullptr;
      L.allow_majority = 0;
      L.allow_frontier = 0;
      if (first) {
        // labels = ids and no repeated neighbour: every label occurs once, so
        // the step is a streaming maximum of dstar*w - vol_r[neighbour]
        if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[16], c.s));
        rc = launch_first_keyed(g->plan, a, FirstKeyLayered<W>{vol_r, p.dstar[layer]}, c.s, &c.launches);
        if (!rc && L.ev) GLP_CUDA(cudaEventRecord(L.ev[17], c.s));
      } else if (narrow) {
        if (!lv_fresh) {  // the layer's first step counted: pairs of the reset labels
          k_label_volumes<<<lv_grid, 256, 0, c.s>>>(lin, vol_r, g->n, g->d_lv);
          ++c.launches;
        }
        rc = launch_step<W>(L, a, ScoreLayered32{vol_r, p.dstar[layer], g->d_lv}, &c.launches);
      } else {
        rc = launch_step<W>(L, a, ScoreLayered{vol_r, (int64_t)p.dstar[layer]}, &c.launches);
      }
      if (rc) return rc;
      if ((rc = c.aux_mark(0))) return rc;
      k_histogram<<<(unsigned)cdiv(g->n, 256), 256, 0, c.s>>>(lout, g->n, vol_w);
      ++c.launches;
      // the next step of this layer reads (lout, vol_w) pairs
      lv_fresh = narrow && it + 1 < niter && g->n > 0;
      if (lv_fresh) {
        k_label_volumes<<<lv_grid, 256, 0, c.s>>>(lout, vol_w, g->n, g->d_lv);
        ++c.launches;
      }
      if ((rc = c.aux_mark(1))) return rc;
      GLP_CUDA(cudaGetLastError());
      if ((rc = after_iter(c, step, lout))) return rc;
      final_lab = lout;
    }
  }
  // the final labels must sit in d_lab[0] or d_lab[1]; report which
  c.iter_base = final_lab == g->d_lab[0] ? 0 : 1;
  g->d_vol[0] = vol_r;
  g->d_vol[1] = vol_w;  // vol_w = volumes after the last iteration
  return GLP_OK;
}

template <bool W>
static int run_slpa(RunCtx& c, const glp_params& p, int32_t niter, glp_outputs* out) {
  glp_graph* g = c.g;
  const int32_t T = p.slpa_T;
  int rc;
  if ((rc = grow(&g->d_mem, &g->mem_elems, (int64_t)T * g->n))) return rc;
  if (!g->d_spoken) GLP_CUDA(dev_alloc(&g->d_spoken, sizeof(int32_t) * std::max(g->n, 1)));
  GLP_CUDA(cudaMemsetAsync(g->d_mem, 0xff, sizeof(int32_t) * (size_t)T * g->n, c.s));
  if ((rc = init_labels(c))) return rc;
  set_l2_window(c, g->d_spoken);
  for (int32_t it = 0; it < niter; ++it) {
    int32_t* lcur = g->d_lab[it & 1];
    int32_t* lout = g->d_lab[(it + 1) & 1];
    StepLaunch L = c.launch();
    if ((rc = c.aux_mark(0))) return rc;
    k_slpa_speak<<<(unsigned)cdiv(g->n, 256), 256, 0, c.s>>>(lcur, g->d_mem, g->d_spoken, g->n, T, it, p.seed);
    ++c.launches;
    if ((rc = c.aux_mark(1))) return rc;
    GLP_CUDA(cudaGetLastError());
    StepArgs a{g->d_off, g->d_cols, g->d_w, g->d_spoken, lcur, lout, g->d_changed + it, g->d_err,
               g->plan.d_mode, g->n, nullptr, nullptr};
    L.prev_changed = it > 0 ? g->d_changed + it - 1 : nullptr;
    L.allow_majority = 1;  // the listener mode; spoken labels change every step: no frontier
    if (it == 0 && g->rows_sorted == 1) {
      // the step's events were taken by c.launch() above; the first step records them
      if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[16], c.s));
      if ((rc = launch_first_step<W>(g->plan, a, c.s, &c.launches))) return rc;
      if (L.ev) GLP_CUDA(cudaEventRecord(L.ev[17], c.s));
    } else if ((rc = launch_step<W>(L, a, ScoreClassic{}, &c.launches))) {
      return rc;
    }
    if ((rc = after_iter(c, it, lout))) return rc;
  }
  if (out->slpa_comm && g->n) {
    const bool dev = out->on_device != 0;
    int32_t* comm = out->slpa_comm;
    int32_t* ncomm = out->slpa_ncomm;
    int32_t *tmp_c = nullptr, *tmp_n = nullptr;
    if (!dev) {
      GLP_CUDA(dev_alloc(&tmp_c, sizeof(int32_t) * (size_t)T * g->n));
      GLP_CUDA(dev_alloc(&tmp_n, sizeof(int32_t) * g->n));
      comm = tmp_c;
      ncomm = tmp_n;
    }
    k_slpa_post<64><<<(unsigned)cdiv(g->n, 128), 128, 0, c.s>>>(g->d_mem, g->n, T, p.slpa_r, comm, ncomm);
    ++c.launches;
    GLP_CUDA(cudaGetLastError());
    if (!dev) {
      GLP_CUDA(cudaMemcpyAsync(out->slpa_comm, tmp_c, sizeof(int32_t) * (size_t)T * g->n, cudaMemcpyDeviceToHost, c.s));
      if (out->slpa_ncomm)
        GLP_CUDA(cudaMemcpyAsync(out->slpa_ncomm, tmp_n, sizeof(int32_t) * g->n, cudaMemcpyDeviceToHost, c.s));
      GLP_CUDA(cudaStreamSynchronize(c.s));
      dev_free(tmp_c);
      dev_free(tmp_n);
    }
  }
  if (out->slpa_mem && g->n)
    GLP_CUDA(cudaMemcpyAsync(out->slpa_mem, g->d_mem, sizeof(int32_t) * (size_t)T * g->n,
                             out->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.s));
  return GLP_OK;
}

// ------------------------------------------------------------ validation
// Offsets: off[0] = 0, off[n] = m, monotone (bad 16 / 8); also the largest
// degree and whether degrees never increase along the ids (sorted = 0 when
// some degree is larger than its predecessor's).
__global__ void k_validate_offsets(const int32_t* __restrict__ off, int32_t n, int64_t m, uint32_t* bad,
                                   int32_t* maxdeg, uint32_t* unsorted) {
  for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
    if (v == 0 && off[0] != 0) atomicOr(bad, 16u);
    if (v == n) {
      if ((int64_t)off[n] != m) atomicOr(bad, 16u);
      continue;
    }
    const int32_t d = off[v + 1] - off[v];
    if (d < 0) atomicOr(bad, 8u);
    atomicMax(maxdeg, d);
    if (v + 1 < n && off[v + 2] - off[v + 1] > d) atomicOr(unsorted, 1u);
  }
}

// Columns in [0, n) (bad 1), weights >= 0 (bad 2), per-vertex weight sums
// below 2^31 (bad 4).  Runs only on valid offsets.
// mid_wsum: the largest weight sum of a vertex of degree <= kMidCap / 2 (a
// bound on any of its label counts); max_wsum: the largest of any vertex.
__global__ void k_validate(const int32_t* __restrict__ off, const int32_t* __restrict__ cols,
                           const int32_t* __restrict__ w, int64_t m, int32_t n, uint32_t* bad, uint32_t* mid_wsum,
                           uint32_t* max_wsum) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cols[j];
    if (c < 0 || c >= n) atomicOr(bad, 1u);
    if (w && w[j] < 0) atomicOr(bad, 2u);
  }
  // the engine sums a vertex's weights in 32 bits
  if (w) {
    uint32_t mid_max = 0, all_max = 0;
    const int32_t nv = (n + 31) & ~31;  // whole warps for the reduction
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
      if (v < n) {
        int64_t sum = 0;
        for (int32_t j = off[v]; j < off[v + 1]; ++j) sum += w[j];
        if (sum >= 2147483648LL) atomicOr(bad, 4u);
        const uint32_t s32 = sum < 0xffffffffLL ? (uint32_t)sum : 0xffffffffu;
        if (off[v + 1] - off[v] <= kMidCap / 2 && sum > 0) mid_max = max(mid_max, s32);
        all_max = max(all_max, s32);
      }
    }
    mid_max = __reduce_max_sync(kFull, mid_max);
    all_max = __reduce_max_sync(kFull, all_max);
    if ((threadIdx.x & 31) == 0 && mid_max) atomicMax(mid_wsum, mid_max);
    if ((threadIdx.x & 31) == 0 && all_max) atomicMax(max_wsum, all_max);
  }
}

int validate_csr_device(glp_graph* g) {
  struct Flags {
    uint32_t bad;
    int32_t maxdeg;
    uint32_t unsorted;
    uint32_t mid_wsum;
    uint32_t max_wsum;
  };
  Flags* d_f = nullptr;
  GLP_CUDA(dev_alloc(&d_f, sizeof(Flags)));
  GLP_CUDA(cudaMemset(d_f, 0, sizeof(Flags)));
  k_validate_offsets<<<1184, 256>>>(g->d_off, g->n, g->m, &d_f->bad, &d_f->maxdeg, &d_f->unsorted);
  Flags f{};
  cudaError_t e = cudaMemcpy(&f, d_f, sizeof f, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && !f.bad && g->m) {
    k_validate<<<1184, 256>>>(g->d_off, g->d_cols, g->d_w, g->m, g->n, &d_f->bad, &d_f->mid_wsum, &d_f->max_wsum);
    e = cudaMemcpy(&f, d_f, sizeof f, cudaMemcpyDeviceToHost);
  }
  dev_free(d_f);
  if (e != cudaSuccess) return cuda_fail(e, "validate");
  if (f.bad & 16u) {
    set_error("offsets[0] must be 0 and offsets[n] must be m");
    return GLP_EINVAL;
  }
  if (f.bad & 8u) {
    set_error("offsets not monotone");
    return GLP_EINVAL;
  }
  if (f.bad & 1u) {
    set_error("column index outside [0, n)");
    return GLP_EINVAL;
  }
  if (f.bad & 2u) {
    set_error("negative edge weight");
    return GLP_EINVAL;
  }
  if (f.bad & 4u) {
    set_error("a vertex's weight sum reaches 2^31");
    return GLP_EINVAL;
  }
  g->max_degree = f.maxdeg;
  g->deg_sorted = f.unsorted ? 0 : 1;
  g->mid_wsum = f.mid_wsum;
  g->max_wsum = g->d_w ? f.max_wsum : (uint32_t)f.maxdeg;
  return GLP_OK;
}

// First vertex whose degree is <= t, for each threshold (degrees must not
// increase along the ids).
__global__ void k_tier_bounds(const int32_t* __restrict__ off, int32_t n, const int32_t* thr, int32_t k,
                              int32_t* out) {
  const int i = threadIdx.x;
  if (i >= k) return;
  const int32_t t = thr[i];
  int32_t lo = 0, hi = n;
  while (lo < hi) {
    const int32_t mid = (int32_t)(((int64_t)lo + hi) >> 1);
    if (off[mid + 1] - off[mid] <= t) hi = mid; else lo = mid + 1;
  }
  out[i] = lo;
}

// Host copy of the offsets, made on first need (unsorted graphs, reports).
static int ensure_host_offsets(glp_graph* g) {
  if (!g->h_off.empty()) return GLP_OK;
  g->h_off.resize((size_t)g->n + 1);
  GLP_CUDA(cudaMemcpy(g->h_off.data(), g->d_off, sizeof(int32_t) * ((size_t)g->n + 1), cudaMemcpyDeviceToHost));
  return GLP_OK;
}

static int device_bounds(glp_graph* g, const int32_t* thr, int k, int32_t* out) {
  int32_t* d = nullptr;
  GLP_CUDA(dev_alloc(&d, sizeof(int32_t) * 2 * k));
  cudaError_t e = cudaMemcpy(d, thr, sizeof(int32_t) * k, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_tier_bounds<<<1, 32>>>(g->d_off, g->n, d, k, d + k);
    e = cudaMemcpy(out, d + k, sizeof(int32_t) * k, cudaMemcpyDeviceToHost);
  }
  dev_free(d);
  if (e != cudaSuccess) return cuda_fail(e, "tier bounds");
  return GLP_OK;
}

// --------------------------------------------------------------- method 4
template <class H>
static int hooks_iterations(RunCtx& c, H h, int32_t niter, int32_t step0, bool layered, int32_t** vol_r,
                            int32_t** vol_w) {
  glp_graph* g = c.g;
  int rc;
  for (int32_t it = 0; it < niter; ++it) {
    const int32_t step = step0 + it;
    if (layered) {
      if (step > 0) {
        std::swap(*vol_r, *vol_w);
        GLP_CUDA(cudaMemsetAsync(*vol_w, 0, sizeof(int32_t) * g->n, c.s));
      }
      h.st.vol_r = *vol_r;
      h.st.vol_w = *vol_w;
    }
    glp_hooks::k_pick<H><<<(unsigned)cdiv(g->n, 256), 256, 0, c.s>>>(h, g->n);
    glp_hooks::k_prop<H><<<(unsigned)std::min<int64_t>(cdiv(g->n, 4), (int64_t)device_sms() * 64), 128, 0, c.s>>>(
        h, h.st, g->d_hook_keys, g->d_hook_vals, g->d_changed + step, g->d_err);
    c.launches += 2;
    GLP_CUDA(cudaGetLastError());
    if ((rc = after_iter(c, step, h.st.Lnext))) return rc;
  }
  return GLP_OK;
}

static int run_hooks(RunCtx& c, const glp_params& p, int32_t niter) {
  glp_graph* g = c.g;
  if (g->max_degree > kHookSmemCap / 2 && !g->d_hook_keys) {
    GLP_CUDA(dev_alloc(&g->d_hook_keys, sizeof(uint32_t) * 2 * (size_t)g->m));
    GLP_CUDA(dev_alloc(&g->d_hook_vals, sizeof(double) * 2 * (size_t)g->m));
  }
  HookState st{g->d_off, g->d_cols, g->d_w, g->n, g->d_lab[0], g->d_lab[1], nullptr, nullptr, 1.0, nullptr};
  c.iter_base = 1;  // Lnext holds the final labels
  int rc;
  if (p.hooks == GLP_HOOKS_LAYERED) {
    int64_t have0 = 0, have1 = 0;
    if (!g->d_vol[0]) {
      if ((rc = grow(&g->d_vol[0], &have0, g->n)) || (rc = grow(&g->d_vol[1], &have1, g->n))) return rc;
    }
    int32_t* vol_r = g->d_vol[0];
    int32_t* vol_w = g->d_vol[1];
    GLP_CUDA(cudaMemsetAsync(vol_r, 0, sizeof(int32_t) * g->n, c.s));
    GLP_CUDA(cudaMemsetAsync(vol_w, 0, sizeof(int32_t) * g->n, c.s));
    for (int32_t layer = 0; layer < p.nlayers; ++layer) {
      if ((rc = init_labels(c))) return rc;
      st.dstar = (double)p.dstar[layer];
      if ((rc = hooks_iterations(c, HooksLayered{st}, niter, layer * niter, true, &vol_r, &vol_w))) return rc;
    }
    g->d_vol[0] = vol_r;
    g->d_vol[1] = vol_w;
    return GLP_OK;
  }
  if ((rc = init_labels(c))) return rc;
  int32_t* vr = nullptr;
  int32_t* vw = nullptr;
  if (p.hooks == GLP_HOOKS_CLASSIC) return hooks_iterations(c, HooksClassic{st}, niter, 0, false, &vr, &vw);
  return hooks_iterations(c, HooksWeightedDegree{st}, niter, 0, false, &vr, &vw);
}


// --------------------------------------------------------------- method 5
// Seeded LP (prop/seedLprop.cuh): seeds fixed at their ids, every other
// vertex starts unlabelled and takes the mode of its labelled neighbours.
template <bool W>
static int run_seeded(RunCtx& c, int32_t niter) {
  glp_graph* g = c.g;
  if (!g->d_seeds) {
    set_error("method 5 needs seeds: call glp_graph_set_seeds first");
    return GLP_EINVAL;
  }
  if (g->max_degree > kSeedSmem / 2 && !g->d_seed_keys) {
    GLP_CUDA(dev_alloc(&g->d_seed_keys, sizeof(uint32_t) * 2 * (size_t)g->m));
    GLP_CUDA(dev_alloc(&g->d_seed_vals, sizeof(uint32_t) * 2 * (size_t)g->m));
  }
  k_seeded_init<<<(unsigned)cdiv(g->n, 256), 256, 0, c.s>>>(g->d_seeds, g->d_lab[0], g->d_lab[1], g->n);
  ++c.launches;
  const unsigned grid = (unsigned)std::min<int64_t>(cdiv(g->n, 8), (int64_t)device_sms() * 16);
  int rc;
  for (int32_t it = 0; it < niter; ++it) {
    k_seeded_step<W><<<grid, 256, 0, c.s>>>(g->d_off, g->d_cols, g->d_w, g->d_seeds, g->d_lab[it & 1],
                                            g->d_lab[(it + 1) & 1], g->n, g->d_seed_keys, g->d_seed_vals,
                                            g->d_changed + it, g->d_err);
    ++c.launches;
    GLP_CUDA(cudaGetLastError());
    if ((rc = after_iter(c, it, g->d_lab[(it + 1) & 1]))) return rc;
  }
  return GLP_OK;
}

// ------------------------------------------------- allocation-free classic LP
// Scratch of glp_run_classic_noalloc: one copy per device (module globals are
// per context), found with cudaGetSymbolAddress.
constexpr int32_t kNoAllocMaxVertices = 1 << 20;
constexpr int32_t kNoAllocMaxIters = 4096;
constexpr int32_t kNoAllocMaxDegree = 4096;
constexpr int kNoAllocNT = 128;
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
  int32_t labels[kNoAllocMaxVertices];           // the second label buffer
  unsigned long long changed[kNoAllocMaxIters];  // per-iteration change counts
  uint32_t err;                                  // kErr* bits of the steps
  uint32_t bad;                                  // validation bits
  int32_t maxdeg;
  uint32_t unsorted;
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];
static std::atomic<int> g_noalloc_attr[kNoAllocMaxDevices];  // 1: shared-memory limit raised

static inline size_t pow2_host(int32_t x) {
  size_t p = 1;
  while (p < (size_t)x) p <<= 1;
  return p;
}

// One classic step over every vertex, a block per vertex: the k_big counting
// (shared table of pow2(2*degree) slots, running maxima) extended to degree 0,
// where the vertex keeps its label.
template <int NT>
__global__ void __launch_bounds__(NT) k_noalloc_step(const int32_t* __restrict__ off,
                                                      const int32_t* __restrict__ cols,
                                                      const int32_t* __restrict__ lin, int32_t* __restrict__ lout,
                                                      int32_t n, unsigned long long* changed, uint32_t* err) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ Best red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const ScoreClassic score;
  for (int32_t v = blockIdx.x; v < n; v += gridDim.x) {
    const int32_t b = off[v], e = off[v + 1];
    if (b == e) {  // block-uniform
      if (threadIdx.x == 0) lout[v] = lin[v];
      continue;
    }
    const uint32_t cap = pow2_ceil(2u * (uint32_t)(e - b));
    uint32_t* keys = smem;
    uint32_t* vals = smem + cap;
    for (uint32_t s = threadIdx.x; s < 2 * cap; s += NT) smem[s] = 0;
    __syncthreads();
    Best best = best_none();
    bool fail = false;
    auto ins = [&](uint32_t key, uint32_t k) {
      return table_insert_bounded(keys, vals, cap - 1, key, k, cap, nullptr, nullptr);
    };
    for (int32_t j0 = b + warp * 32; j0 < e; j0 += 4 * NT) {
      int32_t lab[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + q * NT + lane;
        lab[q] = j < e ? ld_stream(cols + j) : -1;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (lab[q] >= 0) lab[q] = ld_label(lin + lab[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + q * NT < e) count_chunk<false>(lab[q] >= 0, lab[q], 1u, score, ins, best, fail);
    }
    if (fail) atomicOr(err, kErrProbe);
    best = block_max<NT>(best, red);
    if (threadIdx.x == 0) {
      lout[v] = best.l;
      if (best.l != lin[v]) atomicAdd(changed, 1ull);
    }
  }
}

}  // namespace glp

using namespace glp;

// ================================================================ C ABI
extern "C" {

const char* glp_last_error(void) { return g_err.c_str(); }
const char* glp_version(void) { return "glp_b200 0.1 (sm_100a)"; }

int glp_params_default(glp_params* p) {
  if (!p) {
    set_error("params is NULL");
    return GLP_EINVAL;
  }
  std::memset(p, 0, sizeof *p);
  p->struct_size = (int32_t)sizeof(glp_params);
  p->backend = GLP_BACKEND_EXACT;
  // gamma in {1, 1/2, 1/4, 1/8, 1/16} -> dstar = 1/gamma + 1
  p->nlayers = 5;
  const int32_t ds[5] = {2, 3, 5, 9, 17};
  for (int i = 0; i < 5; ++i) p->dstar[i] = ds[i];
  p->slpa_T = 20;
  p->slpa_r = 0.1;
  p->seed = 4;
  p->hooks = GLP_HOOKS_CLASSIC;
  p->use_graph = 0;
  p->async = 0;
  return GLP_OK;
}

int glp_graph_create(const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n, int64_t m,
                     int32_t on_device, glp_graph** out) {
  return glp_graph_create_ex(offsets, cols, weights, n, m, on_device, 0u, out);
}

int glp_graph_create_ex(const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n, int64_t m,
                        int32_t on_device, uint32_t flags, glp_graph** out) {
  if (!out) {
    set_error("out is NULL");
    return GLP_EINVAL;
  }
  *out = nullptr;
  if (n < 0 || m < 0 || m > INT32_MAX || !offsets || (m > 0 && !cols)) {
    set_error("bad graph arguments (n=%d, m=%lld)", n, (long long)m);
    return GLP_EINVAL;
  }
  int rc = require_device();
  if (rc) return rc;
  std::unique_ptr<glp_graph> g(new glp_graph());
  g->n = n;
  g->m = m;
  GLP_CUDA(cudaGetDevice(&g->device));
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  GLP_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  GLP_CUDA(cudaStreamCreateWithFlags(&g->aux[0], cudaStreamNonBlocking));
  GLP_CUDA(cudaStreamCreateWithFlags(&g->aux[1], cudaStreamNonBlocking));
  GLP_CUDA(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
  GLP_CUDA(cudaEventCreateWithFlags(&g->join[0], cudaEventDisableTiming));
  GLP_CUDA(cudaEventCreateWithFlags(&g->join[1], cudaEventDisableTiming));
  GLP_CUDA(dev_alloc(&g->d_off, sizeof(int32_t) * ((size_t)n + 1)));
  GLP_CUDA(cudaMemcpy(g->d_off, offsets, sizeof(int32_t) * ((size_t)n + 1), kind));
  // 4 padding entries: tile kernels read columns as aligned 16-byte quads
  GLP_CUDA(dev_alloc(&g->d_cols, sizeof(int32_t) * (m + 4)));
  GLP_CUDA(cudaMemset(g->d_cols + m, 0, sizeof(int32_t) * 4));
  if (m) GLP_CUDA(cudaMemcpy(g->d_cols, cols, sizeof(int32_t) * m, kind));
  if (weights) {
    GLP_CUDA(dev_alloc(&g->d_w, sizeof(int32_t) * (m + 4)));
    GLP_CUDA(cudaMemset(g->d_w + m, 0, sizeof(int32_t) * 4));
    if (m) GLP_CUDA(cudaMemcpy(g->d_w, weights, sizeof(int32_t) * m, kind));
  }
  // validate columns (and weights) on the device
  if ((rc = validate_csr_device(g.get()))) return rc;
  if (flags & GLP_GRAPH_SYMMETRIC) g->symmetric = 1;
  *out = g.release();
  return GLP_OK;
}

void glp_graph_destroy(glp_graph* g) {
  if (!g) return;
  quiesce(g);  // no kernel of this handle may still use what is freed
  free_plan(&g->plan);
  dev_free(g->d_off);
  dev_free(g->d_cols);
  dev_free(g->d_w);
  dev_free(g->d_lab[0]);
  dev_free(g->d_lab[1]);
  dev_free(g->d_vol[0]);
  dev_free(g->d_vol[1]);
  dev_free(g->d_lv);
  dev_free(g->d_spoken);
  dev_free(g->d_mem);
  dev_free(g->d_changed);
  dev_free(g->d_err);
  dev_free(g->d_hook_keys);
  dev_free(g->d_hook_vals);
  dev_free(g->d_seeds);
  dev_free(g->d_seed_keys);
  dev_free(g->d_seed_vals);
  if (g->h_cycle) cudaFreeHost(g->h_cycle);
  for (cudaEvent_t e : g->cyc_ev)
    if (e) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  for (cudaStream_t st : g->aux)
    if (st) cudaStreamDestroy(st);
  if (g->fork) cudaEventDestroy(g->fork);
  for (cudaEvent_t e : g->join)
    if (e) cudaEventDestroy(e);
  delete g;
}

int glp_graph_export(const glp_graph* g, int32_t* offsets, int32_t* cols, int32_t* weights, int32_t on_device) {
  if (!g || !offsets || (g->m > 0 && !cols)) {
    set_error("graph, offsets and cols are required");
    return GLP_EINVAL;
  }
  GLP_CUDA(cudaSetDevice(g->device));
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  GLP_CUDA(cudaMemcpyAsync(offsets, g->d_off, sizeof(int32_t) * ((size_t)g->n + 1), k, g->stream));
  if (g->m) GLP_CUDA(cudaMemcpyAsync(cols, g->d_cols, sizeof(int32_t) * (size_t)g->m, k, g->stream));
  if (g->m && weights && g->d_w)
    GLP_CUDA(cudaMemcpyAsync(weights, g->d_w, sizeof(int32_t) * (size_t)g->m, k, g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  return GLP_OK;
}

int glp_graph_info(const glp_graph* g, int32_t* n, int64_t* m, int32_t* max_degree) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (max_degree) *max_degree = g->max_degree;
  return GLP_OK;
}

static int plan_counts(const int32_t* offsets, int32_t n, const TierParams& t, int64_t out[16]);

int glp_plan_offsets(const int32_t* offsets, int32_t n, const glp_params* p, int64_t out[16]) {
  if (!offsets || !out || n < 0) {
    set_error("NULL argument or n < 0");
    return GLP_EINVAL;
  }
  for (int32_t v = 0; v < n; ++v)
    if (offsets[v + 1] < offsets[v]) {
      set_error("offsets not monotone at vertex %d", v);
      return GLP_EINVAL;
    }
  TierParams t;
  int rc = tiers_for_graph(p, false, &t);
  if (rc) return rc;
  return plan_counts(offsets, n, t, out);
}

static int plan_counts(const int32_t* offsets, int32_t n, const TierParams& t, int64_t out[16]) {
  HostPlan hp;
  build_host_plan(offsets, n, t, &hp);
  out[0] = hp.isolated;
  out[1] = (int64_t)hp.tiny.size();
  out[2] = (int64_t)hp.g16.size();
  out[3] = (int64_t)hp.g32.size();
  out[4] = (int64_t)hp.mid.size();
  out[5] = (int64_t)hp.big.size();
  out[6] = (int64_t)hp.hub_v.size();
  out[7] = (int64_t)hp.item_hub.size();
  for (int i = 0; i < 7; ++i) out[8 + i] = hp.edges[i];
  out[15] = (int64_t)hp.chunk_hub.size();
  return GLP_OK;
}

int glp_graph_plan(glp_graph* g, const glp_params* p, int64_t out[16]) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  if (!out) {
    set_error("out is NULL");
    return GLP_EINVAL;
  }
  TierParams t;
  int rc = tiers_for_graph(p, g->d_w != nullptr, &t);
  if (rc || (rc = ensure_host_offsets(g))) return rc;
  return plan_counts(g->h_off.data(), g->n, t, out);
}

int glp_graph_check(glp_graph* g) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  if (!g->d_err) return GLP_OK;
  return check_err(g, g->stream);
}

int glp_graph_set_seeds(glp_graph* g, const uint8_t* seeds, int32_t on_device) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  GLP_CUDA(cudaSetDevice(g->device));
  int rc;
  if ((rc = quiesce(g))) return rc;
  if (!seeds) {
    if (g->d_seeds) dev_free(g->d_seeds);
    g->d_seeds = nullptr;
    return GLP_OK;
  }
  if (!g->d_seeds) GLP_CUDA(dev_alloc(&g->d_seeds, std::max<size_t>((size_t)g->n, 1)));
  if (g->n) {
    GLP_CUDA(cudaMemcpyAsync(g->d_seeds, seeds, (size_t)g->n,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, g->stream));
    GLP_CUDA(cudaStreamSynchronize(g->stream));
  }
  return GLP_OK;
}

int glp_graph_set_cancel_flag(glp_graph* g, const volatile int32_t* flag) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  g->cancel = flag;
  return GLP_OK;
}

int glp_graph_device_view(glp_graph* g, int32_t niter, glp_device_view* out) {
  if (!g || !out || niter < 0) {
    set_error("graph, output and niter >= 0 are required");
    return GLP_EINVAL;
  }
  GLP_CUDA(cudaSetDevice(g->device));
  int rc;
  if ((rc = quiesce(g))) return rc;
  if ((rc = ensure_work(g, niter))) return rc;
  if (g->max_degree > kHookSmemCap / 2 && !g->d_hook_keys) {
    GLP_CUDA(dev_alloc(&g->d_hook_keys, sizeof(uint32_t) * 2 * (size_t)g->m));
    GLP_CUDA(dev_alloc(&g->d_hook_vals, sizeof(double) * 2 * (size_t)g->m));
  }
  if (g->n) {
    k_iota<<<(unsigned)cdiv(g->n, 256), 256, 0, g->stream>>>(g->d_lab[0], g->d_lab[1], g->n);
    GLP_CUDA(cudaGetLastError());
  }
  GLP_CUDA(cudaMemsetAsync(g->d_changed, 0, sizeof(unsigned long long) * (niter + 1), g->stream));
  GLP_CUDA(cudaMemsetAsync(g->d_err, 0, sizeof(uint32_t), g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  glp_device_view v{};
  v.n = g->n;
  v.max_degree = g->max_degree;
  v.m = g->m;
  v.device = g->device;
  v.sms = device_sms();
  v.off = g->d_off;
  v.cols = g->d_cols;
  v.w = g->d_w;
  v.labels[0] = g->d_lab[0];
  v.labels[1] = g->d_lab[1];
  v.changed = g->d_changed;
  v.err = g->d_err;
  v.hook_keys = g->d_hook_keys;
  v.hook_vals = g->d_hook_vals;
  v.stream = g->stream;
  *out = v;
  return GLP_OK;
}

// Device buffers of one summary inspection call, freed on every return path.
struct InspectBufs {
  std::vector<void*> held;
  ~InspectBufs() {
    for (void* p : held) dev_free(p);
  }
  int alloc(void** p, size_t bytes) {
    GLP_CUDA(dev_alloc_raw(p, bytes));
    held.push_back(*p);
    return GLP_OK;
  }
};

// Shared argument checks and uploads of glp_graph_cm_sketch / _fa_summary:
// the labels (unless already on the device) and the vertex list.
static int inspect_inputs(glp_graph* g, const int32_t* labels, int32_t on_device, const int32_t* vertices,
                          int32_t nv, InspectBufs& bufs, const int32_t** d_lab, int32_t** d_verts) {
  for (int32_t i = 0; i < nv; ++i)
    if (vertices[i] < 0 || vertices[i] >= g->n) {
      set_error("vertices[%d] = %d outside [0, %d)", i, vertices[i], g->n);
      return GLP_EINVAL;
    }
  int rc = require_device();
  if (rc) return rc;
  GLP_CUDA(cudaSetDevice(g->device));
  if ((rc = quiesce(g))) return rc;
  if (on_device) {
    *d_lab = labels;
  } else {
    int32_t* d = nullptr;
    if ((rc = bufs.alloc((void**)&d, sizeof(int32_t) * (size_t)g->n))) return rc;
    GLP_CUDA(cudaMemcpyAsync(d, labels, sizeof(int32_t) * (size_t)g->n, cudaMemcpyHostToDevice, g->stream));
    *d_lab = d;
  }
  if ((rc = bufs.alloc((void**)d_verts, sizeof(int32_t) * (size_t)nv))) return rc;
  GLP_CUDA(cudaMemcpyAsync(*d_verts, vertices, sizeof(int32_t) * (size_t)nv, cudaMemcpyHostToDevice, g->stream));
  return GLP_OK;
}

int glp_graph_cm_sketch(glp_graph* g, const int32_t* labels, int32_t labels_on_device, const int32_t* vertices,
                        int32_t nv, int32_t width, int32_t ref_compat, uint32_t* rows) {
  if (!g || !labels || nv < 0 || (nv > 0 && (!vertices || !rows))) {
    set_error("graph, labels, vertices and rows are required (nv=%d)", nv);
    return GLP_EINVAL;
  }
  if (width < 1 || width > 4096) {
    set_error("width %d outside [1, 4096]", width);
    return GLP_EINVAL;
  }
  if (nv == 0 || g->n == 0) return GLP_OK;
  InspectBufs bufs;
  const int32_t* d_lab = nullptr;
  int32_t* d_verts = nullptr;
  uint32_t* d_rows = nullptr;
  const size_t cells = 3ull * (size_t)width * (size_t)nv;
  int rc = inspect_inputs(g, labels, labels_on_device, vertices, nv, bufs, &d_lab, &d_verts);
  if (rc || (rc = bufs.alloc((void**)&d_rows, sizeof(uint32_t) * cells))) return rc;
  k_cm_sketch<<<(unsigned)std::min<int32_t>(nv, device_sms() * 8), 256, 3u * (unsigned)width * sizeof(uint32_t), g->stream>>>(
      g->d_off, g->d_cols, g->d_w, d_lab, d_verts, nv, width, ref_compat ? 1 : 0, d_rows);
  GLP_CUDA(cudaGetLastError());
  GLP_CUDA(cudaMemcpyAsync(rows, d_rows, sizeof(uint32_t) * cells, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  return GLP_OK;
}

int glp_graph_fa_summary(glp_graph* g, const int32_t* labels, int32_t labels_on_device, const int32_t* vertices,
                         int32_t nv, int32_t capacity, int32_t ref_compat, uint32_t* keys, uint32_t* vals,
                         int32_t* rounds) {
  if (!g || !labels || nv < 0 || (nv > 0 && (!vertices || !keys || !vals || !rounds))) {
    set_error("graph, labels, vertices, keys, vals and rounds are required (nv=%d)", nv);
    return GLP_EINVAL;
  }
  if (capacity < 1 || capacity > 65536) {
    set_error("capacity %d outside [1, 65536]", capacity);
    return GLP_EINVAL;
  }
  if (nv == 0 || g->n == 0) return GLP_OK;
  InspectBufs bufs;
  const int32_t* d_lab = nullptr;
  int32_t* d_verts = nullptr;
  uint32_t *d_keys = nullptr, *d_vals = nullptr;
  int32_t* d_rounds = nullptr;
  const size_t slots = (size_t)capacity * (size_t)nv;
  int rc = inspect_inputs(g, labels, labels_on_device, vertices, nv, bufs, &d_lab, &d_verts);
  if (rc || (rc = bufs.alloc((void**)&d_keys, sizeof(uint32_t) * slots)) ||
      (rc = bufs.alloc((void**)&d_vals, sizeof(uint32_t) * slots)) ||
      (rc = bufs.alloc((void**)&d_rounds, sizeof(int32_t) * (size_t)nv)))
    return rc;
  k_fa_summary<<<(unsigned)cdiv(nv, 128), 128, 0, g->stream>>>(g->d_off, g->d_cols, d_lab, d_verts, nv, capacity,
                                                                 ref_compat ? 1 : 0, d_keys, d_vals, d_rounds);
  GLP_CUDA(cudaGetLastError());
  GLP_CUDA(cudaMemcpyAsync(keys, d_keys, sizeof(uint32_t) * slots, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaMemcpyAsync(vals, d_vals, sizeof(uint32_t) * slots, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaMemcpyAsync(rounds, d_rounds, sizeof(int32_t) * (size_t)nv, cudaMemcpyDeviceToHost, g->stream));
  GLP_CUDA(cudaStreamSynchronize(g->stream));
  return GLP_OK;
}

int glp_run(glp_graph* g, int32_t method, const glp_params* pin, int32_t niter, glp_outputs* out, glp_iter_cb cb,
            void* cb_user, void* stream) {
  if (!g || !out || !out->labels) {
    set_error("graph, outputs and outputs->labels are required");
    return GLP_EINVAL;
  }
  if (niter < 0) {
    set_error("niter %d < 0", niter);
    return GLP_EINVAL;
  }
  glp_params p;
  glp_params_default(&p);
  if (pin) {
    if (pin->struct_size != (int32_t)sizeof(glp_params)) {
      set_error("glp_params.struct_size %d != %d", pin->struct_size, (int)sizeof(glp_params));
      return GLP_EINVAL;
    }
    p = *pin;
  }
  if (p.async && (cb || !out->on_device || out->changed || out->tier_ms || out->slpa_comm || out->slpa_mem)) {
    set_error("async runs take device outputs only (labels/vol), no callback, no host-side reports");
    return GLP_EINVAL;
  }
  int32_t total = niter;
  switch (method) {
    case GLP_METHOD_CLASSIC:
      break;
    case GLP_METHOD_LAYERED:
      if (p.nlayers < 1 || p.nlayers > GLP_MAX_LAYERS) {
        set_error("nlayers %d outside [1, %d]", p.nlayers, GLP_MAX_LAYERS);
        return GLP_EINVAL;
      }
      for (int i = 0; i < p.nlayers; ++i)
        if (p.dstar[i] < 1 || p.dstar[i] > 65536) {
          set_error("dstar[%d] = %d outside [1, 65536]", i, p.dstar[i]);
          return GLP_EINVAL;
        }
      total = p.nlayers * niter;
      break;
    case GLP_METHOD_SLPA:
      if (p.slpa_T < 1 || p.slpa_T > 64) {
        set_error("slpa_T %d outside [1, 64]", p.slpa_T);
        return GLP_EINVAL;
      }
      if (!(p.slpa_r >= 0.0 && p.slpa_r <= 1.0)) {
        set_error("slpa_r outside [0, 1]");
        return GLP_EINVAL;
      }
      break;
    case GLP_METHOD_USER:
      if (p.hooks < GLP_HOOKS_CLASSIC || p.hooks > GLP_HOOKS_WEIGHTED_DEGREE) {
        set_error("unknown hook set %d", p.hooks);
        return GLP_EINVAL;
      }
      if (p.hooks == GLP_HOOKS_LAYERED) total = p.nlayers * niter;
      break;
    case GLP_METHOD_SEEDED:
      if (!g->d_seeds) {
        set_error("method 5 needs seeds: call glp_graph_set_seeds first");
        return GLP_EINVAL;
      }
      break;
    default:
      set_error("method %d not in 1..5", method);
      return GLP_ENOTSUP;
  }
  if (p.backend != GLP_BACKEND_EXACT && p.backend != GLP_BACKEND_CM && p.backend != GLP_BACKEND_FA) {
    set_error("unknown backend %d", p.backend);
    return GLP_EINVAL;
  }
  TierParams t;
  int rc = tiers_for_graph(&p, g->d_w != nullptr, &t);
  if (rc) return rc;
  if (g->n == 0) {
    if (out->changed)
      for (int32_t i = 0; i < total; ++i) out->changed[i] = 0;
    if (out->launches) *out->launches = 0;
    return GLP_OK;
  }
  GLP_CUDA(cudaSetDevice(g->device));
  if ((rc = quiesce(g))) return rc;  // set-up may free buffers an earlier async run still uses
  if ((rc = ensure_plan(g, t))) return rc;
  if ((rc = ensure_work(g, total))) return rc;
  RunCtx c;
  c.g = g;
  c.s = stream ? (cudaStream_t)stream : g->stream;
  // a synchronous run has finished on return; an async one may still run on c.s
  g->last_stream = p.async ? c.s : nullptr;
  c.cb = cb;
  c.user = cb_user;
  c.backend = p.backend;
  c.serial = p.serial_step != 0;
  if (p.majority_permille > 0) c.majority_pm = (uint32_t)std::min(p.majority_permille, 1000);
  if (p.frontier_permille > 0) c.frontier_pm = (uint32_t)std::min(p.frontier_permille, 1000);
  if (p.frontier_permille < 0) c.frontier_pm = 0;  // never
  c.l2_window = p.l2_window != 0;
  c.cycle = !p.async && p.cycle_stop == 0;
  c.mid_prefetch = p.mid_prefetch == 0;
  c.big_staged = p.big_staged > 0;
  c.timing = out->tier_ms != nullptr;
  GLP_CUDA(cudaMemsetAsync(g->d_changed, 0, sizeof(unsigned long long) * (total + 1), c.s));
  const bool W = g->d_w != nullptr;
  if ((method == GLP_METHOD_CLASSIC || method == GLP_METHOD_SLPA || method == GLP_METHOD_LAYERED) &&
      (rc = ensure_sorted(g)))
    return rc;
  if (method == GLP_METHOD_CLASSIC && (rc = ensure_symmetric(g))) return rc;
  switch (method) {
    case GLP_METHOD_CLASSIC:
      rc = W ? run_classic<true>(c, niter) : run_classic<false>(c, niter);
      c.iter_base = niter & 1;
      break;
    case GLP_METHOD_LAYERED:
      rc = W ? run_layered<true>(c, p, niter) : run_layered<false>(c, p, niter);
      break;
    case GLP_METHOD_SLPA:
      rc = W ? run_slpa<true>(c, p, niter, out) : run_slpa<false>(c, p, niter, out);
      c.iter_base = niter & 1;
      break;
    case GLP_METHOD_USER:
      rc = run_hooks(c, p, niter);
      break;
    case GLP_METHOD_SEEDED:
      rc = W ? run_seeded<true>(c, niter) : run_seeded<false>(c, niter);
      c.iter_base = niter & 1;
      break;
  }
  set_l2_window(c, nullptr);
  if (rc) return rc;
  const int32_t* final_lab = g->d_lab[c.iter_base];
  if (g->n)
    GLP_CUDA(cudaMemcpyAsync(out->labels, final_lab, sizeof(int32_t) * g->n,
                             out->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.s));
  if (out->vol && g->n && (method == GLP_METHOD_LAYERED || (method == GLP_METHOD_USER && p.hooks == GLP_HOOKS_LAYERED)))
    GLP_CUDA(cudaMemcpyAsync(out->vol, g->d_vol[1], sizeof(int32_t) * g->n,
                             out->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.s));
  if (out->launches) *out->launches = c.launches;
  if (p.async) return GLP_OK;
  if (out->changed && total > 0) {
    std::vector<unsigned long long> tmp(total);
    GLP_CUDA(cudaMemcpyAsync(tmp.data(), g->d_changed, sizeof(unsigned long long) * total, cudaMemcpyDeviceToHost,
                             c.s));
    GLP_CUDA(cudaStreamSynchronize(c.s));
    // iterations after a detected two-step cycle change what the last one did
    if (c.cycle_from > 0)
      for (int32_t i = c.cycle_from; i < total; ++i) tmp[i] = tmp[c.cycle_from - 1];
    for (int32_t i = 0; i < total; ++i) out->changed[i] = (int64_t)tmp[i];
  }
  if (out->tier_ms) {
    if ((rc = c.harvest())) return rc;
    for (int i = 0; i < 8; ++i) out->tier_ms[i] = c.tier_ms[i];
    if (out->iter_ms)
      for (size_t i = 0; i < c.step_ms.size() && (int32_t)i < total; ++i) out->iter_ms[i] = c.step_ms[i];
    if (out->step_tier_ms)
      for (size_t i = 0; i < c.step_ms.size() && (int32_t)i < total; ++i)
        for (int t = 0; t < 8; ++t) out->step_tier_ms[i * 8 + t] = c.step_tier[i * 8 + t];
  }
  return check_err(g, c.s);
}

void glp_free_host(void* p) { std::free(p); }

int glp_run_classic_noalloc(const int32_t* d_offsets, const int32_t* d_cols, int32_t n, int64_t m, int32_t niter,
                            int32_t* d_labels, int64_t* changed, void* stream) {
  if (n < 0 || m < 0 || niter < 0 || !d_offsets || !d_labels || (m > 0 && !d_cols)) {
    set_error("bad arguments (n=%d, m=%lld, niter=%d)", n, (long long)m, niter);
    return GLP_EINVAL;
  }
  if (n > kNoAllocMaxVertices) {
    set_error("n=%d exceeds the allocation-free limit of %d vertices", n, kNoAllocMaxVertices);
    return GLP_EINVAL;
  }
  if (niter > kNoAllocMaxIters) {
    set_error("niter=%d exceeds the allocation-free limit of %d iterations", niter, kNoAllocMaxIters);
    return GLP_EINVAL;
  }
  if (m > INT32_MAX) {
    set_error("m=%lld exceeds int32 CSR", (long long)m);
    return GLP_EINVAL;
  }
  int rc = require_device();
  if (rc) return rc;
  int dev = 0;
  GLP_CUDA(cudaGetDevice(&dev));
  if (dev >= kNoAllocMaxDevices) {
    set_error("device %d beyond the %d devices the allocation-free path tracks", dev, kNoAllocMaxDevices);
    return GLP_ENOTSUP;
  }
  // The scratch's device address, looked up on every call with the device
  // current (the lookup allocates nothing): a cached address would go stale
  // if the context were reset and the module loaded again elsewhere.
  void* sp = nullptr;
  {
    const cudaError_t e = cudaGetSymbolAddress(&sp, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(allocation-free scratch)");
  }
  if (!g_noalloc_attr[dev].load(std::memory_order_acquire)) {
    GLP_CUDA(cudaFuncSetAttribute(k_noalloc_step<kNoAllocNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * pow2_host(2 * kNoAllocMaxDegree) * sizeof(uint32_t))));
    g_noalloc_attr[dev].store(1, std::memory_order_release);
  }
  NoAllocScratch* sc = static_cast<NoAllocScratch*>(sp);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // counters and flags start at zero; the label buffers are written below
  GLP_CUDA(cudaMemsetAsync(sc->changed, 0, sizeof(NoAllocScratch) - offsetof(NoAllocScratch, changed), st));
  if (n == 0) {
    if (m != 0) {
      set_error("offsets[0] must be 0 and offsets[n] must be m");
      return GLP_EINVAL;
    }
    GLP_CUDA(cudaStreamSynchronize(st));
    for (int32_t i = 0; changed && i < niter; ++i) changed[i] = 0;
    return GLP_OK;
  }
  k_validate_offsets<<<1184, 256, 0, st>>>(d_offsets, n, m, &sc->bad, &sc->maxdeg, &sc->unsorted);
  if (m) k_validate<<<1184, 256, 0, st>>>(d_offsets, d_cols, nullptr, m, n, &sc->bad, nullptr, nullptr);
  GLP_CUDA(cudaGetLastError());
  uint32_t flags[2] = {0, 0};  // bad, maxdeg
  GLP_CUDA(cudaMemcpyAsync(flags, &sc->bad, sizeof flags, cudaMemcpyDeviceToHost, st));
  GLP_CUDA(cudaStreamSynchronize(st));
  if (flags[0] & 16u) {
    set_error("offsets[0] must be 0 and offsets[n] must be m");
    return GLP_EINVAL;
  }
  if (flags[0] & 8u) {
    set_error("offsets not monotone");
    return GLP_EINVAL;
  }
  if (flags[0] & 1u) {
    set_error("column index outside [0, n)");
    return GLP_EINVAL;
  }
  const int32_t maxdeg = (int32_t)flags[1];
  if (maxdeg > kNoAllocMaxDegree) {
    set_error("a vertex of degree %d exceeds the allocation-free limit of %d", maxdeg, kNoAllocMaxDegree);
    return GLP_EINVAL;
  }
  int32_t* buf[2] = {d_labels, sc->labels};
  k_iota<<<(unsigned)cdiv(n, 256), 256, 0, st>>>(buf[0], buf[1], n);
  const size_t smem = 2 * pow2_host(2 * std::max(maxdeg, 1)) * sizeof(uint32_t);
  const unsigned grid = (unsigned)std::min<int64_t>(n, device_sms() * 16);
  for (int32_t it = 0; it < niter; ++it)
    k_noalloc_step<kNoAllocNT><<<grid, kNoAllocNT, smem, st>>>(d_offsets, d_cols, buf[it & 1], buf[(it + 1) & 1], n,
                                                               sc->changed + it, &sc->err);
  GLP_CUDA(cudaGetLastError());
  if (niter & 1) GLP_CUDA(cudaMemcpyAsync(d_labels, sc->labels, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
  uint32_t err = 0;
  GLP_CUDA(cudaMemcpyAsync(&err, &sc->err, sizeof err, cudaMemcpyDeviceToHost, st));
  static_assert(sizeof(int64_t) == sizeof(unsigned long long), "changed counts are 64-bit");
  if (changed && niter)
    GLP_CUDA(cudaMemcpyAsync(changed, sc->changed, sizeof(int64_t) * niter, cudaMemcpyDeviceToHost, st));
  GLP_CUDA(cudaStreamSynchronize(st));
  if (err) {
    set_error("kernel error flags 0x%x", err);
    return GLP_EKERNEL;
  }
  return GLP_OK;
}

}  // extern "C"

namespace glp {
// Recreates a handle's three streams at `priority` (the order of
// cudaDeviceGetStreamPriorityRange: lower is more urgent) once its work has
// finished.  Not part of the C ABI: the server runs short requests at the
// device's highest priority, so that the block scheduler dispatches their
// blocks ahead of the queued blocks of a long solve sharing the GPU.
int graph_set_stream_priority(glp_graph* g, int priority) {
  if (!g) {
    set_error("graph is NULL");
    return GLP_EINVAL;
  }
  int rc = quiesce(g);
  if (rc) return rc;
  g->last_stream = nullptr;
  for (cudaStream_t* st : {&g->stream, &g->aux[0], &g->aux[1]}) {
    cudaStream_t fresh = nullptr;
    GLP_CUDA(cudaStreamCreateWithPriority(&fresh, cudaStreamNonBlocking, priority));
    if (*st) cudaStreamDestroy(*st);
    *st = fresh;
  }
  return GLP_OK;
}
}  // namespace glp
