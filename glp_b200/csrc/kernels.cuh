// kernels.cuh -- degree-tiered synchronous label-propagation step kernels.
//
// One synchronous step computes, for every non-isolated vertex v,
//   L'(v) = argmax_l score(l, k_l(v)),  k_l(v) = sum of w(u,v) over u in N(v)
//   with L(u) = l (w = 1 when unweighted), ties -> the largest label,
// which is the rule of the reference's bin kernels (header/kernel.cuh:
// 864-911, 1033-1056, 1655-1739, 3124-3222, 4365-4426, 5187-5234: packed
// (count<<32)|(label+1) max).  Isolated vertices are never launched; both
// label buffers hold their label, so they keep it (kernel.cuh:4387-4390).
//
// Tiers (chosen by the host planner from the degree):
//   tiny  (1..8)       : one thread per vertex, labels in registers
//   group (9..32)      : 16 or 32 lanes per vertex, one __match_any_sync round
//   mid   (33..256)    : one warp per vertex, per-warp shared-memory table
//   big   (257..24576) : one block per vertex, block shared-memory table
//   hub   (above big)  : labels gathered once and sorted into hash buckets,
//                        one block per (hub, bucket) with a shared table
// Majority shortcut (classic, weighted, SLPA listener): when a vertex's own
// label holds more than half of its neighbourhood weight it is the unique
// mode.  Once the previous step changed few labels, a streaming pre-pass
// decides those vertices and lists the others for exact counting.
//
// Every table insert returns the running total after the add; the maximum
// of score(l, total) over all inserts equals the maximum over labels of
// score(l, final total) because score is non-decreasing in the count.  So a
// thread keeps only its best candidate and one reduction finishes the vertex,
// independent of the order of the atomics: results are deterministic.
#pragma once
#include <type_traits>

#include "device.cuh"

namespace glp {

// Count bounds of a contiguous big tier, vertices base .. base+n-1 (n = 0:
// off).  For big vertex base + i: lbl[i] is a label and lb[i] a lower bound
// on its count among the current step's input labels (-1: none; written by
// the majority pre-pass and the frontier majority test, cleared by full
// steps); nchg[i] counts its neighbours changed by the previous step
// (k_frontier_push adds them, the big-tier launch of the frontier step takes
// and clears them).  Only unweighted classic runs set it: their gathered
// labels are the current labels, and a changed neighbour moves a count by
// at most one.
struct BigBound {
  int32_t* lbl = nullptr;
  uint32_t* lb = nullptr;
  uint32_t* nchg = nullptr;
  int32_t base = 0, n = 0;
  __device__ __forceinline__ bool has(int32_t v) const { return (uint32_t)(v - base) < (uint32_t)n; }
};

// Neighbour labels, own labels and the output of one step.
struct StepArgs {
  const int32_t* off;
  const int32_t* cols;
  const int32_t* w;     // nullable when !W
  const int32_t* lin;   // labels gathered from neighbours (SLPA: spoken labels)
  const int32_t* lcur;  // own current label (changed count, majority candidate)
  int32_t* lout;
  unsigned long long* changed;
  uint32_t* err;
  // this step's mode, set on the device by k_step_mode (nullptr: full)
  const int32_t* mode;
  int32_t n;
  // vertices whose label changed this step are appended here (nullable)
  int32_t* chg_out;
  uint32_t* chg_out_n;
  BigBound bb{};
};

// Counts (and, when a.chg_out is set, lists) the vertices whose label changed.
// Every lane of the warp calls it; v is only read when changed.
__device__ __forceinline__ void record_changes(const StepArgs& a, bool changed, int32_t v) {
  const uint32_t m = __ballot_sync(kFull, changed);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) {
    atomicAdd(a.changed, (unsigned long long)__popc(m));
    if (a.chg_out) base = atomicAdd(a.chg_out_n, (uint32_t)__popc(m));
  }
  if (a.chg_out) {
    base = __shfl_sync(kFull, base, leader);
    if (changed) a.chg_out[base + __popc(m & ((1u << lane) - 1u))] = v;
  }
}

// The same for one thread deciding alone.
__device__ __forceinline__ void record_change(const StepArgs& a, int32_t v) {
  atomicAdd(a.changed, 1ull);
  if (a.chg_out) a.chg_out[atomicAdd(a.chg_out_n, 1u)] = v;
}

// Batched recording for kernels that decide one vertex per warp: lane 0
// keeps the warp's changed vertices in a 32-entry shared buffer, and a full
// (or final) buffer costs one add to the counter and one reservation in the
// list, written by the whole warp.  Almost every vertex changes in the first
// steps, and a per-vertex atomic on the two shared counters would serialise
// there.
__device__ __forceinline__ void warp_flush_changes(const StepArgs& a, const int32_t* buf, uint32_t nb) {
  if (!nb) return;
  const int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (lane == 0) {
    atomicAdd(a.changed, (unsigned long long)nb);
    if (a.chg_out) base = atomicAdd(a.chg_out_n, nb);
  }
  if (a.chg_out) {
    base = __shfl_sync(kFull, base, 0);
    __syncwarp();
    if ((uint32_t)lane < nb) a.chg_out[base + lane] = buf[lane];
  }
  __syncwarp();
}
// Called by every lane after each vertex; `changed` and v matter on lane 0.
__device__ __forceinline__ void warp_note_change(const StepArgs& a, int32_t* buf, uint32_t& nb, bool changed,
                                                 int32_t v) {
  if ((threadIdx.x & 31) == 0 && changed) buf[nb] = v;
  nb += __shfl_sync(kFull, changed ? 1u : 0u, 0);
  if (nb == 32) {
    warp_flush_changes(a, buf, nb);
    nb = 0;
  }
}

// Step modes.  Full: every vertex counts exactly.  Majority: a streaming
// pre-pass decides vertices whose own label holds a strict majority and
// lists the others.  Frontier: only vertices with a neighbour that changed in
// the previous step are recomputed; the others provably keep their label.
enum : int32_t { kModeFull = 0, kModeMajority = 1, kModeFrontier = 2 };

__device__ __forceinline__ int32_t step_mode(const StepArgs& a) { return a.mode ? *a.mode : kModeFull; }
__device__ __forceinline__ bool use_majority(const StepArgs& a) { return step_mode(a) == kModeMajority; }

// Picks the mode from the previous step's changed count: frontier below
// frontier_pm changes per 1000 vertices (default 50), majority below
// majority_pm (default 500), when the method allows them; else full.
// mode[1] (scores that need a per-label lookup, layered LP): 1 = score each
// distinct label once from the finished table, worth it once fewer than half
// of the n_active non-isolated vertices changed (their neighbourhoods hold
// few distinct labels); 0 = score at every insert, the lookup issued before
// the insert so that its latency overlaps the hashing.
__global__ void k_step_mode(const unsigned long long* prev_changed, int32_t n, int32_t n_active, int allow_majority,
                            int allow_frontier, uint32_t majority_pm, uint32_t frontier_pm, int32_t* mode) {
  int32_t m = kModeFull, scan = 0;
  if (prev_changed) {
    const unsigned long long c = *prev_changed;
    if (allow_frontier && c * 1000ull < (unsigned long long)frontier_pm * (unsigned long long)n) m = kModeFrontier;
    else if (allow_majority && c * 1000ull < (unsigned long long)majority_pm * (unsigned long long)n) m = kModeMajority;
    scan = c * 2ull < (unsigned long long)n_active ? 1 : 0;
  }
  mode[0] = m;
  mode[1] = scan;
}
__device__ __forceinline__ bool scan_scores(const StepArgs& a) { return a.mode && a.mode[1] != 0; }

// The vertices of one tier: explicit ids, or the contiguous range
// [base, base+n) (degree-sorted graphs make every tier contiguous).
struct Verts {
  const int32_t* ids;
  int32_t base;
  int32_t n;
  __device__ __forceinline__ int32_t operator[](int64_t i) const { return ids ? ids[i] : base + (int32_t)i; }
};

// A device-built vertex list (majority failures, frontier members).
struct FailList {
  int32_t* ids;
  uint32_t* count;
};

// The vertices an exact-count kernel works on this step: the whole tier
// (full mode), the tier's majority failures (majority mode, mid/big only) or
// the tier's frontier members (frontier mode).
struct TierWork {
  Verts all;
  FailList major;  // ids == nullptr: the tier has no pre-pass
  FailList front;
  int full_only;   // 1: works only in full mode (a sub-range of a tier)
  int listed = 0;  // 1: works on the `major` list in every mode (screen fallbacks)
  __device__ __forceinline__ int32_t size(int32_t mode) const {
    if (listed) return (int32_t)*major.count;
    if (full_only) return mode == kModeFull ? all.n : 0;
    if (mode == kModeFrontier && front.ids) return (int32_t)*front.count;
    if (mode == kModeMajority && major.ids) return (int32_t)*major.count;
    return all.n;
  }
  __device__ __forceinline__ int32_t at(int32_t mode, int64_t i) const {
    if (listed) return major.ids[i];
    if (mode == kModeFrontier && front.ids) return front.ids[i];
    if (mode == kModeMajority && major.ids) return major.ids[i];
    return all[i];
  }
};

// score(l, k) for classic LP: the count itself.  A label holding more than
// half of the neighbourhood weight is then the unique maximum, so the
// majority shortcut applies.
struct ScoreClassic {
  static constexpr bool kMajority = true;
  // (count << 32 | label) orders candidates as better() does: a block can
  // reduce with one 64-bit shared atomicMax
  static constexpr bool kPacked = true;
  static constexpr bool kScan = false;  // no lookup: running maximum at every insert
  // threads per SM the unweighted mid / big kernels are compiled for (32
  // registers a thread); their 16-bit count tables fit as many
  static constexpr int kSMThreads = 2048;
  __device__ __forceinline__ int64_t operator()(int32_t, uint32_t k) const { return (int64_t)k; }
  __device__ __forceinline__ int32_t vol_of(int32_t) const { return 0; }
  __device__ __forceinline__ int64_t from_vol(uint32_t k, int32_t) const { return (int64_t)k; }
  // the largest score a label of count <= k can have
  __device__ __forceinline__ int64_t bound(uint32_t k) const { return (int64_t)k; }
  // the packed form: counts are non-negative, so (count << 32 | label) is monotone
  static __device__ __forceinline__ unsigned long long pack(const Best& b) {
    return ((unsigned long long)b.s << 32) | (uint32_t)b.l;
  }
  // the monotone 32-bit key of a score (PackedCand)
  __device__ __forceinline__ uint32_t key32(uint32_t k, int32_t) const { return k; }
  // the label of neighbour c (and, for scores that carry it, its volume)
  static constexpr bool kLV = false;
  __device__ __forceinline__ void load(const StepArgs& a, int32_t c, int32_t& lab, int32_t&) const {
    lab = ld_label(a.lin + c);
  }
};

// score(l, k) for layered LP: dstar*k - vol_r[l] (kernel.cuh:2575-2600).
// The volume term breaks the majority argument: no shortcut.
struct ScoreLayered {
  static constexpr bool kMajority = false;
  static constexpr bool kPacked = false;  // signed 64-bit scores: block_max
  // the volume is a global lookup per label: prefetched per insert, or (step
  // mode word 1) looked up once per distinct label by a scan of the table
  static constexpr bool kScan = true;
  static constexpr int kSMThreads = 1024;  // 64 registers a thread
  const int32_t* vol;
  int64_t dstar;
  __device__ __forceinline__ int64_t operator()(int32_t l, uint32_t k) const {
    return dstar * (int64_t)k - (int64_t)__ldg(vol + l);
  }
  // the same split in two, so that callers can issue the loads together
  __device__ __forceinline__ int32_t vol_of(int32_t l) const { return __ldg(vol + l); }
  __device__ __forceinline__ int64_t from_vol(uint32_t k, int32_t v) const { return dstar * (int64_t)k - (int64_t)v; }
  // the largest score a label of count <= k can have (volumes are >= 0)
  __device__ __forceinline__ int64_t bound(uint32_t k) const { return dstar * (int64_t)k; }
  static __device__ __forceinline__ unsigned long long pack(const Best&) { return 0ull; }  // not packed
  static constexpr bool kLV = false;
  __device__ __forceinline__ void load(const StepArgs& a, int32_t c, int32_t& lab, int32_t&) const {
    lab = ld_label(a.lin + c);
  }
};

// The same layered score in 32-bit arithmetic, for graphs where every score
// lies in [-2^31, 2^31): the host checks |dstar| * (largest weight sum of a
// row) + n < 2^31 (counts never exceed a row's weight sum, volumes never
// exceed n).  Scores then pack with their label into one 64-bit word
// ((score + 2^31) << 32 | label, monotone in (score, label)), so the big tier
// reduces with one shared atomicMax and the unweighted tables take 16-bit
// counts, as in classic LP: fewer registers and smaller tables, more blocks
// per SM.  The mid and big tiers read each neighbour's (label, volume of
// that label) as one 8-byte pair from lv, which the step before wrote
// (k_label_volumes): one random gather per entry instead of two.
struct ScoreLayered32 {
  static constexpr bool kMajority = false;
  static constexpr bool kPacked = true;
  static constexpr bool kScan = true;
  static constexpr int kSMThreads = 1536;  // 40 registers a thread: 32 would spill
  static constexpr bool kLV = true;
  const int32_t* vol;
  int32_t dstar;
  const int2* lv;  // [n] (label of v, vol[label of v]); .x equals lin[v]
  __device__ __forceinline__ void load(const StepArgs&, int32_t c, int32_t& lab, int32_t& vl) const {
    const int2 x = __ldg(lv + c);
    lab = x.x;
    vl = x.y;
  }
  __device__ __forceinline__ int64_t operator()(int32_t l, uint32_t k) const {
    return (int64_t)(dstar * (int32_t)k - __ldg(vol + l));
  }
  __device__ __forceinline__ int32_t vol_of(int32_t l) const { return __ldg(vol + l); }
  __device__ __forceinline__ int64_t from_vol(uint32_t k, int32_t v) const { return (int64_t)(dstar * (int32_t)k - v); }
  __device__ __forceinline__ int64_t bound(uint32_t k) const { return (int64_t)(dstar * (int32_t)k); }
  static __device__ __forceinline__ unsigned long long pack(const Best& b) {
    return ((unsigned long long)((uint32_t)(int32_t)b.s ^ 0x80000000u) << 32) | (uint32_t)b.l;
  }
  __device__ __forceinline__ uint32_t key32(uint32_t k, int32_t v) const {
    return (uint32_t)(dstar * (int32_t)k - v) ^ 0x80000000u;
  }
};

template <bool W>
__device__ __forceinline__ void load_edge(const StepArgs& a, int64_t j, int32_t& lab, uint32_t& wt) {
  lab = ld_label(a.lin + ld_stream(a.cols + j));
  wt = W ? (uint32_t)ld_stream(a.w + j) : 1u;
}

// Monotone packing of (score, label) into 64 bits for atomicMax: the score is
// offset by 2^31 and must lie in [-2^31, 2^31).
__device__ __forceinline__ unsigned long long pack_best(const Best& b, uint32_t* err) {
  if (b.l < 0) return 0ull;
  const int64_t s = b.s + 2147483648LL;
  if (s < 0 || s > 0xffffffffLL) {
    atomicOr(err, kErrScoreRange);
    return 0ull;
  }
  return ((unsigned long long)s << 32) | (uint32_t)b.l;
}

// ---------------------------------------------------------------- tiny tier
template <int TMAX, bool W, class S>
__global__ void __launch_bounds__(256, TMAX >= 32 ? 2 : 1) k_tiny(StepArgs a, TierWork tw, S score) {
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  // grid-stride over whole warps so record_changes sees full warps
  for (int32_t t0 = blockIdx.x * blockDim.x; t0 < nwork; t0 += gridDim.x * blockDim.x) {
  const int32_t t = t0 + threadIdx.x;
  bool chg = false;
  int32_t v = 0;
  if (t < nwork) {
    v = tw.at(mode, t);
    const int32_t b = a.off[v];
    const int32_t d = a.off[v + 1] - b;
    int32_t lab[TMAX];
    uint32_t wt[TMAX];
#pragma unroll
    for (int i = 0; i < TMAX; ++i) {
      lab[i] = INT32_MAX;  // past the degree: sorts last, never scored
      wt[i] = 0;
      if (i < d) load_edge<W>(a, (int64_t)b + i, lab[i], wt[i]);
    }
    sort_labels<TMAX, W>(lab, wt);
    // a run's total is scored at its last element.  Layered LP needs the
    // label's volume there: loaded for run ends only, eight slots a round so
    // that the loads of a round are in flight together without holding a
    // register per slot
    constexpr int U = TMAX < 8 ? TMAX : 8;
    Best best = best_none();
    uint32_t run = 0;
#pragma unroll
    for (int i0 = 0; i0 < TMAX; i0 += U) {
      int32_t vl[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + u;
        const bool end = (i == TMAX - 1) || lab[(i + 1) & (TMAX - 1)] != lab[i];
        vl[u] = (S::kScan && end && lab[i] != INT32_MAX) ? score.vol_of(lab[i]) : 0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + u;
        run = (i > 0 && lab[i] == lab[i > 0 ? i - 1 : 0]) ? run + wt[i] : wt[i];
        const bool end = (i == TMAX - 1) || lab[(i + 1) & (TMAX - 1)] != lab[i];
        if (end && lab[i] != INT32_MAX) {
          const Best c{score.from_vol(run, vl[u]), lab[i]};
          if (better(c, best)) best = c;
        }
      }
    }
    a.lout[v] = best.l;
    chg = best.l != a.lcur[v];
  }
  record_changes(a, chg, v);
  }
}

// --------------------------------------------------------------- group tier
// G lanes per vertex (degree <= G); each warp handles U rounds of 32/G
// vertices with all loads issued before any counting.  The match key carries
// the group index so equal labels of different vertices do not merge.
template <int G, int U, bool W, class S>
__global__ void __launch_bounds__(256) k_group(StepArgs a, TierWork tw, S score) {
  constexpr int PER = 32 / G;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp * U * PER < nwork;
       warp += nwarps) {
  int32_t v[U], lab[U];
  uint32_t wt[U];
  bool act[U], has[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int64_t grp = (warp * U + u) * PER + lane / G;
    act[u] = grp < nwork;
    has[u] = false;
    v[u] = 0;
    wt[u] = 0;
    int32_t col = 0;
    if (act[u]) {
      v[u] = tw.at(mode, grp);
      const int32_t b = a.off[v[u]], e = a.off[v[u] + 1];
      const int32_t j = b + (lane & (G - 1));
      has[u] = j < e;
      if (has[u]) {
        col = ld_stream(a.cols + j);
        if (W) wt[u] = (uint32_t)ld_stream(a.w + j);
      }
    }
    lab[u] = col;
  }
#pragma unroll
  for (int u = 0; u < U; ++u) lab[u] = has[u] ? ld_label(a.lin + lab[u]) : -1;
  uint32_t chg = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const unsigned long long key = ((unsigned long long)(lane / G) << 32) | (uint32_t)lab[u];
    const uint32_t m = __match_any_sync(kFull, key);
    const uint32_t k = W ? __reduce_add_sync(m, wt[u]) : (uint32_t)__popc(m);
    Best c = best_none();
    if (has[u] && lane == __ffs(m) - 1) c = Best{score(lab[u], k), lab[u]};
    c = group_max<G>(c);
    const bool writer = act[u] && (lane & (G - 1)) == 0;
    bool ch = false;
    if (writer) {
      a.lout[v[u]] = c.l;
      ch = c.l != a.lcur[v[u]];
    }
    record_changes(a, ch, v[u]);
  }
  (void)chg;
  }
}

// Count one 32-edge chunk: every lane adds its own label to the table and
// keeps the best (score, label) of the running totals it saw.  Lanes holding
// lane 0's label add once, through lane 0 (a hot label of a forming
// community costs one atomic per warp).  Other lanes are not merged:
// __match_any_sync costs a round per distinct value on B200, while a 32-bit
// shared atomicAdd stays cheap under moderate contention.  Called by all
// lanes of the warp.
// VIN: vl_in is the volume of lab, loaded with it (S::load of an S::kLV score).
// merge (warp-uniform): fold lane 0's label as above; off, every lane adds
// its own (measured faster in rows of mostly distinct labels, where the fold
// rarely finds a copy).
// B: Best, or PackedCand for S::kPacked scores.
template <bool W, bool VIN = false, class S, class Ins, class B>
__device__ __forceinline__ void count_chunk(bool has, int32_t lab, uint32_t wt, const S& score, const Ins& insert,
                                            B& best, bool& fail, bool scan = false, int32_t vl_in = 0,
                                            bool merge = true) {
  const int lane = threadIdx.x & 31;
  uint32_t k = W ? wt : 1u;
  if (merge) {
    const int32_t l0 = __shfl_sync(kFull, has ? lab : -1, 0);
    const uint32_t m0 = __ballot_sync(kFull, has && lab == l0);
    if (l0 >= 0) {
      const uint32_t k0 = W ? __reduce_add_sync(kFull, lab == l0 && has ? wt : 0u) : (uint32_t)__popc(m0);
      if (lane == 0) k = k0;
      else if (has && lab == l0) has = false;  // counted by lane 0
    }
  }
  if (!has) return;
  // the volume (S::kLV: loaded with the label) is in flight during the insert
  const int32_t vl = (S::kScan && !scan) ? (VIN ? vl_in : score.vol_of(lab)) : 0;
  const uint32_t tot = insert((uint32_t)lab + 1u, k);
  if (tot == kNoSlot) {
    fail = true;
  } else if (!scan) {
    offer(best, score, tot, vl, lab);
  }
}

// The best (score, label) over the occupied slots of a finished table, slots
// t, t+stride, ... of it (scores with kScan).
// Eight slots a round (four in kernels held to 40 registers), their volume
// loads in flight together.
// CF: a claim-first table (table_claim_insert), whose vals hold count - 1.
template <bool C16 = false, bool CF = false, class S, class B>
__device__ __forceinline__ void scan_table(const uint32_t* keys, const uint32_t* vals, uint32_t cap, uint32_t t,
                                           uint32_t stride, const S& score, B& best) {
  constexpr int U = S::kSMThreads > 1024 ? 4 : 8;
  for (uint32_t s0 = t; s0 < cap; s0 += U * stride) {
    uint32_t key[U], val[U];
    int32_t vl[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t s = s0 + u * stride;
      key[u] = s < cap ? keys[s] : 0u;
      val[u] = s < cap ? (CF ? claim_count_at<C16>(keys, vals, s) : count_at<C16>(vals, s)) : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) vl[u] = key[u] ? score.vol_of((int32_t)(key[u] - 1u)) : 0;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (key[u]) offer(best, score, val[u], vl[u], (int32_t)(key[u] - 1u));
  }
}

// ---------------------------------------------------- majority pre-pass
// One warp per vertex of the mid and big tiers: count the weight of the vertex's
// own label with 4 independent column/label loads in flight per lane.  A
// strict majority is written; other vertices go to the mid or big fail list.
template <bool W>
__global__ void __launch_bounds__(256) k_major_warp(StepArgs a, Verts vs, int32_t mid_max, FailList fmid,
                                                    FailList fbig) {
  constexpr int U = 8;  // column loads in flight per lane
  if (!use_majority(a)) return;
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // the next vertex's offsets and label are fetched while this one streams
  int32_t nv_b = 0, nv_e = 0, nv_c = 0, nv_v = 0;
  if (gw < vs.n) {
    nv_v = vs[gw];
    nv_b = a.off[nv_v];
    nv_e = a.off[nv_v + 1];
    nv_c = a.lcur[nv_v];
  }
  for (int64_t i = gw; i < vs.n; i += nw) {
    const int32_t v = nv_v, b = nv_b, e = nv_e, cand = nv_c;
    if (i + nw < vs.n) {
      nv_v = vs[i + nw];
      nv_b = a.off[nv_v];
      nv_e = a.off[nv_v + 1];
      nv_c = a.lcur[nv_v];
    }
    uint32_t cnt = 0, tot = 0;
    // unweighted rows stop at the first chunk after which the own label's
    // count proves a strict majority (2 cnt > d) or rules it out (even every
    // unread entry could not lift it above d / 2): the answer is the same as
    // after the whole row, and a formed community's big rows are decided
    // after a little more than half of their entries
    const uint32_t d = (uint32_t)(e - b);
    for (int32_t c0 = b; c0 < e; c0 += 32 * U) {  // warp-uniform chunks
      const int32_t j0 = c0 + lane;
      int32_t c[U];
      uint32_t wt[U];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int32_t j = j0 + 32 * q;
        c[q] = j < e ? ld_stream(a.cols + j) : -1;
        wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int32_t l = c[q] >= 0 ? ld_label(a.lin + c[q]) : -1;
        cnt += l == cand ? wt[q] : 0u;
        tot += wt[q];
      }
      if (!W && c0 + 32 * U < e) {
        const uint32_t seen = (uint32_t)(c0 + 32 * U - b);
        const uint32_t sc = __reduce_add_sync(kFull, cnt);
        if (2ull * sc > d || 2ull * (sc + (d - seen)) <= d) {
          cnt = lane == 0 ? sc : 0u;  // the reduction below returns sc
          break;
        }
      }
    }
    cnt = __reduce_add_sync(kFull, cnt);
    tot = W ? __reduce_add_sync(kFull, tot) : d;
    if (lane == 0) {
      // the count (partial after an early stop: still a lower bound) bounds
      // the frontier step that may follow
      if (!W && a.bb.has(v)) {
        a.bb.lbl[v - a.bb.base] = cand;
        a.bb.lb[v - a.bb.base] = cnt;
      }
      if (2ull * cnt > (unsigned long long)tot) {
        a.lout[v] = cand;
      } else {
        const FailList& f = (e - b) <= mid_max ? fmid : fbig;
        f.ids[atomicAdd(f.count, 1u)] = v;
      }
    }
  }
}

// ----------------------------------------------------------------- mid tier
// Exact count, one warp per vertex (degree <= CAP/2): per-warp shared table
// sized to the power of two >= 2*degree; batches of 4 chunks of 32 edges are
// loaded before they are counted.
// C16: 16-bit counts (unweighted: a count never exceeds the degree;
// weighted: the caller knows every mid vertex's weights sum below 2^16), so
// that the tables and 32 registers a thread fit eight blocks per SM.
// PF: the first batch of the warp's next vertex (its columns, then its
// neighbour labels) is loaded before the current vertex is counted, so the
// label gathers are in flight while the table work runs; it costs registers
// (at most 40 a thread: six blocks per SM).
template <int CAP, int NT, bool W, class S, bool C16 = (S::kPacked && !W), bool PF = false>
__global__ void __launch_bounds__(NT, PF ? (S::kPacked ? 1536 : 1024) / NT
                                         : (C16 ? S::kSMThreads : S::kSMThreads == 2048 ? 1536 : 1024) / NT)
    k_mid(StepArgs a, TierWork tw, S score) {
  constexpr int NW = NT / 32;
  // unweighted 16-bit tables count claim-first; the lane-0 fold runs outside
  // full-count steps, where listed vertices hold few distinct labels, and
  // for classic-type scores in every step
  constexpr bool CF = C16 && !W;
  const bool scan = S::kScan && scan_scores(a);
  __shared__ __align__(16) uint32_t skeys[NW][CAP];
  __shared__ __align__(16) uint32_t svals[NW][C16 ? CAP / 2 : CAP];
  __shared__ int32_t cbuf[NW][32];  // changed vertices not yet listed
  uint32_t ncb = 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  const int32_t stride = gridDim.x * NW;
  // classic-type scores fold lane 0's label in full-count steps too (the
  // third full-count step of R-MAT s24, whose labels have begun to gather,
  // 1.12 -> 1.00 ms, the first two unchanged); the layered score does not
  // (measured slower)
  const bool merge = !CF || mode != kModeFull || S::kMajority;
  uint32_t* kk = skeys[warp];
  uint32_t* vv = svals[warp];
  // batch loader: columns (and weights) of entries j0 + 32q + lane below e,
  // then their labels (-1 past the row)
  auto load_batch = [&](int32_t j0, int32_t e, int32_t (&lab)[4], uint32_t (&wt)[4], int32_t (&vl)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int32_t j = j0 + 32 * q + lane;
      lab[q] = j < e ? ld_stream(a.cols + j) : -1;
      wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (lab[q] >= 0) score.load(a, lab[q], lab[q], vl[q]);
  };
  int32_t pv = 0, pb = 0, pe = 0;  // PF: the next vertex and its first batch
  int32_t plab[4], pvl[4];
  uint32_t pwt[4];
  auto prefetch = [&](int32_t idx) {
    pb = pe = 0;
    if (idx < nwork) {
      pv = tw.at(mode, idx);
      pb = a.off[pv];
      pe = a.off[pv + 1];
    }
    load_batch(pb, pe, plab, pwt, pvl);
  };
  int32_t i = blockIdx.x * NW + warp;
  if (PF) prefetch(i);
  for (; i < nwork; i += stride) {
    int32_t v, b, e;
    int32_t lab0[4], vl0[4];
    uint32_t wt0[4];
    if (PF) {
      v = pv;
      b = pb;
      e = pe;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        lab0[q] = plab[q];
        wt0[q] = pwt[q];
        vl0[q] = pvl[q];
      }
      prefetch(i + stride);  // in flight while this vertex is counted
    } else {
      v = tw.at(mode, i);
      b = a.off[v];
      e = a.off[v + 1];
    }
    // four slots a neighbour where the warp's table holds them, else two: a
    // quarter-full table probes less (measured: rows of degree 33..128 8.2 ->
    // 7.3 ps per entry); degree > 32: cap >= 128
    const uint32_t cap = min(pow2_ceil(4u * (uint32_t)(e - b)), (uint32_t)CAP);
    zero_words16(kk, cap, lane, 32);
    zero_words16(vv, C16 ? cap / 2 : cap, lane, 32);
    __syncwarp();
    std::conditional_t<S::kPacked, PackedCand, Best> best{};
    if constexpr (!S::kPacked) best = best_none();
    bool fail = false;
    auto ins = [&](uint32_t key, uint32_t k) {
      return CF ? table_claim_insert<C16>(kk, vv, cap - 1, key, k, cap)
                : table_insert_bounded<C16>(kk, vv, cap - 1, key, k, cap, nullptr, nullptr);
    };
    for (int32_t j0 = b; j0 < e; j0 += 128) {
      int32_t lab[4], vl[4];
      uint32_t wt[4];
      if (PF && j0 == b) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          lab[q] = lab0[q];
          wt[q] = wt0[q];
          vl[q] = vl0[q];
        }
      } else {
        load_batch(j0, e, lab, wt, vl);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + 32 * q < e)
          count_chunk<W, S::kLV>(lab[q] >= 0, lab[q], wt[q], score, ins, best, fail, scan, vl[q], merge);
    }
    if (fail) atomicOr(a.err, kErrProbe);
    if (scan) {
      __syncwarp();
      scan_table<C16, CF>(kk, vv, cap, lane, 32, score, best);
    }
    int32_t lbest;
    if constexpr (S::kPacked) {
      lbest = (int32_t)(uint32_t)warp_best(best);
    } else {
      best = group_max<32>(best);
      lbest = best.l;
    }
    bool chg = false;
    if (lane == 0) {
      a.lout[v] = lbest;
      chg = lbest != a.lcur[v];
    }
    warp_note_change(a, cbuf[warp], ncb, chg, v);
    __syncwarp();  // the table is cleared for the next vertex
  }
  warp_flush_changes(a, cbuf[warp], ncb);
}

// One thread's batch of changed vertices: one add to the counter and one
// reservation in the list for the whole batch.
__device__ __forceinline__ void flush_big_changes(const StepArgs& a, const int32_t* buf, uint32_t& nb) {
  if (!nb) return;
  atomicAdd(a.changed, (unsigned long long)nb);
  if (a.chg_out) {
    const uint32_t base = atomicAdd(a.chg_out_n, nb);
    for (uint32_t i = 0; i < nb; ++i) a.chg_out[base + i] = buf[i];
  }
  nb = 0;
}

// ----------------------------------------------------------------- big tier
// Exact count, one block per vertex: block shared table (dynamic) sized per
// vertex to the power of two >= 2*degree.  C16 (unweighted counts only):
// claim-first 16-bit counts, and at most kBig16Slots slots (three quarters
// full at degree 24576), so 24576 labels fit 192 KB of shared memory.
// 32-bit tables hold at most kBig32Slots slots (three quarters full at
// degree 12288, the weighted tier's largest): 128 KB.
// Unweighted blocks are held to S::kSMThreads threads per SM (classic: 32
// registers, 32-bit layered: 40), weighted classic blocks of up to 512
// threads to 40 (1536), which they fit without spilling; the other
// instantiations to 64 (1024 threads per SM).
constexpr uint32_t kBig16Slots = 32768, kBig32Slots = 16384;
// Rows above this degree fold lane 0's label in full-count steps too.
constexpr int32_t kMergeDegree = 8192;
// CF (with C16): claim-first inserts (table_claim_insert).  Off, a C16
// table counts load-first; the top degree range runs so, its tables up to
// three quarters full, where a CAS per probe measured slower.
// 1024-thread blocks of packed scores run two to an SM at 32 registers; the
// 32-bit layered score spills there (36-52 bytes) and still measured faster
// than one block at 64 (layered R-MAT s24 big tier 2.88 -> 2.70 ms per
// iteration)
template <int NT, bool W, class S, bool C16 = false, bool CF = C16>
__global__ void __launch_bounds__(NT, (!W ? ((NT == 1024 && S::kPacked) ? 2048 : S::kSMThreads)
                                          : (S::kSMThreads == 2048 && NT <= 512) ? 1536 : 1024) / NT)
    k_big(StepArgs a, TierWork tw, S score) {
  static_assert(!(C16 && W), "16-bit counts hold unweighted counts only");
  static_assert(C16 || !CF, "claim-first tables are the 16-bit ones");
  const bool scan = S::kScan && scan_scores(a);
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ int32_t cbuf[64];  // changed vertices not yet listed (thread 0's)
  uint32_t ncb = 0;
  __shared__ Best red[32];
  // packed scores: one slot per vertex parity, so thread 0 can read vertex
  // i's result while the block already counts vertex i+1 into the other
  __shared__ unsigned long long sbest[2];
  __shared__ uint32_t msum[2][2];  // majority test: (own-label weight, total weight) per vertex parity
  __shared__ uint32_t sdec[2];     // frontier vertex decided by its count bound, per vertex parity
  int par = 0, mpar = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  for (int32_t i = blockIdx.x; i < nwork; i += gridDim.x) {
    const int32_t v = tw.at(mode, i);
    const int32_t b = a.off[v], e = a.off[v + 1];
    // the vertex's own label, loaded here so that thread 0 does not wait for
    // it after the reduction barrier while the block waits for thread 0
    const int32_t cur = a.lcur[v];
    if (S::kMajority && mode == kModeFrontier) {
      // a frontier vertex of this tier has many neighbours and usually keeps
      // its label: a strict majority of its own label decides it without a
      // table (the majority pre-pass does this for every tier in majority
      // steps)
      const int32_t cand = cur;
      if (threadIdx.x == 0) {
        msum[mpar][0] = msum[mpar][1] = 0u;
        // count bound: the last count of its label, less the neighbours
        // that changed since, is still a strict majority -> keeps it unread
        uint32_t dec = 0u;
        if (!W && a.bb.has(v)) {
          const int32_t bi = v - a.bb.base;
          const uint32_t nc = a.bb.nchg[bi];
          a.bb.nchg[bi] = 0u;
          if (a.bb.lbl[bi] == cand) {
            const uint32_t lb0 = a.bb.lb[bi];
            const uint32_t lb = nc >= lb0 ? 0u : lb0 - nc;
            if (2ull * lb > (unsigned long long)(e - b)) {
              a.bb.lb[bi] = lb;
              dec = 1u;
            }
          }
        }
        sdec[mpar] = dec;
      }
      __syncthreads();
      if (sdec[mpar]) {  // block-uniform
        if (threadIdx.x == 0) a.lout[v] = cand;
        mpar ^= 1;
        continue;
      }
      uint32_t cnt = 0, tot = 0;
      for (int32_t j0 = b + threadIdx.x; j0 < e; j0 += 4 * NT) {
        int32_t c[4];
        uint32_t wt[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int32_t j = j0 + q * NT;
          c[q] = j < e ? ld_stream(a.cols + j) : -1;
          wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          cnt += (c[q] >= 0 && ld_label(a.lin + c[q]) == cand) ? wt[q] : 0u;
          tot += wt[q];
        }
      }
      cnt = __reduce_add_sync(kFull, cnt);
      tot = __reduce_add_sync(kFull, tot);
      if (lane == 0) {
        atomicAdd(&msum[mpar][0], cnt);
        atomicAdd(&msum[mpar][1], tot);
      }
      __syncthreads();
      const bool major = 2ull * msum[mpar][0] > (unsigned long long)msum[mpar][1];
      if (!W && threadIdx.x == 0 && a.bb.has(v)) {  // the exact count of this step's input
        a.bb.lbl[v - a.bb.base] = cand;
        a.bb.lb[v - a.bb.base] = msum[mpar][0];
      }
      mpar ^= 1;  // the next vertex resets the other pair while this one is read
      if (major) {  // block-uniform
        if (threadIdx.x == 0) a.lout[v] = cand;
        continue;
      }
    }
    // a full-count step keeps no own-label count: the bounds go stale
    if (!W && mode == kModeFull && threadIdx.x == 0 && a.bb.has(v)) a.bb.lbl[v - a.bb.base] = -1;
    // two slots a neighbour (four, where a launch's table had room for them,
    // measured no faster in this tier)
    const uint32_t cap = min(pow2_ceil(2u * (uint32_t)(e - b)), C16 ? kBig16Slots : kBig32Slots);
    const uint32_t words = C16 ? cap + cap / 2 : 2 * cap;
    if (4ull * words > dynamic_smem_bytes()) {  // a planning error: report it, touch nothing (block-uniform)
      if (threadIdx.x == 0) atomicOr(a.err, kErrTable);
      continue;
    }
    uint32_t* keys = smem;
    uint32_t* vals = smem + cap;
    zero_words16(smem, words, threadIdx.x, NT);  // degree > 32: cap >= 128
    if (S::kPacked && threadIdx.x == 0) sbest[par] = 0ull;
    __syncthreads();
    std::conditional_t<S::kPacked, PackedCand, Best> best{};
    if constexpr (!S::kPacked) best = best_none();
    bool fail = false;
    auto ins = [&](uint32_t key, uint32_t k) {
      return CF ? table_claim_insert<C16>(keys, vals, cap - 1, key, k, cap)
                : table_insert_bounded<C16>(keys, vals, cap - 1, key, k, cap, nullptr, nullptr);
    };
    // the lane-0 fold pays off on listed vertices (few distinct labels) and
    // on the largest rows, where one label (a hub's own id, carried by its
    // degree-1 neighbours) fills many lanes of a chunk: without it those
    // lanes' adds to one slot serialise
    const bool merge = !CF || mode != kModeFull || (e - b) > kMergeDegree;
    for (int32_t j0 = b + warp * 32; j0 < e; j0 += 4 * NT) {
      int32_t lab[4], vl[4];
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + q * NT + lane;
        lab[q] = j < e ? ld_stream(a.cols + j) : -1;
        wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (lab[q] >= 0) score.load(a, lab[q], lab[q], vl[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + q * NT < e)
          count_chunk<W, S::kLV>(lab[q] >= 0, lab[q], wt[q], score, ins, best, fail, scan, vl[q], merge);
    }
    if (fail) atomicOr(a.err, kErrProbe);
    if (scan) {  // block-uniform
      __syncthreads();
      scan_table<C16, CF>(keys, vals, cap, threadIdx.x, NT, score, best);
    }
    int32_t lbest = 0;
    if constexpr (S::kPacked) {
      // (key << 32 | label) is monotone in (score, label)
      const unsigned long long wb = warp_best(best);
      if (lane == 0 && wb) atomicMax(&sbest[par], wb);
      __syncthreads();
      if (threadIdx.x == 0) lbest = (int32_t)(uint32_t)sbest[par];
      par ^= 1;
    } else {
      lbest = block_max<NT>(best, red).l;
    }
    if (threadIdx.x == 0) {
      a.lout[v] = lbest;
      if (lbest != cur) {
        cbuf[ncb++] = v;
        if (ncb == 64) flush_big_changes(a, cbuf, ncb);
      }
    }
  }
  if (threadIdx.x == 0) flush_big_changes(a, cbuf, ncb);
}

// ------------------------------------------------------- big tier, staged
// Full-count steps, degrees up to kStagedRow (one 256-thread block per
// vertex, at most four entries a thread): the row's column segment is staged
// in shared memory by one bulk copy (cp.async.bulk, completing on an
// mbarrier), issued one vertex ahead into the other of two buffers, so the
// next row's columns stream in while the block gathers and counts the
// current one -- without holding them in registers.  The copy takes the
// 16-byte-aligned superset of the row (the column array carries four pad
// entries past m).  Counting is k_big's: claim-first 16-bit table, packed
// candidates, no lane-0 fold (full-count rows of this range hold mostly
// distinct labels).  Every mbarrier wait is bounded (kErrWait); after one
// runs out a thread stops waiting, and at the end thread 0 waits, bounded,
// for the copy it issued last.
constexpr int32_t kStagedRow = 1024;
constexpr uint32_t kStagedBuf = (uint32_t)kStagedRow + 8;  // ints: the aligned superset of a row

template <int NT, class S>
__global__ void __launch_bounds__(NT, S::kSMThreads / NT) k_big_staged(StepArgs a, TierWork tw, S score) {
  static_assert(S::kPacked, "packed scores only");
  constexpr int ITEMS = kStagedRow / NT;
  extern __shared__ __align__(16) uint32_t smem[];  // table: 2*kStagedRow keys + their 16-bit counts
  __shared__ __align__(128) int32_t scol[2][kStagedBuf];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ unsigned long long sbest[2];
  __shared__ int32_t cbuf[64];
  uint32_t ncb = 0;
  const int lane = threadIdx.x & 31;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  if ((int32_t)blockIdx.x >= nwork) return;  // block-uniform, before any barrier exists
  const bool scan = S::kScan && scan_scores(a);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
    sbest[0] = sbest[1] = 0ull;
  }
  __syncthreads();
  // thread 0: stage the row of work item idx into buffer bi
  auto issue = [&](int32_t idx, int bi) {
    const int32_t u = tw.at(mode, idx);
    const int32_t lo = a.off[u] & ~3, hi = (a.off[u + 1] + 3) & ~3;
    const uint32_t bytes = (uint32_t)(hi - lo) * 4u;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bar[bi], bytes);
    bulk_copy_g2s(scol[bi], a.cols + lo, bytes, &bar[bi]);
  };
  if (threadIdx.x == 0) issue(blockIdx.x, 0);
  uint32_t ph[2] = {0u, 0u};
  bool waited_out = false;
  // thread 0 after a wait ran out: the copies it left in flight (buffer,
  // phase), waited for (bounded) before the block leaves; it issues no more
  int pend_b[2] = {-1, -1};
  uint32_t pend_p[2] = {0u, 0u};
  int bi = 0, par = 0;
  for (int32_t i = blockIdx.x; i < nwork; i += gridDim.x, bi ^= 1) {
    const int32_t v = tw.at(mode, i);
    const int32_t b = a.off[v], e = a.off[v + 1];
    const int32_t cur = a.lcur[v];
    if (threadIdx.x == 0 && a.bb.has(v)) a.bb.lbl[v - a.bb.base] = -1;  // a full-count step keeps no count
    const uint32_t cap = pow2_ceil(2u * (uint32_t)(e - b));
    uint32_t* keys = smem;
    uint32_t* vals = smem + cap;
    zero_words16(smem, cap + cap / 2, threadIdx.x, NT);  // degree > 32: cap >= 128
    if (threadIdx.x == 0) sbest[par] = 0ull;
    __syncthreads();  // every thread is done with the previous row and its buffer
    const bool next = threadIdx.x == 0 && !waited_out && i + (int32_t)gridDim.x < nwork;
    if (next) issue(i + gridDim.x, bi ^ 1);
    if (!waited_out && !mbar_wait_bounded(&bar[bi], ph[bi])) {
      waited_out = true;
      atomicOr(a.err, kErrWait);
      pend_b[0] = bi;
      pend_p[0] = ph[bi];
      if (next) {
        pend_b[1] = bi ^ 1;
        pend_p[1] = ph[bi ^ 1];
      }
    }
    ph[bi] ^= 1u;
    const int32_t lo = b & ~3;
    int32_t lab[ITEMS], vl[ITEMS];
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
      const int32_t j = b + q * NT + (int32_t)threadIdx.x;
      lab[q] = j < e ? scol[bi][j - lo] : -1;
    }
#pragma unroll
    for (int q = 0; q < ITEMS; ++q)
      if (lab[q] >= 0) score.load(a, lab[q], lab[q], vl[q]);
    PackedCand best{};
    bool fail = false;
    auto ins = [&](uint32_t key, uint32_t k) { return table_claim_insert<true>(keys, vals, cap - 1, key, k, cap); };
#pragma unroll
    for (int q = 0; q < ITEMS; ++q)
      if (b + q * NT + (threadIdx.x & ~31u) < (uint32_t)e)  // warp-uniform
        count_chunk<false, S::kLV>(lab[q] >= 0, lab[q], 1u, score, ins, best, fail, scan, vl[q], false);
    if (fail) atomicOr(a.err, kErrProbe);
    if (scan) {  // block-uniform
      __syncthreads();
      scan_table<true, true>(keys, vals, cap, threadIdx.x, NT, score, best);
    }
    const unsigned long long wb = warp_best(best);
    if (lane == 0 && wb) atomicMax(&sbest[par], wb);
    __syncthreads();
    if (threadIdx.x == 0) {
      const int32_t l = (int32_t)(uint32_t)sbest[par];
      a.lout[v] = l;
      if (l != cur) {
        cbuf[ncb++] = v;
        if (ncb == 64) flush_big_changes(a, cbuf, ncb);
      }
    }
    par ^= 1;
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; ++k)
      if (pend_b[k] >= 0) (void)mbar_wait_bounded(&bar[pend_b[k]], pend_p[k]);
    flush_big_changes(a, cbuf, ncb);
  }
}

// ----------------------------------------------------------------- hub tier
// Vertices above the big tier.  Hub h gets nb_h = ceil(3*deg/kHubTable) hash
// buckets, so a bucket averages at most kHubTable/3 labels and its distinct
// labels fit a shared table of kHubTable slots at most half full.  Every
// pass is its own launch; no block waits on another:
//   k_hub_majority : chunks add (own-label weight, total weight) per hub;
//   k_hub_decide   : a strict majority decides the hub (state 1);
//   k_hub_gather   : chunks of undecided hubs gather their labels (one random
//                    gather per edge) and count them per bucket;
//   k_hub_offsets  : per hub, bucket counts -> bucket starts (and cursors);
//   k_hub_scatter  : chunks place their labels bucket-contiguously;
//   k_hub_bucket   : one block per (hub, bucket) counts its own labels in a
//                    shared table and folds its (score, label) maximum into
//                    the hub's best (a bucket too large for the table is
//                    counted in exact hashed sub-passes);
//   k_hub_finalize : undecided hubs take their best label.
constexpr int kHubTable = 8192;  // shared slots per bucket block

struct HubPlan {
  const int32_t* chunk_hub;    // [nchunks] hub index of each chunk
  const int32_t* chunk_begin;  // [nchunks] first edge of the chunk
  const int32_t* chunk_end;    // [nchunks] one past the last edge
  const int32_t* hub_v;        // [nhubs] vertex id
  const int64_t* hub_lbase;    // [nhubs] first entry of the hub in the label scratch
  const int32_t* hub_nb;       // [nhubs] hash buckets
  const int32_t* hub_item0;    // [nhubs] first (hub, bucket) item of the hub
  const int32_t* item_hub;     // [nitems] (hub, bucket) work items
  const int32_t* item_bucket;
  int32_t* hlab;               // [labels] gathered labels (edge order)
  int32_t* hsort;              // [labels] labels in bucket order
  int32_t* hw;                 // [labels] weights in edge order (weighted graphs)
  int32_t* hsw;                // [labels] weights in bucket order (weighted graphs)
  uint32_t* bcnt;              // [nitems] labels per bucket
  uint32_t* bstart;            // [nitems] bucket start (relative to the hub)
  uint32_t* bcur;              // [nitems] scatter cursor
  int32_t nhubs, nitems, max_nb;
  unsigned long long* hub_best;  // [nhubs] packed best (0 = none)
  unsigned long long* hub_cand;  // [nhubs] (own-label weight << 32) + total weight
  uint32_t* hub_state;           // [nhubs] 0 = count exactly this step; 1 = decided by the majority pass
                                 // (or inactive); 2 = take the majority pass; 3 = decided by the count bound
  int32_t* hub_lbl;              // [nhubs] label whose count hub_lb bounds (-1: none)
  uint32_t* hub_lb;              // [nhubs] lower bound on that label's count among this step's input labels
};

// Bucket of a key: the high bits of its hash (table slots use the low bits).
__device__ __forceinline__ uint32_t hub_bucket_of(uint32_t key, uint32_t nb) {
  return (uint32_t)(((unsigned long long)fmix32(key) * nb) >> 32);
}

// Before the majority pass of a majority or frontier step: every hub that
// takes part gets state 2, unless the count bound decides it (state 3).
// The bound (unweighted classic steps, `use`): the majority pass of an
// earlier step counted label l = hub_lbl at c = hub_lb of the hub's
// neighbours; a step changes prev_changed labels in all, so l's count among
// the next step's input is at least c - prev_changed.  A hub still holding l
// whose bound is a strict majority keeps l without reading its row (exact:
// the majority argument holds for the bound, hence for the count).  Hubs
// that no changed vertex touches (frontier state 1) keep both their label
// and their count, so their bound stays as it is; a full step, whose hub
// counts are not kept, clears every bound.
template <bool W>
__global__ void k_hub_bound(StepArgs a, HubPlan hp, const unsigned long long* prev_changed, int use) {
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= hp.nhubs) return;
  const int32_t mode = step_mode(a);
  if (mode == kModeFull) {
    hp.hub_lbl[h] = -1;
    return;
  }
  if (mode == kModeFrontier && hp.hub_state[h] != 2u) return;
  uint32_t st = 2u;
  if (!W && use && prev_changed) {
    const int32_t v = hp.hub_v[h];
    const int32_t cand = a.lcur[v];
    if (hp.hub_lbl[h] == cand) {
      const unsigned long long chg = *prev_changed;
      const uint32_t lb0 = hp.hub_lb[h];
      const uint32_t lb = chg >= lb0 ? 0u : lb0 - (uint32_t)chg;
      const uint32_t d = (uint32_t)(a.off[v + 1] - a.off[v]);
      if (2ull * lb > d) {
        hp.hub_lb[h] = lb;
        a.lout[v] = cand;
        st = 3u;
      }
    }
  }
  hp.hub_state[h] = st;
}

template <int NT, bool W>
__global__ void __launch_bounds__(NT) k_hub_majority(StepArgs a, HubPlan hp, int32_t nchunks) {
  __shared__ uint32_t red[2][NT / 32];
  const int32_t mode = step_mode(a);
  if (mode == kModeFull) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int32_t h = hp.chunk_hub[c];
    if (hp.hub_state[h] != 2u) continue;  // block-uniform: inactive or decided by the bound
    const int32_t cand = a.lcur[hp.hub_v[h]];
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    uint32_t cnt = 0, tot = 0;
    for (int32_t j0 = cb + threadIdx.x; j0 < ce; j0 += 8 * NT) {
      int32_t col[8];
      uint32_t wt[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int32_t j = j0 + q * NT;
        col[q] = j < ce ? ld_stream(a.cols + j) : -1;
        wt[q] = j < ce ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int32_t l = col[q] >= 0 ? ld_label(a.lin + col[q]) : -1;
        cnt += l == cand ? wt[q] : 0u;
        tot += wt[q];
      }
    }
    cnt = __reduce_add_sync(kFull, cnt);
    tot = __reduce_add_sync(kFull, tot);
    if (lane == 0) {
      red[0][warp] = cnt;
      red[1][warp] = tot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long sc = 0, st = 0;
      for (int w2 = 0; w2 < NT / 32; ++w2) {
        sc += red[0][w2];
        st += red[1][w2];
      }
      atomicAdd(hp.hub_cand + h, (sc << 32) + st);
    }
    __syncthreads();
  }
}

// State after the step's majority pass: 1 = decided (or inactive), 0 = count
// exactly.  Outside full steps only hubs in state 2 took the pass; the
// others keep state 1 or 3.  The pass's count is kept for k_hub_bound.
__global__ void k_hub_decide(StepArgs a, HubPlan hp) {
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= hp.nhubs) return;
  const int32_t mode = step_mode(a);
  if (mode != kModeFull && hp.hub_state[h] != 2u) return;
  const int32_t v = hp.hub_v[h];
  bool major = false;
  if (mode != kModeFull) {
    const unsigned long long p = hp.hub_cand[h];
    hp.hub_cand[h] = 0ull;
    const uint32_t kc = (uint32_t)(p >> 32), kt = (uint32_t)(p & 0xffffffffull);
    major = 2ull * kc > (unsigned long long)kt;
    hp.hub_lbl[h] = a.lcur[v];
    hp.hub_lb[h] = kc;
  }
  if (major) a.lout[v] = a.lcur[v];
  hp.hub_state[h] = major ? 1u : 0u;
}

// Gathers the labels of undecided hubs and counts them per bucket
// (block-local histogram, one global add per nonzero bucket).
template <int NT, bool W>
__global__ void __launch_bounds__(NT) k_hub_gather(StepArgs a, HubPlan hp, int32_t nchunks) {
  extern __shared__ uint32_t hist[];  // [max_nb]
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int32_t h = hp.chunk_hub[c];
    if (hp.hub_state[h]) continue;  // block-uniform
    const uint32_t nb = (uint32_t)hp.hub_nb[h];
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    const int64_t base = hp.hub_lbase[h] - a.off[hp.hub_v[h]];
    for (uint32_t b = threadIdx.x; b < nb; b += NT) hist[b] = 0;
    __syncthreads();
    for (int32_t j0 = cb + threadIdx.x; j0 < ce; j0 += 4 * NT) {
      int32_t col[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) col[q] = j0 + q * NT < ce ? ld_stream(a.cols + j0 + q * NT) : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (col[q] < 0) continue;
        const int32_t j = j0 + q * NT;
        const int32_t l = ld_label(a.lin + col[q]);
        hp.hlab[base + j] = l;
        if (W) hp.hw[base + j] = ld_stream(a.w + j);
        atomicAdd(hist + (nb > 1 ? hub_bucket_of((uint32_t)l + 1u, nb) : 0u), 1u);
      }
    }
    __syncthreads();
    const int32_t item0 = hp.hub_item0[h];
    for (uint32_t b = threadIdx.x; b < nb; b += NT)
      if (hist[b]) atomicAdd(hp.bcnt + item0 + b, hist[b]);
    __syncthreads();
  }
}

// Bucket starts from the counts (exclusive scan per hub); counts stay.
__global__ void k_hub_offsets(HubPlan hp) {
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= hp.nhubs || hp.hub_state[h]) return;
  const int32_t item0 = hp.hub_item0[h], nb = hp.hub_nb[h];
  uint32_t run = 0;
  for (int32_t b = 0; b < nb; ++b) {
    hp.bstart[item0 + b] = run;
    hp.bcur[item0 + b] = run;
    run += hp.bcnt[item0 + b];
  }
}

// Places the gathered labels bucket-contiguously: a block counts its labels
// per bucket, reserves each bucket's range with one global add, then every
// label takes a slot of its bucket's range.
template <int NT, bool W>
__global__ void __launch_bounds__(NT) k_hub_scatter(StepArgs a, HubPlan hp, int32_t nchunks) {
  extern __shared__ uint32_t sh[];  // [max_nb] counts, then [max_nb] cursors
  uint32_t* cnt = sh;
  uint32_t* cur = sh + hp.max_nb;
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int32_t h = hp.chunk_hub[c];
    if (hp.hub_state[h]) continue;  // block-uniform
    const uint32_t nb = (uint32_t)hp.hub_nb[h];
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    const int64_t lb = hp.hub_lbase[h];
    const int64_t base = lb - a.off[hp.hub_v[h]];
    const int32_t item0 = hp.hub_item0[h];
    for (uint32_t b = threadIdx.x; b < nb; b += NT) cnt[b] = 0;
    __syncthreads();
    for (int32_t j = cb + threadIdx.x; j < ce; j += NT) {
      const int32_t l = hp.hlab[base + j];
      atomicAdd(cnt + (nb > 1 ? hub_bucket_of((uint32_t)l + 1u, nb) : 0u), 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nb; b += NT) cur[b] = cnt[b] ? atomicAdd(hp.bcur + item0 + b, cnt[b]) : 0u;
    __syncthreads();
    for (int32_t j = cb + threadIdx.x; j < ce; j += NT) {
      const int32_t l = hp.hlab[base + j];
      const uint32_t b = nb > 1 ? hub_bucket_of((uint32_t)l + 1u, nb) : 0u;
      const uint32_t pos = atomicAdd(cur + b, 1u);
      hp.hsort[lb + pos] = l;
      if (W) hp.hsw[lb + pos] = hp.hw[base + j];
    }
    __syncthreads();
  }
}

// One block per (hub, bucket): exact count of the bucket's labels in one
// pass; if its distinct labels overflow the table (an insert gives up after
// kHubProbe probes), the bucket is recounted in 2, 4, ... hashed sub-passes.
constexpr uint32_t kHubProbe = 64;

template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_hub_bucket(StepArgs a, HubPlan hp, S score) {
  const bool scan = S::kScan && scan_scores(a);
  extern __shared__ __align__(16) uint32_t hsm[];
  __shared__ Best red[32];
  __shared__ int overflow;
  for (int32_t it = blockIdx.x; it < hp.nitems; it += gridDim.x) {
    const int32_t h = hp.item_hub[it];
    if (hp.hub_state[h]) continue;  // block-uniform
    const uint32_t size = hp.bcnt[it];
    const int64_t beg = hp.hub_lbase[h] + hp.bstart[it];
    Best best = best_none();
    for (uint32_t nsub = 1;; nsub *= 2) {
      best = best_none();
      if (threadIdx.x == 0) overflow = 0;
      const uint32_t cap = nsub > 1 ? (uint32_t)kHubTable
                                    : (size * 2u < (uint32_t)kHubTable ? pow2_ceil(2u * (size ? size : 1u))
                                                                        : (uint32_t)kHubTable);
      for (uint32_t sub = 0; sub < nsub; ++sub) {
        uint32_t* keys = hsm;
        uint32_t* vals = hsm + cap;
        zero_words16(hsm, 2 * cap, threadIdx.x, NT);  // cap >= 2
        __syncthreads();
        bool fail = false;
        auto ins = [&](uint32_t key, uint32_t k) {
          return table_insert_bounded(keys, vals, cap - 1, key, k, kHubProbe, nullptr, nullptr);
        };
        // warp-uniform trip count: the lanes of a warp read 32 consecutive labels
        for (uint32_t k0 = threadIdx.x & ~31u; k0 < size; k0 += 4 * NT) {
          int32_t l[4];
          uint32_t wt[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t k = k0 + q * NT + (threadIdx.x & 31);
            l[q] = k < size ? __ldcg(hp.hsort + beg + k) : -1;
            wt[q] = k < size ? (W ? (uint32_t)__ldcg(hp.hsw + beg + k) : 1u) : 0u;
            // sub-pass filter: another hash of the key (bucket bits are high bits)
            if (nsub > 1 && l[q] >= 0 && (fmix32(((uint32_t)l[q] + 1u) ^ 0x2545f491u) & (nsub - 1)) != sub) l[q] = -1;
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (k0 + q * NT < size) count_chunk<W>(l[q] >= 0, l[q], wt[q], score, ins, best, fail, scan);
        }
        if (fail) overflow = 1;
        __syncthreads();
        if (overflow) break;  // block-uniform
        if (scan) {  // block-uniform
          scan_table(keys, vals, cap, threadIdx.x, NT, score, best);
          __syncthreads();  // the next sub-pass clears the table
        }
      }
      if (!overflow) break;
      if (nsub >= 1024u) {  // cannot happen for int32 sizes; stop rather than loop
        if (threadIdx.x == 0) atomicOr(a.err, kErrProbe);
        break;
      }
    }
    best = block_max<NT>(best, red);
    if (threadIdx.x == 0 && best.l >= 0) atomicMax(hp.hub_best + h, pack_best(best, a.err));
    __syncthreads();
  }
}

__global__ void k_hub_finalize(StepArgs a, HubPlan hp) {
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= hp.nhubs) return;
  if (hp.hub_state[h]) return;
  const unsigned long long p = hp.hub_best[h];
  hp.hub_best[h] = 0ull;
  const int32_t v = hp.hub_v[h];
  const int32_t l = p ? (int32_t)(uint32_t)(p & 0xffffffffull) : a.lcur[v];
  if (!p) atomicOr(a.err, kErrHubPlan);
  a.lout[v] = l;
  if (l != a.lcur[v]) record_change(a, v);
}

// ------------------------------------------------- two-step cycle detection
// Synchronous LP on a symmetric graph often ends in a cycle of two labelings
// (L_{t+1} = L_{t-1} for every vertex): a few vertices flip between two
// labels for ever.  Once a step ends in that cycle every later labeling is
// known exactly, so a run can stop there.  With S_t the vertices step t
// changes (L_{t+1}(v) != L_t(v)), L_{t+1} = L_{t-1} holds iff S_t = S_{t-1}
// and every v in S_t returns to L_{t-1}(v).  k_cycle_save keeps L_{t-1}(v)
// for v in S_{t-1} before step t overwrites it; k_cycle_check compares after
// the step; k_cycle_verdict publishes the answer to the host.  The lists are
// walked only while they are short (at most `cap` entries); a longer list
// marks the step as not cyclic.
__global__ void k_cycle_save(const int32_t* __restrict__ chg_prev, const uint32_t* n_prev, uint32_t cap,
                             const int32_t* __restrict__ lab_prev2, int32_t* __restrict__ old,
                             uint32_t* __restrict__ stamp, uint32_t tag, uint32_t* mism) {
  const uint32_t c = *n_prev;
  if (c > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(mism, 1u);
    return;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const int32_t v = chg_prev[i];
    old[v] = lab_prev2[v];
    stamp[v] = tag;
  }
}

__global__ void k_cycle_check(const int32_t* __restrict__ chg, const uint32_t* n_now, const uint32_t* n_prev,
                              uint32_t cap, const int32_t* __restrict__ lab_next, const int32_t* __restrict__ old,
                              const uint32_t* __restrict__ stamp, uint32_t tag, uint32_t* mism) {
  const uint32_t c = *n_now;
  if (c != *n_prev || c > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(mism, 1u);
    return;
  }
  bool bad = false;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const int32_t v = chg[i];
    bad |= stamp[v] != tag || lab_next[v] != old[v];
  }
  if (__any_sync(kFull, bad) && (threadIdx.x & 31) == 0) atomicOr(mism, 1u);
}

// flag: host-mapped word; 1 = the step ended in a two-step cycle.
__global__ void k_cycle_verdict(const uint32_t* mism, volatile uint32_t* flag) {
  *flag = *mism == 0u ? 1u : 0u;
  __threadfence_system();
}

// ------------------------------------------------------- first-step shortcut
// Before the first step every label is its vertex id.  When every row lists
// strictly ascending columns (no repeated neighbour), every neighbour label
// occurs once, so all counts are 1 and the tie rule picks the largest label:
// the row's last column.  Exact for classic LP and the SLPA listener
// (unweighted).
__global__ void __launch_bounds__(256) k_first_step(StepArgs a) {
  for (int32_t v0 = blockIdx.x * blockDim.x; v0 < a.n; v0 += gridDim.x * blockDim.x) {
    const int32_t v = v0 + threadIdx.x;
    bool chg = false;
    if (v < a.n) {
      const int32_t e = a.off[v + 1];
      if (e > a.off[v]) {
        const int32_t l = a.lin[a.cols[e - 1]];
        a.lout[v] = l;
        chg = l != a.lcur[v];
      }
    }
    record_changes(a, chg, v);
  }
}

// The weighted form of the same shortcut: every neighbour label occurs once,
// so its count is the edge's weight, and the step takes the neighbour label
// of largest (weight, label).  G lanes per vertex (1 or 32); the rows of the
// big tier and the hubs go to k_first_step_w_block.  The key of an entry is
// a 64-bit word monotone in (score, label) and never 0 for a candidate.
struct FirstKeyW {
  __device__ __forceinline__ unsigned long long operator()(const StepArgs& a, int32_t j) const {
    return ((unsigned long long)(uint32_t)a.w[j] << 32) | (uint32_t)a.lin[a.cols[j]];
  }
};
// Layered LP at the start of a layer: every label is its vertex id and
// occurs once, so neighbour c of edge weight k (1 unweighted) scores
// dstar*k - vol_r[c], in 32 bits (the host checks the range) and packed as
// ScoreLayered32::pack does.  No label gather: the label is the column.
template <bool W>
struct FirstKeyLayered {
  const int32_t* vol;
  int32_t dstar;
  __device__ __forceinline__ unsigned long long operator()(const StepArgs& a, int32_t j) const {
    const int32_t l = ld_stream(a.cols + j);
    const int32_t k = W ? ld_stream(a.w + j) : 1;
    const int32_t sc = dstar * k - __ldg(vol + l);
    return ((unsigned long long)((uint32_t)sc ^ 0x80000000u) << 32) | (uint32_t)l;
  }
};
template <int G, class K = FirstKeyW>
__global__ void __launch_bounds__(256) k_first_step_w(StepArgs a, Verts vs, K key = K{}) {
  const int lane = threadIdx.x & (G - 1);
  for (int64_t t0 = (int64_t)blockIdx.x * blockDim.x; t0 < (int64_t)vs.n * G; t0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = (t0 + threadIdx.x) / G;
    bool chg = false;
    int32_t v = 0;
    unsigned long long best = 0ull;
    if (i < vs.n) {
      v = vs[i];
      const int32_t b = a.off[v], e = a.off[v + 1];
      if (G == 1) {
        // eight entries a round, their loads in flight together
        for (int32_t j0 = b; j0 < e; j0 += 8) {
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (j0 + q < e) best = max(best, key(a, j0 + q));
        }
      } else {
        for (int32_t j = b + lane; j < e; j += G) best = max(best, key(a, j));
      }
    }
#pragma unroll
    for (int m = G / 2; m >= 1; m >>= 1) best = max(best, __shfl_xor_sync(kFull, best, m));
    if (i < vs.n && lane == 0 && a.off[v + 1] > a.off[v]) {
      const int32_t l = (int32_t)(uint32_t)best;
      a.lout[v] = l;
      chg = l != a.lcur[v];
    }
    record_changes(a, chg, v);
  }
}
template <int NT, class K = FirstKeyW>
__global__ void __launch_bounds__(NT) k_first_step_w_block(StepArgs a, Verts vs, K key = K{}) {
  __shared__ unsigned long long sb;
  for (int32_t i = blockIdx.x; i < vs.n; i += gridDim.x) {
    const int32_t v = vs[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
    if (threadIdx.x == 0) sb = 0ull;
    __syncthreads();
    unsigned long long best = 0ull;
    for (int32_t j = b + threadIdx.x; j < e; j += NT) best = max(best, key(a, j));
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) best = max(best, __shfl_xor_sync(kFull, best, m));
    if ((threadIdx.x & 31) == 0) atomicMax(&sb, best);
    __syncthreads();
    if (threadIdx.x == 0 && e > b) {
      const int32_t l = (int32_t)(uint32_t)sb;
      a.lout[v] = l;
      if (l != a.lcur[v]) record_change(a, v);
    }
    __syncthreads();  // sb is reset for the next vertex
  }
}

// bad |= 1 when some row is not strictly ascending.  One warp per row, 8
// column pairs in flight per lane.
__global__ void __launch_bounds__(256) k_check_sorted(const int32_t* __restrict__ off,
                                                      const int32_t* __restrict__ cols, int32_t n, uint32_t* bad) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
    const int32_t b = off[v], e = off[v + 1];
    bool ok = true;
    for (int32_t j0 = b + 1 + lane; j0 < e; j0 += 256) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int32_t j = j0 + 32 * q;
        if (j < e && ld_stream(cols + j - 1) >= ld_stream(cols + j)) ok = false;
      }
    }
    if (__any_sync(kFull, !ok) && lane == 0) atomicOr(bad, 1u);
  }
}

// ----------------------------------------------------------- frontier mode
// A vertex's new label is a function of its neighbours' labels; if none of
// them changed in the previous step the result is its current label.  On a
// symmetric CSR (every edge stored both ways) the vertices to recompute are
// exactly the neighbours of the vertices that changed.  The previous step
// listed its changed vertices (chg_in); marks carry this step's epoch, so
// nothing is ever cleared.  The output buffer already holds the labels of
// two steps back, which equal the current ones except for chg_in: those that
// are not recomputed are copied.  No pass touches all n vertices.
struct Frontier {
  uint32_t* act;           // [n] epoch of the last step that marked the vertex
  uint32_t epoch;          // this step's mark (unique per step of the handle)
  const int32_t* chg_in;   // vertices changed in the previous step
  const uint32_t* chg_in_n;
  int32_t tiny_max, mid_max, big_max;
  FailList tier[5];        // frontier members of tiny, g16, g32, mid, big
};

// One warp per changed vertex marks its neighbours; the first marker of a
// vertex lists it in its tier (hubs are picked up by k_frontier_hubs).
__global__ void __launch_bounds__(256) k_frontier_push(StepArgs a, Frontier f) {
  if (step_mode(a) != kModeFrontier) return;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t nc = *f.chg_in_n;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += nw) {
    const int32_t u = f.chg_in[i];
    const int32_t b = a.off[u], e = a.off[u + 1];
    for (int32_t j0 = b; j0 < e; j0 += 32) {
      const int32_t j = j0 + lane;
      int tier = -1;
      int32_t x = 0;
      if (j < e) {
        x = ld_stream(a.cols + j);
        if (a.bb.has(x)) atomicAdd(a.bb.nchg + (x - a.bb.base), 1u);
        if (atomicExch(f.act + x, f.epoch) != f.epoch) {
          const int32_t d = a.off[x + 1] - a.off[x];
          tier = d <= f.tiny_max ? 0 : d <= 16 ? 1 : d <= 32 ? 2 : d <= f.mid_max ? 3 : d <= f.big_max ? 4 : -1;
        }
      }
#pragma unroll
      for (int t = 0; t < 5; ++t) {
        const uint32_t m = __ballot_sync(kFull, tier == t);
        if (!m) continue;
        uint32_t base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(f.tier[t].count, (uint32_t)__popc(m));
        base = __shfl_sync(kFull, base, __ffs(m) - 1);
        if (tier == t) f.tier[t].ids[base + __popc(m & ((1u << lane) - 1u))] = x;
      }
    }
  }
}

// Changed vertices that are not recomputed keep their (new) label.
__global__ void __launch_bounds__(256) k_frontier_copy(StepArgs a, Frontier f) {
  if (step_mode(a) != kModeFrontier) return;
  const uint32_t nc = *f.chg_in_n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = f.chg_in[i];
    if (f.act[v] != f.epoch) a.lout[v] = a.lin[v];
  }
}

// Marked hubs go through the majority check (state 2), unmarked ones are
// done (state 1).
__global__ void k_frontier_hubs(StepArgs a, Frontier f, HubPlan hp) {
  if (step_mode(a) != kModeFrontier) return;
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h < hp.nhubs) hp.hub_state[h] = f.act[hp.hub_v[h]] == f.epoch ? 2u : 1u;
}

// Symmetry check of a CSR with strictly ascending rows, one thread per edge:
// every (v, u) needs (u, v).  bad |= 1 for an unsorted row, 2 for a missing
// reverse edge.
__global__ void k_check_symmetric(const int32_t* __restrict__ off, const int32_t* __restrict__ cols, int32_t n,
                                  int64_t m, uint32_t* bad) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {  // the row of edge j: last v with off[v] <= j
      const int32_t mid = (int32_t)(((int64_t)lo + hi + 1) >> 1);
      if (off[mid] <= j) lo = mid; else hi = mid - 1;
    }
    const int32_t v = lo, u = cols[j];
    if (j > off[v] && cols[j - 1] >= u) {
      atomicOr(bad, 1u);
      continue;
    }
    int32_t a = off[u], b = off[u + 1] - 1;
    bool found = false;
    while (a <= b) {
      const int32_t mid = (a + b) >> 1;
      const int32_t x = cols[mid];
      if (x == v) {
        found = true;
        break;
      }
      if (x < v) a = mid + 1; else b = mid - 1;
    }
    if (!found) atomicOr(bad, 2u);
  }
}

// --------------------------------------------------------- layered volumes
// vol[l] += #vertices whose label is l (warp-aggregated atomics).
// Lanes holding lane 0's label add once for all (hot labels of converged
// communities); the others add directly.
__global__ void __launch_bounds__(256) k_histogram(const int32_t* __restrict__ lab, int32_t n, int32_t* vol) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t l = v < n ? lab[v] : -1;
  const int32_t l0 = __shfl_sync(kFull, l, 0);
  const uint32_t m0 = __ballot_sync(kFull, l == l0);
  if (l < 0) return;
  if (l != l0) atomicAdd(vol + l, 1);
  else if ((threadIdx.x & 31) == 0) atomicAdd(vol + l, __popc(m0));
}

// lv[v] = (lab[v], vol[lab[v]]): the pairs the next layered step gathers,
// one 8-byte load per neighbour (ScoreLayered32::load).
__global__ void __launch_bounds__(256) k_label_volumes(const int32_t* __restrict__ lab, const int32_t* __restrict__ vol,
                                                       int32_t n, int2* __restrict__ lv) {
  for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int32_t l = lab[v];
    lv[v] = make_int2(l, __ldg(vol + l));
  }
}

// ------------------------------------------------------------------- SLPA
// Store the current label into the speaker memory and pick the spoken label
// (tutorial/Base5prop.cuh:161-208).  Every vertex stores once per iteration,
// so all memories fill alike: before the store of iteration `it` the filled
// slots are [T-min(it,T), T); the store goes to the last empty slot T-1-it,
// or slot 0 once full.  The cyclic scan from h = H(seed,it,v) mod T to the
// first non-empty slot then lands on max(h, T-f) with f = min(it+1, T).
// mem is slot-major [T][n].
__global__ void __launch_bounds__(256) k_slpa_speak(const int32_t* __restrict__ lab, int32_t* __restrict__ mem,
                                                    int32_t* __restrict__ spoken, int32_t n, int32_t T, int32_t it,
                                                    uint64_t seed) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t pos = it < T ? T - 1 - it : 0;
  const int32_t cur = lab[v];
  mem[(int64_t)pos * n + v] = cur;
  const int32_t f = it + 1 < T ? it + 1 : T;
  const int32_t h = (int32_t)(slpa_hash(seed, (uint32_t)it, (uint32_t)v) % (uint64_t)T);
  const int32_t pick = h >= T - f ? h : T - f;
  spoken[v] = pick == pos ? cur : mem[(int64_t)pick * n + v];
}

// Post-processing (Xie et al. 2011): keep labels whose memory frequency is
// >= r of the filled slots; ascending, -1 padded.  comm is [n][T].
template <int TMAXP>
__global__ void __launch_bounds__(128) k_slpa_post(const int32_t* __restrict__ mem, int32_t n, int32_t T, double r,
                                                   int32_t* __restrict__ comm, int32_t* __restrict__ ncomm) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  int32_t x[TMAXP];
  int filled = 0;
  for (int s = 0; s < T; ++s) {
    const int32_t y = mem[(int64_t)s * n + v];
    if (y != -1) x[filled++] = y;
  }
  for (int i = 1; i < filled; ++i) {  // insertion sort, at most 64 entries
    const int32_t y = x[i];
    int j = i - 1;
    while (j >= 0 && x[j] > y) {
      x[j + 1] = x[j];
      --j;
    }
    x[j + 1] = y;
  }
  int k = 0;
  int i = 0;
  while (i < filled) {
    int j = i;
    while (j < filled && x[j] == x[i]) ++j;
    if ((double)(j - i) >= r * (double)filled) comm[(int64_t)v * T + k++] = x[i];
    i = j;
  }
  if (ncomm) ncomm[v] = k;
  for (int s = k; s < T; ++s) comm[(int64_t)v * T + s] = -1;
}

__global__ void k_iota(int32_t* __restrict__ a, int32_t* __restrict__ b, int32_t n) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    a[v] = v;
    if (b) b[v] = v;
  }
}

}  // namespace glp
