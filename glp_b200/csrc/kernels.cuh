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
//   big   (257..4096)  : one block per vertex, block shared-memory table
//   hub   (> 4096)     : labels gathered once, then counted per hash bucket,
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
#include "device.cuh"

namespace glp {

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
  // majority pre-pass switch: on when prev_changed is set and the previous
  // step changed fewer than n/20 labels
  const unsigned long long* prev_changed;
  int32_t n;
};

__device__ __forceinline__ bool use_majority(const StepArgs& a) {
  return a.prev_changed != nullptr && (*a.prev_changed) * 20ull < (unsigned long long)a.n;
}

// The vertices of one tier: explicit ids, or the contiguous range
// [base, base+n) (degree-sorted graphs make every tier contiguous).
struct Verts {
  const int32_t* ids;
  int32_t base;
  int32_t n;
  __device__ __forceinline__ int32_t operator[](int64_t i) const { return ids ? ids[i] : base + (int32_t)i; }
};

// Vertices the majority pre-pass could not decide.
struct FailList {
  int32_t* ids;
  uint32_t* count;
};

// The work of an exact-count kernel: its tier, or the tier's fail list when
// the pre-pass ran.
__device__ __forceinline__ int32_t work_size(const StepArgs& a, const Verts& vs, const FailList& fl, bool* listed) {
  *listed = use_majority(a);
  return *listed ? (int32_t)*fl.count : vs.n;
}

// score(l, k) for classic LP: the count itself.  A label holding more than
// half of the neighbourhood weight is then the unique maximum, so the
// majority shortcut applies.
struct ScoreClassic {
  static constexpr bool kMajority = true;
  __device__ __forceinline__ int64_t operator()(int32_t, uint32_t k) const { return (int64_t)k; }
};

// score(l, k) for layered LP: dstar*k - vol_r[l] (kernel.cuh:2575-2600).
// The volume term breaks the majority argument: no shortcut.
struct ScoreLayered {
  static constexpr bool kMajority = false;
  const int32_t* vol;
  int64_t dstar;
  __device__ __forceinline__ int64_t operator()(int32_t l, uint32_t k) const {
    return dstar * (int64_t)k - (int64_t)__ldg(vol + l);
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
__global__ void __launch_bounds__(256) k_tiny(StepArgs a, Verts vs, S score) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  bool chg = false;
  if (t < vs.n) {
    const int32_t v = vs[t];
    const int32_t b = a.off[v];
    const int32_t d = a.off[v + 1] - b;
    int32_t lab[TMAX];
    uint32_t wt[TMAX];
#pragma unroll
    for (int i = 0; i < TMAX; ++i) {
      lab[i] = -1;
      wt[i] = 0;
      if (i < d) load_edge<W>(a, (int64_t)b + i, lab[i], wt[i]);
    }
    Best best = best_none();
#pragma unroll
    for (int i = 0; i < TMAX; ++i) {
      if (i < d) {
        uint32_t k = 0;
#pragma unroll
        for (int j = 0; j < TMAX; ++j) k += (lab[j] == lab[i]) ? wt[j] : 0u;
        const Best c{score(lab[i], k), lab[i]};
        if (better(c, best)) best = c;
      }
    }
    a.lout[v] = best.l;
    chg = best.l != a.lcur[v];
  }
  warp_count_add(a.changed, chg);
}

// --------------------------------------------------------------- group tier
// G lanes per vertex (degree <= G); each warp handles U rounds of 32/G
// vertices with all loads issued before any counting.  The match key carries
// the group index so equal labels of different vertices do not merge.
template <int G, int U, bool W, class S>
__global__ void __launch_bounds__(256) k_group(StepArgs a, Verts vs, S score) {
  constexpr int PER = 32 / G;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int32_t v[U], lab[U];
  uint32_t wt[U];
  bool act[U], has[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int64_t grp = (warp * U + u) * PER + lane / G;
    act[u] = grp < vs.n;
    has[u] = false;
    v[u] = 0;
    wt[u] = 0;
    int32_t col = 0;
    if (act[u]) {
      v[u] = vs[grp];
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
    if (act[u] && (lane & (G - 1)) == 0) {
      a.lout[v[u]] = c.l;
      chg += c.l != a.lcur[v[u]];
    }
  }
  warp_count_add(a.changed, chg);
}

// Count one 32-edge chunk: lanes with equal labels are merged by
// __match_any_sync and their leader adds the group's count to the table.
template <bool W, class S, class Ins>
__device__ __forceinline__ void count_chunk(bool has, int32_t lab, uint32_t wt, const S& score, const Ins& insert,
                                            Best& best, bool& fail) {
  const int lane = threadIdx.x & 31;
  const uint32_t m = __match_any_sync(kFull, (uint32_t)lab);
  const uint32_t k = W ? __reduce_add_sync(m, wt) : (uint32_t)__popc(m);
  if (has && lane == __ffs(m) - 1) {
    const uint32_t tot = insert((uint32_t)lab + 1u, k);
    if (tot == kNoSlot) {
      fail = true;
    } else {
      const Best c{score(lab, tot), lab};
      if (better(c, best)) best = c;
    }
  }
}

// ---------------------------------------------------- majority pre-pass
// One warp per vertex of degree 33..4096: count the weight of the vertex's
// own label with 4 independent column/label loads in flight per lane.  A
// strict majority is written; other vertices go to the mid or big fail list.
template <bool W>
__global__ void __launch_bounds__(256) k_major_warp(StepArgs a, Verts vs, int32_t mid_max, FailList fmid,
                                                    FailList fbig) {
  if (!use_majority(a)) return;
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = gw; i < vs.n; i += nw) {
    const int32_t v = vs[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
    const int32_t cand = a.lcur[v];
    uint32_t cnt = 0, tot = 0;
    for (int32_t j0 = b + lane; j0 < e; j0 += 128) {
      int32_t c[4];
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + 32 * q;
        c[q] = j < e ? ld_stream(a.cols + j) : -1;
        wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t l = c[q] >= 0 ? ld_label(a.lin + c[q]) : -1;
        cnt += l == cand ? wt[q] : 0u;
        tot += wt[q];
      }
    }
    cnt = __reduce_add_sync(kFull, cnt);
    tot = W ? __reduce_add_sync(kFull, tot) : (uint32_t)(e - b);
    if (lane == 0) {
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
template <int CAP, int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_mid(StepArgs a, Verts vs, FailList fl, S score) {
  constexpr int NW = NT / 32;
  __shared__ uint32_t skeys[NW][CAP];
  __shared__ uint32_t svals[NW][CAP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool listed;
  const int32_t nwork = work_size(a, vs, fl, &listed);
  uint32_t* kk = skeys[warp];
  uint32_t* vv = svals[warp];
  for (int32_t i = blockIdx.x * NW + warp; i < nwork; i += gridDim.x * NW) {
    const int32_t v = listed ? fl.ids[i] : vs[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
    const uint32_t cap = pow2_ceil(2u * (uint32_t)(e - b));
    for (uint32_t s = lane; s < cap; s += 32) {
      kk[s] = 0;
      vv[s] = 0;
    }
    __syncwarp();
    Best best = best_none();
    bool fail = false;
    auto ins = [&](uint32_t key, uint32_t k) {
      return table_insert_bounded(kk, vv, cap - 1, key, k, cap, nullptr, nullptr);
    };
    for (int32_t j0 = b; j0 < e; j0 += 128) {
      int32_t lab[4];
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + 32 * q + lane;
        lab[q] = j < e ? ld_stream(a.cols + j) : -1;
        wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (lab[q] >= 0) lab[q] = ld_label(a.lin + lab[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + 32 * q < e) count_chunk<W>(lab[q] >= 0, lab[q], wt[q], score, ins, best, fail);
    }
    if (fail) atomicOr(a.err, kErrProbe);
    best = group_max<32>(best);
    bool chg = false;
    if (lane == 0) {
      a.lout[v] = best.l;
      chg = best.l != a.lcur[v];
    }
    warp_count_add(a.changed, chg);
    __syncwarp();
  }
}

// ----------------------------------------------------------------- big tier
// Exact count, one block per vertex (degree <= CAP/2): block shared table
// (dynamic, CAP slots) sized per vertex to the power of two >= 2*degree.
template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_big(StepArgs a, Verts vs, FailList fl, S score) {
  extern __shared__ uint32_t smem[];
  __shared__ Best red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool listed;
  const int32_t nwork = work_size(a, vs, fl, &listed);
  for (int32_t i = blockIdx.x; i < nwork; i += gridDim.x) {
    const int32_t v = listed ? fl.ids[i] : vs[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
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
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + q * NT + lane;
        lab[q] = j < e ? ld_stream(a.cols + j) : -1;
        wt[q] = j < e ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (lab[q] >= 0) lab[q] = ld_label(a.lin + lab[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + q * NT < e) count_chunk<W>(lab[q] >= 0, lab[q], wt[q], score, ins, best, fail);
    }
    if (fail) atomicOr(a.err, kErrProbe);
    best = block_max<NT>(best, red);
    if (threadIdx.x == 0) {
      a.lout[v] = best.l;
      if (best.l != a.lcur[v]) atomicAdd(a.changed, 1ull);
    }
  }
}

// ----------------------------------------------------------------- hub tier
// Vertices above the big tier.  Each hub h has P_h hash buckets (about
// kHubBucket labels each).  Every pass is its own launch; no block waits on
// another:
//   k_hub_majority : chunks add (own-label weight, total weight) per hub;
//   k_hub_decide   : a strict majority decides the hub (state 1);
//   k_hub_gather   : chunks of undecided hubs gather their labels into a
//                    compact scratch array (one random gather per edge);
//   k_hub_bucket   : one block per (hub, bucket) streams the hub's gathered
//                    labels, counts those hashing to its bucket in a shared
//                    table (at most twice the expected size), and folds its
//                    (score, label) maximum into the hub's best;
//   k_hub_finalize : undecided hubs take their best label.
constexpr int kHubBucket = 8192;           // target labels per bucket
constexpr int kHubTable = 2 * kHubBucket;  // shared slots per bucket block

struct HubPlan {
  const int32_t* chunk_hub;    // [nchunks] hub index of each chunk
  const int32_t* chunk_begin;  // [nchunks] first edge of the chunk
  const int32_t* chunk_end;    // [nchunks] one past the last edge
  const int32_t* hub_v;        // [nhubs] vertex id
  const int64_t* hub_lbase;    // [nhubs] first entry of the hub in the label scratch
  const int32_t* hub_nb;       // [nhubs] hash buckets
  const int32_t* item_hub;     // [nitems] (hub, bucket) work items
  const int32_t* item_bucket;
  int32_t* hlab;               // gathered labels of undecided hubs
  int32_t nhubs, nitems;
  unsigned long long* hub_best;  // [nhubs] packed best (0 = none)
  unsigned long long* hub_cand;  // [nhubs] (own-label weight << 32) + total weight
  uint32_t* hub_state;           // [nhubs] 1 = decided by the majority pass this step
};

// Bucket of a key (high bits of one hash) and its table slot (another hash).
__device__ __forceinline__ uint32_t hub_bucket_of(uint32_t key, uint32_t nb) {
  return (uint32_t)(((unsigned long long)fmix32(key) * nb) >> 32);
}
__device__ __forceinline__ uint32_t hub_slot_of(uint32_t key) { return fmix32(key ^ 0x9e3779b9u); }

template <int NT, bool W>
__global__ void __launch_bounds__(NT) k_hub_majority(StepArgs a, HubPlan hp, int32_t nchunks) {
  __shared__ uint32_t red[2][NT / 32];
  if (!use_majority(a)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int32_t h = hp.chunk_hub[c];
    const int32_t cand = a.lcur[hp.hub_v[h]];
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    uint32_t cnt = 0, tot = 0;
    for (int32_t j0 = cb + threadIdx.x; j0 < ce; j0 += 4 * NT) {
      int32_t col[4];
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t j = j0 + q * NT;
        col[q] = j < ce ? ld_stream(a.cols + j) : -1;
        wt[q] = j < ce ? (W ? (uint32_t)ld_stream(a.w + j) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
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

__global__ void k_hub_decide(StepArgs a, HubPlan hp) {
  const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= hp.nhubs) return;
  bool major = false;
  if (use_majority(a)) {
    const unsigned long long p = hp.hub_cand[h];
    hp.hub_cand[h] = 0ull;
    const uint32_t kc = (uint32_t)(p >> 32), kt = (uint32_t)(p & 0xffffffffull);
    major = 2ull * kc > (unsigned long long)kt;
  }
  const int32_t v = hp.hub_v[h];
  if (major) a.lout[v] = a.lcur[v];
  hp.hub_state[h] = major ? 1u : 0u;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_hub_gather(StepArgs a, HubPlan hp, int32_t nchunks) {
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int32_t h = hp.chunk_hub[c];
    if (hp.hub_state[h]) continue;  // block-uniform
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    const int64_t base = hp.hub_lbase[h] - a.off[hp.hub_v[h]];
    for (int32_t j0 = cb + threadIdx.x; j0 < ce; j0 += 4 * NT) {
      int32_t col[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) col[q] = j0 + q * NT < ce ? ld_stream(a.cols + j0 + q * NT) : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (col[q] >= 0) hp.hlab[base + j0 + q * NT] = ld_label(a.lin + col[q]);
    }
  }
}

template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_hub_bucket(StepArgs a, HubPlan hp, S score) {
  extern __shared__ uint32_t smem[];
  uint32_t* keys = smem;
  uint32_t* vals = smem + kHubTable;
  __shared__ Best red[32];
  for (int32_t it = blockIdx.x; it < hp.nitems; it += gridDim.x) {
    const int32_t h = hp.item_hub[it];
    if (hp.hub_state[h]) continue;  // block-uniform
    const uint32_t p = (uint32_t)hp.item_bucket[it], nb = (uint32_t)hp.hub_nb[h];
    const int32_t v = hp.hub_v[h];
    const int32_t b = a.off[v], d = a.off[v + 1] - b;
    const int32_t* lab = hp.hlab + hp.hub_lbase[h];
    for (uint32_t s = threadIdx.x; s < 2 * kHubTable; s += NT) smem[s] = 0;
    __syncthreads();
    Best best = best_none();
    bool fail = false;
    for (int32_t k0 = threadIdx.x; k0 < d; k0 += 4 * NT) {
      int32_t l[4];
      uint32_t wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int32_t k = k0 + q * NT;
        l[q] = k < d ? __ldcg(lab + k) : -1;
        wt[q] = k < d ? (W ? (uint32_t)ld_stream(a.w + b + k) : 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (l[q] < 0) continue;
        const uint32_t key = (uint32_t)l[q] + 1u;
        if (nb > 1 && hub_bucket_of(key, nb) != p) continue;
        uint32_t sl = hub_slot_of(key) & (kHubTable - 1);
        uint32_t tot = kNoSlot;
        for (uint32_t probe = 0; probe < kHubTable; ++probe) {
          const uint32_t kc = keys[sl];
          if (kc == key) {
            tot = atomicAdd(vals + sl, wt[q]) + wt[q];
            break;
          }
          if (kc == 0) {
            const uint32_t prev = atomicCAS(keys + sl, 0u, key);
            if (prev == 0u || prev == key) {
              tot = atomicAdd(vals + sl, wt[q]) + wt[q];
              break;
            }
          }
          sl = (sl + 1) & (kHubTable - 1);
        }
        if (tot == kNoSlot) {
          fail = true;
          continue;
        }
        const Best c{score(l[q], tot), l[q]};
        if (better(c, best)) best = c;
      }
    }
    if (fail) atomicOr(a.err, kErrProbe);
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
  if (l != a.lcur[v]) atomicAdd(a.changed, 1ull);
}

// --------------------------------------------------------- layered volumes
// vol[l] += #vertices whose label is l (warp-aggregated atomics).
__global__ void __launch_bounds__(256) k_histogram(const int32_t* __restrict__ lab, int32_t n, int32_t* vol) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t l = v < n ? lab[v] : -1;
  const uint32_t m = __match_any_sync(kFull, (uint32_t)l);
  if (l >= 0 && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(vol + l, __popc(m));
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
