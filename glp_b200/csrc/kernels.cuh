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
//   tiny  : one thread per vertex, labels in registers, pairwise counts
//   group : G = 16 or 32 lanes per vertex, one __match_any_sync round
//   mid   : one warp per vertex, per-warp shared-memory count table
//   big   : one block per vertex, block shared-memory count table
//   hub   : several blocks per vertex; each counts a chunk in shared memory
//           and merges its distinct labels into a per-hub global table; the
//           last block to finish a hub writes its label (no spin waits).
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
  const int32_t* lcur;  // own current label, for the changed count
  int32_t* lout;
  unsigned long long* changed;
  uint32_t* err;
};

// score(l, k) for classic LP: the count itself.
struct ScoreClassic {
  __device__ __forceinline__ int64_t operator()(int32_t, uint32_t k) const { return (int64_t)k; }
};

// score(l, k) for layered LP: dstar*k - vol_r[l] (kernel.cuh:2575-2600).
struct ScoreLayered {
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

// ---------------------------------------------------------------- tiny tier
template <int TMAX, bool W, class S>
__global__ void __launch_bounds__(256) k_tiny(StepArgs a, const int32_t* __restrict__ verts, int32_t nv, S score) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  bool chg = false;
  if (t < nv) {
    const int32_t v = verts[t];
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
// G lanes per vertex (degree <= G).  The match key carries the group index so
// equal labels of different vertices in one warp do not merge.
template <int G, bool W, class S>
__global__ void __launch_bounds__(256) k_group(StepArgs a, const int32_t* __restrict__ verts, int32_t nv, S score) {
  const int lane = threadIdx.x & 31;
  const int64_t grp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = grp < nv;
  int32_t v = 0, b = 0, e = 0;
  if (act) {
    v = verts[grp];
    b = a.off[v];
    e = a.off[v + 1];
  }
  const int32_t j = b + (lane & (G - 1));
  const bool has = act && j < e;
  int32_t lab = -1;
  uint32_t wt = 0;
  if (has) load_edge<W>(a, j, lab, wt);
  const unsigned long long key = ((unsigned long long)(lane / G) << 32) | (uint32_t)lab;
  const uint32_t m = __match_any_sync(kFull, key);
  const uint32_t k = W ? __reduce_add_sync(m, wt) : (uint32_t)__popc(m);
  Best c = best_none();
  if (has && lane == __ffs(m) - 1) c = Best{score(lab, k), lab};
  c = group_max<G>(c);
  bool chg = false;
  if (act && (lane & (G - 1)) == 0) {
    a.lout[v] = c.l;
    chg = c.l != a.lcur[v];
  }
  warp_count_add(a.changed, chg);
}

// ----------------------------------------------------------------- mid tier
// One warp per vertex; per-warp table of CAP slots in static shared memory.
template <int CAP, int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_mid(StepArgs a, const int32_t* __restrict__ verts, int32_t nv, S score) {
  constexpr int NW = NT / 32;
  __shared__ uint32_t skeys[NW][CAP];
  __shared__ uint32_t svals[NW][CAP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const CountTable tab{skeys[warp], svals[warp], (uint32_t)(CAP - 1)};
  for (int32_t i = blockIdx.x * NW + warp; i < nv; i += gridDim.x * NW) {
#pragma unroll
    for (int s = lane; s < CAP; s += 32) {
      skeys[warp][s] = 0;
      svals[warp][s] = 0;
    }
    __syncwarp();
    const int32_t v = verts[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
    Best best = best_none();
    for (int32_t j0 = b; j0 < e; j0 += 64) {
      const int32_t ja = j0 + lane, jb = j0 + 32 + lane;
      int32_t la = -1, lb = -1;
      uint32_t wa = 0, wb = 0;
      if (ja < e) load_edge<W>(a, ja, la, wa);
      if (jb < e) load_edge<W>(a, jb, lb, wb);
      {
        const uint32_t m = __match_any_sync(kFull, (uint32_t)la);
        const uint32_t k = W ? __reduce_add_sync(m, wa) : (uint32_t)__popc(m);
        if (ja < e && lane == __ffs(m) - 1) {
          const uint32_t tot = tab.insert((uint32_t)la + 1u, k, a.err);
          const Best c{score(la, tot), la};
          if (better(c, best)) best = c;
        }
      }
      if (j0 + 32 < e) {
        const uint32_t m = __match_any_sync(kFull, (uint32_t)lb);
        const uint32_t k = W ? __reduce_add_sync(m, wb) : (uint32_t)__popc(m);
        if (jb < e && lane == __ffs(m) - 1) {
          const uint32_t tot = tab.insert((uint32_t)lb + 1u, k, a.err);
          const Best c{score(lb, tot), lb};
          if (better(c, best)) best = c;
        }
      }
    }
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
// One block per vertex; block table of `cap` slots in dynamic shared memory.
template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_big(StepArgs a, const int32_t* __restrict__ verts, int32_t nv, uint32_t cap,
                                            S score) {
  extern __shared__ uint32_t smem[];
  __shared__ Best red[32];
  uint32_t* keys = smem;
  uint32_t* vals = smem + cap;
  const CountTable tab{keys, vals, cap - 1};
  const int lane = threadIdx.x & 31;
  for (int32_t i = blockIdx.x; i < nv; i += gridDim.x) {
    for (uint32_t s = threadIdx.x; s < cap; s += NT) {
      keys[s] = 0;
      vals[s] = 0;
    }
    __syncthreads();
    const int32_t v = verts[i];
    const int32_t b = a.off[v], e = a.off[v + 1];
    Best best = best_none();
    for (int32_t j0 = b; j0 < e; j0 += NT) {
      const int32_t j = j0 + threadIdx.x;
      int32_t lab = -1;
      uint32_t wt = 0;
      if (j < e) load_edge<W>(a, j, lab, wt);
      const uint32_t m = __match_any_sync(kFull, (uint32_t)lab);
      const uint32_t k = W ? __reduce_add_sync(m, wt) : (uint32_t)__popc(m);
      if (j < e && lane == __ffs(m) - 1) {
        const uint32_t tot = tab.insert((uint32_t)lab + 1u, k, a.err);
        const Best c{score(lab, tot), lab};
        if (better(c, best)) best = c;
      }
    }
    best = block_max<NT>(best, red);
    if (threadIdx.x == 0) {
      a.lout[v] = best.l;
      if (best.l != a.lcur[v]) atomicAdd(a.changed, 1ull);
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- hub tier
struct HubPlan {
  const int32_t* chunk_hub;    // [nchunks] hub index of each chunk
  const int32_t* chunk_begin;  // [nchunks] first edge of the chunk
  const int32_t* chunk_end;    // [nchunks] one past the last edge
  const int32_t* hub_v;        // [nhubs] vertex id
  const int32_t* hub_nchunks;  // [nhubs]
  const int64_t* hub_tbase;    // [nhubs] first slot of the hub's global table
  const uint32_t* hub_tmask;   // [nhubs] table capacity - 1 (power of two)
  const int64_t* hub_ubase;    // [nhubs] first entry of the hub's used-slot list
  uint32_t* gkeys;             // global tables (label+1, 0 = empty)
  uint32_t* gvals;
  uint32_t* used;              // used-slot lists
  uint32_t* used_n;            // [nhubs] entries in the used list
  unsigned long long* hub_best;  // [nhubs] packed best (0 = none)
  uint32_t* hub_done;            // [nhubs] chunks finished this step
};

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

// Insert into a hub's global table; newly claimed slots are appended to the
// hub's used list so the finishing block can clear exactly those.  Probes use
// L2 loads (__ldcg) since other blocks write the table concurrently.
__device__ __forceinline__ uint32_t hub_insert(const HubPlan& hp, int32_t h, uint32_t key, uint32_t c, uint32_t* err) {
  const int64_t base = hp.hub_tbase[h];
  const uint32_t mask = hp.hub_tmask[h];
  uint32_t s = fmix32(key) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t* kp = hp.gkeys + base + s;
    const uint32_t cur = __ldcg(kp);
    if (cur == key) return atomicAdd(hp.gvals + base + s, c) + c;
    if (cur == 0) {
      const uint32_t prev = atomicCAS(kp, 0u, key);
      if (prev == 0u) {
        const uint32_t idx = atomicAdd(hp.used_n + h, 1u);
        hp.used[hp.hub_ubase[h] + idx] = s;
        return atomicAdd(hp.gvals + base + s, c) + c;
      }
      if (prev == key) return atomicAdd(hp.gvals + base + s, c) + c;
    }
    s = (s + 1) & mask;
  }
  atomicOr(err, kErrProbe);
  return 0;
}

template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_hub(StepArgs a, HubPlan hp, int32_t nchunks, uint32_t cap, S score) {
  extern __shared__ uint32_t smem[];
  __shared__ Best red[32];
  __shared__ int last;
  __shared__ uint32_t s_nused;
  uint32_t* keys = smem;
  uint32_t* vals = smem + cap;
  const CountTable tab{keys, vals, cap - 1};
  const int lane = threadIdx.x & 31;
  for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    for (uint32_t s = threadIdx.x; s < cap; s += NT) {
      keys[s] = 0;
      vals[s] = 0;
    }
    __syncthreads();
    const int32_t h = hp.chunk_hub[c];
    const int32_t cb = hp.chunk_begin[c], ce = hp.chunk_end[c];
    for (int32_t j0 = cb; j0 < ce; j0 += NT) {
      const int32_t j = j0 + threadIdx.x;
      int32_t lab = -1;
      uint32_t wt = 0;
      if (j < ce) load_edge<W>(a, j, lab, wt);
      const uint32_t m = __match_any_sync(kFull, (uint32_t)lab);
      const uint32_t k = W ? __reduce_add_sync(m, wt) : (uint32_t)__popc(m);
      if (j < ce && lane == __ffs(m) - 1) tab.insert((uint32_t)lab + 1u, k, a.err);
    }
    __syncthreads();
    // merge this chunk's distinct labels into the hub's global table
    Best best = best_none();
    for (uint32_t s = threadIdx.x; s < cap; s += NT) {
      const uint32_t key = keys[s];
      if (key) {
        const uint32_t tot = hub_insert(hp, h, key, vals[s], a.err);
        const Best cnd{score((int32_t)(key - 1u), tot), (int32_t)(key - 1u)};
        if (better(cnd, best)) best = cnd;
      }
    }
    // every thread's used-list stores are ordered before the done counter
    __threadfence();
    best = block_max<NT>(best, red);
    if (threadIdx.x == 0) {
      atomicMax(hp.hub_best + h, pack_best(best, a.err));
      __threadfence();
      const uint32_t done = atomicAdd(hp.hub_done + h, 1u);
      last = (done + 1u == (uint32_t)hp.hub_nchunks[h]);
      if (last) {
        __threadfence();
        s_nused = atomicAdd(hp.used_n + h, 0u);
      }
    }
    __syncthreads();
    if (last) {
      // the last block of this hub: all other chunks have merged
      const int64_t ub = hp.hub_ubase[h], tb = hp.hub_tbase[h];
      for (uint32_t i = threadIdx.x; i < s_nused; i += NT) {
        const uint32_t s = __ldcg(hp.used + ub + i);
        hp.gkeys[tb + s] = 0;
        hp.gvals[tb + s] = 0;
      }
      if (threadIdx.x == 0) {
        const unsigned long long p = atomicExch(hp.hub_best + h, 0ull);
        const int32_t v = hp.hub_v[h];
        const int32_t l = p ? (int32_t)(uint32_t)(p & 0xffffffffull) : a.lcur[v];
        if (!p) atomicOr(a.err, kErrHubPlan);
        a.lout[v] = l;
        if (l != a.lcur[v]) atomicAdd(a.changed, 1ull);
        atomicExch(hp.used_n + h, 0u);
        atomicExch(hp.hub_done + h, 0u);
      }
    }
    __syncthreads();
  }
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
