// hooks_engine.cuh -- method 4: label propagation driven by the four user
// hooks of README.md:72-101 (PickLabel, LoadNeighbor, LabelScore,
// UpdateVertex), which the reference declares as __device__ stubs in
// header/kernel.cuh:6071-6085 and drives from prop/UserdefinedLprop.cuh.
//
// A hook set is a struct with four __device__ members:
//   void   pick(int32_t vid)                                   PickLabel
//   void   load(int32_t vid, int32_t sid, int64_t e,
//               int32_t* label, double* freq)                  LoadNeighbor
//   double score(int32_t vid, int32_t l, double freq)          LabelScore
//   void   update(int32_t vid, int32_t l, double score)        UpdateVertex
// and the engine runs, per iteration:
//   1. pick(v) for every vertex (classic: L[v] = Lnext[v]);
//   2. per vertex, freq(l) = sum of LoadNeighbor freqs over neighbours with
//      label l; the winner maximises LabelScore(v, l, freq(l)), ties ->
//      largest label; Lnext[v] = winner and update(v, winner, score).  An
//      isolated vertex keeps L[v] and gets update(v, L[v], -inf).
// LabelScore may be any function of the final frequency, so the engine
// scores every distinct label after accumulation (no running maximum).
// Frequencies are summed in a fixed order -- within a 32-edge chunk in lane
// order, chunks in CSR order -- so FP64 results are deterministic.
//
// The same template is public (include/glp_hooks.cuh) for users who compile
// their own hook sets against this library.
#pragma once
#include <cmath>

#include "engine.h"

namespace glp {

struct HookState {
  const int32_t* off;
  const int32_t* cols;
  const int32_t* w;
  int32_t* L;
  int32_t* Lnext;
  const int32_t* vol_r;
  int32_t* vol_w;
  double dstar;
};

// README.md:83-101: copy Lnext -> L, (L[sid], 1.0), score = freq, no update.
struct HooksClassic {
  HookState st;
  __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
  __device__ void load(int32_t, int32_t sid, int64_t e, int32_t* l, double* f) const {
    *l = st.L[sid];
    *f = st.w ? (double)st.w[e] : 1.0;
  }
  __device__ double score(int32_t, int32_t, double f) const { return f; }
  __device__ void update(int32_t, int32_t, double) const {}
};

// Layered LP as hooks: score = dstar*freq - vol_r[l] (FP64, exact for these
// magnitudes); UpdateVertex counts the volume of the chosen label.
struct HooksLayered {
  HookState st;
  __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
  __device__ void load(int32_t, int32_t sid, int64_t e, int32_t* l, double* f) const {
    *l = st.L[sid];
    *f = st.w ? (double)st.w[e] : 1.0;
  }
  __device__ double score(int32_t, int32_t l, double f) const { return st.dstar * f - (double)st.vol_r[l]; }
  __device__ void update(int32_t, int32_t l, double) const { atomicAdd(st.vol_w + l, 1); }
};

// Degree-normalised frequencies: freq = w(e) / deg(sid) in FP64.
struct HooksWeightedDegree {
  HookState st;
  __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
  __device__ void load(int32_t, int32_t sid, int64_t e, int32_t* l, double* f) const {
    *l = st.L[sid];
    const double d = (double)(st.off[sid + 1] - st.off[sid]);
    *f = (st.w ? (double)st.w[e] : 1.0) / d;
  }
  __device__ double score(int32_t, int32_t, double f) const { return f; }
  __device__ void update(int32_t, int32_t, double) const {}
};

template <class H>
__global__ void __launch_bounds__(256) k_hooks_pick(H h, int32_t n) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) h.pick(v);
}

// Per-vertex accumulation table: label+1 keys with FP64 frequencies.  The
// global spill region of vertex v is [2*off[v], 2*off[v] + cap) with cap the
// largest power of two <= 2*deg (so cap >= deg >= distinct labels).
constexpr int kHookSmemCap = 512;  // per warp; degrees <= 256 stay in shared memory

template <class H>
__global__ void __launch_bounds__(128) k_hooks_prop(H h, int32_t n, uint32_t* gkeys, double* gvals,
                                                    unsigned long long* changed, uint32_t* err) {
  constexpr int NW = 4;
  __shared__ uint32_t skeys[NW][kHookSmemCap];
  __shared__ double svals[NW][kHookSmemCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const HookState& st = h.st;
  for (int32_t v = blockIdx.x * NW + warp; v < n; v += gridDim.x * NW) {
    const int32_t b = st.off[v], e = st.off[v + 1], d = e - b;
    if (d == 0) {
      if (lane == 0) {
        const int32_t l = st.L[v];
        st.Lnext[v] = l;
        h.update(v, l, -INFINITY);
      }
      continue;  // warp-uniform
    }
    uint32_t* keys;
    double* vals;
    uint32_t cap;
    if (d <= kHookSmemCap / 2) {
      keys = skeys[warp];
      vals = svals[warp];
      cap = kHookSmemCap;
    } else {
      cap = 1;
      while (cap * 2 <= 2u * (uint32_t)d) cap *= 2;
      keys = gkeys + 2ll * b;
      vals = gvals + 2ll * b;
    }
    for (uint32_t s = lane; s < cap; s += 32) {
      keys[s] = 0;
      vals[s] = 0.0;
    }
    __syncwarp();
    for (int32_t j0 = b; j0 < e; j0 += 32) {
      const int32_t j = j0 + lane;
      int32_t lab = -1;
      double f = 0.0;
      if (j < e) h.load(v, st.cols[j], j, &lab, &f);
      const uint32_t m = __match_any_sync(kFull, (uint32_t)lab);
      // lane-ordered sum over the lanes holding the same label
      double s = 0.0;
      for (int k = 0; k < 32; ++k) {
        const double x = __shfl_sync(kFull, f, k);
        if ((m >> k) & 1u) s += x;
      }
      if (j < e && lane == __ffs(m) - 1) {
        const uint32_t key = (uint32_t)lab + 1u;
        uint32_t slot = fmix32(key) & (cap - 1);
        bool done = false;
        for (uint32_t probe = 0; probe < cap; ++probe) {
          const uint32_t prev = atomicCAS(&keys[slot], 0u, key);
          if (prev == 0u || prev == key) {
            vals[slot] += s;  // one writer per label per chunk; chunks in order
            done = true;
            break;
          }
          slot = (slot + 1) & (cap - 1);
        }
        if (!done) atomicOr(err, kErrProbe);
      }
      __syncwarp();
    }
    // score every distinct label on its final frequency
    double bs = -INFINITY;
    int32_t bl = -1;
    for (uint32_t s = lane; s < cap; s += 32) {
      const uint32_t key = keys[s];
      if (key) {
        const int32_t l = (int32_t)(key - 1u);
        const double sc = h.score(v, l, vals[s]);
        if (bl < 0 || sc > bs || (sc == bs && l > bl)) {
          bs = sc;
          bl = l;
        }
      }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      const double os = __shfl_xor_sync(kFull, bs, o);
      const int32_t ol = __shfl_xor_sync(kFull, bl, o);
      if (ol >= 0 && (bl < 0 || os > bs || (os == bs && ol > bl))) {
        bs = os;
        bl = ol;
      }
    }
    if (lane == 0) {
      st.Lnext[v] = bl;
      h.update(v, bl, bs);
      if (bl != st.L[v]) atomicAdd(changed, 1ull);
    }
    __syncwarp();
  }
}

}  // namespace glp
