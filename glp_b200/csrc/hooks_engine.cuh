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
// The propagation template itself (k_pick / k_prop) is the public one of
// include/glp_hooks.cuh, which users include to compile hook sets of their
// own against a resident graph; the built-in sets below use it too.
#pragma once
#include <cmath>

#include "../../include/glp_hooks.cuh"
#include "engine.h"

namespace glp {

using HookState = glp_hooks::State;

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

// Degrees up to this count in shared memory; above it the spill tables.
constexpr int kHookSmemCap = glp_hooks::kSmemCap;

}  // namespace glp
