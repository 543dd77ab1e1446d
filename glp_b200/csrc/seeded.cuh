// seeded.cuh -- seeded (semi-supervised) label propagation, method 5.
//
// Reference: prop/seedLprop.cuh (driver) with the *_seed kernels of
// header/kernel.cuh:914-1031 (huge), :1742-1836 (big), :3224-3331 (medium),
// :5236-5290 (tiny), and initialize_labels_by_seeds (:453-466): seed
// vertices are labelled with their own id and keep it; every other vertex
// starts unlabelled (-1) and takes the mode of its neighbours' labels.
//
// The rule implemented here, for every vertex v in one synchronous step:
//   seed v           : L'(v) = L(v) (its own id);
//   otherwise        : L'(v) = argmax_l k_l(v) over the LABELLED neighbours
//                      (label >= 0; weights summed exactly when the graph is
//                      weighted), ties -> the largest label; with no labelled
//                      neighbour, L'(v) = L(v).
// The reference's tiers disagree on unlabelled neighbours and on a vertex
// with none labelled: its tiny kernel counts the unlabelled ones as a label
// of their own, which can win (kernel.cuh:5253-5269), and its big and huge
// kernels skip them but then give the vertex its own id (:1767-1768); the
// rule above is the hard-clamping label propagation those kernels approach
// (Zhu and Ghahramani, CMU-CALD-02-107, 2002), the same on every tier.
//
// One warp per vertex.  Counts live in a per-warp shared table for degrees
// up to kSeedSmem / 2, else in the vertex's own region of a global spill
// table (2 slots per CSR entry).  Running totals make the result independent
// of the order of the atomics, as in the other exact-count kernels.
#pragma once
#include "device.cuh"

namespace glp {

constexpr int kSeedSmem = 512;  // shared slots per warp

template <bool W>
__global__ void __launch_bounds__(256) k_seeded_step(const int32_t* __restrict__ off, const int32_t* __restrict__ cols,
                                                     const int32_t* __restrict__ w, const uint8_t* __restrict__ seeds,
                                                     const int32_t* __restrict__ lin, int32_t* __restrict__ lout,
                                                     int32_t n, uint32_t* gkeys, uint32_t* gvals,
                                                     unsigned long long* changed, uint32_t* err) {
  constexpr int NW = 8;
  __shared__ __align__(16) uint32_t skeys[NW][kSeedSmem];
  __shared__ __align__(16) uint32_t svals[NW][kSeedSmem];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t v0 = (int64_t)blockIdx.x * NW + warp; v0 < n; v0 += (int64_t)gridDim.x * NW) {
    const int32_t v = (int32_t)v0;
    const int32_t cur = lin[v];
    if (seeds[v]) {  // warp-uniform
      if (lane == 0) lout[v] = cur;
      continue;
    }
    const int32_t b = off[v], e = off[v + 1];
    uint32_t *keys, *vals, cap;
    if (e - b <= kSeedSmem / 2) {
      keys = skeys[warp];
      vals = svals[warp];
      cap = kSeedSmem;
    } else {
      cap = pow2_ceil(2u * (uint32_t)(e - b)) >> 1;  // the largest power of two <= 2*degree
      keys = gkeys + 2ll * b;
      vals = gvals + 2ll * b;
    }
    for (uint32_t s = lane; s < cap; s += 32) {
      keys[s] = 0u;
      vals[s] = 0u;
    }
    __syncwarp();
    const CountTable table{keys, vals, cap - 1};
    Best best = best_none();
    for (int32_t j0 = b; j0 < e; j0 += 32) {
      const int32_t j = j0 + lane;
      if (j < e) {
        const int32_t l = ld_label(lin + ld_stream(cols + j));
        if (l >= 0) {  // unlabelled neighbours are not counted
          const uint32_t k = W ? (uint32_t)ld_stream(w + j) : 1u;
          const uint32_t tot = table.insert((uint32_t)l + 1u, k, err);
          const Best c{(int64_t)tot, l};
          if (better(c, best)) best = c;
        }
      }
    }
    best = group_max<32>(best);
    if (lane == 0) {
      const int32_t nl = best.l >= 0 ? best.l : cur;
      lout[v] = nl;
      if (nl != cur) atomicAdd(changed, 1ull);
    }
    __syncwarp();  // the table is cleared for the next vertex
  }
}

// Labels at the start: a seed gets its id, every other vertex -1.
__global__ void k_seeded_init(const uint8_t* __restrict__ seeds, int32_t* __restrict__ a, int32_t* __restrict__ b,
                              int32_t n) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) a[v] = b[v] = seeds[v] ? v : -1;
}

}  // namespace glp
