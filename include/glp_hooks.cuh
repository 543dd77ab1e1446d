/*
 * glp_hooks.cuh -- method 4 of the label-propagation engine as a header-only
 * CUDA template: user-written PickLabel / LoadNeighbor / LabelScore /
 * UpdateVertex hooks run on a graph handle of libglp_b200.so.
 *
 * Reference surface: README.md:72-101 asks users to fill in four __device__
 * functions (stubs at header/kernel.cuh:6071-6085) and run method=4
 * (prop/UserdefinedLprop.cuh, main.cu:96-100).  Here a hook set is any
 * struct with these four __device__ members:
 *
 *   void   pick(int32_t vid)                               PickLabel
 *   void   load(int32_t vid, int32_t sid, int64_t e,
 *               int32_t* label, double* freq)              LoadNeighbor
 *   double score(int32_t vid, int32_t label, double freq)  LabelScore
 *   void   update(int32_t vid, int32_t label, double score) UpdateVertex
 *
 * and glp_hooks::run() drives, per iteration:
 *   1. pick(v) for every vertex (the classic hook set copies Lnext to L);
 *   2. per vertex v, freq(l) = the sum of the freq values LoadNeighbor gives
 *      for the neighbours (CSR entries e of v, neighbour sid) whose label is
 *      l; the winner maximises LabelScore(v, l, freq(l)), ties -> the
 *      largest label; Lnext[v] = winner, then update(v, winner, score).  An
 *      isolated vertex keeps L[v] and gets update(v, L[v], -inf).
 * LabelScore may be any function of the final frequency: every distinct
 * label is scored once its frequency is complete.  Frequencies are summed in
 * a fixed order -- within a chunk of 32 consecutive CSR entries in entry
 * order, chunks in CSR order -- so FP64 results are deterministic and can be
 * restated exactly on the host.
 *
 * Build a hook set into your own shared object or program with nvcc
 * (-gencode arch=compute_100a,code=sm_100a) and link -lglp_b200; the graph
 * stays resident in the library's handle, so nothing is copied.  The hooks
 * get the device view (glp_hooks::State, filled from glp_graph_device_view)
 * through a member of their own, as in the example below.
 *
 *   struct MyHooks {
 *     glp_hooks::State st;
 *     __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
 *     __device__ void load(int32_t, int32_t sid, int64_t, int32_t* l, double* f) const {
 *       *l = st.L[sid];
 *       *f = 1.0 / (1.0 + (st.off[sid + 1] - st.off[sid]));
 *     }
 *     __device__ double score(int32_t, int32_t, double f) const { return f; }
 *     __device__ void update(int32_t, int32_t, double) const {}
 *   };
 *   ...
 *   glp_hooks::run(g, [](const glp_hooks::State& s) { return MyHooks{s}; }, niter, labels, 0, nullptr,
 *                  stream);
 */
#ifndef GLP_B200_GLP_HOOKS_CUH
#define GLP_B200_GLP_HOOKS_CUH

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "glp.h"

namespace glp_hooks {

/* What a hook set sees: the resident CSR, the two label buffers (L read,
 * Lnext written by the step) and, for layered-style scores, two volume
 * arrays (vol_r read, vol_w written).  dstar and user are free for the hook
 * set's own use. */
struct State {
  const int32_t* off;
  const int32_t* cols;
  const int32_t* w;  /* NULL when the graph is unweighted */
  int32_t n;
  int32_t* L;
  int32_t* Lnext;
  const int32_t* vol_r;
  int32_t* vol_w;
  double dstar;
  void* user;
};

constexpr uint32_t kFullMask = 0xffffffffu;
constexpr int kSmemCap = 512; /* per warp; degrees <= kSmemCap/2 count in shared memory */
constexpr uint32_t kErrProbe = 1u;

/* The 32-bit finaliser of MurmurHash3 (Appleby): slot of a key. */
__device__ __forceinline__ uint32_t slot_hash(uint32_t k) {
  k ^= k >> 16;
  k *= 0x85ebca6bu;
  k ^= k >> 13;
  k *= 0xc2b2ae35u;
  k ^= k >> 16;
  return k;
}

template <class H>
__global__ void __launch_bounds__(256) k_pick(H h, int32_t n) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) h.pick(v);
}

/* One warp per vertex.  The per-vertex table holds label+1 keys and FP64
 * frequencies: in shared memory up to degree kSmemCap/2, else in the global
 * spill region [2*off[v], 2*off[v] + cap) of gkeys/gvals (cap = the largest
 * power of two <= 2*degree, so it holds every distinct label). */
template <class H>
__global__ void __launch_bounds__(128) k_prop(H h, const State st, uint32_t* gkeys, double* gvals,
                                              unsigned long long* changed, uint32_t* err) {
  constexpr int NW = 4;
  __shared__ uint32_t skeys[NW][kSmemCap];
  __shared__ double svals[NW][kSmemCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int32_t v = blockIdx.x * NW + warp; v < st.n; v += gridDim.x * NW) {
    const int32_t b = st.off[v], e = st.off[v + 1], d = e - b;
    if (d == 0) {
      if (lane == 0) {
        const int32_t l = st.L[v];
        st.Lnext[v] = l;
        h.update(v, l, -INFINITY);
      }
      continue; /* warp-uniform */
    }
    uint32_t* keys;
    double* vals;
    uint32_t cap;
    if (d <= kSmemCap / 2) {
      keys = skeys[warp];
      vals = svals[warp];
      cap = kSmemCap;
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
      const uint32_t m = __match_any_sync(kFullMask, (uint32_t)lab);
      /* entry-ordered sum over the lanes holding the same label */
      double s = 0.0;
      for (int k = 0; k < 32; ++k) {
        const double x = __shfl_sync(kFullMask, f, k);
        if ((m >> k) & 1u) s += x;
      }
      if (j < e && lane == __ffs(m) - 1) {
        const uint32_t key = (uint32_t)lab + 1u;
        uint32_t slot = slot_hash(key) & (cap - 1);
        bool done = false;
        for (uint32_t probe = 0; probe < cap; ++probe) {
          const uint32_t prev = atomicCAS(&keys[slot], 0u, key);
          if (prev == 0u || prev == key) {
            vals[slot] += s; /* one writer per label per chunk; chunks in order */
            done = true;
            break;
          }
          slot = (slot + 1) & (cap - 1);
        }
        if (!done) atomicOr(err, kErrProbe);
      }
      __syncwarp();
    }
    /* score every distinct label on its final frequency */
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
      const double os = __shfl_xor_sync(kFullMask, bs, o);
      const int32_t ol = __shfl_xor_sync(kFullMask, bl, o);
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

/* Launches one iteration (pick, then the propagation step) on `stream`. */
template <class H>
inline cudaError_t launch_iteration(const H& h, const State& st, const glp_device_view& vw, int32_t iter,
                                    cudaStream_t stream) {
  if (st.n == 0) return cudaSuccess;
  k_pick<H><<<(unsigned)((st.n + 255) / 256), 256, 0, stream>>>(h, st.n);
  unsigned grid = (unsigned)((st.n + 3) / 4);
  const unsigned cap = (unsigned)(vw.sms > 0 ? vw.sms : 1) * 64u;
  if (grid > cap) grid = cap;
  k_prop<H><<<grid, 128, 0, stream>>>(h, st, vw.hook_keys, vw.hook_vals, vw.changed + iter, vw.err);
  return cudaGetLastError();
}

/* Runs niter iterations of the hook set that make(state) returns, on the
 * resident graph g, from label = vertex id.  L is labels[0] and Lnext
 * labels[1] in every iteration: PickLabel moves the previous result into L
 * (the classic hooks copy Lnext to L), so the final labels are in Lnext.
 * labels_out receives them (a device pointer when on_device, else host);
 * changed (nullable, host) the number of labels changed per iteration.
 * Returns a GLP_* code.  The call is synchronous. */
template <class Make>
inline int run(glp_graph* g, Make make, int32_t niter, int32_t* labels_out, int32_t on_device, int64_t* changed,
               cudaStream_t stream) {
  if (!g || !labels_out || niter < 0) return GLP_EINVAL;
  glp_device_view vw;
  int rc = glp_graph_device_view(g, niter, &vw);
  if (rc) return rc;
  cudaStream_t s = stream ? stream : (cudaStream_t)vw.stream;
  cudaError_t e = cudaSuccess;
  if (vw.n > 0) {
    const State st{vw.off, vw.cols, vw.w, vw.n, vw.labels[0], vw.labels[1], nullptr, nullptr, 1.0, nullptr};
    const auto h = make(st);
    for (int32_t it = 0; it < niter && e == cudaSuccess; ++it) e = launch_iteration(h, st, vw, it, s);
    const int32_t* fin = vw.labels[1];
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(labels_out, fin, sizeof(int32_t) * (size_t)vw.n,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess && changed && niter > 0)
    e = cudaMemcpyAsync(changed, vw.changed, sizeof(int64_t) * (size_t)niter, cudaMemcpyDeviceToHost, s);
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, vw.err, sizeof err, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return GLP_ECUDA;
  return err ? GLP_EKERNEL : GLP_OK;
}

} /* namespace glp_hooks */

#endif /* GLP_B200_GLP_HOOKS_CUH */
