// graphgen.cu -- deterministic synthetic-graph samplers and the reference
// edge-list loader.
//
// Samplers are counter based: sample i depends only on (seed, i), every
// random draw is a SplitMix64 word, and every decision is integer
// arithmetic, so the host (OpenMP) and device (CUDA) paths emit identical
// edge lists.  Building the CSR from the samples (symmetrise, drop self
// loops, dedupe, degree-descending relabel) is done by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/glp.h"
#include "device.cuh"

namespace glp {
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
int device_sms();
}  // namespace glp

namespace {

using glp::mix64;

// uniform integer in [0, range) from 32 random bits (multiply-shift)
__host__ __device__ __forceinline__ uint32_t bounded(uint32_t r, uint32_t range) {
  return (uint32_t)(((uint64_t)r * (uint64_t)range) >> 32);
}

struct RmatP {
  int32_t scale;
  uint64_t ta, tab, tabc;  // cumulative quadrant thresholds on 32-bit draws
  uint64_t key;
};

__host__ __device__ __forceinline__ void rmat_sample(const RmatP& p, int64_t i, int32_t* su, int32_t* sv) {
  const uint64_t k = mix64(p.key ^ (uint64_t)i);
  uint32_t u = 0, v = 0;
  uint64_t word = 0;
  for (int32_t lvl = 0; lvl < p.scale; ++lvl) {
    if ((lvl & 1) == 0) word = mix64(k + (uint64_t)(lvl >> 1));
    const uint64_t r = (lvl & 1) ? (word >> 32) : (word & 0xffffffffull);
    uint32_t bu, bv;
    if (r < p.ta) {
      bu = 0; bv = 0;
    } else if (r < p.tab) {
      bu = 0; bv = 1;
    } else if (r < p.tabc) {
      bu = 1; bv = 0;
    } else {
      bu = 1; bv = 1;
    }
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
  *su = (int32_t)u;
  *sv = (int32_t)v;
}

struct PlantedP {
  int32_t n, k, csize;
  int64_t n_intra;
  uint64_t key;
};

__host__ __device__ __forceinline__ void planted_sample(const PlantedP& p, int64_t i, int32_t* su, int32_t* sv) {
  const uint64_t k = mix64(p.key ^ (uint64_t)i);
  const uint64_t w0 = mix64(k), w1 = mix64(k + 1);
  const int32_t u = (int32_t)bounded((uint32_t)(w0 >> 32), (uint32_t)p.n);
  const int32_t c = u / p.csize;
  const int32_t cs = c * p.csize;
  const int32_t ce = cs + p.csize < p.n ? cs + p.csize : p.n;
  const int32_t size = ce - cs;
  int32_t v;
  if (i < p.n_intra) {
    v = cs + (int32_t)bounded((uint32_t)w0, (uint32_t)size);
  } else {
    const int32_t other = p.n - size;
    if (other == 0) {
      v = u;
    } else {
      const int32_t x = (int32_t)bounded((uint32_t)w1, (uint32_t)other);
      v = x < cs ? x : x + size;
    }
  }
  *su = u;
  *sv = v;
}

struct OverlapP {
  int32_t n, k, csize;
  uint64_t key;
  uint64_t thresh;          // overlap fraction on 32-bit draws
  const int32_t* sec_of;    // [n] second community or -1
  const int64_t* sec_off;   // [k+1]
  const int32_t* sec_list;  // members by second community
};

__host__ __device__ __forceinline__ int32_t second_community(uint64_t key, int32_t v, int32_t k, int32_t csize,
                                                             uint64_t thresh) {
  const uint64_t w = mix64(key ^ 0x5bd1e995ull ^ ((uint64_t)v << 20));
  if (k < 2 || (w & 0xffffffffull) >= thresh) return -1;
  const int32_t home = v / csize;
  return (home + 1 + (int32_t)bounded((uint32_t)(w >> 32), (uint32_t)(k - 1))) % k;
}

__host__ __device__ __forceinline__ void overlap_sample(const OverlapP& p, int64_t i, int32_t* su, int32_t* sv) {
  const uint64_t k = mix64(p.key ^ (uint64_t)i);
  const uint64_t w0 = mix64(k), w1 = mix64(k + 1);
  const int32_t u = (int32_t)bounded((uint32_t)(w0 >> 32), (uint32_t)p.n);
  int32_t c = u / p.csize;
  const int32_t s2 = p.sec_of[u];
  if (s2 >= 0 && (w0 & 1ull)) c = s2;
  const int32_t cs = c * p.csize;
  const int32_t ce = cs + p.csize < p.n ? cs + p.csize : p.n;
  const int32_t home_size = ce > cs ? ce - cs : 0;
  const int64_t nsec = p.sec_off[c + 1] - p.sec_off[c];
  const uint32_t total = (uint32_t)(home_size + nsec);
  const uint32_t idx = bounded((uint32_t)w1, total);
  *su = u;
  *sv = (int32_t)idx < home_size ? cs + (int32_t)idx : p.sec_list[p.sec_off[c] + ((int64_t)idx - home_size)];
}

template <class P, void (*F)(const P&, int64_t, int32_t*, int32_t*)>
__global__ void k_sample(P p, int64_t first, int64_t count, int32_t* src, int32_t* dst) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
    F(p, first + t, src + t, dst + t);
}

template <class P, void (*F)(const P&, int64_t, int32_t*, int32_t*)>
int run_sampler(const P& p, int64_t first, int64_t count, int32_t* src, int32_t* dst, int32_t on_device) {
  if (count < 0 || (count > 0 && (!src || !dst))) {
    glp::set_error("bad sample range or NULL output");
    return GLP_EINVAL;
  }
  if (on_device) {
    if (count == 0) return GLP_OK;
    k_sample<P, F><<<glp::device_sms() * 16, 256>>>(p, first, count, src, dst);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return glp::cuda_fail(e, "sampler kernel");
    return GLP_OK;
  }
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < count; ++t) F(p, first + t, src + t, dst + t);
  return GLP_OK;
}

uint64_t thresh32(double x) {
  if (x <= 0) return 0;
  if (x >= 1) return 1ull << 32;
  return (uint64_t)std::floor(x * 4294967296.0);
}

}  // namespace

extern "C" {

int glp_sample_rmat(int32_t scale, double a, double b, double c, uint64_t seed, int64_t first, int64_t count,
                    int32_t* src, int32_t* dst, int32_t on_device) {
  if (scale < 1 || scale > 30 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) {
    glp::set_error("bad R-MAT parameters");
    return GLP_EINVAL;
  }
  RmatP p{scale, thresh32(a), thresh32(a + b), thresh32(a + b + c), mix64(seed)};
  return run_sampler<RmatP, rmat_sample>(p, first, count, src, dst, on_device);
}

int glp_sample_planted(int32_t n, int32_t k, int64_t n_intra, uint64_t seed, int64_t first, int64_t count,
                       int32_t* src, int32_t* dst, int32_t on_device) {
  if (n < 1 || k < 1 || k > n || n_intra < 0) {
    glp::set_error("bad planted-partition parameters");
    return GLP_EINVAL;
  }
  const int32_t csize = (int32_t)(((int64_t)n + k - 1) / k);
  PlantedP p{n, k, csize, n_intra, mix64(seed ^ 0x9d2c5680ull)};
  return run_sampler<PlantedP, planted_sample>(p, first, count, src, dst, on_device);
}

int glp_sample_overlap(int32_t n, int32_t k, double overlap, uint64_t seed, int64_t first, int64_t count,
                       int32_t* src, int32_t* dst, int32_t on_device) {
  if (n < 1 || k < 1 || k > n || overlap < 0 || overlap > 1) {
    glp::set_error("bad overlap parameters");
    return GLP_EINVAL;
  }
  const int32_t csize = (int32_t)(((int64_t)n + k - 1) / k);
  const uint64_t key = mix64(seed ^ 0xefc60000ull);
  const uint64_t th = thresh32(overlap);
  std::vector<int32_t> sec_of(n);
  std::vector<int64_t> sec_off((size_t)k + 1, 0);
  for (int32_t v = 0; v < n; ++v) {
    sec_of[v] = second_community(key, v, k, csize, th);
    if (sec_of[v] >= 0) sec_off[sec_of[v] + 1]++;
  }
  for (int32_t c = 0; c < k; ++c) sec_off[c + 1] += sec_off[c];
  std::vector<int32_t> sec_list(std::max<int64_t>(sec_off[k], 1));
  {
    std::vector<int64_t> fill(sec_off.begin(), sec_off.end() - 1);
    for (int32_t v = 0; v < n; ++v)
      if (sec_of[v] >= 0) sec_list[fill[sec_of[v]]++] = v;
  }
  OverlapP p{n, k, csize, key, th, sec_of.data(), sec_off.data(), sec_list.data()};
  if (!on_device) return run_sampler<OverlapP, overlap_sample>(p, first, count, src, dst, 0);
  int32_t *d_sec_of = nullptr, *d_sec_list = nullptr;
  int64_t* d_sec_off = nullptr;
  int rc = GLP_OK;
  cudaError_t e = cudaMalloc(&d_sec_of, sizeof(int32_t) * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_sec_off, sizeof(int64_t) * sec_off.size());
  if (e == cudaSuccess) e = cudaMalloc(&d_sec_list, sizeof(int32_t) * sec_list.size());
  if (e == cudaSuccess) e = cudaMemcpy(d_sec_of, sec_of.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_sec_off, sec_off.data(), sizeof(int64_t) * sec_off.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_sec_list, sec_list.data(), sizeof(int32_t) * sec_list.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    rc = glp::cuda_fail(e, "overlap sampler tables");
  } else {
    p.sec_of = d_sec_of;
    p.sec_off = d_sec_off;
    p.sec_list = d_sec_list;
    rc = run_sampler<OverlapP, overlap_sample>(p, first, count, src, dst, 1);
  }
  cudaFree(d_sec_of);
  cudaFree(d_sec_off);
  cudaFree(d_sec_list);
  return rc;
}

}  // extern "C"

namespace {
__host__ __device__ __forceinline__ int32_t edge_weight(uint64_t key, int32_t u, int32_t v, int32_t wmax) {
  const uint32_t a = (uint32_t)(u < v ? u : v), b = (uint32_t)(u < v ? v : u);
  return 1 + (int32_t)(mix64(key ^ (((uint64_t)a << 32) | b)) % (uint64_t)wmax);
}

__global__ void k_weights(const int32_t* off, const int32_t* cols, int32_t n, int32_t wmax, uint64_t key, int32_t* w) {
  for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    for (int32_t j = off[v]; j < off[v + 1]; ++j) w[j] = edge_weight(key, v, cols[j], wmax);
}
}  // namespace

extern "C" {

int glp_edge_weights(const int32_t* off, const int32_t* cols, int32_t n, int64_t m, int32_t wmax, uint64_t seed,
                     int32_t* w, int32_t on_device) {
  if (n < 0 || m < 0 || wmax < 1 || !off || (m > 0 && (!cols || !w))) {
    glp::set_error("bad edge-weight arguments");
    return GLP_EINVAL;
  }
  const uint64_t key = mix64(seed ^ 0x27d4eb2full);
  if (on_device) {
    if (n == 0) return GLP_OK;
    k_weights<<<glp::device_sms() * 8, 256>>>(off, cols, n, wmax, key, w);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return glp::cuda_fail(e, "weights kernel");
    return GLP_OK;
  }
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t v = 0; v < n; ++v)
    for (int32_t j = off[v]; j < off[v + 1]; ++j) w[j] = edge_weight(key, v, cols[j], wmax);
  return GLP_OK;
}

// header/graph.h:69-147 + :226-258 semantics for undirected input: read int32
// (u,v) pairs, drop u == v, append v to u's list and u to v's list in file
// order, n = largest id seen in a kept pair + 1, no dedupe.  Directed input
// keeps only u -> v and takes n = largest id in any pair + 1.
int glp_load_edgelist_bin(const char* path, int32_t direct, int32_t** offsets, int32_t** cols, int32_t* n,
                          int64_t* m) {
  if (!path || !offsets || !cols || !n || !m) {
    glp::set_error("NULL argument");
    return GLP_EINVAL;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    glp::set_error("cannot open %s", path);
    return GLP_EINVAL;
  }
  std::vector<std::vector<int32_t>> adj;
  int32_t buf[2];
  int32_t maxid = -1;
  while (std::fread(buf, sizeof(int32_t), 2, f) == 2) {
    const int32_t u = buf[0], v = buf[1];
    if (u < 0 || v < 0) {
      std::fclose(f);
      glp::set_error("negative vertex id in %s", path);
      return GLP_EINVAL;
    }
    maxid = std::max(maxid, std::max(u, v));
    if (u == v) continue;
    if ((int64_t)adj.size() <= u) adj.resize((size_t)u + 1);
    adj[u].push_back(v);
    if (!direct) {
      if ((int64_t)adj.size() <= v) adj.resize((size_t)v + 1);
      adj[v].push_back(u);
    }
  }
  std::fclose(f);
  const int64_t nn = direct ? (int64_t)maxid + 1 : (int64_t)adj.size();
  if ((int64_t)adj.size() < nn) adj.resize((size_t)nn);
  int64_t mm = 0;
  for (const auto& l : adj) mm += (int64_t)l.size();
  if (mm > INT32_MAX) {
    glp::set_error("graph has %lld CSR entries (> int32)", (long long)mm);
    return GLP_EINVAL;
  }
  int32_t* off = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)(nn + 1));
  int32_t* cc = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(mm, 1));
  if (!off || !cc) {
    std::free(off);
    std::free(cc);
    glp::set_error("host allocation failed");
    return GLP_ENOMEM;
  }
  int64_t cur = 0;
  off[0] = 0;
  for (int64_t u = 0; u < nn; ++u) {
    for (int32_t v : adj[u]) cc[cur++] = v;
    off[u + 1] = (int32_t)cur;
  }
  *offsets = off;
  *cols = cc;
  *n = (int32_t)nn;
  *m = mm;
  return GLP_OK;
}

}  // extern "C"
