// ingest.cu -- building the int32 CSR of an edge list on the device.
//
// Reference semantics: tools/normalize.cpp:262-348 (degree-descending
// relabel) and header/graph.h:226-258 (edge list -> CSR: self loops dropped,
// both directions stored for an undirected graph).  Here, on the device:
//   1. every edge (u,v), u != v, becomes the key (u << 32 | v), and for an
//      undirected graph also (v << 32 | u);
//   2. the keys are sorted (stable LSD radix sort, 8-bit digits, only the
//      digits an id can occupy) and duplicates dropped;
//   3. unless ids are kept, vertices are renumbered by degree descending,
//      ties by the smaller original id (normalize.cpp's order, made
//      deterministic), the keys rewritten and sorted again;
//   4. offsets come from a binary search of each row's first key; columns
//      are the low halves of the keys, so every row is ascending.
// The result equals, bit for bit, the host construction the tests and the
// samplers use (symmetrise, drop self loops, sort, dedupe, relabel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/glp.h"
#include "device.cuh"

namespace glp {
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
int device_sms();
}  // namespace glp

namespace {

using glp::kFull;

#define ICUDA(call)                                            \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return glp::cuda_fail(e_, #call);   \
  } while (0)

constexpr int kNT = 256;             // threads per block
constexpr int kItems = 16;           // rounds of kNT keys per tile
constexpr int kTile = kNT * kItems;  // 4096 keys per tile
constexpr int kRadix = 256;
constexpr int kScanNT = 256, kScanPer = 8, kScanBlock = kScanNT * kScanPer;

int bit_length(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

// ------------------------------------------------------------------ scan
// Exclusive scan of uint32 counts, in place, block by block; sums[b] gets
// block b's total.
__global__ void __launch_bounds__(kScanNT) k_scan_blocks(uint32_t* __restrict__ a, int64_t len,
                                                         uint32_t* __restrict__ sums) {
  __shared__ uint32_t wsum[kScanNT / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanPer;
  uint32_t x[kScanPer], run = 0;
#pragma unroll
  for (int i = 0; i < kScanPer; ++i) {
    x[i] = base + i < len ? a[base + i] : 0u;
    const uint32_t t = x[i];
    x[i] = run;
    run += t;
  }
  // exclusive scan of the thread totals
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  uint32_t wbase = 0, total = 0;
  for (int w = 0; w < kScanNT / 32; ++w) {
    if (w < warp) wbase += wsum[w];
    total += wsum[w];
  }
  const uint32_t off = wbase + inc - run;
#pragma unroll
  for (int i = 0; i < kScanPer; ++i)
    if (base + i < len) a[base + i] = x[i] + off;
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_add(uint32_t* __restrict__ a, int64_t len, const uint32_t* __restrict__ sums) {
  const int64_t b = blockIdx.x;
  const uint32_t add = sums[b];
  for (int64_t i = b * kScanBlock + threadIdx.x; i < std::min(len, (b + 1) * kScanBlock); i += blockDim.x)
    a[i] += add;
}

// Exclusive scan of len counts (total < 2^32).  scratch: >= scan_scratch(len)
// words.
int64_t scan_scratch(int64_t len) {
  int64_t need = 0;
  while (len > 1) {
    len = (len + kScanBlock - 1) / kScanBlock;
    need += len;
  }
  return need + 1;
}

int scan_u32(uint32_t* a, int64_t len, uint32_t* scratch, cudaStream_t s) {
  if (len <= 0) return GLP_OK;
  const int64_t nb = (len + kScanBlock - 1) / kScanBlock;
  k_scan_blocks<<<(unsigned)nb, kScanNT, 0, s>>>(a, len, scratch);
  ICUDA(cudaGetLastError());
  if (nb > 1) {
    int rc = scan_u32(scratch, nb, scratch + nb, s);
    if (rc) return rc;
    k_scan_add<<<(unsigned)nb, 256, 0, s>>>(a, len, scratch);
    ICUDA(cudaGetLastError());
  }
  return GLP_OK;
}

// ------------------------------------------------------------ radix sort
// Per tile, the count of each 8-bit digit: hist[digit * ntiles + tile]
// (digit-major, so one exclusive scan gives every tile's first position of
// every digit).
__global__ void __launch_bounds__(kNT) k_digit_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                    uint32_t* __restrict__ hist, int64_t ntiles) {
  __shared__ uint32_t h[kRadix];
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (int d = threadIdx.x; d < kRadix; d += kNT) h[d] = 0;
    __syncthreads();
    const int64_t base = t * kTile;
#pragma unroll 4
    for (int r = 0; r < kItems; ++r) {
      const int64_t i = base + (int64_t)r * kNT + threadIdx.x;
      if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kNT) hist[(int64_t)d * ntiles + t] = h[d];
    __syncthreads();
  }
}

// Stable scatter by one digit.  A tile is read in kItems rounds of kNT keys
// (key r*kNT + thread); within a round, lanes holding the same digit are
// found with eight ballots, ranked by lane, and the warps' counts are turned
// into running offsets per digit in warp order, so equal digits keep their
// input order.
__global__ void __launch_bounds__(kNT) k_digit_scatter(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                       int64_t n, int shift, const uint32_t* __restrict__ offs,
                                                       int64_t ntiles) {
  constexpr int NW = kNT / 32;
  __shared__ uint32_t base[kRadix];
  __shared__ uint32_t wcnt[NW][kRadix];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (int d = threadIdx.x; d < kRadix; d += kNT) base[d] = offs[(int64_t)d * ntiles + t];
    for (int r = 0; r < kItems; ++r) {
      for (int x = threadIdx.x; x < NW * kRadix; x += kNT) (&wcnt[0][0])[x] = 0u;
      __syncthreads();
      const int64_t i = t * kTile + (int64_t)r * kNT + threadIdx.x;
      const bool valid = i < n;
      const uint64_t key = valid ? in[i] : 0ull;
      const uint32_t dig = (uint32_t)(key >> shift) & 0xffu;
      uint32_t peers = __ballot_sync(kFull, valid);
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const bool bit = (dig >> b) & 1u;
        const uint32_t m = __ballot_sync(kFull, bit);
        peers &= bit ? m : ~m;
      }
      const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
      if (valid && rank == 0) wcnt[warp][dig] = __popc(peers);
      __syncthreads();
      for (int d = threadIdx.x; d < kRadix; d += kNT) {
        uint32_t run = base[d];
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          const uint32_t c = wcnt[w][d];
          wcnt[w][d] = run;
          run += c;
        }
        base[d] = run;
      }
      __syncthreads();
      if (valid) out[wcnt[warp][dig] + rank] = key;
      __syncthreads();  // the next round clears wcnt
    }
  }
}

struct Sorter {
  uint32_t* hist = nullptr;
  uint32_t* scratch = nullptr;
  int64_t cap_keys = 0;
};

// Sorts n keys by the given bit ranges [lo, lo + width) (8-bit digits, least
// significant range first).  keys and tmp hold n keys; the result ends in
// *keys (the pointers swap when the digit count is odd).
int radix_sort(uint64_t** keys, uint64_t** tmp, int64_t n, const std::vector<std::pair<int, int>>& ranges,
               const Sorter& so, cudaStream_t s) {
  if (n <= 1) return GLP_OK;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)glp::device_sms() * 8);
  for (const auto& rg : ranges) {
    for (int shift = rg.first; shift < rg.first + rg.second; shift += 8) {
      k_digit_hist<<<grid, kNT, 0, s>>>(*keys, n, shift, so.hist, ntiles);
      ICUDA(cudaGetLastError());
      int rc = scan_u32(so.hist, (int64_t)kRadix * ntiles, so.scratch, s);
      if (rc) return rc;
      k_digit_scatter<<<grid, kNT, 0, s>>>(*keys, *tmp, n, shift, so.hist, ntiles);
      ICUDA(cudaGetLastError());
      std::swap(*keys, *tmp);
    }
  }
  return GLP_OK;
}

// ------------------------------------------------------------- CSR steps
// Keys of the valid edges, appended through a warp-aggregated counter; bad
// ids (outside [0, n)) set bad.
__global__ void k_edge_keys(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t count,
                            int32_t n, int both, uint64_t* __restrict__ keys, unsigned long long* nkeys,
                            uint32_t* bad) {
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < count; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    int32_t u = 0, v = 0;
    bool ok = false;
    if (i < count) {
      u = src[i];
      v = dst[i];
      if (u < 0 || u >= n || v < 0 || v >= n) atomicOr(bad, 1u);
      else ok = u != v;
    }
    const uint32_t per = ok ? (both ? 2u : 1u) : 0u;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t incl = per;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    unsigned long long base = 0;
    if (lane == 0 && total) base = atomicAdd(nkeys, (unsigned long long)total);
    base = __shfl_sync(kFull, base, 0);
    if (ok) {
      const unsigned long long at = base + incl - per;
      keys[at] = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
      if (both) keys[at + 1] = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
    }
  }
}

__global__ void k_mark_unique(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ keep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    keep[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_compact(const uint64_t* __restrict__ in, int64_t n, const uint32_t* __restrict__ pos,
                          uint64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (i == 0 || in[i] != in[i - 1]) out[pos[i]] = in[i];
}

// off[u] = index of the first key of row u (a lower bound on u << 32), u in
// [0, n]; keys sorted.
__global__ void k_row_offsets(const uint64_t* __restrict__ keys, int64_t m, int32_t n, int32_t* __restrict__ off) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u <= n; u += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t want = (uint64_t)u << 32;
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < want) lo = mid + 1;
      else hi = mid;
    }
    off[u] = (int32_t)lo;
  }
}

// Relabel keys ((maxd - degree) << 32 | id) and the largest degree.
__global__ void k_degree_keys(const int32_t* __restrict__ off, int32_t n, int32_t maxd, uint64_t* __restrict__ keys) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    keys[v] = ((uint64_t)(uint32_t)(maxd - (off[v + 1] - off[v])) << 32) | (uint32_t)v;
}

__global__ void k_max_degree(const int32_t* __restrict__ off, int32_t n, int32_t* maxd) {
  int32_t best = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    best = max(best, off[v + 1] - off[v]);
  best = __reduce_max_sync(kFull, best);
  if ((threadIdx.x & 31) == 0) atomicMax(maxd, best);
}

// From the sorted relabel keys: old id of each new vertex, new id of each old.
__global__ void k_perm(const uint64_t* __restrict__ keys, int32_t n, int32_t* __restrict__ old_of,
                       int32_t* __restrict__ new_of) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t old = (int32_t)(uint32_t)keys[r];
    old_of[r] = old;
    new_of[old] = (int32_t)r;
  }
}

__global__ void k_remap(uint64_t* __restrict__ keys, int64_t m, const int32_t* __restrict__ new_of) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    keys[i] = ((uint64_t)(uint32_t)new_of[(uint32_t)(k >> 32)] << 32) | (uint32_t)new_of[(uint32_t)k];
  }
}

__global__ void k_ids(int32_t* __restrict__ a, int32_t n) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    a[v] = (int32_t)v;
}

__global__ void k_low_halves(const uint64_t* __restrict__ keys, int64_t m, int32_t* __restrict__ cols) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    cols[i] = (int32_t)(uint32_t)keys[i];
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(int64_t count) { return cudaMalloc(&p, sizeof(T) * (size_t)std::max<int64_t>(count, 1)); }
};

}  // namespace

namespace glp {

// Builds the CSR of an edge list on the current device.  *d_off ([n+1]) and
// *d_cols ([m], at least one entry) are cudaMalloc'd for the caller; d_old
// (nullable, device, [n]) receives the original id of each vertex.
int ingest_edges(const int32_t* src, const int32_t* dst, int64_t count, int32_t n, int32_t on_device, uint32_t flags,
                 int32_t** d_off_out, int32_t** d_cols_out, int64_t* m_out, int32_t* d_old, cudaStream_t s) {
  if (n < 1 || count < 0 || count >= (1ll << 30) || (count > 0 && (!src || !dst))) {
    set_error("bad edge list (n >= 1, 0 <= count < 2^30, src and dst given)");
    return GLP_EINVAL;
  }
  const bool both = (flags & GLP_EDGES_DIRECTED) == 0;
  const bool relabel = (flags & GLP_EDGES_KEEP_IDS) == 0;
  const int64_t cap = both ? 2 * count : count;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((cap + 255) / 256, (int64_t)device_sms() * 32));
  DevBuf<int32_t> in_src, in_dst;
  const int32_t* s_src = src;
  const int32_t* s_dst = dst;
  if (!on_device && count) {
    ICUDA(in_src.alloc(count));
    ICUDA(in_dst.alloc(count));
    ICUDA(cudaMemcpyAsync(in_src.p, src, sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
    ICUDA(cudaMemcpyAsync(in_dst.p, dst, sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
    s_src = in_src.p;
    s_dst = in_dst.p;
  }
  DevBuf<uint64_t> ka, kb;
  DevBuf<uint32_t> keep, hist, scratch, flags_d;
  DevBuf<unsigned long long> nk;
  ICUDA(ka.alloc(cap));
  ICUDA(kb.alloc(cap));
  ICUDA(nk.alloc(1));
  ICUDA(flags_d.alloc(2));
  ICUDA(cudaMemsetAsync(nk.p, 0, sizeof(unsigned long long), s));
  ICUDA(cudaMemsetAsync(flags_d.p, 0, 2 * sizeof(uint32_t), s));
  if (count) {
    k_edge_keys<<<grid, 256, 0, s>>>(s_src, s_dst, count, n, both ? 1 : 0, ka.p, nk.p, flags_d.p);
    ICUDA(cudaGetLastError());
  }
  unsigned long long nkeys = 0;
  uint32_t bad = 0;
  ICUDA(cudaMemcpyAsync(&nkeys, nk.p, sizeof nkeys, cudaMemcpyDeviceToHost, s));
  ICUDA(cudaMemcpyAsync(&bad, flags_d.p, sizeof bad, cudaMemcpyDeviceToHost, s));
  ICUDA(cudaStreamSynchronize(s));
  if (bad) {
    set_error("an edge names a vertex outside [0, n)");
    return GLP_EINVAL;
  }
  const int64_t nk0 = (int64_t)nkeys;
  const int64_t work = std::max<int64_t>(nk0, n);
  const int64_t ntiles = (work + kTile - 1) / kTile;
  ICUDA(hist.alloc((int64_t)kRadix * ntiles));
  ICUDA(scratch.alloc(std::max(scan_scratch((int64_t)kRadix * ntiles), scan_scratch(work))));
  ICUDA(keep.alloc(work));
  const Sorter so{hist.p, scratch.p, work};
  const int idb = (bit_length((uint64_t)(n - 1)) + 7) / 8 * 8;  // bits an id can occupy, whole digits
  std::vector<std::pair<int, int>> id_ranges{{0, idb}, {32, idb}};
  uint64_t* keys = ka.p;
  uint64_t* tmp = kb.p;
  int rc = radix_sort(&keys, &tmp, nk0, id_ranges, so, s);
  if (rc) return rc;
  // dedupe
  int64_t m = 0;
  if (nk0) {
    k_mark_unique<<<grid, 256, 0, s>>>(keys, nk0, keep.p);
    ICUDA(cudaGetLastError());
    uint32_t last_keep = 0, last_pos = 0;
    ICUDA(cudaMemcpyAsync(&last_keep, keep.p + nk0 - 1, sizeof last_keep, cudaMemcpyDeviceToHost, s));
    if ((rc = scan_u32(keep.p, nk0, scratch.p, s))) return rc;
    ICUDA(cudaMemcpyAsync(&last_pos, keep.p + nk0 - 1, sizeof last_pos, cudaMemcpyDeviceToHost, s));
    k_compact<<<grid, 256, 0, s>>>(keys, nk0, keep.p, tmp);
    ICUDA(cudaGetLastError());
    ICUDA(cudaStreamSynchronize(s));
    m = (int64_t)last_pos + last_keep;
    std::swap(keys, tmp);
  }
  if (m >= (1ll << 31)) {
    set_error("the graph exceeds an int32 CSR");
    return GLP_EINVAL;
  }
  int32_t* d_off = nullptr;
  int32_t* d_cols = nullptr;
  ICUDA(cudaMalloc(&d_off, sizeof(int32_t) * ((size_t)n + 1)));
  cudaError_t e = cudaMalloc(&d_cols, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  if (e != cudaSuccess) {
    cudaFree(d_off);
    return cuda_fail(e, "cudaMalloc(cols)");
  }
  auto fail = [&](int code) {
    cudaFree(d_off);
    cudaFree(d_cols);
    return code;
  };
  const unsigned vgrid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n + 256) / 256, (int64_t)device_sms() * 32));
  k_row_offsets<<<vgrid, 256, 0, s>>>(keys, m, n, d_off);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(e, "row offsets"));
  DevBuf<int32_t> new_of, old_of;
  if (relabel) {
    DevBuf<int32_t> maxd_d;
    if ((e = maxd_d.alloc(1)) != cudaSuccess || (e = new_of.alloc(n)) != cudaSuccess ||
        (e = old_of.alloc(n)) != cudaSuccess || (e = cudaMemsetAsync(maxd_d.p, 0, sizeof(int32_t), s)) != cudaSuccess)
      return fail(cuda_fail(e, "relabel buffers"));
    k_max_degree<<<vgrid, 256, 0, s>>>(d_off, n, maxd_d.p);
    int32_t maxd = 0;
    if ((e = cudaMemcpyAsync(&maxd, maxd_d.p, sizeof maxd, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fail(cuda_fail(e, "largest degree"));
    // (maxd - degree, id) keys, sorted: the new order of the vertices
    DevBuf<uint64_t> r1, r2;
    if ((e = r1.alloc(n)) != cudaSuccess || (e = r2.alloc(n)) != cudaSuccess)
      return fail(cuda_fail(e, "relabel sort buffers"));
    k_degree_keys<<<vgrid, 256, 0, s>>>(d_off, n, maxd, r1.p);
    const int degb = (bit_length((uint64_t)maxd) + 7) / 8 * 8;
    std::vector<std::pair<int, int>> rel{{0, idb}, {32, degb}};
    uint64_t* a = r1.p;
    uint64_t* b = r2.p;
    if ((rc = radix_sort(&a, &b, n, rel, so, s))) return fail(rc);
    k_perm<<<vgrid, 256, 0, s>>>(a, n, old_of.p, new_of.p);
    if (m) {
      k_remap<<<grid, 256, 0, s>>>(keys, m, new_of.p);
      uint64_t* other = (keys == ka.p) ? kb.p : ka.p;
      if ((rc = radix_sort(&keys, &other, m, id_ranges, so, s))) return fail(rc);
    }
    k_row_offsets<<<vgrid, 256, 0, s>>>(keys, m, n, d_off);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(e, "relabel"));
    if (d_old &&
        (e = cudaMemcpyAsync(d_old, old_of.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
      return fail(cuda_fail(e, "old ids"));
  } else if (d_old) {
    k_ids<<<vgrid, 256, 0, s>>>(d_old, n);
  }
  if (m) k_low_halves<<<grid, 256, 0, s>>>(keys, m, d_cols);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail(cuda_fail(e, "columns"));
  *d_off_out = d_off;
  *d_cols_out = d_cols;
  *m_out = m;
  return GLP_OK;
}

}  // namespace glp

extern "C" {

int glp_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t count, int32_t n, int32_t on_device,
                         uint32_t flags, int32_t* old_id, glp_graph** out) {
  if (!out) {
    glp::set_error("out is NULL");
    return GLP_EINVAL;
  }
  *out = nullptr;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    cudaGetLastError();
    glp::set_error("no usable CUDA device");
    return GLP_ENODEV;
  }
  cudaStream_t s = nullptr;
  ICUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int32_t *d_off = nullptr, *d_cols = nullptr, *d_old = nullptr;
  int64_t m = 0;
  int rc = GLP_OK;
  if (old_id) {
    if (on_device) {
      d_old = old_id;
    } else if (cudaMalloc(&d_old, sizeof(int32_t) * (size_t)std::max(n, 1)) != cudaSuccess) {
      glp::set_error("cudaMalloc(old ids)");
      rc = GLP_ENOMEM;
    }
  }
  if (!rc) rc = glp::ingest_edges(src, dst, count, n, on_device, flags, &d_off, &d_cols, &m, d_old, s);
  if (!rc && old_id && !on_device) {
    if (cudaMemcpyAsync(old_id, d_old, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      glp::set_error("copying the old ids to the host failed");
      rc = GLP_ECUDA;
    }
  }
  if (!rc)
    rc = glp_graph_create_ex(d_off, d_cols, nullptr, n, m, 1,
                             (flags & GLP_EDGES_DIRECTED) ? 0u : GLP_GRAPH_SYMMETRIC, out);
  if (old_id && !on_device && d_old) cudaFree(d_old);
  cudaFree(d_off);
  cudaFree(d_cols);
  cudaStreamDestroy(s);
  return rc;
}

}  // extern "C"
