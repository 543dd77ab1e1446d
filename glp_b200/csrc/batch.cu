// batch.cu -- batched classic LP: many independent graphs propagated by one
// persistent cooperative kernel launch over a packed multi-CSR.
//
// Layout.  G graphs are packed into one CSR of N = sum n_g vertices: global
// row offsets int64[N+1] and global column ids int32[M] (vertex i of graph g
// is vbase_g + i).  Labels stay LOCAL to their graph (0..n_g-1, what a solo
// run of that graph holds): every neighbour of a vertex lies in its graph, so
// the counts and the largest-label tie rule see exactly the labels of the
// solo run, and the packed label array is the per-graph result as it stands.
// This is the disjoint union of the graphs, so one synchronous step of the
// union is one synchronous step of every graph (the reference's single-graph
// rule, header/kernel.cuh:1655-1739, :4365-4426, :5187-5234).
//
// Work.  At creation the vertices are sorted, stably, into degree buckets
// (bounds 8, 16, 32, 64, 128, 256), high degree first; inside a bucket they
// keep id order, which is graph-major, so every sweep walks the graphs in
// order and the labels it gathers stay in L2.  A step is three static
// grid-stride sweeps over that order:
//   block tier  (WMAX < d <= 4096): a CTA per vertex, shared table of
//                                   pow2(2d) slots;
//   warp tier   (TT < d <= WMAX)  : a warp per vertex, its <= 8 labels per
//                                   lane held in registers: a strict-majority
//                                   test of the own label, else a per-warp
//                                   shared table;
//   thread tier (1 <= d <= TT)    : a thread per vertex, labels sorted in
//                                   registers (bitonic network), counts read
//                                   off the runs.
// Every step also writes a change flag per vertex (1 byte).  Once few labels
// still change (fewer than frontier_permille, default 10, per 1000 vertices
// in the previous step), a vertex first reads
// its neighbours' flags of the previous step: if none changed, its
// neighbourhood is what it was, so is its label (exact on any CSR); it keeps
// the label without gathering or counting.
// Neighbouring entries of the order have similar degrees, so the sweeps are
// balanced without a work queue.  Steps are separated by a grid
// barrier; the cooperative launch makes every CTA resident, and the barrier
// gives up after a time limit with an error bit instead of waiting forever.
// The first step, when every row is strictly ascending, is the closed form
// "last column" (labels are the ids, every count is 1, the largest wins).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/glp.h"
#include "device.cuh"
#include "smem_attr.h"

namespace glp {
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
}  // namespace glp

#define GLP_BCUDA(call)                                     \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return glp::cuda_fail(e_, #call); \
  } while (0)

namespace glp {
namespace {

constexpr int32_t kBatchMaxDegree = 4096;
constexpr uint32_t kErrBarrier = 8u;   // a grid barrier ran out of time
constexpr uint32_t kBadOffsets = 1u, kBadCols = 2u, kBadDegree = 4u, kUnsortedRow = 8u;
constexpr unsigned long long kBarrierLimitNs = 5000000000ull;  // default wait limit: 5 s

struct BatchArgs {
  const int64_t* off;      // [N+1] global row offsets
  const int32_t* cols;     // [M] global column ids
  const int32_t* order;    // [N] vertices by degree, descending
  const int64_t* vbase;    // [G+1]
  int32_t ngraphs;
  int32_t n;               // N
  int32_t nclass;          // iteration classes (graphs grouped by iteration count)
  int32_t class_niter[8];  // iterations of each class in this run
  int64_t class_v[9];      // class c owns vertices [class_v[c], class_v[c+1])
  int64_t bstart[8][9];    // class c, bucket q: order[bstart[c][q], bstart[c][q+1])
  uint32_t mode;           // kB* strategy bits
  uint32_t warp_words;     // shared words per warp for group tables
  uint32_t blk_cap;        // table slots of the block tier
  int32_t* lab0;
  int32_t* lab1;
  uint8_t* chg0;           // [N] changed in the last even / odd step (1) or not (0)
  uint8_t* chg1;
  uint32_t flag_pm;        // change-flag skips below this many changes per 1000 vertices
  unsigned long long* changed;  // [niter]
  unsigned int* bar;
  uint32_t* err;
  int32_t niter;
  int32_t first_step;      // rows strictly ascending
  unsigned long long barrier_ns;  // how long a grid barrier waits before giving up
  int32_t skip_cta;        // failure tests: 1 + a CTA that never arrives at the first barrier (0: none)
};

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier of a cooperative launch: CTA leaders add to a counter that
// never resets (phase p waits for (p+1)*gridDim.x arrivals).  A leader gives
// up after limit_ns of %globaltimer, or as soon as another CTA has given up;
// either way the kernel then returns with kErrBarrier set.  `arrive` = false
// withholds this CTA's arrival (failure tests: nobody's wait can be met).
__device__ bool grid_barrier(unsigned int* bar, unsigned int target, uint32_t* err,
                             unsigned long long limit_ns = kBarrierLimitNs, bool arrive = true) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (arrive) atomicAdd(bar, 1u);
    const uint64_t t0 = globaltimer();
    int ok = 1;
    while (ld_acquire(bar) < target) {
      if (*(volatile uint32_t*)err & kErrBarrier) {
        ok = 0;
        break;
      }
      if (globaltimer() - t0 > limit_ns) {
        atomicOr(err, kErrBarrier);
        ok = 0;
        break;
      }
      __nanosleep(256);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Graph of a global id: the last g with base[g] <= x (base non-decreasing).
__device__ __forceinline__ int32_t graph_of(const int64_t* base, int32_t ng, int64_t x) {
  int32_t lo = 0, hi = ng - 1;
  while (lo < hi) {
    const int32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(base + mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One vertex per group of G lanes (G | 32), at most G*L neighbours, L labels
// per lane in registers.  v < 0: this group has no vertex (it still takes
// part in the warp-wide shuffles).  keys/vals: the group's table slice of
// at least pow2(2*G*L) slots.  A strict majority of the own label decides
// the vertex when `majority` is set; otherwise (or when it fails) the labels
// are counted in the table, lanes holding the group leader's label adding
// once through the leader.  Returns "changed" on the group leader.
template <int G, int L>
__device__ __forceinline__ bool group_vertex(const BatchArgs& a, int32_t v, const int32_t* __restrict__ lin,
                                             int32_t* __restrict__ lout, uint32_t* keys, uint32_t* vals,
                                             bool majority, const uint8_t* __restrict__ fin,
                                             uint8_t* __restrict__ fout) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const uint32_t gmask = G == 32 ? kFull : (((1u << G) - 1u) << (lane & ~(G - 1)));
  int64_t b = 0;
  int32_t d = 0;
  if (v >= 0) {
    b = a.off[v];
    d = (int32_t)(a.off[v + 1] - b);
  }
  const int32_t dmax = __reduce_max_sync(kFull, d);
  int32_t lab[L];
#pragma unroll
  for (int q = 0; q < L; ++q) {
    const int32_t j = q * G + gl;
    lab[q] = (q * G < dmax && j < d) ? ld_stream(a.cols + b + j) : -1;
  }
  const int32_t own = v >= 0 ? lin[v] : -1;
  bool done = v < 0;
  if (fin) {  // no neighbour changed in the previous step: the label stays
    bool any = false;
#pragma unroll
    for (int q = 0; q < L; ++q)
      if (lab[q] >= 0) any = any || fin[lab[q]] != 0;
    const uint32_t group_any = __ballot_sync(kFull, any) & gmask;  // every lane takes part
    if (!done && !group_any) {
      if (gl == 0) {
        lout[v] = own;
        fout[v] = 0;
      }
      done = true;
    }
  }
#pragma unroll
  for (int q = 0; q < L; ++q)
    if (lab[q] >= 0 && !done) lab[q] = ld_label(lin + lab[q]);
  if (majority) {
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < L; ++q)
      if (q * G < dmax) c += __popc(__ballot_sync(kFull, lab[q] >= 0 && lab[q] == own) & gmask);
    if (!done && 2 * c > (uint32_t)d) {  // own label is the unique mode
      if (gl == 0) {
        lout[v] = own;
        fout[v] = 0;
      }
      done = true;
    }
  }
  const uint32_t cap = done ? 0u : pow2_ceil(2u * (uint32_t)d);
  __syncwarp();
  for (uint32_t s = gl; s < cap; s += G) {
    keys[s] = 0;
    vals[s] = 0;
  }
  __syncwarp();
  Best best = best_none();
  bool fail = false;
#pragma unroll
  for (int q = 0; q < L; ++q) {
    if (q * G >= dmax) break;  // warp-uniform
    bool has = !done && lab[q] >= 0;
    const int32_t l0 = __shfl_sync(kFull, has ? lab[q] : -1, 0, G);
    const uint32_t m0 = __ballot_sync(kFull, has && lab[q] == l0) & gmask;
    uint32_t k = 1;
    if (l0 >= 0) {
      if (gl == 0) k = (uint32_t)__popc(m0);
      else if (has && lab[q] == l0) has = false;
    }
    if (has) {
      const uint32_t tot = table_insert_bounded(keys, vals, cap - 1, (uint32_t)lab[q] + 1u, k, cap, nullptr, nullptr);
      if (tot == kNoSlot) {
        fail = true;
      } else {
        const Best c{(int64_t)tot, lab[q]};
        if (better(c, best)) best = c;
      }
    }
  }
  if (fail) atomicOr(a.err, kErrProbe);
  best = group_max<G>(best);
  if (done) return false;
  if (gl == 0) {
    lout[v] = best.l;
    fout[v] = best.l != own;
  }
  return gl == 0 && best.l != own;
}

template <int G, int L>
constexpr uint32_t group_slots() {  // pow2(2*G*L)
  uint32_t p = 1;
  while (p < 2u * G * L) p <<= 1;
  return p;
}

// Sweep order[lo, hi) with groups of G lanes; smem_warp: this warp's slice.
template <int NT, int G, int L>
__device__ __forceinline__ uint32_t sweep_groups(const BatchArgs& a, int64_t lo, int64_t hi,
                                                 const int32_t* __restrict__ lin, int32_t* __restrict__ lout,
                                                 uint32_t* smem_warp, bool majority, const uint8_t* fin,
                                                 uint8_t* fout) {
  constexpr int kGroups = 32 / G;
  constexpr uint32_t kSlots = group_slots<G, L>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int grp = lane / G;
  uint32_t* keys = smem_warp + (size_t)grp * 2 * kSlots;
  uint32_t* vals = keys + kSlots;
  const int64_t nw = (int64_t)gridDim.x * (NT / 32);
  uint32_t chg = 0;
  for (int64_t i0 = lo + ((int64_t)blockIdx.x * (NT / 32) + warp) * kGroups; i0 < hi; i0 += nw * kGroups) {
    const int64_t i = i0 + grp;
    const int32_t v = i < hi ? a.order[i] : -1;
    chg += group_vertex<G, L>(a, v, lin, lout, keys, vals, majority, fin, fout) ? 1u : 0u;
  }
  return chg;
}

// One vertex, one CTA (degree <= kBatchMaxDegree).  Returns "changed" on
// thread 0.
template <int NT>
__device__ __forceinline__ bool block_vertex(const BatchArgs& a, int32_t v, const int32_t* __restrict__ lin,
                                             int32_t* __restrict__ lout, uint32_t* smem, Best* red,
                                             const uint8_t* __restrict__ fin, uint8_t* __restrict__ fout) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t b = a.off[v];
  const int32_t d = (int32_t)(a.off[v + 1] - b);
  if (fin) {  // block-uniform: no neighbour changed in the previous step, the label stays
    bool any = false;
    for (int32_t j = threadIdx.x; j < d && !any; j += NT) any = fin[ld_stream(a.cols + b + j)] != 0;
    if (!__syncthreads_or(any)) {
      if (threadIdx.x == 0) {
        lout[v] = lin[v];
        fout[v] = 0;
      }
      return false;
    }
  }
  const uint32_t cap = pow2_ceil(2u * (uint32_t)d);
  uint32_t* keys = smem;
  uint32_t* vals = smem + cap;
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < 2 * cap; s += NT) smem[s] = 0;
  __syncthreads();
  Best best = best_none();
  bool fail = false;
  for (int32_t j0 = warp * 32; j0 < d; j0 += 4 * NT) {
    int32_t lab[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int32_t j = j0 + q * NT + lane;
      lab[q] = j < d ? ld_stream(a.cols + b + j) : -1;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (lab[q] >= 0) lab[q] = ld_label(lin + lab[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j0 + q * NT >= d) break;  // warp-uniform
      bool has = lab[q] >= 0;
      const int32_t l0 = __shfl_sync(kFull, has ? lab[q] : -1, 0);
      const uint32_t m0 = __ballot_sync(kFull, has && lab[q] == l0);
      uint32_t k = 1;
      if (l0 >= 0) {
        if (lane == 0) k = (uint32_t)__popc(m0);
        else if (has && lab[q] == l0) has = false;
      }
      if (has) {
        const uint32_t tot =
            table_insert_bounded(keys, vals, cap - 1, (uint32_t)lab[q] + 1u, k, cap, nullptr, nullptr);
        if (tot == kNoSlot) {
          fail = true;
        } else {
          const Best c{(int64_t)tot, lab[q]};
          if (better(c, best)) best = c;
        }
      }
    }
  }
  if (fail) atomicOr(a.err, kErrProbe);
  best = block_max<NT>(best, red);
  if (threadIdx.x == 0) {
    lout[v] = best.l;
    fout[v] = best.l != lin[v];
  }
  return threadIdx.x == 0 && best.l != lin[v];
}

// One vertex per thread (1 <= degree <= TT): its labels sorted in registers,
// counts read off the runs (sort_labels).
template <int TT>
__device__ __forceinline__ bool thread_vertex(const BatchArgs& a, int32_t v, const int32_t* __restrict__ lin,
                                              int32_t* __restrict__ lout, const uint8_t* __restrict__ fin,
                                              uint8_t* __restrict__ fout) {
  const int64_t b = a.off[v];
  const int32_t d = (int32_t)(a.off[v + 1] - b);
  int32_t lab[TT];
  uint32_t one[TT];
#pragma unroll
  for (int i = 0; i < TT; ++i) lab[i] = i < d ? ld_stream(a.cols + b + i) : -1;
  if (fin) {  // no neighbour changed in the previous step: the label stays
    bool any = false;
#pragma unroll
    for (int i = 0; i < TT; ++i)
      if (lab[i] >= 0) any = any || fin[lab[i]] != 0;
    if (!any) {
      lout[v] = lin[v];
      fout[v] = 0;
      return false;
    }
  }
#pragma unroll
  for (int i = 0; i < TT; ++i) lab[i] = lab[i] >= 0 ? ld_label(lin + lab[i]) : INT32_MAX;
  sort_labels<TT, false>(lab, one);
  Best best = best_none();
  uint32_t run = 0;
#pragma unroll
  for (int i = 0; i < TT; ++i) {
    run = (i > 0 && lab[i] == lab[i > 0 ? i - 1 : 0]) ? run + 1u : 1u;
    const bool end = (i == TT - 1) || lab[(i + 1) & (TT - 1)] != lab[i];
    if (end && lab[i] != INT32_MAX) {
      const Best c{(int64_t)run, lab[i]};
      if (better(c, best)) best = c;
    }
  }
  const int32_t own = lin[v];
  lout[v] = best.l;
  fout[v] = best.l != own;
  return best.l != own;
}

template <int NT, int TT>
__device__ __forceinline__ uint32_t sweep_threads(const BatchArgs& a, int64_t lo, int64_t hi,
                                                  const int32_t* __restrict__ lin, int32_t* __restrict__ lout,
                                                  const uint8_t* fin, uint8_t* fout) {
  uint32_t chg = 0;
  for (int64_t i = lo + (int64_t)blockIdx.x * NT + threadIdx.x; i < hi; i += (int64_t)gridDim.x * NT)
    chg += thread_vertex<TT>(a, a.order[i], lin, lout, fin, fout) ? 1u : 0u;
  return chg;
}

// Adds the CTA's changed count for a step (one atomic per CTA).
template <int NT>
__device__ __forceinline__ void block_count_add(unsigned long long* counter, uint32_t mine, uint32_t* red_u) {
  const uint32_t w = __reduce_add_sync(kFull, mine);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red_u[warp] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int i = 0; i < NT / 32; ++i) t += red_u[i];
    if (t) atomicAdd(counter, (unsigned long long)t);
  }
}

// Strategy bits of a run (how buckets 3..5 are counted).
constexpr uint32_t kB4Threads = 1u;  // degrees 17..32: a thread each (else 8-lane groups)
constexpr uint32_t kB5Threads = 2u;  // degrees 9..16: a thread each (else 4-lane groups)
constexpr uint32_t kB3Half = 4u;     // degrees 33..64: 16-lane groups (else whole warps)

template <int NT>
__global__ void __launch_bounds__(NT) k_batch(BatchArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ Best red[32];
  __shared__ uint32_t red_u[32];
  const int warp = threadIdx.x >> 5;
  const int64_t gthreads = (int64_t)gridDim.x * NT;
  unsigned int phase = 0;

  // labels = local ids in both buffers; with ascending rows the first step
  // is the last column of each row
  {
    uint32_t chg = 0;
    for (int64_t v = (int64_t)blockIdx.x * NT + threadIdx.x; v < a.n; v += gthreads) {
      const int32_t g = graph_of(a.vbase, a.ngraphs, v);
      const int32_t own = (int32_t)(v - a.vbase[g]);
      a.lab0[v] = own;
      int32_t nxt = own;
      if (a.first_step) {
        const int64_t e = a.off[v + 1];
        if (e > a.off[v]) nxt = (int32_t)(a.cols[e - 1] - a.vbase[g]);
        chg += nxt != own;
      }
      a.lab1[v] = nxt;
      a.chg0[v] = nxt != own;  // the first step's flags (none without it)
      a.chg1[v] = 0;
      if (nxt != own) {  // count it only for graphs that run a step
        int c = 0;
        while (c + 1 < a.nclass && v >= a.class_v[c + 1]) ++c;
        if (a.class_niter[c] == 0) --chg;
      }
    }
    if (a.first_step && a.niter > 0) block_count_add<NT>(a.changed, chg, red_u);
  }
  if (!grid_barrier(a.bar, ++phase * gridDim.x, a.err, a.barrier_ns, (int32_t)blockIdx.x + 1 != a.skip_cta))
    return;

  uint32_t* smem_warp = smem + (size_t)warp * a.warp_words;
  for (int32_t it = a.first_step ? 1 : 0; it < a.niter; ++it) {
    const int32_t* lin = (it & 1) ? a.lab1 : a.lab0;
    int32_t* lout = (it & 1) ? a.lab0 : a.lab1;
    // a vertex's own label decides it when it holds a strict majority; worth
    // testing once few labels still change
    const unsigned long long prev = it > 0 ? *(volatile unsigned long long*)(a.changed + it - 1) : ~0ull;
    const bool majority = prev < (unsigned long long)(a.n / 4);
    // the previous step's flags (written by every vertex it counted; the
    // first step's by the set-up above), once few labels still change
    const uint8_t* fin =
        prev * 1000ull < (unsigned long long)a.flag_pm * (unsigned long long)a.n ? ((it & 1) ? a.chg0 : a.chg1)
                                                                                 : nullptr;
    uint8_t* fout = (it & 1) ? a.chg1 : a.chg0;
    uint32_t chg = 0;
    for (int c = 0; c < a.nclass; ++c) {
      if (it >= a.class_niter[c]) continue;  // this class has finished
      const int64_t* B = a.bstart[c];
      for (int64_t i = B[0] + blockIdx.x; i < B[1]; i += gridDim.x)
        chg += block_vertex<NT>(a, a.order[i], lin, lout, smem, red, fin, fout) ? 1u : 0u;
      chg += sweep_groups<NT, 32, 8>(a, B[1], B[2], lin, lout, smem_warp, majority, fin, fout);
      chg += sweep_groups<NT, 32, 4>(a, B[2], B[3], lin, lout, smem_warp, majority, fin, fout);
      if (a.mode & kB3Half) chg += sweep_groups<NT, 16, 4>(a, B[3], B[4], lin, lout, smem_warp, majority, fin, fout);
      else chg += sweep_groups<NT, 32, 2>(a, B[3], B[4], lin, lout, smem_warp, majority, fin, fout);
      if (a.mode & kB4Threads) chg += sweep_threads<NT, 32>(a, B[4], B[5], lin, lout, fin, fout);
      else chg += sweep_groups<NT, 8, 4>(a, B[4], B[5], lin, lout, smem_warp, majority, fin, fout);
      if (a.mode & kB5Threads) chg += sweep_threads<NT, 16>(a, B[5], B[6], lin, lout, fin, fout);
      else chg += sweep_groups<NT, 4, 4>(a, B[5], B[6], lin, lout, smem_warp, majority, fin, fout);
      chg += sweep_threads<NT, 8>(a, B[6], B[7], lin, lout, fin, fout);
    }
    block_count_add<NT>(a.changed + it, chg, red_u);
    if (it + 1 < a.niter && !grid_barrier(a.bar, ++phase * gridDim.x, a.err, a.barrier_ns)) return;
  }
}

// ------------------------------------------------------------ packing
// Vertex pass: global offsets from the staged local ones (graph g's n_g+1
// local offsets start at vbase_g + g), offset checks, degree histogram and
// the strictly-ascending-rows test.
__global__ void k_pack_vertices(const int32_t* __restrict__ loc_off, const int64_t* __restrict__ vbase,
                                const int64_t* __restrict__ ebase, int32_t ng, int64_t n, int64_t* __restrict__ off,
                                unsigned long long* __restrict__ hist, uint32_t* flags) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = graph_of(vbase, ng, v);
    const int64_t i = v - vbase[g];
    const int64_t s = vbase[g] + g + i;  // staged index of local offset i
    const int32_t o0 = loc_off[s], o1 = loc_off[s + 1];
    const int64_t ng_v = vbase[g + 1] - vbase[g];
    const int64_t mg = ebase[g + 1] - ebase[g];
    if ((i == 0 && o0 != 0) || (i + 1 == ng_v && (int64_t)o1 != mg) || o1 < o0 || o0 < 0 || (int64_t)o1 > mg) {
      atomicOr(flags, kBadOffsets);
      continue;
    }
    off[v] = ebase[g] + o0;
    if (v + 1 == n) off[n] = ebase[g] + o1;
    const int32_t d = o1 - o0;
    if (d > kBatchMaxDegree) {
      atomicOr(flags, kBadDegree);
      continue;
    }
    atomicAdd(hist + d, 1ull);
  }
}

// Edge pass (after the vertex pass succeeded): columns in [0, n_g), to
// global ids.
__global__ void k_pack_cols(int32_t* __restrict__ cols, const int64_t* __restrict__ vbase,
                            const int64_t* __restrict__ ebase, int32_t ng, int64_t m, uint32_t* flags) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = graph_of(ebase, ng, e);
    const int32_t c = cols[e];
    if (c < 0 || (int64_t)c >= vbase[g + 1] - vbase[g]) {
      atomicOr(flags, kBadCols);
      continue;
    }
    cols[e] = (int32_t)(vbase[g] + c);
  }
}

// Rows strictly ascending (first-step closed form), a warp per row.
__global__ void k_pack_sorted(const int64_t* __restrict__ off, const int32_t* __restrict__ cols, int64_t n,
                              uint32_t* flags) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; v < n; v += nw) {
    const int64_t b = off[v], e = off[v + 1];
    bool bad = false;
    for (int64_t j = b + 1 + lane; j < e; j += 32) bad |= cols[j] <= cols[j - 1];
    if (__any_sync(kFull, bad)) {
      if (lane == 0) atomicOr(flags, kUnsortedRow);
    }
  }
}

// Work order: vertices stably sorted into degree buckets, from high degree to
// low; inside a bucket they keep id order, which is graph-major, so each
// sweep walks the graphs in order and the labels it gathers stay in L2.
// Bucket bounds are the only tier bounds a run may pick.
constexpr int kBuckets = 8;
__host__ __device__ __forceinline__ int bucket_of(int32_t d) {
  return d > 256 ? 0 : d > 128 ? 1 : d > 64 ? 2 : d > 32 ? 3 : d > 16 ? 4 : d > 8 ? 5 : d > 0 ? 6 : 7;
}
constexpr int kOrderChunk = 2048;  // vertices per block in the two passes below
constexpr int kMaxClasses = 8;     // distinct iteration counts in one batch
constexpr int kKeys = kMaxClasses * kBuckets;

struct ClassRanges {
  int64_t vstart[kMaxClasses + 1];  // class c owns vertices [vstart[c], vstart[c+1])
  int32_t nclass;
};
__device__ __forceinline__ int class_of(const ClassRanges& cr, int64_t v) {
  int c = 0;
  while (c + 1 < cr.nclass && v >= cr.vstart[c + 1]) ++c;
  return c;
}
__device__ __forceinline__ int order_key(const int64_t* __restrict__ off, const ClassRanges& cr, int64_t v) {
  return class_of(cr, v) * kBuckets + bucket_of((int32_t)(off[v + 1] - off[v]));
}

// Pass 1: per block (a chunk of kOrderChunk consecutive vertices) the number
// of its vertices under each (class, bucket) key.
__global__ void __launch_bounds__(256) k_order_count(const int64_t* __restrict__ off, int64_t n, ClassRanges cr,
                                                     uint32_t* __restrict__ counts) {
  __shared__ uint32_t c[kKeys];
  if (threadIdx.x < kKeys) c[threadIdx.x] = 0;
  __syncthreads();
  const int64_t v0 = (int64_t)blockIdx.x * kOrderChunk;
  for (int64_t v = v0 + threadIdx.x; v < n && v < v0 + kOrderChunk; v += 256) atomicAdd(&c[order_key(off, cr, v)], 1u);
  __syncthreads();
  if (threadIdx.x < kKeys) counts[(size_t)blockIdx.x * kKeys + threadIdx.x] = c[threadIdx.x];
}

// Pass 2: each block places its vertices at start[block][key] onwards in id
// order (ranks inside a warp from __match_any_sync, then by warp).
__global__ void __launch_bounds__(256) k_order_scatter(const int64_t* __restrict__ off, int64_t n, ClassRanges cr,
                                                       const int64_t* __restrict__ start,
                                                       int32_t* __restrict__ order) {
  __shared__ uint32_t wc[8][kKeys];  // per warp, per key
  __shared__ int64_t run[kKeys];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < kKeys) run[threadIdx.x] = start[(size_t)blockIdx.x * kKeys + threadIdx.x];
  const int64_t v0 = (int64_t)blockIdx.x * kOrderChunk;
  for (int64_t s0 = v0; s0 < v0 + kOrderChunk && s0 < n; s0 += 256) {
    for (int i = threadIdx.x; i < 8 * kKeys; i += 256) (&wc[0][0])[i] = 0;
    __syncthreads();
    const int64_t v = s0 + threadIdx.x;
    const int key = v < n ? order_key(off, cr, v) : -1;
    const uint32_t peers = __match_any_sync(kFull, key);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (key >= 0 && rank == 0) wc[warp][key] = __popc(peers);
    __syncthreads();
    if (key >= 0) {
      int64_t pos = run[key] + rank;
      for (int w = 0; w < warp; ++w) pos += wc[w][key];
      order[pos] = (int32_t)v;
    }
    __syncthreads();
    if (threadIdx.x < kKeys) {
      uint32_t t = 0;
      for (int w = 0; w < 8; ++w) t += wc[w][threadIdx.x];
      run[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

struct Config {
  int nt = 1024;   // threads per CTA
  int tt = 32;     // degrees <= tt: a thread per vertex (8, 16 or 32)
  int half = 1;    // degrees 33..64: 16-lane groups (else whole warps)
  unsigned long long barrier_ns = kBarrierLimitNs;  // grid-barrier wait limit
  int skip_cta = 0;  // failure tests: 1 + a CTA withholding its first arrival
  int blocks = 0;    // CTAs of the cooperative grid (0: as many as fit every SM)
  uint32_t flag_pm = 10;  // change-flag skips below this many changes per 1000 vertices (0: never)
  bool operator==(const Config& o) const {
    return nt == o.nt && tt == o.tt && half == o.half && barrier_ns == o.barrier_ns && skip_cta == o.skip_cta &&
           blocks == o.blocks && flag_pm == o.flag_pm;
  }
};

}  // namespace
}  // namespace glp

struct glp_batch {
  int device = 0;
  int32_t ngraphs = 0;
  int64_t n = 0, m = 0;
  int32_t max_degree = 0;
  int first_step = 0;
  int64_t* d_off = nullptr;
  int32_t* d_cols = nullptr;
  int32_t* d_order = nullptr;
  int64_t* d_vbase = nullptr;
  int64_t* d_ebase = nullptr;
  int32_t* d_stage = nullptr;        // staged local offsets
  uint32_t* d_counts = nullptr;      // per-block (class, bucket) counts
  int64_t* d_start = nullptr;        // per-block (class, bucket) starts
  unsigned long long* d_hist = nullptr;
  uint32_t* d_flags = nullptr;
  size_t cap_off = 0, cap_cols = 0, cap_order = 0, cap_vbase = 0, cap_ebase = 0, cap_stage = 0, cap_counts = 0,
         cap_start = 0, cap_lab[2] = {0, 0};
  std::vector<uint32_t> h_counts;
  std::vector<int64_t> h_starts;
  std::vector<int64_t> h_vbase, h_ebase;
  std::vector<unsigned long long> hist;  // vertices per degree 0..kBatchMaxDegree
  // iteration classes: graphs with equal iteration counts, contiguous
  int32_t nclass = 1;
  int32_t class_niter[8] = {0};
  int64_t class_v[9] = {0};
  int64_t bstart[8][9] = {{0}};
  int32_t* d_lab[2] = {nullptr, nullptr};
  uint8_t* d_chg[2] = {nullptr, nullptr};  // per-vertex change flags of the last even / odd step
  size_t cap_chg[2] = {0, 0};
  unsigned long long* d_changed = nullptr;
  int32_t changed_cap = 0;
  unsigned int* d_bar = nullptr;
  uint32_t* d_err = nullptr;
  cudaStream_t stream = nullptr;
  int nsm = 1;  // the device's SM count, queried when the batch is created
  glp::Config cfg;
  bool tuned = false;
  // captured launch
  cudaGraphExec_t gexec = nullptr;
  int32_t g_niter = -1;
  glp::Config g_cfg;
  int32_t* g_labels = nullptr;
  cudaStream_t g_stream = nullptr;
};

namespace glp {
namespace {

uint32_t pow2_host(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

int max_degree_in(const glp_batch* b, int lo, int hi) {  // largest degree d with lo < d <= hi present
  for (int d = std::min(hi, kBatchMaxDegree); d > lo; --d)
    if (b->hist[d]) return d;
  return 0;
}

template <int NT>
int launch_k(glp_batch* b, const BatchArgs& a, size_t smem, cudaStream_t s, int max_blocks) {
  auto kern = k_batch<NT>;
  GLP_BCUDA(raise_smem_limit((const void*)kern, smem));
  int per_sm = 0;
  GLP_BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  if (per_sm < 1) {
    set_error("batch kernel does not fit an SM (%d threads, %zu B shared)", NT, smem);
    return GLP_ENOTSUP;
  }
  cudaLaunchConfig_t lc = {};
  // a smaller grid leaves SMs to other work: its CTAs can all become resident
  // while other kernels still hold the rest of the GPU
  const int fit = per_sm * b->nsm;
  lc.gridDim = dim3((unsigned)(max_blocks > 0 ? std::min(max_blocks, fit) : fit));
  lc.blockDim = dim3(NT);
  lc.dynamicSmemBytes = smem;
  lc.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  GLP_BCUDA(cudaLaunchKernelEx(&lc, kern, a));
  return GLP_OK;
}

int launch_cfg(glp_batch* b, const Config& c, const BatchArgs& a, cudaStream_t s) {
  const size_t smem = std::max<size_t>((size_t)(c.nt / 32) * a.warp_words, 2 * (size_t)a.blk_cap) * sizeof(uint32_t);
  if (c.nt == 512) return launch_k<512>(b, a, smem, s, c.blocks);
  if (c.nt == 1024) return launch_k<1024>(b, a, smem, s, c.blocks);
  set_error("no batch kernel for %d threads per block", c.nt);
  return GLP_EINVAL;
}

// niter >= 0: every graph runs niter iterations; GLP_BATCH_OWN_ITERATIONS:
// each graph runs the count it was created with.
int32_t run_niter(const glp_batch* b, int32_t niter, int c) { return niter >= 0 ? niter : b->class_niter[c]; }
int32_t max_niter(const glp_batch* b, int32_t niter) {
  int32_t mx = 0;
  for (int c = 0; c < b->nclass; ++c) mx = std::max(mx, run_niter(b, niter, c));
  return mx;
}

BatchArgs make_args(glp_batch* b, const Config& c, int32_t niter) {
  BatchArgs a{};
  a.off = b->d_off;
  a.cols = b->d_cols;
  a.order = b->d_order;
  a.vbase = b->d_vbase;
  a.ngraphs = b->ngraphs;
  a.n = (int32_t)b->n;
  a.nclass = b->nclass;
  for (int k = 0; k < b->nclass; ++k) {
    a.class_niter[k] = run_niter(b, niter, k);
    for (int q = 0; q <= kBuckets; ++q) a.bstart[k][q] = b->bstart[k][q];
  }
  for (int k = 0; k <= b->nclass; ++k) a.class_v[k] = b->class_v[k];
  a.mode = (c.tt >= 32 ? kB4Threads : 0u) | (c.tt >= 16 ? kB5Threads : 0u) | (c.half ? kB3Half : 0u);
  a.warp_words = max_degree_in(b, 128, 256) ? 2 * group_slots<32, 8>() : 2 * group_slots<32, 4>();
  const int bdeg = max_degree_in(b, 256, kBatchMaxDegree);
  a.blk_cap = bdeg ? pow2_host(2u * (uint32_t)bdeg) : 0u;
  a.lab0 = b->d_lab[0];
  a.lab1 = b->d_lab[1];
  a.chg0 = b->d_chg[0];
  a.chg1 = b->d_chg[1];
  a.flag_pm = c.flag_pm;
  a.changed = b->d_changed;
  a.bar = b->d_bar;
  a.err = b->d_err;
  a.niter = max_niter(b, niter);
  a.first_step = b->first_step;
  a.barrier_ns = c.barrier_ns;
  a.skip_cta = c.skip_cta;
  return a;
}

int ensure_changed(glp_batch* b, int32_t niter) {
  if (niter <= b->changed_cap) return GLP_OK;
  cudaFree(b->d_changed);
  b->d_changed = nullptr;
  b->changed_cap = 0;
  GLP_BCUDA(cudaMalloc(&b->d_changed, sizeof(unsigned long long) * std::max(niter, 1)));
  b->changed_cap = std::max(niter, 1);
  return GLP_OK;
}

// Enqueues one whole run (reset of counters and barrier, the persistent
// launch) on s.
int enqueue_run(glp_batch* b, const Config& c, int32_t niter, cudaStream_t s) {
  GLP_BCUDA(cudaMemsetAsync(b->d_changed, 0, sizeof(unsigned long long) * std::max(max_niter(b, niter), 1), s));
  GLP_BCUDA(cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned int), s));
  GLP_BCUDA(cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), s));
  if (b->n == 0) return GLP_OK;
  return launch_cfg(b, c, make_args(b, c, niter), s);
}

int check_batch_err(glp_batch* b, cudaStream_t s) {
  uint32_t err = 0;
  GLP_BCUDA(cudaMemcpyAsync(&err, b->d_err, sizeof err, cudaMemcpyDeviceToHost, s));
  GLP_BCUDA(cudaStreamSynchronize(s));
  if (err & kErrBarrier) {
    set_error("a grid barrier of the batch kernel timed out");
    return GLP_ETIMEOUT;
  }
  if (err) {
    set_error("batch kernel error flags 0x%x", err);
    return GLP_EKERNEL;
  }
  return GLP_OK;
}

Config config_from(const glp_batch* b, const glp_params* p) {
  Config c = b->cfg;
  if (p) {
    if (p->tiny_max == 8 || p->tiny_max == 16 || p->tiny_max == 32) c.tt = p->tiny_max;
    if (p->mid_max == 32) c.half = 0;
    if (p->mid_max == 64) c.half = 1;
    if (p->batch_threads == 512 || p->batch_threads == 1024) c.nt = p->batch_threads;
    c.barrier_ns = p->barrier_limit_us > 0 ? 1000ull * (unsigned long long)p->barrier_limit_us : kBarrierLimitNs;
    c.skip_cta = p->fault_skip_cta > 0 ? p->fault_skip_cta : 0;
    c.blocks = p->batch_blocks > 0 ? p->batch_blocks : 0;
    c.flag_pm = p->frontier_permille > 0 ? (uint32_t)std::min(p->frontier_permille, 1000)
                : p->frontier_permille < 0 ? 0u : 10u;
  }
  return c;
}

void free_graph_exec(glp_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->g_niter = -1;
}

// Grow-only device buffer: reallocated only when a larger one is needed, so
// repacking a batch allocates nothing once it has seen its largest round.
template <class T>
int grow(T** p, size_t* cap, size_t need) {
  need = std::max<size_t>(need, 1);
  if (*p && *cap >= need) return GLP_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t want = need + need / 4;
  GLP_BCUDA(cudaMalloc(p, sizeof(T) * want));
  *cap = want;
  return GLP_OK;
}

int init_device(glp_batch* b) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    set_error("no usable CUDA device");
    return GLP_ENODEV;
  }
  GLP_BCUDA(cudaGetDevice(&b->device));
  GLP_BCUDA(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device));
  int coop = 0;
  GLP_BCUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->device));
  if (!coop) {
    set_error("device %d has no cooperative launch", b->device);
    return GLP_ENOTSUP;
  }
  GLP_BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  GLP_BCUDA(cudaMalloc(&b->d_bar, sizeof(unsigned int)));
  GLP_BCUDA(cudaMalloc(&b->d_err, sizeof(uint32_t)));
  GLP_BCUDA(cudaMalloc(&b->d_flags, sizeof(uint32_t)));
  GLP_BCUDA(cudaMalloc(&b->d_hist, sizeof(unsigned long long) * (kBatchMaxDegree + 1)));
  return ensure_changed(b, 32);
}

// (Re)packs the graphs into b's buffers and builds the work order.
int pack(glp_batch* b, int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols, const int32_t* n,
         const int64_t* m, int32_t on_device, const int32_t* niter) {
  if (ngraphs < 0 || (ngraphs > 0 && (!offsets || !cols || !n || !m))) {
    set_error("bad batch arguments");
    return GLP_EINVAL;
  }
  b->ngraphs = ngraphs;
  b->n = b->m = 0;
  b->h_vbase.assign((size_t)ngraphs + 1, 0);
  b->h_ebase.assign((size_t)ngraphs + 1, 0);
  for (int32_t g = 0; g < ngraphs; ++g) {
    if (n[g] < 0 || m[g] < 0 || !offsets[g] || (m[g] > 0 && !cols[g])) {
      set_error("graph %d: bad arguments (n=%d, m=%lld)", g, n[g], (long long)m[g]);
      b->ngraphs = 0;
      return GLP_EINVAL;
    }
    b->h_vbase[g + 1] = b->h_vbase[g] + n[g];
    b->h_ebase[g + 1] = b->h_ebase[g] + m[g];
  }
  const int64_t N = b->h_vbase[ngraphs], M = b->h_ebase[ngraphs];
  if (N >= INT32_MAX) {
    set_error("batch of %lld vertices exceeds the packed layout", (long long)N);
    b->ngraphs = 0;
    return GLP_EINVAL;
  }
  // iteration classes: runs of equal counts (graphs sorted by count)
  b->nclass = 1;
  b->class_v[0] = 0;
  b->class_niter[0] = 0;
  if (niter) {
    for (int32_t g = 0; g < ngraphs; ++g) {
      if (niter[g] < 0 || (g > 0 && niter[g] < niter[g - 1])) {
        set_error("per-graph iteration counts must be >= 0 and non-decreasing (graph %d)", g);
        b->ngraphs = 0;
        return GLP_EINVAL;
      }
      if (g == 0) {
        b->class_niter[0] = niter[0];
      } else if (niter[g] != niter[g - 1]) {
        if (b->nclass == kMaxClasses) {
          set_error("more than %d distinct iteration counts in one batch", kMaxClasses);
          b->ngraphs = 0;
          return GLP_ENOTSUP;
        }
        b->class_v[b->nclass] = b->h_vbase[g];
        b->class_niter[b->nclass++] = niter[g];
      }
    }
  }
  b->class_v[b->nclass] = N;
  int rc;
  const int64_t nblocks = std::max<int64_t>((N + kOrderChunk - 1) / kOrderChunk, 1);
  if ((rc = grow(&b->d_off, &b->cap_off, (size_t)N + 1)) || (rc = grow(&b->d_cols, &b->cap_cols, (size_t)M)) ||
      (rc = grow(&b->d_order, &b->cap_order, (size_t)N)) || (rc = grow(&b->d_vbase, &b->cap_vbase, (size_t)ngraphs + 1)) ||
      (rc = grow(&b->d_ebase, &b->cap_ebase, (size_t)ngraphs + 1)) ||
      (rc = grow(&b->d_lab[0], &b->cap_lab[0], (size_t)N)) || (rc = grow(&b->d_lab[1], &b->cap_lab[1], (size_t)N)) ||
      (rc = grow(&b->d_chg[0], &b->cap_chg[0], (size_t)N)) || (rc = grow(&b->d_chg[1], &b->cap_chg[1], (size_t)N)) ||
      (rc = grow(&b->d_stage, &b->cap_stage, (size_t)(N + ngraphs + 1))) ||
      (rc = grow(&b->d_counts, &b->cap_counts, (size_t)nblocks * kKeys)) ||
      (rc = grow(&b->d_start, &b->cap_start, (size_t)nblocks * kKeys))) {
    b->ngraphs = 0;
    return rc;
  }
  b->n = N;
  b->m = M;
  cudaStream_t s = b->stream;
  auto bad = [&](int code, const char* msg) {
    set_error("%s", msg);
    b->ngraphs = 0;
    b->n = b->m = 0;
    return code;
  };
  cudaError_t e;
  auto fail = [&](cudaError_t err, const char* what) {
    b->ngraphs = 0;
    b->n = b->m = 0;
    return cuda_fail(err, what);
  };
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  // staging: local offsets of graph g at [vbase_g + g, vbase_g + g + n_g]
  for (int32_t g = 0; g < ngraphs; ++g) {
    if ((e = cudaMemcpyAsync(b->d_stage + b->h_vbase[g] + g, offsets[g], sizeof(int32_t) * ((size_t)n[g] + 1), kind,
                             s)) != cudaSuccess)
      return fail(e, "batch offsets copy");
    if (m[g] && (e = cudaMemcpyAsync(b->d_cols + b->h_ebase[g], cols[g], sizeof(int32_t) * (size_t)m[g], kind, s)) !=
                    cudaSuccess)
      return fail(e, "batch columns copy");
  }
  if ((e = cudaMemcpyAsync(b->d_vbase, b->h_vbase.data(), sizeof(int64_t) * (ngraphs + 1), cudaMemcpyHostToDevice,
                           s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_ebase, b->h_ebase.data(), sizeof(int64_t) * (ngraphs + 1), cudaMemcpyHostToDevice,
                           s)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_hist, 0, sizeof(unsigned long long) * (kBatchMaxDegree + 1), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_flags, 0, sizeof(uint32_t), s)) != cudaSuccess)
    return fail(e, "batch set-up");
  const unsigned grid = (unsigned)std::max(1, b->nsm * 8);
  if (N)
    k_pack_vertices<<<grid, 256, 0, s>>>(b->d_stage, b->d_vbase, b->d_ebase, ngraphs, N, b->d_off, b->d_hist,
                                         b->d_flags);
  else if ((e = cudaMemsetAsync(b->d_off, 0, sizeof(int64_t), s)) != cudaSuccess)
    return fail(e, "batch offsets");
  uint32_t flags = 0;
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(&flags, b->d_flags, sizeof flags, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail(e, "batch vertex pass");
  if (flags & kBadOffsets)
    return bad(GLP_EINVAL, "a graph's offsets are malformed (offsets[0] = 0, non-decreasing, offsets[n] = m)");
  if (flags & kBadDegree)
    return bad(GLP_ENOTSUP, "a vertex degree exceeds the batch limit of 4096 (run that graph through glp_run)");
  if (M) k_pack_cols<<<grid, 256, 0, s>>>(b->d_cols, b->d_vbase, b->d_ebase, ngraphs, M, b->d_flags);
  if (N) k_pack_sorted<<<grid, 256, 0, s>>>(b->d_off, b->d_cols, N, b->d_flags);
  b->hist.assign(kBatchMaxDegree + 1, 0ull);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(&flags, b->d_flags, sizeof flags, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->hist.data(), b->d_hist, sizeof(unsigned long long) * (kBatchMaxDegree + 1),
                           cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail(e, "batch edge pass");
  if (flags & kBadCols) return bad(GLP_EINVAL, "a column index lies outside its graph's [0, n)");
  b->first_step = (flags & kUnsortedRow) ? 0 : 1;
  b->max_degree = 0;
  for (int d = kBatchMaxDegree; d >= 0; --d)
    if (b->hist[d]) {
      b->max_degree = d;
      break;
    }
  // work order (two passes, per-block (class, bucket) starts from the host):
  // class-major, then bucket-major, then vertex id
  ClassRanges cr{};
  cr.nclass = b->nclass;
  for (int c = 0; c <= b->nclass; ++c) cr.vstart[c] = b->class_v[c];
  for (int c = 0; c < kMaxClasses; ++c)
    for (int q = 0; q <= kBuckets; ++q) b->bstart[c][q] = 0;
  if (N) {
    std::vector<uint32_t>& counts = b->h_counts;
    std::vector<int64_t>& starts = b->h_starts;
    counts.resize((size_t)nblocks * kKeys);
    starts.resize((size_t)nblocks * kKeys);
    k_order_count<<<(unsigned)nblocks, 256, 0, s>>>(b->d_off, N, cr, b->d_counts);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(counts.data(), b->d_counts, sizeof(uint32_t) * counts.size(), cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fail(e, "batch order count");
    int64_t acc = 0;
    for (int key = 0; key < kKeys; ++key) {
      const int c = key / kBuckets, q = key % kBuckets;
      if (c < b->nclass) b->bstart[c][q] = acc;
      for (int64_t k = 0; k < nblocks; ++k) {
        starts[(size_t)k * kKeys + key] = acc;
        acc += counts[(size_t)k * kKeys + key];
      }
      if (c < b->nclass) b->bstart[c][q + 1] = acc;
    }
    if ((e = cudaMemcpyAsync(b->d_start, starts.data(), sizeof(int64_t) * starts.size(), cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
      return fail(e, "batch order starts");
    k_order_scatter<<<(unsigned)nblocks, 256, 0, s>>>(b->d_off, N, cr, b->d_start, b->d_order);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fail(e, "batch order scatter");
  }
  return GLP_OK;
}

}  // namespace
}  // namespace glp

using namespace glp;

extern "C" {

int glp_batch_create(int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols, const int32_t* n,
                     const int64_t* m, int32_t on_device, glp_batch** out) {
  return glp_batch_create_ex(ngraphs, offsets, cols, n, m, on_device, nullptr, out);
}

int glp_batch_create_ex(int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols, const int32_t* n,
                        const int64_t* m, int32_t on_device, const int32_t* niter, glp_batch** out) {
  if (!out) {
    set_error("out is NULL");
    return GLP_EINVAL;
  }
  *out = nullptr;
  std::unique_ptr<glp_batch> b(new glp_batch());
  int rc = init_device(b.get());
  if (rc) {
    glp_batch_destroy(b.release());
    return rc;
  }
  if ((rc = pack(b.get(), ngraphs, offsets, cols, n, m, on_device, niter))) {
    glp_batch_destroy(b.release());
    return rc;
  }
  *out = b.release();
  return GLP_OK;
}

int glp_batch_repack(glp_batch* b, int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols,
                     const int32_t* n, const int64_t* m, int32_t on_device, const int32_t* niter) {
  if (!b) {
    set_error("batch is NULL");
    return GLP_EINVAL;
  }
  free_graph_exec(b);
  return pack(b, ngraphs, offsets, cols, n, m, on_device, niter);
}

void glp_batch_destroy(glp_batch* b) {
  if (!b) return;
  free_graph_exec(b);
  cudaFree(b->d_off);
  cudaFree(b->d_cols);
  cudaFree(b->d_order);
  cudaFree(b->d_vbase);
  cudaFree(b->d_ebase);
  cudaFree(b->d_stage);
  cudaFree(b->d_counts);
  cudaFree(b->d_start);
  cudaFree(b->d_hist);
  cudaFree(b->d_flags);
  cudaFree(b->d_lab[0]);
  cudaFree(b->d_lab[1]);
  cudaFree(b->d_chg[0]);
  cudaFree(b->d_chg[1]);
  cudaFree(b->d_changed);
  cudaFree(b->d_bar);
  cudaFree(b->d_err);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int glp_batch_info(const glp_batch* b, int64_t* n, int64_t* m, int32_t* max_degree, int32_t* ngraphs) {
  if (!b) {
    set_error("batch is NULL");
    return GLP_EINVAL;
  }
  if (n) *n = b->n;
  if (m) *m = b->m;
  if (max_degree) *max_degree = b->max_degree;
  if (ngraphs) *ngraphs = b->ngraphs;
  return GLP_OK;
}

int glp_batch_run(glp_batch* b, const glp_params* p, int32_t niter, int32_t* labels, int32_t on_device,
                  int64_t* changed, void* stream) {
  if (!b || niter < GLP_BATCH_OWN_ITERATIONS || (!labels && b->n > 0)) {
    set_error("bad arguments to glp_batch_run");
    return GLP_EINVAL;
  }
  if (p && p->struct_size != (int32_t)sizeof(glp_params)) {
    set_error("glp_params.struct_size mismatch");
    return GLP_EINVAL;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  const Config c = config_from(b, p);
  const int32_t total = max_niter(b, niter);
  int rc = ensure_changed(b, total);
  if (rc) return rc;
  // graph g's labels end in the buffer of its iteration count's parity
  auto copy_out = [&](cudaMemcpyKind kind) -> cudaError_t {
    for (int k = 0; k < b->nclass; ++k) {
      const int64_t lo = b->class_v[k], hi = b->class_v[k + 1];
      if (hi <= lo) continue;
      const int32_t* src = b->d_lab[run_niter(b, niter, k) & 1];
      const cudaError_t e = cudaMemcpyAsync(labels + lo, src + lo, sizeof(int32_t) * (size_t)(hi - lo), kind, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  const bool use_graph = p && p->use_graph;
  if (use_graph) {
    const bool hit = b->gexec && b->g_niter == niter && b->g_cfg == c && b->g_stream == s &&
                     b->g_labels == (on_device ? labels : nullptr);
    if (!hit) {
      free_graph_exec(b);
      cudaGraph_t graph = nullptr;
      GLP_BCUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      rc = enqueue_run(b, c, niter, s);
      if (!rc && on_device && b->n) rc = copy_out(cudaMemcpyDeviceToDevice) == cudaSuccess ? GLP_OK : GLP_ECUDA;
      const cudaError_t ee = cudaStreamEndCapture(s, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
      const cudaError_t ei = cudaGraphInstantiate(&b->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        b->gexec = nullptr;
        return cuda_fail(ei, "cudaGraphInstantiate");
      }
      b->g_niter = niter;
      b->g_cfg = c;
      b->g_stream = s;
      b->g_labels = on_device ? labels : nullptr;
    }
    GLP_BCUDA(cudaGraphLaunch(b->gexec, s));
  } else {
    if ((rc = enqueue_run(b, c, niter, s))) return rc;
    if (on_device && b->n) GLP_BCUDA(copy_out(cudaMemcpyDeviceToDevice));
  }
  if (!on_device && b->n) GLP_BCUDA(copy_out(cudaMemcpyDeviceToHost));
  if (changed && total) {
    std::vector<unsigned long long> tmp((size_t)total);
    GLP_BCUDA(cudaMemcpyAsync(tmp.data(), b->d_changed, sizeof(unsigned long long) * total, cudaMemcpyDeviceToHost, s));
    GLP_BCUDA(cudaStreamSynchronize(s));
    for (int32_t i = 0; i < total; ++i) changed[i] = (int64_t)tmp[i];
  }
  return check_batch_err(b, s);
}

int glp_batch_tune(glp_batch* b, int32_t probe_iters, glp_params* best, float* times_ms, int32_t* ncand) {
  if (!b || probe_iters <= 0) {
    set_error("bad arguments to glp_batch_tune");
    return GLP_EINVAL;
  }
  std::vector<Config> cands;
  for (int nt : {512, 1024})
    for (int tt : {8, 16, 32})
      for (int half : {0, 1}) cands.push_back(Config{nt, tt, half});
  if (ncand) *ncand = (int32_t)cands.size();
  int rc = ensure_changed(b, probe_iters);
  if (rc) return rc;
  cudaStream_t s = b->stream;
  cudaEvent_t e0, e1;
  GLP_BCUDA(cudaEventCreate(&e0));
  GLP_BCUDA(cudaEventCreate(&e1));
  float best_ms = 0;
  Config best_c = b->cfg;
  bool have = false;
  for (size_t i = 0; i < cands.size(); ++i) {
    float ms = -1.f;
    // one untimed run warms the launch, then one timed run
    rc = enqueue_run(b, cands[i], probe_iters, s);
    if (!rc) rc = check_batch_err(b, s);
    if (!rc) {
      cudaEventRecord(e0, s);
      rc = enqueue_run(b, cands[i], probe_iters, s);
      cudaEventRecord(e1, s);
      if (!rc) rc = check_batch_err(b, s);
      if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (rc == GLP_ENOTSUP) {  // does not fit: skip the candidate
      rc = GLP_OK;
      ms = -1.f;
    } else if (rc) {
      break;
    }
    if (times_ms) times_ms[i] = ms;
    if (ms >= 0 && (!have || ms < best_ms)) {
      best_ms = ms;
      best_c = cands[i];
      have = true;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->cfg = best_c;
  b->tuned = true;
  free_graph_exec(b);
  if (best) {
    glp_params_default(best);
    best->tiny_max = best_c.tt;
    best->mid_max = best_c.half ? 64 : 32;
    best->batch_threads = best_c.nt;
  }
  return GLP_OK;
}

}  // extern "C"

namespace glp {
// Recreates a batch's stream at `priority` once its work has finished (the
// server's batched rounds run at the device's highest priority).  Not part of
// the C ABI.
int batch_set_stream_priority(glp_batch* b, int priority) {
  if (!b) {
    set_error("batch is NULL");
    return GLP_EINVAL;
  }
  GLP_BCUDA(cudaStreamSynchronize(b->stream));
  cudaStream_t fresh = nullptr;
  GLP_BCUDA(cudaStreamCreateWithPriority(&fresh, cudaStreamNonBlocking, priority));
  cudaStreamDestroy(b->stream);
  b->stream = fresh;
  return GLP_OK;
}
}  // namespace glp
