// backends.cuh -- the count-min and frequent-items counting back-ends.
//
// The reference has three counting structures (method/hashtable.cuh,
// method/countmin.cuh, method/frequent.cuh).  The exact one is the engine's
// default (kernels.cuh).  The other two are approximate summaries; the
// reference's only kernel that uses one (l_big_update_syn3,
// header/kernel.cuh:1420-1566) screens with a sketch and re-counts exactly
// when the sketch cannot rule a label out.  Here both summaries work the
// same way, on the big tier (one block or warp per vertex of degree
// mid_max+1 .. big_max):
//
//   count-min (k_big_cm): every label goes to a one-probe shared table; a
//     label whose slot another label holds goes to a 3-row count-min sketch
//     instead (all of its occurrences do, so table counts are exact).  No
//     label outside the table can count more than B = min over rows of the
//     row's largest cell, so when the best table score beats score(B) the
//     vertex is decided; otherwise it is listed for the exact kernel.
//   frequent items (k_big_fa): one warp builds a Misra-Gries summary of at
//     most kFaCap labels in edge order, 32 edges a round, keeps it sorted,
//     and on overflow subtracts the smallest count from every entry and every
//     pending label (D accumulates the subtractions).  Every label counts at
//     most (summary estimate + D); a second pass counts the summary's labels
//     exactly, and when the best of them beats score(D) the vertex is
//     decided; otherwise it is listed for the exact kernel.
//
// Both therefore return the exact labels, bit for bit; the summaries only
// decide how much of the tier needs a full exact count.  The sketch
// arithmetic itself (row hashes, and the reference's row-3 defect on
// request) is exposed by k_cm_sketch, the reference's sequential frequent
// table by k_fa_summary, for parity checks of the summaries.
#pragma once
#include "kernels.cuh"

namespace glp {

// ------------------------------------------------------------ count-min rows
// Row hash r of a key (label + 1): multiply-xorshift with per-row constants,
// the three row hashes cm_hash1..3 of method/countmin.cuh:97-125 (the same
// constants, so that sketch cells agree with the reference's).
struct CmRowConst {
  uint32_t m1, m2;
};
__host__ __device__ __forceinline__ uint32_t cm_row_hash(int r, uint32_t k) {
  const CmRowConst c = r == 0 ? CmRowConst{0x12ebcb3bu, 0xc123ae53u}
                     : r == 1 ? CmRowConst{0x21eb21bbu, 0x2cb2ea35u}
                              : CmRowConst{0x8febce61u, 0xa2b2be25u};
  k = (k ^ (k >> 16)) * c.m1;
  k = (k ^ (k >> 13)) * c.m2;
  return k ^ (k >> 16);
}

// Row that row r's increments land in.  ref_compat reproduces
// method/countmin.cuh:190, where the third increment indexes the second row.
__device__ __forceinline__ int cm_dest_row(int r, bool ref_compat) { return (ref_compat && r == 2) ? 1 : r; }

// Count-min sketch of whole neighbourhoods: one block per listed vertex,
// rows [3][width] in dynamic shared memory, written to out[i][3][width].
// Every neighbour adds its weight (1 when unweighted) to one cell per row;
// cell totals do not depend on the order of the adds.
__global__ void k_cm_sketch(const int32_t* off, const int32_t* cols, const int32_t* w, const int32_t* labels,
                            const int32_t* verts, int32_t nv, int32_t width, int ref_compat, uint32_t* out) {
  extern __shared__ uint32_t rows[];
  const uint32_t cells = 3u * (uint32_t)width;
  for (int32_t i = blockIdx.x; i < nv; i += gridDim.x) {
    for (uint32_t s = threadIdx.x; s < cells; s += blockDim.x) rows[s] = 0;
    __syncthreads();
    const int32_t v = verts[i];
    for (int32_t j = off[v] + threadIdx.x; j < off[v + 1]; j += blockDim.x) {
      const uint32_t key = (uint32_t)labels[cols[j]] + 1u;
      const uint32_t x = w ? (uint32_t)w[j] : 1u;
#pragma unroll
      for (int r = 0; r < 3; ++r)
        atomicAdd(&rows[cm_dest_row(r, ref_compat != 0) * width + cm_row_hash(r, key) % (uint32_t)width], x);
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < cells; s += blockDim.x) out[(size_t)i * cells + s] = rows[s];
    __syncthreads();
  }
}

// The reference's frequent table (method/frequent.cuh:77-105) applied to a
// neighbourhood in edge order by one thread per listed vertex: a key (label
// + 1) is added by linear probing from fmix32(key) % cap to a free or equal
// slot; when every slot holds another key, a decrement round runs and the
// key is dropped.  Clean rounds subtract one from every count and free the
// keys reaching zero; ref_compat rounds do what the reference's atomicDec
// with limit 0 does: every count becomes 0, and only keys whose count was 1
// are freed.  keys/vals: [nv][cap] in global memory; rounds: [nv].
__global__ void k_fa_summary(const int32_t* off, const int32_t* cols, const int32_t* labels, const int32_t* verts,
                             int32_t nv, int32_t cap, int ref_compat, uint32_t* keys, uint32_t* vals,
                             int32_t* rounds) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  uint32_t* kk = keys + (size_t)i * cap;
  uint32_t* vv = vals + (size_t)i * cap;
  for (int32_t s = 0; s < cap; ++s) kk[s] = vv[s] = 0;
  int32_t nr = 0;
  const int32_t v = verts[i];
  for (int32_t j = off[v]; j < off[v + 1]; ++j) {
    const uint32_t key = (uint32_t)labels[cols[j]] + 1u;
    uint32_t s = fmix32(key) % (uint32_t)cap;
    bool placed = false;
    for (int32_t probe = 0; probe < cap && !placed; ++probe) {
      if (kk[s] == 0u || kk[s] == key) {
        kk[s] = key;
        vv[s] += 1u;
        placed = true;
      }
      s = s + 1u == (uint32_t)cap ? 0u : s + 1u;
    }
    if (placed) continue;
    ++nr;
    for (int32_t t = 0; t < cap; ++t) {
      const uint32_t prev = vv[t];
      if (ref_compat) vv[t] = 0u;
      else if (prev > 0u) vv[t] = prev - 1u;
      if (prev == 1u) kk[t] = 0u;
    }
  }
  rounds[i] = nr;
}

// ------------------------------------------------------ count-min screen
constexpr uint32_t kCmTable = 2048;  // one-probe shared table slots
constexpr uint32_t kCmWidth = 1024;  // sketch cells per row

// Big-tier vertices of `tw`: decided by the table when no label outside it
// can reach the table's best score, else appended to `fb` for exact counting.
template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_big_cm(StepArgs a, TierWork tw, S score, FailList fb) {
  __shared__ __align__(16) uint32_t tkeys[kCmTable];
  __shared__ __align__(16) uint32_t tvals[kCmTable];
  __shared__ __align__(16) uint32_t rows[3 * kCmWidth];
  __shared__ Best red[32];
  __shared__ uint32_t rmax[3][NT / 32];
  __shared__ uint32_t spilled;
  __shared__ int32_t cbuf[64];
  uint32_t ncb = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  for (int32_t i = blockIdx.x; i < nwork; i += gridDim.x) {
    const int32_t v = tw.at(mode, i);
    const int32_t b = a.off[v], e = a.off[v + 1];
    zero_words16(tkeys, kCmTable, threadIdx.x, NT);
    zero_words16(tvals, kCmTable, threadIdx.x, NT);
    zero_words16(rows, 3 * kCmWidth, threadIdx.x, NT);
    if (threadIdx.x == 0) spilled = 0;
    __syncthreads();
    auto ins = [&](uint32_t key, uint32_t k) -> uint32_t {
      const uint32_t s = __umulhi(key * 0x9E3779B1u, kCmTable);
      uint32_t cur = tkeys[s];
      if (cur == 0u) {
        cur = atomicCAS(&tkeys[s], 0u, key);
        if (cur == 0u) cur = key;
      }
      if (cur == key) {
        atomicAdd(&tvals[s], k);
      } else {  // the slot belongs to another label for the rest of the vertex
#pragma unroll
        for (int r = 0; r < 3; ++r) atomicAdd(&rows[r * kCmWidth + cm_row_hash(r, key) % kCmWidth], k);
        spilled = 1u;
      }
      return 0u;
    };
    Best best = best_none();
    bool fail = false;
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
        if (j0 + q * NT < e) count_chunk<W>(lab[q] >= 0, lab[q], wt[q], score, ins, best, fail, true);
    }
    __syncthreads();
    scan_table(tkeys, tvals, kCmTable, threadIdx.x, NT, score, best);
    // the largest cell of each row
    uint32_t m[3] = {0u, 0u, 0u};
    if (spilled) {  // block-uniform
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        for (uint32_t s = threadIdx.x; s < kCmWidth; s += NT) m[r] = max(m[r], rows[r * kCmWidth + s]);
        m[r] = __reduce_max_sync(kFull, m[r]);
        if (lane == 0) rmax[r][warp] = m[r];
      }
    }
    best = block_max<NT>(best, red);  // its barriers publish rmax
    if (threadIdx.x == 0) {
      bool decided = true;
      if (spilled) {
        uint32_t bound = 0xffffffffu;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          uint32_t x = 0u;
          for (int w8 = 0; w8 < NT / 32; ++w8) x = max(x, rmax[r][w8]);
          bound = min(bound, x);
        }
        decided = best.s > score.bound(bound);
      }
      if (decided) {
        a.lout[v] = best.l;
        if (best.l != a.lcur[v]) {
          cbuf[ncb++] = v;
          if (ncb == 64) flush_big_changes(a, cbuf, ncb);
        }
      } else {
        fb.ids[atomicAdd(fb.count, 1u)] = v;
      }
    }
    __syncthreads();  // tables are cleared for the next vertex
  }
  if (threadIdx.x == 0) flush_big_changes(a, cbuf, ncb);
}

// ------------------------------------------------ frequent-items screen
constexpr int kFaCap = 256;  // summary entries per warp

// Ascending bitonic sort of one value per lane across the warp; weights move
// with their keys when W.
template <bool W>
__device__ __forceinline__ void warp_sort32(int32_t& k, uint32_t& w) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const int32_t ok = __shfl_xor_sync(kFull, k, stride);
      const uint32_t ow = W ? __shfl_xor_sync(kFull, w, stride) : w;
      const bool up = (lane & size) == 0 || size == 32;
      const bool low = (lane & stride) == 0;
      const bool take = (low == up) ? ok < k : ok > k;
      if (take) {
        k = ok;
        if (W) w = ow;
      }
    }
  }
}

// First index in the sorted keys[0, n) whose key is >= x.
__device__ __forceinline__ int32_t lower_bound_keys(const int32_t* keys, int32_t n, int32_t x) {
  int32_t lo = 0, hi = n;
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (keys[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One warp's Misra-Gries summary, sorted by label, double-buffered: buffer c
// is keys/vals [c * kFaCap, (c + 1) * kFaCap).
struct FaSummary {
  int32_t* keys;
  uint32_t* vals;
  int32_t* plb;    // [32] insertion points of the pending labels
  __device__ __forceinline__ int32_t* key(int c) const { return keys + c * kFaCap; }
  __device__ __forceinline__ uint32_t* val(int c) const { return vals + c * kFaCap; }
  int cur = 0;
  int32_t ns = 0;  // entries in use
  uint32_t dec = 0;  // D: total subtracted from every label
  bool rounds = false;

  // Adds the 32 labels of one chunk (lab = INT32_MAX: no edge).  Warp-wide.
  template <bool W>
  __device__ __forceinline__ void add_chunk(int32_t lab, uint32_t wt) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    warp_sort32<W>(lab, wt);
    // run totals: inclusive prefix of the weights, read at each run's end
    uint32_t pre = wt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, pre, d);
      if (lane >= d) pre += o;
    }
    const int32_t prev = __shfl_up_sync(kFull, lab, 1);
    const int32_t next = __shfl_down_sync(kFull, lab, 1);
    const uint32_t heads = __ballot_sync(kFull, lane == 0 || prev != lab);
    const bool tail = lane == 31 || next != lab;
    const uint32_t upto = lane == 31 ? kFull : ((2u << lane) - 1u);
    const int head = 31 - __clz(heads & upto);
    const uint32_t before = __shfl_sync(kFull, pre, head > 0 ? head - 1 : 0);
    uint32_t x = pre - (head > 0 ? before : 0u);
    bool pending = false;
    if (tail && lab != INT32_MAX) {
      const int32_t p = lower_bound_keys(key(cur), ns, lab);
      if (p < ns && key(cur)[p] == lab) val(cur)[p] += x;
      else pending = true;
    }
    __syncwarp();
    uint32_t pm = __ballot_sync(kFull, pending);
    // overflow rounds: subtract the smallest count from every entry and every
    // pending label until the pending labels fit
    while (__popc(pm) > kFaCap - ns) {
      uint32_t mn = pending ? x : 0xffffffffu;
      for (int32_t s = lane; s < ns; s += 32) mn = min(mn, val(cur)[s]);
      mn = __reduce_min_sync(kFull, mn);
      dec += mn;
      rounds = true;
      int32_t base = 0;
      for (int32_t s0 = 0; s0 < ns; s0 += 32) {
        const int32_t s = s0 + lane;
        const uint32_t nv = s < ns ? val(cur)[s] - mn : 0u;
        const bool keep = s < ns && nv > 0u;
        const uint32_t kb = __ballot_sync(kFull, keep);
        if (keep) {
          const int32_t o = base + __popc(kb & lt);
          key(cur ^ 1)[o] = key(cur)[s];
          val(cur ^ 1)[o] = nv;
        }
        base += __popc(kb);
      }
      ns = base;
      cur ^= 1;
      if (pending) {
        x -= mn;
        pending = x > 0u;
      }
      pm = __ballot_sync(kFull, pending);
      __syncwarp();
    }
    if (!pm) return;
    // merge the pending labels (ascending by lane) into the summary
    const int32_t np = __popc(pm);
    int32_t lb = 0;
    if (pending) {
      lb = lower_bound_keys(key(cur), ns, lab);
      plb[__popc(pm & lt)] = lb;
    }
    __syncwarp();
    for (int32_t s = lane; s < ns; s += 32) {
      // pending labels inserted before entry s: those with insertion point <= s
      int32_t lo = 0, hi = np;
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (plb[mid] <= s) lo = mid + 1;
        else hi = mid;
      }
      key(cur ^ 1)[s + lo] = key(cur)[s];
      val(cur ^ 1)[s + lo] = val(cur)[s];
    }
    if (pending) {
      const int32_t o = lb + __popc(pm & lt);
      key(cur ^ 1)[o] = lab;
      val(cur ^ 1)[o] = x;
    }
    ns += np;
    cur ^= 1;
    __syncwarp();
  }
};

// Big-tier vertices of `tw`, one warp each: decided from the summary when no
// label outside it can reach the best summary label's exact score, else
// appended to `fb` for exact counting.
template <int NT, bool W, class S>
__global__ void __launch_bounds__(NT) k_big_fa(StepArgs a, TierWork tw, S score, FailList fb) {
  constexpr int NW = NT / 32;
  __shared__ __align__(16) int32_t skey[NW][2 * kFaCap];
  __shared__ __align__(16) uint32_t sval[NW][2 * kFaCap];
  __shared__ int32_t splb[NW][32];
  __shared__ int32_t cbuf[NW][32];
  uint32_t ncb = 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t mode = step_mode(a);
  const int32_t nwork = tw.size(mode);
  for (int32_t i = blockIdx.x * NW + warp; i < nwork; i += gridDim.x * NW) {
    const int32_t v = tw.at(mode, i);
    const int32_t b = a.off[v], e = a.off[v + 1];
    FaSummary fs{skey[warp], sval[warp], splb[warp]};
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
      for (int q = 0; q < 4; ++q) lab[q] = lab[q] >= 0 ? ld_label(a.lin + lab[q]) : INT32_MAX;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (j0 + 32 * q < e) fs.add_chunk<W>(lab[q], wt[q]);
    }
    const int32_t* ck = fs.key(fs.cur);
    uint32_t* cnt = fs.val(fs.cur);
    if (fs.rounds) {
      // exact counts of the summary's labels, in the other buffer's counts
      cnt = fs.val(fs.cur ^ 1);
      for (int32_t s = lane; s < fs.ns; s += 32) cnt[s] = 0u;
      __syncwarp();
      for (int32_t j = b + lane; j < e; j += 32) {
        const int32_t l = ld_label(a.lin + ld_stream(a.cols + j));
        const int32_t p = lower_bound_keys(ck, fs.ns, l);
        if (p < fs.ns && ck[p] == l) atomicAdd(&cnt[p], W ? (uint32_t)ld_stream(a.w + j) : 1u);
      }
      __syncwarp();
    }
    Best best = best_none();
    for (int32_t s = lane; s < fs.ns; s += 32) {
      const Best c{score(ck[s], cnt[s]), ck[s]};
      if (better(c, best)) best = c;
    }
    best = group_max<32>(best);
    // without a round the summary holds every label with its exact count
    const bool decided = !fs.rounds || best.s > score.bound(fs.dec);
    bool chg = false;
    if (lane == 0) {
      if (decided) {
        a.lout[v] = best.l;
        chg = best.l != a.lcur[v];
      } else {
        fb.ids[atomicAdd(fb.count, 1u)] = v;
      }
    }
    warp_note_change(a, cbuf[warp], ncb, chg, v);
    __syncwarp();  // the summary is rebuilt for the next vertex
  }
  warp_flush_changes(a, cbuf[warp], ncb);
}

}  // namespace glp
