// device.cuh -- device helpers shared by the label-propagation kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace glp {

constexpr uint32_t kFull = 0xffffffffu;

// Error bits a kernel may raise in the per-handle status word (never traps).
enum : uint32_t {
  kErrProbe = 1u,       // a hash table probe ran past its capacity
  kErrScoreRange = 2u,  // a layered score left the packable range
  kErrHubPlan = 4u,     // hub chunk bookkeeping inconsistent
  kErrTable = 8u,       // a vertex's table would not fit the launch's shared memory
  kErrWait = 16u,       // a bounded wait on a bulk copy's mbarrier ran out
};

// Bulk global -> shared copies (cp.async.bulk, no multicast: this GPU's own
// memory only) completing on a shared-memory mbarrier.  Source, destination
// and size must be multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes the initialised barriers visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this thread's earlier generic accesses to shared memory before
// later bulk copies that write it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of the barrier to complete, at most ~2^20 polls
// (well under a second); false when the wait ran out.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 20); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it >= 32) __nanosleep(64);
  }
  return false;
}

// Dynamic shared memory of the running launch, in bytes.
__device__ __forceinline__ uint32_t dynamic_smem_bytes() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}

// Murmur3 fmix32 finaliser; the reference hashes labels with it too
// (method/hashtable.cuh:19-26).
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t k) {
  k ^= k >> 16;
  k *= 0x85ebca6bu;
  k ^= k >> 13;
  k *= 0xc2b2ae35u;
  k ^= k >> 16;
  return k;
}

// SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// SLPA speaker hash H(seed, iter, v).
__host__ __device__ __forceinline__ uint64_t slpa_hash(uint64_t seed, uint32_t iter, uint32_t v) {
  return mix64(mix64(mix64(seed) ^ (uint64_t)iter) ^ (uint64_t)v);
}

// Streaming load for data read once per iteration (CSR columns, weights).
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) { return __ldcs(p); }
// Read-only cached load for the label gather (reused across edges).
__device__ __forceinline__ int32_t ld_label(const int32_t* p) { return __ldg(p); }

// A (score, label) candidate; larger score wins, then larger label.
struct Best {
  int64_t s;
  int32_t l;
};
__device__ __forceinline__ Best best_none() { return Best{INT64_MIN, -1}; }
__device__ __forceinline__ bool better(const Best& a, const Best& b) {
  return a.s > b.s || (a.s == b.s && a.l > b.l);
}
__device__ __forceinline__ Best shfl_xor_best(const Best& b, int m) {
  Best o;
  o.s = __shfl_xor_sync(kFull, b.s, m);
  o.l = __shfl_xor_sync(kFull, b.l, m);
  return o;
}
// Max over aligned groups of G lanes (G power of two, <= 32).
template <int G>
__device__ __forceinline__ Best group_max(Best b) {
#pragma unroll
  for (int m = G / 2; m >= 1; m >>= 1) {
    Best o = shfl_xor_best(b, m);
    if (better(o, b)) b = o;
  }
  return b;
}

// A thread's running candidate for scores with a monotone 32-bit key
// (S::kPacked): the key and the label, two registers where a Best takes
// three, and a warp reduces it with two __reduce_max_sync instead of fifteen
// shuffles.  Starts at (0, 0): a real candidate never loses to it (its key
// or its label is at least as large), and a row always has one.
struct PackedCand {
  uint32_t s = 0u;
  uint32_t l = 0u;
};
template <class S>
__device__ __forceinline__ void offer(Best& b, const S& score, uint32_t tot, int32_t vl, int32_t lab) {
  const Best c{score.from_vol(tot, vl), lab};
  if (better(c, b)) b = c;
}
template <class S>
__device__ __forceinline__ void offer(PackedCand& b, const S& score, uint32_t tot, int32_t vl, int32_t lab) {
  const uint32_t k = score.key32(tot, vl);
  if (k > b.s || (k == b.s && (uint32_t)lab > b.l)) {
    b.s = k;
    b.l = (uint32_t)lab;
  }
}
// The warp's largest (key, label), as key << 32 | label, on every lane.
__device__ __forceinline__ unsigned long long warp_best(const PackedCand& b) {
  const uint32_t m = __reduce_max_sync(kFull, b.s);
  const uint32_t l = __reduce_max_sync(kFull, b.s == m ? b.l : 0u);
  return ((unsigned long long)m << 32) | l;
}

// Block-wide max; every thread gets the result.  scratch: >= 32 Best.
template <int NT>
__device__ __forceinline__ Best block_max(Best b, Best* scratch) {
  b = group_max<32>(b);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) scratch[warp] = b;
  __syncthreads();
  if (warp == 0) {
    Best x = lane < NT / 32 ? scratch[lane] : best_none();
    x = group_max<32>(x);
    if (lane == 0) scratch[0] = x;
  }
  __syncthreads();
  Best r = scratch[0];
  __syncthreads();
  return r;
}

// Open-addressing counter table (linear probing) in shared or global memory:
// keys hold label+1 (0 = empty), vals the running count or weight sum.
// insert() returns the count AFTER adding c; the largest value returned for a
// key over all of its inserts is its final total, whatever the order.
struct CountTable {
  uint32_t* keys;
  uint32_t* vals;
  uint32_t mask;  // capacity - 1, capacity a power of two

  __device__ __forceinline__ uint32_t insert(uint32_t key, uint32_t c, uint32_t* err) const {
    uint32_t h = fmix32(key) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      uint32_t cur = keys[h];
      if (cur == 0) {
        uint32_t prev = atomicCAS(&keys[h], 0u, key);
        if (prev == 0u || prev == key) return atomicAdd(&vals[h], c) + c;
      } else if (cur == key) {
        return atomicAdd(&vals[h], c) + c;
      }
      h = (h + 1) & mask;
    }
    atomicOr(err, kErrProbe);
    return 0;
  }
};

// Bounded insert: gives up after `max_probe` probes and returns kNoSlot.
// The home slot is the top bits of a Fibonacci (multiplicative) hash, one
// multiply-high; on a collision the probe continues by double hashing with an
// odd stride from other bits of the same product, so the lanes of a warp
// finish their probes close together and the table can be half full.
// Optionally appends newly claimed slots to `claimed`.
// C16: counts are 16-bit, two slots to a word (slot h in half h & 1 of word
// h >> 1), for tables whose every count stays below 2^16.
constexpr uint32_t kNoSlot = 0xffffffffu;
template <bool C16>
__device__ __forceinline__ uint32_t count_add(uint32_t* vals, uint32_t h, uint32_t c) {
  if (!C16) return atomicAdd(&vals[h], c) + c;
  const uint32_t sh = (h & 1u) * 16u;
  return ((atomicAdd(&vals[h >> 1], c << sh) >> sh) & 0xffffu) + c;
}
template <bool C16>
__device__ __forceinline__ uint32_t count_at(const uint32_t* vals, uint32_t h) {
  return C16 ? (vals[h >> 1] >> ((h & 1u) * 16u)) & 0xffffu : vals[h];
}
// HOIST: the probe loop only finds (or claims) the slot and the count is
// added once after it, so lanes that stop at different probes do not each
// run the add as a separate divergent pass (measured on B200: 15-20 % fewer
// cycles per entry in the block-per-vertex tier on rows of mostly distinct
// labels).  Off, each lane adds as soon as it finds its slot: faster on the
// largest rows, whose hot labels make lanes stop early.
template <bool C16 = false, bool HOIST = !C16>
__device__ __forceinline__ uint32_t table_insert_bounded(uint32_t* keys, uint32_t* vals, uint32_t mask, uint32_t key,
                                                         uint32_t c, uint32_t max_probe, uint32_t* claimed,
                                                         uint32_t* nclaimed) {
  const uint32_t hk = key * 0x9E3779B1u;
  uint32_t h = __umulhi(hk, mask + 1u);
  uint32_t step = 0;
  uint32_t probe = 0;
  for (; probe < max_probe; ++probe) {
    const uint32_t cur = keys[h];
    if (cur == key) {
      if (HOIST) break;
      return count_add<C16>(vals, h, c);
    }
    if (cur == 0) {
      const uint32_t prev = atomicCAS(&keys[h], 0u, key);
      if (prev == 0u) {
        if (claimed) claimed[atomicAdd(nclaimed, 1u)] = h;
        if (HOIST) break;
        return count_add<C16>(vals, h, c);
      }
      if (prev == key) {
        if (HOIST) break;
        return count_add<C16>(vals, h, c);
      }
    }
    if (step == 0) {
      step = ((hk >> 9) | 1u) & mask;
      if (step == 0) step = 1u;
    }
    h = (h + step) & mask;
  }
  if (!HOIST || probe == max_probe) return kNoSlot;
  return count_add<C16>(vals, h, c);
}

// Claim-first insert for unweighted counts (c >= 1): the atomicCAS that
// claims a slot is the key's first occurrence, so `extra` holds a key's
// count minus one and a label seen once costs a single shared atomic (a
// key found on its slot costs the CAS plus one add).  The neighbourhoods of
// the first propagation steps hold mostly distinct labels: B200 issues a
// random-address shared CAS at half the rate of an add, and the saved add
// and probe load cut the big-tier count by a quarter to a third.
// Returns the running count after this insert (kNoSlot when no slot was
// found within max_probe probes).
template <bool C16>
__device__ __forceinline__ uint32_t table_claim_insert(uint32_t* keys, uint32_t* extra, uint32_t mask, uint32_t key,
                                                       uint32_t c, uint32_t max_probe) {
  const uint32_t hk = key * 0x9E3779B1u;
  uint32_t h = __umulhi(hk, mask + 1u);
  uint32_t step = ((hk >> 9) | 1u) & mask;
  if (step == 0) step = 1u;
  uint32_t prev = 1u, probe = 0;
  for (; probe < max_probe; ++probe) {
    prev = atomicCAS(&keys[h], 0u, key);
    if (prev == 0u || prev == key) break;
    h = (h + step) & mask;
  }
  if (probe == max_probe) return kNoSlot;
  const uint32_t inc = prev == 0u ? c - 1u : c;
  if (inc == 0u) return 1u;
  return count_add<C16>(extra, h, inc) + 1u;
}
// The count of slot h of a claim-first table (0 for an empty slot).
template <bool C16>
__device__ __forceinline__ uint32_t claim_count_at(const uint32_t* keys, const uint32_t* extra, uint32_t h) {
  return keys[h] ? 1u + count_at<C16>(extra, h) : 0u;
}

// Zeroes n words of shared memory with 16-byte stores (p 16-byte aligned, n a
// multiple of 4); threads t, t+stride, ... of the caller's group take part.
__device__ __forceinline__ void zero_words16(uint32_t* p, uint32_t n, uint32_t t, uint32_t stride) {
  uint4* q = reinterpret_cast<uint4*>(p);
  for (uint32_t s = t; s < n / 4; s += stride) q[s] = make_uint4(0u, 0u, 0u, 0u);
}

// Sorts TMAX (a power of two) labels held in registers, ascending, with a
// bitonic network (every index known at compile time, so nothing leaves the
// registers); weights move with their labels when W.  Equal labels end up
// adjacent, so a row's counts are the lengths (weight sums) of its runs:
// O(TMAX log^2 TMAX) min/max steps instead of O(degree * TMAX) compares.
template <int TMAX, bool W>
__device__ __forceinline__ void sort_labels(int32_t (&lab)[TMAX], uint32_t (&wt)[TMAX]) {
#pragma unroll
  for (int k = 2; k <= TMAX; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < TMAX; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const int32_t x = lab[i], y = lab[l];
          if (W) {
            const bool sw = up ? (x > y) : (x < y);
            const uint32_t wx = wt[i], wy = wt[l];
            lab[i] = sw ? y : x;
            lab[l] = sw ? x : y;
            wt[i] = sw ? wy : wx;
            wt[l] = sw ? wx : wy;
          } else {
            lab[i] = up ? min(x, y) : max(x, y);
            lab[l] = up ? max(x, y) : min(x, y);
          }
        }
      }
    }
  }
}

// Smallest power of two >= x (x >= 1).
__device__ __forceinline__ uint32_t pow2_ceil(uint32_t x) { return x <= 1 ? 1u : 1u << (32 - __clz(x - 1)); }

// Warp-aggregated add of per-lane counts (0..255) to a counter.
__device__ __forceinline__ void warp_count_add(unsigned long long* counter, uint32_t count) {
  const uint32_t total = __reduce_add_sync(kFull, count);
  if ((threadIdx.x & 31) == 0 && total) atomicAdd(counter, (unsigned long long)total);
}

}  // namespace glp
