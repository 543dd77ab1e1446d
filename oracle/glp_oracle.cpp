// glp_oracle.cpp -- CPU ORACLE for the label-propagation hot path.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py may load this library, and
// only as the checker or the timed CPU baseline -- never as the product path.
//
// This file restates, in plain sequential-semantics C++17 (OpenMP across
// vertices where the semantics are synchronous), what the reference computes:
//
//   * classic synchronous LP: header/kernel.cuh:1655-1739 (big),
//     :4365-4426 (small), :5187-5234 (tiny), :864-911 + :1033-1056 (huge):
//     L'(v) = argmax_l #{u in N(v) : L(u) = l}; ties go to the LARGEST label
//     (the packed (count<<32)|(label+1) max, e.g. kernel.cuh:1724-1734);
//     an isolated vertex keeps its label (kernel.cuh:4387-4390).
//   * weighted variant: the same rule with integer weight sums (no reference
//     code exists: parity unpinned for weights beyond the unit-weight case).
//   * layered LP: kernel.cuh:2529-2630 (score delta*.k - vol[l], signed packed
//     max) + the CPU volume bookkeeping of tutorial/CPUlp.cuh:189-248
//     (vol_r <- vol_w, vol_w <- 0 every iteration; labels reset to ids at each
//     layer).  vol_w[l] counts every vertex whose label is l after the step.
//   * SLPA: tutorial/Base5prop.cuh:161-208 (store into the last empty memory
//     slot, else slot 0; speaker = first non-empty slot scanning cyclically
//     from a random index) with rand() replaced by a counter hash, and the
//     listener rule of kernel.cuh:1837-1894 (mode of the spoken labels).
//   * the reference OpenMP CPU path, tutorial/CPUlp.cuh:28-92 (sync_run_1),
//     restated exactly for one thread: labels are read IN PLACE and a tie goes
//     to the first label to reach the maximum in CSR order.  This mode exists
//     to pin the oracle against the reference CPU code compiled from source.
//   * count-min sketch rows (method/countmin.cuh:97-125, :175-195) and the
//     Misra-Gries frequent table (method/frequent.cuh:77-105).
//
// Counting here is by sorting each neighbourhood (not by hashing), so the
// oracle shares no mechanism with the CUDA kernels it checks.

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct LW {
  int32_t label;
  int64_t w;
};

// argmax over labels of (sum of weights), ties -> largest label.
// Returns false when the neighbourhood is empty.
inline bool mode_of(std::vector<LW>& buf, int32_t* best_label, int64_t* best_count) {
  if (buf.empty()) return false;
  std::sort(buf.begin(), buf.end(), [](const LW& a, const LW& b) { return a.label < b.label; });
  int64_t bc = -1;
  int32_t bl = 0;
  size_t i = 0;
  while (i < buf.size()) {
    size_t j = i;
    int64_t s = 0;
    while (j < buf.size() && buf[j].label == buf[i].label) { s += buf[j].w; ++j; }
    // labels ascend, so ">=" keeps the largest label among equal counts
    if (s >= bc) { bc = s; bl = buf[i].label; }
    i = j;
  }
  *best_label = bl;
  *best_count = bc;
  return true;
}

inline int threads_or_default(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).
inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

// Counter-based speaker hash H(seed, iter, v): three chained SplitMix64
// finalisers.  The CUDA engine uses the same function.
uint64_t orc_slpa_hash(uint64_t seed, uint32_t iter, uint32_t v) {
  return mix64(mix64(mix64(seed) ^ (uint64_t)iter) ^ (uint64_t)v);
}

// One synchronous classic step.  weights may be NULL (unit weights).
int orc_classic_step(int32_t n, const int32_t* off, const int32_t* cols, const int32_t* w,
                     const int32_t* lin, int32_t* lout, int nthreads) {
  if (n < 0) return -1;
  const int nt = threads_or_default(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<LW> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int32_t v = 0; v < n; ++v) {
      buf.clear();
      for (int32_t j = off[v]; j < off[v + 1]; ++j) buf.push_back({lin[cols[j]], w ? (int64_t)w[j] : 1});
      int32_t bl;
      int64_t bc;
      lout[v] = mode_of(buf, &bl, &bc) ? bl : lin[v];
    }
  }
  return 0;
}

// niter synchronous classic steps from init (NULL: label = vertex id).
// trace (nullable) receives the labels after every step, [niter][n].
// From the second step on, a vertex none of whose neighbours changed label
// in the previous step keeps its label without recounting: its new label is
// a function of its neighbours' labels only (an isolated vertex keeps its
// own), and those equal the ones its current label was computed from.  This
// is exact, needs no symmetry, and makes converged steps cheap.
int orc_classic_run(int32_t n, const int32_t* off, const int32_t* cols, const int32_t* w, int32_t niter,
                    const int32_t* init, int32_t* lout, int32_t* trace, int nthreads) {
  std::vector<int32_t> a(n), b(n);
  std::vector<uint8_t> chg(n, 1);
  for (int32_t v = 0; v < n; ++v) a[v] = init ? init[v] : v;
  const int nt = threads_or_default(nthreads);
  for (int32_t it = 0; it < niter; ++it) {
    if (it == 0) {
      orc_classic_step(n, off, cols, w, a.data(), b.data(), nthreads);
    } else {
#pragma omp parallel num_threads(nt)
      {
        std::vector<LW> buf;
#pragma omp for schedule(dynamic, 1024)
        for (int32_t v = 0; v < n; ++v) {
          bool dirty = false;
          for (int32_t j = off[v]; j < off[v + 1] && !dirty; ++j) dirty = chg[cols[j]] != 0;
          if (!dirty) {
            b[v] = a[v];
            continue;
          }
          buf.clear();
          for (int32_t j = off[v]; j < off[v + 1]; ++j) buf.push_back({a[cols[j]], w ? (int64_t)w[j] : 1});
          int32_t bl;
          int64_t bc;
          b[v] = mode_of(buf, &bl, &bc) ? bl : a[v];
        }
      }
    }
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int32_t v = 0; v < n; ++v) chg[v] = a[v] != b[v];
    std::swap(a, b);
    if (trace) std::memcpy(trace + (size_t)it * n, a.data(), sizeof(int32_t) * n);
  }
  std::memcpy(lout, a.data(), sizeof(int32_t) * n);
  return 0;
}

// Layered LP.  dstar[s] = delta*+1 ... i.e. the integer score multiplier of
// layer s (delta* = 1/gamma + 1).  Each layer starts from label = id; every
// iteration first sets vol_r <- vol_w (vol_r = 0 before the very first one),
// then scores score(l) = dstar*k_l - vol_r[l], argmax, ties -> largest label,
// and vol_w = histogram of the new labels (all vertices).
// use_fp64 != 0 evaluates the north-star form k - gamma*(vol - k) in double
// (gamma = 1/(dstar-1)); for power-of-two gamma both forms order identically.
// trace (nullable): labels after every iteration, [nlayers*niter][n].
int orc_layered_run(int32_t n, const int32_t* off, const int32_t* cols, const int32_t* w,
                    const int32_t* dstar, int32_t nlayers, int32_t niter, int use_fp64,
                    int32_t* lout, int32_t* vol_out, int32_t* trace, int nthreads) {
  std::vector<int32_t> a(n), b(n);
  std::vector<int64_t> vol_r(n, 0), vol_w(n, 0);
  const int nt = threads_or_default(nthreads);
  int64_t step = 0;
  for (int32_t s = 0; s < nlayers; ++s) {
    for (int32_t v = 0; v < n; ++v) a[v] = v;
    const int64_t ds = dstar[s];
    const double gamma = 1.0 / (double)(ds - 1);
    for (int32_t it = 0; it < niter; ++it, ++step) {
      if (step > 0) vol_r = vol_w;
#pragma omp parallel num_threads(nt)
      {
        std::vector<LW> buf;
#pragma omp for schedule(dynamic, 1024)
        for (int32_t v = 0; v < n; ++v) {
          buf.clear();
          for (int32_t j = off[v]; j < off[v + 1]; ++j) buf.push_back({a[cols[j]], w ? (int64_t)w[j] : 1});
          if (buf.empty()) { b[v] = a[v]; continue; }
          std::sort(buf.begin(), buf.end(), [](const LW& x, const LW& y) { return x.label < y.label; });
          bool have = false;
          int64_t bi = 0;
          double bd = 0;
          int32_t bl = 0;
          size_t i = 0;
          while (i < buf.size()) {
            size_t j = i;
            int64_t k = 0;
            while (j < buf.size() && buf[j].label == buf[i].label) { k += buf[j].w; ++j; }
            const int32_t l = buf[i].label;
            if (use_fp64) {
              const double sc = (double)k - gamma * ((double)vol_r[l] - (double)k);
              if (!have || sc >= bd) { bd = sc; bl = l; have = true; }
            } else {
              const int64_t sc = ds * k - vol_r[l];
              if (!have || sc >= bi) { bi = sc; bl = l; have = true; }
            }
            i = j;
          }
          b[v] = bl;
        }
      }
      std::fill(vol_w.begin(), vol_w.end(), 0);
      for (int32_t v = 0; v < n; ++v) vol_w[b[v]]++;
      std::swap(a, b);
      if (trace) std::memcpy(trace + (size_t)step * n, a.data(), sizeof(int32_t) * n);
    }
  }
  std::memcpy(lout, a.data(), sizeof(int32_t) * n);
  if (vol_out)
    for (int32_t v = 0; v < n; ++v) vol_out[v] = (int32_t)vol_w[v];
  return 0;
}

// SLPA with speaker memory (tutorial/Base5prop.cuh:161-293).
// mem is slot-major [T][n], -1 = empty.  Per iteration it:
//   store  : label -> last empty slot, or slot 0 when full (Base5prop.cuh:187-208)
//   pick   : scan cyclically from H(seed,it,v) mod T to the first non-empty slot
//            (Base5prop.cuh:163-183 with rand() replaced by H)
//   listen : mode of the neighbours' spoken labels, ties -> largest label;
//            an isolated vertex keeps its label.
// After niter iterations the memory is post-processed (Xie et al. 2011): a
// vertex keeps every label whose frequency in its filled slots is >= r
// (compared in double as count >= r*filled).  comm is [n][T] ascending labels
// padded with -1; ncomm[v] the number kept.
int orc_slpa_run(int32_t n, const int32_t* off, const int32_t* cols, const int32_t* w, int32_t T,
                 int32_t niter, uint64_t seed, double r, int32_t* lout, int32_t* mem, int32_t* comm,
                 int32_t* ncomm, int32_t* spoken_trace, int nthreads) {
  if (T <= 0 || T > 64) return -1;
  const int nt = threads_or_default(nthreads);
  std::vector<int32_t> lab(n), spk(n);
  for (int32_t v = 0; v < n; ++v) lab[v] = v;
  for (size_t i = 0; i < (size_t)T * n; ++i) mem[i] = -1;
  for (int32_t it = 0; it < niter; ++it) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int32_t v = 0; v < n; ++v) {
      int filled = 0, insertpos = 0;
      for (int s = 0; s < T; ++s) {
        if (mem[(size_t)s * n + v] != -1) ++filled; else insertpos = s;
      }
      if (filled == T) insertpos = 0;
      mem[(size_t)insertpos * n + v] = lab[v];
      const uint32_t start = (uint32_t)(orc_slpa_hash(seed, (uint32_t)it, (uint32_t)v) % (uint64_t)T);
      int pick = 0;
      for (int s = 0; s < T; ++s) {
        pick = (int)((start + s) % (uint32_t)T);
        if (mem[(size_t)pick * n + v] != -1) break;
      }
      spk[v] = mem[(size_t)pick * n + v];
    }
    if (spoken_trace) std::memcpy(spoken_trace + (size_t)it * n, spk.data(), sizeof(int32_t) * n);
    std::vector<int32_t> nxt(n);
    orc_classic_step(n, off, cols, w, spk.data(), nxt.data(), nthreads);
    // an isolated vertex keeps its own current label, not its spoken one
    for (int32_t v = 0; v < n; ++v)
      if (off[v] == off[v + 1]) nxt[v] = lab[v];
    lab.swap(nxt);
  }
  std::memcpy(lout, lab.data(), sizeof(int32_t) * n);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int32_t v = 0; v < n; ++v) {
    std::vector<int32_t> ls;
    for (int s = 0; s < T; ++s) {
      int32_t x = mem[(size_t)s * n + v];
      if (x != -1) ls.push_back(x);
    }
    std::sort(ls.begin(), ls.end());
    const int filled = (int)ls.size();
    int k = 0;
    size_t i = 0;
    while (i < ls.size()) {
      size_t j = i;
      while (j < ls.size() && ls[j] == ls[i]) ++j;
      if ((double)(j - i) >= r * (double)filled) comm[(size_t)v * T + k++] = ls[i];
      i = j;
    }
    ncomm[v] = k;
    for (int s = k; s < T; ++s) comm[(size_t)v * T + s] = -1;
  }
  return 0;
}

// tutorial/CPUlp.cuh:28-92 (sync_run_1) restated for ONE thread: per
// iteration prelabels <- labels, then for k = 0..n-1 in order the label
// counts read labels[] IN PLACE (CPUlp.cuh:64) and a tie keeps the first
// label to reach the maximum (CPUlp.cuh:67-71); max_label starts at
// prelabels[u] with max_score 0.
int orc_cpulp_sync_run_1(int32_t n, const int32_t* off, const int32_t* cols, int32_t niter, int32_t* lout,
                         int32_t* nupdates_out) {
  std::vector<int32_t> labels(n), pre(n);
  for (int32_t v = 0; v < n; ++v) labels[v] = pre[v] = v;
  for (int32_t it = 0; it < niter; ++it) {
    int32_t nupd = 0;
    for (int32_t k = 0; k < n; ++k) pre[k] = labels[k];
    std::map<int32_t, int> cnt;
    for (int32_t u = 0; u < n; ++u) {
      cnt.clear();
      int32_t max_label = pre[u];
      int max_score = 0;
      for (int32_t j = off[u]; j < off[u + 1]; ++j) {
        const int32_t lab = labels[cols[j]];
        const int c = ++cnt[lab];
        if (c > max_score) { max_score = c; max_label = lab; }
      }
      if (pre[u] != max_label) { labels[u] = max_label; ++nupd; }
    }
    if (nupdates_out) nupdates_out[it] = nupd;
  }
  std::memcpy(lout, labels.data(), sizeof(int32_t) * n);
  return 0;
}

// tutorial/CPUlp.cuh:169-262 (layered_run) restated for ONE thread: 10
// layers; labels reset to ids from the second layer on (prelabels and the
// volume arrays are not reset); delta doubles at EVERY iteration
// (CPUlp.cuh:199) with delta* = delta + 1; per iteration prelabels <- labels,
// gcount_r <- gcount_w, gcount_w <- 0; a vertex scores each neighbour label
// in CSR order as c*delta* - gcount_r[label] with labels read in place and
// keeps the first label to reach the maximum (start INT_MIN); the chosen
// label's gcount_w is incremented.  delta overflows int after 30 doublings,
// so callers keep 10*niter <= 20 and degrees below 2048.
int orc_cpulp_layered_run(int32_t n, const int32_t* off, const int32_t* cols, int32_t niter, int32_t* lout,
                          int32_t* nupdates_out) {
  const int d_iter = 10;
  int delta = 1;
  std::vector<int32_t> labels(n), pre(n), gr(n, 0), gw(n, 0);
  for (int32_t v = 0; v < n; ++v) labels[v] = pre[v] = v;
  std::map<int32_t, int> cnt;
  int idx = 0;
  for (int j = 0; j < d_iter; ++j) {
    if (j != 0)
      for (int32_t v = 0; v < n; ++v) labels[v] = v;
    for (int32_t it = 0; it < niter; ++it, ++idx) {
      int32_t nupd = 0;
      delta = 2 * delta;
      const int delta_star = delta + 1;
      for (int32_t k = 0; k < n; ++k) pre[k] = labels[k];
      gr = gw;
      std::fill(gw.begin(), gw.end(), 0);
      for (int32_t u = 0; u < n; ++u) {
        cnt.clear();
        int32_t max_label = pre[u];
        int max_score = INT_MIN;
        for (int32_t x = off[u]; x < off[u + 1]; ++x) {
          const int32_t lab = labels[cols[x]];
          const int c = ++cnt[lab];
          int s = c * delta_star;
          if (lab < n) s -= gr[lab];
          if (s > max_score) { max_score = s; max_label = lab; }
        }
        if (max_label < n) gw[max_label]++;
        if (pre[u] != max_label) { labels[u] = max_label; ++nupd; }
      }
      if (nupdates_out) nupdates_out[idx] = nupd;
    }
  }
  std::memcpy(lout, labels.data(), sizeof(int32_t) * n);
  return 0;
}

// --- counting back-ends -----------------------------------------------------

// method/countmin.cuh:97-125 row hashes.
static inline uint32_t cm_h1(uint32_t k) { k ^= k >> 16; k *= 0x12ebcb3bu; k ^= k >> 13; k *= 0xc123ae53u; k ^= k >> 16; return k; }
static inline uint32_t cm_h2(uint32_t k) { k ^= k >> 16; k *= 0x21eb21bbu; k ^= k >> 13; k *= 0x2cb2ea35u; k ^= k >> 16; return k; }
static inline uint32_t cm_h3(uint32_t k) { k ^= k >> 16; k *= 0x8febce61u; k ^= k >> 13; k *= 0xa2b2be25u; k ^= k >> 16; return k; }

// Count-min sketch of one neighbourhood: every neighbour contributes key =
// label+1 with weight x (1 or its edge weight).  rows is [3][W].  With
// ref_compat != 0 the third row's increment lands in row 2 at the row-3
// index, as method/countmin.cuh:190 does.
int orc_cm_sketch(int32_t v, const int32_t* off, const int32_t* cols, const int32_t* w, const int32_t* labels,
                  int32_t W, int ref_compat, uint32_t* rows) {
  if (W <= 0) return -1;
  std::memset(rows, 0, sizeof(uint32_t) * 3 * (size_t)W);
  for (int32_t j = off[v]; j < off[v + 1]; ++j) {
    const uint32_t key = (uint32_t)labels[cols[j]] + 1u;
    const uint32_t x = w ? (uint32_t)w[j] : 1u;
    rows[0 * W + cm_h1(key) % (uint32_t)W] += x;
    rows[1 * W + cm_h2(key) % (uint32_t)W] += x;
    rows[(ref_compat ? 1 : 2) * W + cm_h3(key) % (uint32_t)W] += x;
  }
  return 0;
}

// Estimate of one key from a sketch (min over the three rows; in ref_compat
// mode the third probe reads row 2 at the row-3 index).
uint32_t orc_cm_estimate(const uint32_t* rows, int32_t W, int ref_compat, int32_t label) {
  const uint32_t key = (uint32_t)label + 1u;
  uint32_t a = rows[0 * W + cm_h1(key) % (uint32_t)W];
  uint32_t b = rows[1 * W + cm_h2(key) % (uint32_t)W];
  uint32_t c = rows[(ref_compat ? 1 : 2) * W + cm_h3(key) % (uint32_t)W];
  return std::min(a, std::min(b, c));
}

// Misra-Gries frequent-items summary of one neighbourhood in CSR order
// (method/frequent.cuh:77-105, sequential): the key is inserted by linear
// probing from fmix32(key) % C into an empty or equal slot; when all C slots
// hold other keys the summary is decremented and the new key is dropped.
// Clean mode (ref_compat == 0): every count drops by one and keys reaching 0
// are removed.  ref_compat != 0 restates frequent.cuh:96-100 as written:
// atomicDec(&val, 0) stores 0 into every slot, and only keys whose previous
// count was 1 are removed.  keys/vals receive the C slots (key = label+1,
// 0 = empty); the return value is the number of decrement rounds.
static inline uint32_t fmix32(uint32_t k) { k ^= k >> 16; k *= 0x85ebca6bu; k ^= k >> 13; k *= 0xc2b2ae35u; k ^= k >> 16; return k; }

int orc_fa_summary(int32_t v, const int32_t* off, const int32_t* cols, const int32_t* labels, int32_t C,
                   int ref_compat, uint32_t* keys, uint32_t* vals) {
  if (C <= 0) return -1;
  std::memset(keys, 0, sizeof(uint32_t) * C);
  std::memset(vals, 0, sizeof(uint32_t) * C);
  int rounds = 0;
  for (int32_t j = off[v]; j < off[v + 1]; ++j) {
    const uint32_t key = (uint32_t)labels[cols[j]] + 1u;
    bool found = false;
    uint32_t i = fmix32(key);
    for (int32_t step = 0; step < C; ++step, ++i) {
      i = i % (uint32_t)C;
      if (keys[i] == 0 || keys[i] == key) { keys[i] = key; vals[i] += 1; found = true; break; }
    }
    if (!found) {
      ++rounds;
      for (int32_t s = 0; s < C; ++s) {
        const uint32_t prev = vals[s];
        if (ref_compat) {
          vals[s] = 0;
          if (prev == 1) keys[s] = 0;
        } else if (prev > 0) {
          vals[s] = prev - 1;
          if (prev == 1) keys[s] = 0;
        }
      }
    }
  }
  return rounds;
}

// Seeded LP (prop/seedLprop.cuh; seed kernels header/kernel.cuh:914-1031,
// :1742-1836, :5236-5290; start labels initialize_labels_by_seeds, :453-466):
// seeds start with their id and keep it; every other vertex starts at -1 and
// takes, each synchronous step, the label of largest count (weight sum) among
// its labelled (>= 0) neighbours, ties -> the largest label, keeping its own
// label when none is labelled.  (The reference's tiers disagree on
// unlabelled neighbours; this is the rule its big and huge kernels follow
// for labelled ones.)  trace (nullable): labels after every step [niter][n].
int orc_seeded_run(int32_t n, const int32_t* off, const int32_t* cols, const int32_t* w, const uint8_t* seeds,
                   int32_t niter, int32_t* lout, int32_t* trace, int nthreads) {
  const int nt = threads_or_default(nthreads);
  std::vector<int32_t> a(n), b(n);
  for (int32_t v = 0; v < n; ++v) a[v] = seeds[v] ? v : -1;
  for (int32_t it = 0; it < niter; ++it) {
#pragma omp parallel num_threads(nt)
    {
      std::vector<LW> buf;
#pragma omp for schedule(dynamic, 1024)
      for (int32_t v = 0; v < n; ++v) {
        if (seeds[v]) {
          b[v] = a[v];
          continue;
        }
        buf.clear();
        for (int32_t j = off[v]; j < off[v + 1]; ++j)
          if (a[cols[j]] >= 0) buf.push_back({a[cols[j]], w ? (int64_t)w[j] : 1});
        int32_t bl;
        int64_t bc;
        b[v] = mode_of(buf, &bl, &bc) ? bl : a[v];
      }
    }
    std::swap(a, b);
    if (trace) std::memcpy(trace + (size_t)it * n, a.data(), sizeof(int32_t) * n);
  }
  std::memcpy(lout, a.data(), sizeof(int32_t) * n);
  return 0;
}

// ---------------------------------------------------------------- graphs
// The seeded R-MAT workload built on the host, for the CPU legs of the
// benchmark (which must not load the engine library) and to check the
// engine's own sampler + CSR construction: samples as glp_sample_rmat
// (a counter-based SplitMix64 stream, sample i depends on (seed, i) only;
// Chakrabarti, Zhan, Faloutsos, "R-MAT", SDM 2004, quadrant probabilities
// a, b, c, d = 1-a-b-c), then
//   1. symmetrise (u,v) -> (u,v),(v,u) and drop self loops,
//   2. sort every row and drop duplicate entries,
//   3. relabel by degree descending, ties by the smaller original id (the
//      degree-sorted order tools/normalize.cpp:262-348 produces, made
//      deterministic),
//   4. emit int32 offsets[n+1] and int32 columns[m], rows ascending.
// *off and *cols are malloc'd (free with orc_free).  Returns 0, or -1 on
// bad parameters / -2 when the graph exceeds an int32 CSR.
static uint64_t rmat_thresh32(double x) {
  if (x <= 0) return 0;
  if (x >= 1) return 1ull << 32;
  return (uint64_t)std::floor(x * 4294967296.0);
}

int orc_rmat_csr(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, int32_t** off_out,
                 int32_t** cols_out, int64_t* m_out, int nthreads) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  const int nt = threads_or_default(nthreads);
  const int64_t n = 1ll << scale;
  const int64_t count = (int64_t)edge_factor << scale;
  const uint64_t ta = rmat_thresh32(a), tab = rmat_thresh32(a + b), tabc = rmat_thresh32(a + b + c);
  const uint64_t key = mix64(seed);
  std::vector<int32_t> su((size_t)count), sv((size_t)count);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < count; ++i) {
    const uint64_t k = mix64(key ^ (uint64_t)i);
    uint32_t u = 0, v = 0;
    uint64_t word = 0;
    for (int32_t lvl = 0; lvl < scale; ++lvl) {
      if ((lvl & 1) == 0) word = mix64(k + (uint64_t)(lvl >> 1));
      const uint64_t r = (lvl & 1) ? (word >> 32) : (word & 0xffffffffull);
      const uint32_t bu = r < tab ? 0u : 1u;
      const uint32_t bv = r < ta ? 0u : (r < tab ? 1u : (r < tabc ? 0u : 1u));
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    su[(size_t)i] = (int32_t)u;
    sv[(size_t)i] = (int32_t)v;
  }
  // 1. symmetrised rows (with duplicates) by counting and scattering
  std::vector<int64_t> start((size_t)n + 1, 0);
  {
    std::vector<std::atomic<int64_t>> deg((size_t)n);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t v = 0; v < n; ++v) deg[(size_t)v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < count; ++i) {
      if (su[(size_t)i] == sv[(size_t)i]) continue;
      deg[(size_t)su[(size_t)i]].fetch_add(1, std::memory_order_relaxed);
      deg[(size_t)sv[(size_t)i]].fetch_add(1, std::memory_order_relaxed);
    }
    for (int64_t v = 0; v < n; ++v) start[(size_t)v + 1] = start[(size_t)v] + deg[(size_t)v].load();
  }
  std::vector<int32_t> adj((size_t)start[(size_t)n]);
  {
    std::vector<std::atomic<int64_t>> cur((size_t)n);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t v = 0; v < n; ++v) cur[(size_t)v].store(start[(size_t)v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < count; ++i) {
      const int32_t u = su[(size_t)i], v = sv[(size_t)i];
      if (u == v) continue;
      adj[(size_t)cur[(size_t)u].fetch_add(1, std::memory_order_relaxed)] = v;
      adj[(size_t)cur[(size_t)v].fetch_add(1, std::memory_order_relaxed)] = u;
    }
  }
  std::vector<int32_t>().swap(su);
  std::vector<int32_t>().swap(sv);
  // 2. sort + dedupe every row in place; ddeg = deduplicated degree
  std::vector<int64_t> ddeg((size_t)n);
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
  for (int64_t v = 0; v < n; ++v) {
    int32_t* b0 = adj.data() + start[(size_t)v];
    int32_t* e0 = adj.data() + start[(size_t)v + 1];
    std::sort(b0, e0);
    ddeg[(size_t)v] = std::unique(b0, e0) - b0;
  }
  // 3. degree-descending order, stable in the original id (counting sort)
  int64_t maxd = 0;
  for (int64_t v = 0; v < n; ++v) maxd = std::max(maxd, ddeg[(size_t)v]);
  std::vector<int64_t> bucket((size_t)maxd + 2, 0);
  for (int64_t v = 0; v < n; ++v) ++bucket[(size_t)(maxd - ddeg[(size_t)v]) + 1];
  for (int64_t d = 0; d <= maxd; ++d) bucket[(size_t)d + 1] += bucket[(size_t)d];
  std::vector<int32_t> perm((size_t)n), newid((size_t)n);
  for (int64_t v = 0; v < n; ++v) {
    const int64_t pos = bucket[(size_t)(maxd - ddeg[(size_t)v])]++;
    perm[(size_t)pos] = (int32_t)v;
    newid[(size_t)v] = (int32_t)pos;
  }
  // 4. the relabelled CSR, rows ascending
  int64_t m = 0;
  for (int64_t v = 0; v < n; ++v) m += ddeg[(size_t)v];
  if (m > INT32_MAX) return -2;
  int32_t* off = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)(n + 1)));
  int32_t* cols = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1)));
  if (!off || !cols) {
    std::free(off);
    std::free(cols);
    return -3;
  }
  off[0] = 0;
  for (int64_t r = 0; r < n; ++r) off[r + 1] = off[r] + (int32_t)ddeg[(size_t)perm[(size_t)r]];
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
  for (int64_t r = 0; r < n; ++r) {
    const int32_t v = perm[(size_t)r];
    const int32_t* src = adj.data() + start[(size_t)v];
    int32_t* dst = cols + off[r];
    const int64_t d = ddeg[(size_t)v];
    for (int64_t j = 0; j < d; ++j) dst[j] = newid[(size_t)src[j]];
    std::sort(dst, dst + d);
  }
  *off_out = off;
  *cols_out = cols;
  *m_out = m;
  return 0;
}

void orc_free(void* p) { std::free(p); }

// Number of vertices whose label differs between two arrays.
int64_t orc_count_diff(int32_t n, const int32_t* a, const int32_t* b) {
  int64_t c = 0;
  for (int32_t v = 0; v < n; ++v) c += (a[v] != b[v]);
  return c;
}

}  // extern "C"
