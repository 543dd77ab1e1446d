// ref_gpu_harness.cu -- runs the reference's own GPU propagation kernels on a
// CSR with a correct plan and fully initialised buffers.  TEST
// INFRASTRUCTURE ONLY: it is built by oracle/build_ref.sh into
// oracle/_ref/ref_gpu_lp, and only tests/ run it, as a second checker of the
// oracle's synchronous rule.
//
// The kernels come from the reference tree: header/kernel.cuh (copied at
// build time, truncated before its user-defined stub area at line 6071,
// which does not compile, into the ignored folder oracle/_ref/kshim/header/)
// and method/hashtable.cuh (GlobalHT), included where they lie.  The driver
// is this file's own; it replaces prop/classicLprop.cuh:161-452 and
// prop/MultiLprop.cuh:308-374, whose plan and buffers are not usable as
// shipped (labels_write never initialised and copied over the labels every
// iteration, prop/classicLprop.cuh:203, :371; hub block counts scanned from
// uninitialised memory, :241-246; the hub maxima never reset, :255; the tiny
// packing's first offset a vertex id, :275; niter-1 steps, :361).
//
// Plan (vertices must be sorted by non-increasing degree, as the reference's
// binning assumes, prop/classicLprop.cuh:212-220): hubs have degree > 640,
// big 129..640, medium 33..128, small 17..32, tiny 0..16 -- the reference's
// thresholds (huge = 128*5, medium = 32*4, :196-198; small_index at 32,
// tiny at 16, :217-219).  Launch shapes and template arguments are the
// reference's: l_huge_update_syn2_labelload<32,256> on ceil(d/256) blocks per
// hub with l_sub_huge_update_syn<32,128>, l_big_update_syn2_labelload<32,1,
// 128,600>, l_medium_update_syn_labelload<32,1,128,4>, l_small_update_syn_
// labelload<32,1,64>, l_tiny_update_syn2_labelload on 64-thread blocks over
// warps packing up to 32 edges (:235-316, :381-423); the ml_* layered
// kernels likewise (prop/MultiLprop.cuh:330-368).
//
// Every index a kernel will form is checked on the host before the first
// launch: CSR bounds, the degree order, labels in [0, n), and that the
// kernels' signed hash (kernel.cuh:408-415, abs() of a 32-bit mix) is never
// INT_MIN for a key 1..n (a negative value would index shared memory below
// its table in l_big_update_syn2_labelload, kernel.cuh:1694-1696).  The
// tiny kernel reads warp_begin[] for every warp of its last block
// (kernel.cuh:5199), so that array is padded to whole blocks.
//
// usage:
//   ref_gpu_lp classic <graph.csr> <niter> <init.bin|-> <trace.bin>
//   ref_gpu_lp classic-time <graph.csr> <niter> - <labels.bin>   (prints per-step device ms)
//   ref_gpu_lp layered <graph.csr> <niter> <dstar,dstar,...> <trace.bin> [<vol.bin>]
//   ref_gpu_lp slpa    <graph.csr> <niter> <T,seed> <trace.bin> <memory.bin>
// graph.csr: int64 n, int64 m, int32 offsets[n+1], int32 cols[m].
// trace.bin receives int32 labels after every step ([steps][n]); vol.bin
// the layered volumes after the last step.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "method/hashtable.cuh"
#include "method/countmin.cuh"
#include "header/kernel.cuh"
#include "header/graph.h"

#include <thrust/execution_policy.h>
#include <thrust/sort.h>

// SLPA: the reference's own speaker memory (tutorial/Base5prop.cuh:161-208,
// storelabel/picklabel, host code) with its rand() call replaced, for this
// translation unit only, by the counter hash the engine and the oracle use:
// inside picklabel the vertex is the loop variable i.  Every header the file
// pulls in is already included above, so the macro touches its text alone.
static int g_slpa_iter = 0, g_slpa_T = 1;
static uint64_t g_slpa_seed = 0;
static inline uint64_t splitmix64(uint64_t z) {  // Steele, Lea, Flood, OOPSLA 2014
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
// H(seed, iteration, v) mod T: the first memory slot the speaker scan tries
static int glp_speaker_draw(int v) {
  const uint64_t h = splitmix64(splitmix64(splitmix64(g_slpa_seed) ^ (uint64_t)g_slpa_iter) ^ (uint64_t)v);
  return (int)(h % (uint64_t)g_slpa_T);
}
#define rand() glp_speaker_draw(i)
#include "tutorial/Base5prop.cuh"
#undef rand

namespace {

constexpr int kHuge = 640, kMedium = 128, kSmall = 32, kTiny = 16;

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      std::fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #call,           \
                   cudaGetErrorString(e_));                                       \
      std::exit(5);                                                               \
    }                                                                             \
  } while (0)

[[noreturn]] void die(const char* msg) {
  std::fprintf(stderr, "ref_gpu_lp: %s\n", msg);
  std::exit(2);
}

// The kernels' signed hash (kernel.cuh:408-415) evaluated on the host with
// the same 32-bit wrap-around and arithmetic shifts.
int32_t kernel_hash(int32_t k) {
  auto sh = [](int32_t x, int s) { return (int32_t)(x >> s); };  // arithmetic, as on the device
  k ^= sh(k, 16);
  k = (int32_t)((uint32_t)k * 0x85ebca6bu);
  k ^= sh(k, 13);
  k = (int32_t)((uint32_t)k * 0xc2b2ae35u);
  k ^= sh(k, 16);
  return k;  // abs() of INT_MIN stays negative
}

struct Csr {
  int32_t n = 0;
  int64_t m = 0;
  std::vector<int32_t> off, cols;
};

Csr read_csr(const char* path) {
  Csr g;
  FILE* f = std::fopen(path, "rb");
  if (!f) die("cannot open the graph file");
  int64_t hdr[2];
  if (std::fread(hdr, sizeof hdr[0], 2, f) != 2) die("short graph header");
  if (hdr[0] < 0 || hdr[0] > INT_MAX - 1 || hdr[1] < 0 || hdr[1] > INT_MAX) die("graph size outside int32");
  g.n = (int32_t)hdr[0];
  g.m = hdr[1];
  g.off.resize((size_t)g.n + 1);
  g.cols.resize((size_t)std::max<int64_t>(g.m, 1));
  if (std::fread(g.off.data(), 4, g.off.size(), f) != g.off.size()) die("short offsets");
  if (g.m && std::fread(g.cols.data(), 4, (size_t)g.m, f) != (size_t)g.m) die("short columns");
  std::fclose(f);
  if (g.off[0] != 0 || g.off[g.n] != g.m) die("offsets[0] must be 0 and offsets[n] must be m");
  for (int32_t v = 0; v < g.n; ++v) {
    if (g.off[v + 1] < g.off[v]) die("offsets not monotone");
    if (v + 1 < g.n && g.off[v + 2] - g.off[v + 1] > g.off[v + 1] - g.off[v]) die("degrees must not increase");
  }
  for (int64_t j = 0; j < g.m; ++j)
    if (g.cols[j] < 0 || g.cols[j] >= g.n) die("column outside [0, n)");
  for (int32_t k = 1; k <= g.n; ++k)
    if (kernel_hash(k) == INT_MIN) die("a key hashes to INT_MIN (negative shared-memory index): graph refused");
  return g;
}

struct Plan {
  int32_t huge_end = 0, big_end = 0, medium_end = 0, small_end = 0;  // tier ends on the sorted ids
  std::vector<int32_t> block_v, block_id;                              // hub blocks
  std::vector<int32_t> warp_v, warp_begin;                             // tiny packing
  int32_t warps = 0;
};

Plan make_plan(const Csr& g) {
  Plan p;
  auto deg = [&](int32_t v) { return g.off[v + 1] - g.off[v]; };
  int32_t v = 0;
  while (v < g.n && deg(v) > kHuge) ++v;
  p.huge_end = v;
  while (v < g.n && deg(v) > kMedium) ++v;
  p.big_end = v;
  while (v < g.n && deg(v) > kSmall) ++v;
  p.medium_end = v;
  while (v < g.n && deg(v) > kTiny) ++v;
  p.small_end = v;
  for (int32_t h = 0; h < p.huge_end; ++h)
    for (int32_t b = 0; b * 256 < deg(h); ++b) {
      p.block_v.push_back(h);
      p.block_id.push_back(b);
    }
  // tiny packing: consecutive vertices share a warp while their edges fit in
  // 32 lanes; lane i of a warp reads edge warp_begin + i
  int32_t used = 32;
  for (int32_t u = p.small_end; u < g.n; ++u) {
    const int32_t d = deg(u);
    if (d == 0) continue;  // an isolated vertex keeps its label
    if (used + d > 32) {
      while (p.warps > 0 && used < 32) { p.warp_v.push_back(-1); ++used; }
      p.warp_begin.push_back(g.off[u]);
      ++p.warps;
      used = 0;
    }
    for (int32_t k = 0; k < d; ++k) p.warp_v.push_back(u);
    used += d;
  }
  while (p.warps > 0 && used < 32) { p.warp_v.push_back(-1); ++used; }
  // whole 64-thread blocks: the kernel reads warp_begin[] for every warp
  const int32_t padded = ((p.warps + 1) / 2) * 2;
  p.warp_begin.resize((size_t)std::max(padded, 2), 0);
  p.warp_v.resize((size_t)std::max(padded, 2) * 32, -1);
  return p;
}

template <class T>
T* dcopy(const std::vector<T>& h) {
  T* d = nullptr;
  CK(cudaMalloc(&d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) CK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return d;
}

inline int divup(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

struct Dev {
  int *nb, *off, *lr, *lw, *verts, *counter, *block_v, *block_id, *warp_v, *warp_begin;
  int *vol_r, *vol_w;
  unsigned long long* maxc;
  GlobalHT table;
  size_t table_len;
};

Dev upload(const Csr& g, const Plan& p) {
  Dev d{};
  d.nb = dcopy(g.cols);
  d.off = dcopy(g.off);
  std::vector<int32_t> ids(g.n);
  for (int32_t v = 0; v < g.n; ++v) ids[v] = v;
  d.verts = dcopy(ids);
  d.lr = dcopy(ids);
  d.lw = dcopy(ids);
  d.counter = dcopy(std::vector<int32_t>(1, 0));
  d.block_v = dcopy(p.block_v);
  d.block_id = dcopy(p.block_id);
  d.warp_v = dcopy(p.warp_v);
  d.warp_begin = dcopy(p.warp_begin);
  d.vol_r = dcopy(std::vector<int32_t>((size_t)g.n, 0));
  d.vol_w = dcopy(std::vector<int32_t>((size_t)g.n, 0));
  d.maxc = dcopy(std::vector<unsigned long long>((size_t)std::max(p.huge_end, 1), 0ull));
  d.table_len = (size_t)std::max(g.off[p.big_end], 1);
  CK(cudaMalloc(&d.table.keys, sizeof(uint32_t) * d.table_len));
  CK(cudaMalloc(&d.table.vals, sizeof(uint32_t) * d.table_len));
  return d;
}

// One synchronous step of the classic kernels: labels_read <- labels_write,
// global table and hub maxima cleared, every tier launched in the
// reference's order.
void classic_step(const Csr& g, const Plan& p, Dev& d) {
  CK(cudaMemcpy(d.lr, d.lw, sizeof(int) * g.n, cudaMemcpyDeviceToDevice));
  CK(cudaMemset(d.table.keys, 0, sizeof(uint32_t) * d.table_len));
  CK(cudaMemset(d.table.vals, 0, sizeof(uint32_t) * d.table_len));
  CK(cudaMemset(d.maxc, 0, sizeof(unsigned long long) * std::max(p.huge_end, 1)));
  const int nhub = p.huge_end, nbig = p.big_end - p.huge_end, nmed = p.medium_end - p.big_end,
            nsmall = p.small_end - p.medium_end;
  if (nhub) {
    l_huge_update_syn2_labelload<32, 256><<<(unsigned)p.block_v.size(), 256>>>(
        d.nb, d.off, d.lr, d.verts, d.block_v, d.block_id, d.maxc, d.table);
    l_sub_huge_update_syn<32, 128><<<divup(nhub, 128), 128>>>(d.maxc, d.lw, d.counter, nhub);
  }
  if (nbig)
    l_big_update_syn2_labelload<32, 1, 128, 600><<<nbig, 128>>>(p.huge_end, p.big_end, d.nb, d.off, d.lw, d.lr,
                                                                 d.verts, d.counter, d.table);
  if (nmed)
    l_medium_update_syn_labelload<32, 1, 128, 4><<<divup(nmed, 4), 128>>>(p.big_end, p.medium_end, d.nb, d.off, d.lw,
                                                                          d.lr, d.verts, d.counter, kMedium);
  if (nsmall)
    l_small_update_syn_labelload<32, 1, 64><<<divup(nsmall, 2), 64>>>(p.medium_end, p.small_end, d.nb, d.off, d.lw,
                                                                      d.lr, d.verts, d.counter);
  if (p.warps)
    l_tiny_update_syn2_labelload<<<divup(p.warps, 2), 64>>>(d.nb, d.off, d.lw, d.lr, d.counter, d.warp_v,
                                                            d.warp_begin, p.warps);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
}

// One layered step (score delta*k - vol_r[l]); the kernels add each new
// label into vol_w (the tiny kernel adds into vol_r, kernel.cuh:5498, and the
// small kernel counts no isolated vertex, :4720-4722: graphs for a volume
// comparison have neither).
void layered_step(const Csr& g, const Plan& p, Dev& d, int delta) {
  CK(cudaMemcpy(d.lr, d.lw, sizeof(int) * g.n, cudaMemcpyDeviceToDevice));
  CK(cudaMemset(d.table.keys, 0, sizeof(uint32_t) * d.table_len));
  CK(cudaMemset(d.table.vals, 0, sizeof(uint32_t) * d.table_len));
  // the hub maxima are signed (score << 32) + key: start below every score
  std::vector<long long> lo((size_t)std::max(p.huge_end, 1), LLONG_MIN);
  CK(cudaMemcpy(d.maxc, lo.data(), sizeof(long long) * lo.size(), cudaMemcpyHostToDevice));
  long long* maxc = reinterpret_cast<long long*>(d.maxc);
  const int nhub = p.huge_end, nbig = p.big_end - p.huge_end, nmed = p.medium_end - p.big_end,
            nsmall = p.small_end - p.medium_end;
  if (nhub) {
    ml_huge_update_syn_labelload<32, 256><<<(unsigned)p.block_v.size(), 256>>>(
        d.nb, d.off, d.lr, d.verts, d.block_v, d.block_id, maxc, d.table, d.vol_r, delta);
    ml_sub_huge_update_syn<32, 128><<<divup(nhub, 128), 128>>>(maxc, d.lw, d.counter, nhub, d.vol_w);
  }
  if (nbig)
    ml_big_update_syn_labelload<32, 1, 128, 600><<<nbig, 128>>>(p.huge_end, p.big_end, d.nb, d.off, d.lw, d.lr,
                                                                 d.verts, d.counter, d.table, d.vol_r, d.vol_w,
                                                                 delta);
  if (nmed)
    ml_medium_update_syn_labelload<32, 1, 128, 4><<<divup(nmed, 4), 128>>>(
        p.big_end, p.medium_end, d.nb, d.off, d.lw, d.lr, d.verts, d.counter, kMedium, d.vol_r, d.vol_w, delta);
  if (nsmall)
    ml_small_update_syn_labelload<32, 1, 64><<<divup(nsmall, 2), 64>>>(p.medium_end, p.small_end, d.nb, d.off, d.lw,
                                                                       d.lr, d.verts, d.counter, d.vol_r, d.vol_w,
                                                                       delta);
  if (p.warps)
    ml_tiny_update_syn_labelload<<<divup(p.warps, 2), 64>>>(d.nb, d.off, d.lw, d.lr, d.counter, d.warp_v,
                                                            d.warp_begin, p.warps, d.vol_r, d.vol_w, delta);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
}

// Exposes the speaker-memory steps of the reference SLPA propagator.
struct SlpaHarness : Base5prop<int, int> {
  using Base5prop<int, int>::Base5prop;
  using Base5prop<int, int>::init_gmem;
  using Base5prop<int, int>::free_gmem;
  using Base5prop<int, int>::picklabel;
  using Base5prop<int, int>::storelabel;
  using Base5prop<int, int>::labels;
  using Base5prop<int, int>::label_container;
  using Base5prop<int, int>::d_labels;
  using Base5prop<int, int>::myconf;
};

// The listener of one SLPA step on the host: the synchronous rule over the
// spoken labels (mode, ties -> the largest label); an isolated vertex keeps
// its current label.
void listen(const Csr& g, const std::vector<int32_t>& spoken, const std::vector<int32_t>& cur,
            std::vector<int32_t>& out) {
  std::vector<int32_t> buf;
  for (int32_t v = 0; v < g.n; ++v) {
    if (g.off[v] == g.off[v + 1]) {
      out[v] = cur[v];
      continue;
    }
    buf.clear();
    for (int32_t j = g.off[v]; j < g.off[v + 1]; ++j) buf.push_back(spoken[g.cols[j]]);
    std::sort(buf.begin(), buf.end());
    int32_t best = buf[0], bc = 0;
    for (size_t i = 0; i < buf.size();) {
      size_t k = i;
      while (k < buf.size() && buf[k] == buf[i]) ++k;
      if ((int32_t)(k - i) >= bc) {  // ascending labels: ">=" keeps the largest on a tie
        bc = (int32_t)(k - i);
        best = buf[i];
      }
      i = k;
    }
    out[v] = best;
  }
}

void dump(FILE* f, const int* dptr, int32_t n) {
  std::vector<int32_t> h((size_t)n);
  CK(cudaMemcpy(h.data(), dptr, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (std::fwrite(h.data(), 4, h.size(), f) != h.size()) die("short write");
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    std::fprintf(stderr,
                 "usage: %s classic <graph.csr> <niter> <init.bin|-> <trace.bin>\n"
                 "       %s layered <graph.csr> <niter> <dstar,...> <trace.bin> [<vol.bin>]\n"
                 "       %s slpa <graph.csr> <niter> <T,seed> <trace.bin> <memory.bin>\n",
                 argv[0], argv[0], argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  const Csr g = read_csr(argv[2]);
  const int niter = std::atoi(argv[3]);
  if (niter < 0 || niter > 100000) die("niter outside [0, 100000]");
  const Plan p = make_plan(g);
  std::printf("n %d m %lld huge %d big %d medium %d small %d tiny_warps %d\n", g.n, (long long)g.m, p.huge_end,
              p.big_end - p.huge_end, p.medium_end - p.big_end, p.small_end - p.medium_end, p.warps);
  if (g.n == 0) return 0;
  Dev d = upload(g, p);
  FILE* tr = std::fopen(argv[5], "wb");
  if (!tr) die("cannot open the trace file");
  if (mode == "classic-time") {
    // device time of each synchronous step (the reference's per-iteration
    // work: label copy, table and hub-maxima clears, the five bin kernels),
    // CUDA events around the step, no label dump inside the timed span
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double total = 0;
    for (int it = 0; it < niter; ++it) {
      CK(cudaEventRecord(e0));
      classic_step(g, p, d);
      CK(cudaEventRecord(e1));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      total += ms;
      std::printf("iter %d ms %.4f\n", it, ms);
    }
    std::printf("total_ms %.4f\n", total);
    dump(tr, d.lw, g.n);
  } else if (mode == "classic") {
    if (std::strcmp(argv[4], "-") != 0) {
      std::vector<int32_t> init((size_t)g.n);
      FILE* f = std::fopen(argv[4], "rb");
      if (!f || std::fread(init.data(), 4, init.size(), f) != init.size()) die("cannot read the initial labels");
      std::fclose(f);
      for (int32_t x : init)
        if (x < 0 || x >= g.n) die("initial label outside [0, n)");
      CK(cudaMemcpy(d.lw, init.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
    }
    for (int it = 0; it < niter; ++it) {
      classic_step(g, p, d);
      dump(tr, d.lw, g.n);
    }
  } else if (mode == "layered") {
    std::vector<int> dstar;
    for (const char* s = argv[4]; *s;) {
      char* e = nullptr;
      const long x = std::strtol(s, &e, 10);
      if (e == s || x < 1 || x > 65536) die("bad dstar list");
      dstar.push_back((int)x);
      s = *e == ',' ? e + 1 : e;
    }
    if (dstar.empty()) die("empty dstar list");
    // scores must stay inside int (kernel arithmetic): dstar * degree < 2^31
    for (int x : dstar)
      if ((int64_t)x * (g.n ? (g.off[1] - g.off[0]) : 0) + g.n >= INT_MAX) die("layered scores overflow int");
    std::vector<int32_t> ids((size_t)g.n);
    for (int32_t v = 0; v < g.n; ++v) ids[v] = v;
    bool first = true;
    for (int delta : dstar) {
      CK(cudaMemcpy(d.lw, ids.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
      for (int it = 0; it < niter; ++it) {
        // vol_r <- vol_w (0 before the very first step), vol_w <- 0
        if (first) {
          CK(cudaMemset(d.vol_r, 0, sizeof(int) * g.n));
          first = false;
        } else {
          std::swap(d.vol_r, d.vol_w);
        }
        CK(cudaMemset(d.vol_w, 0, sizeof(int) * g.n));
        layered_step(g, p, d, delta);
        dump(tr, d.lw, g.n);
      }
    }
    if (argc > 6) {
      FILE* vf = std::fopen(argv[6], "wb");
      if (!vf) die("cannot open the volume file");
      dump(vf, d.vol_w, g.n);
      std::fclose(vf);
    }
  } else if (mode == "slpa") {
    // argv[4] = "T,seed"; trace = labels after every step; argv[6] = memory [n][T]
    int T = 0;
    unsigned long long seed = 0;
    if (std::sscanf(argv[4], "%d,%llu", &T, &seed) != 2 || T < 1 || T > 64) die("slpa wants T,seed with T in 1..64");
    if (argc < 7) die("slpa wants a memory output file");
    g_slpa_T = T;
    g_slpa_seed = seed;
    CSRGraph<int, int> G;
    G.n = g.n;
    G.m = (int)g.m;
    G.startvalue = 0;
    G.direct = false;
    G.offsets = g.off;
    G.neighbors.assign(g.cols.begin(), g.cols.begin() + g.m);
    SlpaHarness lp(&G);
    lp.myconf.label_size = T;
    lp.init_gmem(g.n, (int)std::max<int64_t>(g.m, 1));
    std::vector<int32_t> cur((size_t)g.n), spoken((size_t)g.n), next((size_t)g.n);
    for (int32_t v = 0; v < g.n; ++v) cur[v] = v;
    CK(cudaMemcpy(lp.d_labels, cur.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
    for (int it = 0; it < niter; ++it) {
      g_slpa_iter = it;
      lp.storelabel();  // the current labels into memory (Base5prop.cuh:187-208)
      lp.picklabel();   // the speakers (Base5prop.cuh:161-183): lp.labels, copied to d_labels
      std::copy(lp.labels, lp.labels + g.n, spoken.begin());
      listen(g, spoken, cur, next);
      cur.swap(next);
      CK(cudaMemcpy(lp.d_labels, cur.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
      if (std::fwrite(cur.data(), 4, cur.size(), tr) != cur.size()) die("short write");
    }
    FILE* mf = std::fopen(argv[6], "wb");
    if (!mf) die("cannot open the memory file");
    for (int32_t v = 0; v < g.n; ++v)
      if (std::fwrite(lp.label_container[v], 4, (size_t)T, mf) != (size_t)T) die("short write");
    std::fclose(mf);
    lp.free_gmem();
  } else {
    die("mode must be classic, layered or slpa");
  }
  std::fclose(tr);
  return 0;
}
