// ref_cpulp_harness.cpp -- drives the reference's OpenMP CPU path
// (tutorial/CPUlp.cuh, compiled unmodified from the reference tree) on a
// binary int32 edge-list file, through the reference's own loader
// (header/graph.h CSRGraph).  TEST INFRASTRUCTURE: builds oracle/_ref/.
//
// CPUlp::sync_run_1 / layered_run / slpa_run free their label array before
// returning and print only per-iteration update counts, so the harness
// captures the labels with an array operator new[]/delete[] pair: after
// arm(n) the first `new int[n]` is the label array (CPUlp.cuh:32, :175,
// :268), and its contents are copied out when it is deleted[].
//
// usage: ref_cpulp <sync|layered|slpa> <edges.bin> <niter> <labels_out.bin>
//        ref_cpulp <sync-csr|layered-csr> <graph.csr> <niter> <labels_out.bin>
//   prints "seconds <t>" (the value the reference returns) and "n <n> m <m>".
//   A .csr file is int64 n, int64 m, int32 offsets[n+1], int32 cols[m]; it
//   fills the reference's CSRGraph members directly (they are public,
//   header/graph.h:21-44, :193-194) instead of re-parsing an edge list.
//   OMP_THREAD_LIMIT=1 makes the run deterministic (num_threads(20) is
//   hard-coded at CPUlp.cuh:50).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

static size_t g_watch_bytes = 0;
static void* g_watch_ptr = nullptr;
static std::vector<int32_t> g_captured;

void* operator new[](size_t sz) {
  void* p = std::malloc(sz ? sz : 1);
  if (!p) throw std::bad_alloc();
  if (g_watch_bytes && !g_watch_ptr && sz == g_watch_bytes) g_watch_ptr = p;
  return p;
}
void operator delete[](void* p) noexcept {
  if (p && p == g_watch_ptr) {
    g_captured.assign((int32_t*)p, (int32_t*)p + g_watch_bytes / sizeof(int32_t));
    g_watch_ptr = nullptr;
    g_watch_bytes = 0;
  }
  std::free(p);
}
void operator delete[](void* p, size_t) noexcept { operator delete[](p); }

#include "tutorial/CPUlp.cuh"

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <sync|layered|slpa> <edges.bin> <niter> <labels_out.bin>\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  const int niter = std::atoi(argv[3]);
  CSRGraph<int32_t, int32_t>* G = nullptr;
  if (mode.size() > 4 && mode.compare(mode.size() - 4, 4, "-csr") == 0) {
    mode = mode.substr(0, mode.size() - 4);
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) return 3;
    int64_t hdr[2];
    if (std::fread(hdr, sizeof(int64_t), 2, f) != 2) return 3;
    G = new CSRGraph<int32_t, int32_t>();
    G->n = (int32_t)hdr[0];
    G->m = (int32_t)hdr[1];
    G->startvalue = 0;
    G->direct = false;
    G->offsets.resize((size_t)hdr[0] + 1);
    G->neighbors.resize((size_t)hdr[1]);
    if (std::fread(G->offsets.data(), sizeof(int32_t), G->offsets.size(), f) != G->offsets.size()) return 3;
    if (std::fread(G->neighbors.data(), sizeof(int32_t), G->neighbors.size(), f) != G->neighbors.size()) return 3;
    std::fclose(f);
  } else {
    G = new CSRGraph<int32_t, int32_t>(argv[2], 0, false);
  }
  std::printf("n %d m %d\n", (int)G->n, (int)G->m);
  CPUlp<int32_t, int32_t> lp(G);
  g_watch_bytes = sizeof(int32_t) * (size_t)G->n;
  g_watch_ptr = nullptr;
  double t = 0;
  if (mode == "sync") t = lp.sync_run_1(niter);
  else if (mode == "layered") t = lp.layered_run(niter);
  else if (mode == "slpa") t = lp.slpa_run(niter);
  else {
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  }
  std::printf("\nseconds %.9f\n", t);
  FILE* f = std::fopen(argv[4], "wb");
  if (!f) return 3;
  std::fwrite(g_captured.data(), sizeof(int32_t), g_captured.size(), f);
  std::fclose(f);
  return g_captured.size() == (size_t)G->n ? 0 : 4;
}
