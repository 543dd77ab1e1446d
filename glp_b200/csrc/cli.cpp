// cli.cpp -- command-line driver over the C ABI, in the form of the
// reference's executable (main.cu:38-56, :63-101, :106-119):
//
//   glp_cli method niter graph.bin outfile ifdirect [options]
//
// method 1 classic, 2 layered, 3 SLPA, 4 user hooks; graph.bin is a binary
// int32 (u, v) pair file read with the reference's loader semantics
// (glp_load_edgelist_bin: self loops dropped, symmetrised unless ifdirect);
// one line "graph: ... method: ... iteration: ... time: ..." is appended to
// outfile, as the reference does.  Unlike the reference, the labels can be
// written out, and the layered / SLPA constants are options instead of
// compiled-in values.
//
// Options:
//   --labels FILE     write the final labels (int32, n entries)
//   --gammas g1,g2..  layered: one layer per gamma (dstar = 1/gamma + 1)
//   --slpa-T T        SLPA memory slots (default 20)
//   --slpa-r R        SLPA post-processing threshold (default 0.1)
//   --seed S          SLPA speaker hash seed
//   --hooks K         method 4 hook set: 0 classic, 1 layered, 2 weighted degree
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "glp.h"

static int usage() {
  std::fprintf(stderr,
               "usage: glp_cli method niter graph.bin outfile ifdirect [--labels FILE] [--gammas g1,g2,..]\n"
               "               [--slpa-T T] [--slpa-r R] [--seed S] [--hooks K]\n");
  return 2;
}

static int fail(const char* what, int rc) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, glp_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 6) return usage();
  const int method = std::atoi(argv[1]);
  const int niter = std::atoi(argv[2]);
  const std::string graph_path = argv[3], out_path = argv[4];
  const int direct = std::atoi(argv[5]);
  std::string labels_path;
  glp_params p;
  glp_params_default(&p);
  for (int i = 6; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
    const char* v = next();
    if (!v) return usage();
    if (a == "--labels") {
      labels_path = v;
    } else if (a == "--gammas") {
      p.nlayers = 0;
      for (const char* s = v; *s && p.nlayers < GLP_MAX_LAYERS;) {
        const double g = std::strtod(s, const_cast<char**>(&s));
        if (!(g > 0)) return usage();
        p.dstar[p.nlayers++] = (int32_t)std::lround(1.0 / g) + 1;
        if (*s == ',') ++s;
      }
    } else if (a == "--slpa-T") {
      p.slpa_T = std::atoi(v);
    } else if (a == "--slpa-r") {
      p.slpa_r = std::atof(v);
    } else if (a == "--seed") {
      p.seed = std::strtoull(v, nullptr, 10);
    } else if (a == "--hooks") {
      p.hooks = std::atoi(v);
    } else {
      return usage();
    }
  }
  if (method < 1 || method > 4 || niter < 0) return usage();

  const auto t0 = std::chrono::steady_clock::now();
  int32_t *off = nullptr, *cols = nullptr, n = 0;
  int64_t m = 0;
  int rc = glp_load_edgelist_bin(graph_path.c_str(), direct, &off, &cols, &n, &m);
  if (rc) return fail("loading the graph", rc);
  std::printf("n = %d m = %lld\n\n", n, (long long)m);
  glp_graph* g = nullptr;
  rc = glp_graph_create(off, cols, nullptr, n, m, 0, &g);
  glp_free_host(off);
  glp_free_host(cols);
  if (rc) return fail("glp_graph_create", rc);
  const auto t1 = std::chrono::steady_clock::now();

  std::vector<int32_t> labels((size_t)(n > 0 ? n : 1));
  glp_outputs out;
  std::memset(&out, 0, sizeof out);
  out.labels = labels.data();
  rc = glp_run(g, method, &p, niter, &out, nullptr, nullptr, nullptr);
  const auto t2 = std::chrono::steady_clock::now();
  glp_graph_destroy(g);
  if (rc) return fail("glp_run", rc);
  std::printf("success run\n");

  const double load_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  const double lp_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
  if (FILE* f = std::fopen(out_path.c_str(), "a")) {
    std::fprintf(f, "graph: %s method: %d iteration: %d time: %.3f load graph to GPU: %.3f LP: %.3f\n",
                 graph_path.c_str(), method, niter, lp_ms, load_ms, lp_ms);
    std::fclose(f);
  } else {
    std::fprintf(stderr, "cannot append to %s\n", out_path.c_str());
    return 1;
  }
  if (!labels_path.empty()) {
    FILE* f = std::fopen(labels_path.c_str(), "wb");
    if (!f || std::fwrite(labels.data(), sizeof(int32_t), (size_t)n, f) != (size_t)n) {
      std::fprintf(stderr, "cannot write %s\n", labels_path.c_str());
      if (f) std::fclose(f);
      return 1;
    }
    std::fclose(f);
  }
  return 0;
}
