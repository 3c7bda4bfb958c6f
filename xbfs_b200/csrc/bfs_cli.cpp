// bfs — command line with the reference's argument contract
// (bfs_gpu_update.cu:33-48):
//
//   bfs beg csr weight BlockDim GridDim gpu_id results alpha src workload padding
//       [--out levels.bin] [--parents parents.bin] [--policy heuristic|beamer|mlp]
//       [--forced td_queue,bu,...] [--no-async] [--trace] [--repeat N]
//
// It loads the CSR pair, runs one single-source BFS through libxbfs.so and
// appends "workload;td_seconds;bu_seconds;total_seconds" to <results>, the
// line the reference writes to its timing CSV (bfs_gpu_update.cu:282-285).
// <weight> is accepted and ignored, as in the reference (run.sh passes "x").
// BlockDim is accepted for compatibility; the traversal kernel's CTA shape is
// fixed at compile time, and GridDim (> 0) caps the number of resident CTAs.
// Unlike the reference, the level array can be written out (--out: raw
// little-endian int32[V]), and no CPU BFS is run: correctness is the test
// suite's job, not the tool's.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "xbfs.h"

static int die(xbfs_status st, const char* what) {
  fprintf(stderr, "bfs: %s failed: %s (%s)\n", what, xbfs_strerror(st), xbfs_last_error());
  return 1;
}

static int parse_strategy(const std::string& s) {
  if (s == "td_queue") return XBFS_TD_QUEUE;
  if (s == "td_scan") return XBFS_TD_SCAN;
  if (s == "bu") return XBFS_BU;
  return -1;
}

int main(int argc, char** argv) {
  printf("Input: ./exe beg csr weight BlockDim GridDim gpu_id results alpha src workload padding\n");
  std::vector<std::string> pos;
  const char* out_path = nullptr;
  const char* par_path = nullptr;
  std::string policy = "heuristic";
  std::vector<int8_t> forced;
  int async_bu = 1, trace = 0, repeat = 1;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&](const char* flag) -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "bfs: %s needs a value\n", flag);
        exit(2);
      }
      return argv[++i];
    };
    if (a == "--out") out_path = next("--out");
    else if (a == "--parents") par_path = next("--parents");
    else if (a == "--policy") policy = next("--policy");
    else if (a == "--forced") {
      policy = "forced";
      std::string list = next("--forced");
      size_t st = 0;
      while (st <= list.size()) {
        size_t c = list.find(',', st);
        std::string tok = list.substr(st, c == std::string::npos ? std::string::npos : c - st);
        int v = parse_strategy(tok);
        if (v < 0) {
          fprintf(stderr, "bfs: unknown strategy '%s'\n", tok.c_str());
          return 2;
        }
        forced.push_back((int8_t)v);
        if (c == std::string::npos) break;
        st = c + 1;
      }
    } else if (a == "--no-async") async_bu = 0;
    else if (a == "--trace") trace = 1;
    else if (a == "--repeat") repeat = atoi(next("--repeat"));
    else pos.push_back(a);
  }
  if (pos.size() != 11) {
    printf("Wrong input\n");
    return 255;  // the reference returns -1 (bfs_gpu_update.cu:34)
  }
  const char* beg_file = pos[0].c_str();
  const char* csr_file = pos[1].c_str();
  const int block_dim = atoi(pos[3].c_str());
  const int grid_dim = atoi(pos[4].c_str());
  const int gpu = atoi(pos[5].c_str());
  const char* results = pos[6].c_str();
  const float alpha = (float)atof(pos[7].c_str());
  const int src = atoi(pos[8].c_str());
  const std::string workload = pos[9];
  const int padding = atoi(pos[10].c_str());
  printf("alpha = %g\n", alpha);
  // refused before any device work: the reference's bottom-up update is only
  // correct for padding 1 (bfs_adaptiveFQ_wb_async.cuh:739-775)
  if (padding != 1) {
    fprintf(stderr, "bfs: padding = %d: only 1 is supported\n", padding);
    return 2;
  }
  if (src < 0) {
    fprintf(stderr, "bfs: source %d is negative\n", src);
    return 2;
  }

  xbfs_graph* g = nullptr;
  xbfs_status st = xbfs_graph_load(beg_file, csr_file, gpu, &g);
  if (st) return die(st, "loading the graph");
  int64_t V = 0, E = 0, maxd = 0, niso = 0;
  xbfs_graph_info(g, &V, &E, &maxd, &niso);
  printf("Graph load (success): %lld verts, %lld edges, max degree %lld, %lld isolated\n", (long long)V,
         (long long)E, (long long)maxd, (long long)niso);

  xbfs_opts o;
  xbfs_opts_init(&o);
  o.alpha = alpha;
  o.block_dim = block_dim;
  o.grid_dim = grid_dim;
  o.padding = padding;
  o.async_bu = async_bu;
  o.trace = 1;
  if (policy == "heuristic") o.policy = XBFS_POLICY_HEURISTIC;
  else if (policy == "beamer") o.policy = XBFS_POLICY_BEAMER;
  else if (policy == "mlp") o.policy = XBFS_POLICY_MLP;
  else if (policy == "forced") {
    o.policy = XBFS_POLICY_FORCED;
    o.forced = forced.data();
    o.n_forced = (int32_t)forced.size();
  } else {
    fprintf(stderr, "bfs: unknown policy '%s'\n", policy.c_str());
    return 2;
  }
  std::vector<int32_t> levels((size_t)V);
  std::vector<int32_t> parents(par_path ? (size_t)V : 0);
  xbfs_stats s;
  memset(&s, 0, sizeof(s));
  printf("\nStarting BFS graph traversal from node %d......\n", src);
  for (int r = 0; r < (repeat > 0 ? repeat : 1); ++r) {
    st = xbfs_bfs(g, src, levels.data(), par_path ? parents.data() : nullptr, &o, &s);
    if (st) return die(st, "xbfs_bfs");
  }
  std::vector<xbfs_level_trace> tr((size_t)s.depth + 1);
  int32_t ntr = 0;
  xbfs_last_trace(g, tr.data(), (int32_t)tr.size(), &ntr);
  double td_us = 0, bu_us = 0;
  for (int i = 0; i < ntr; ++i) {
    (tr[i].strategy == XBFS_BU ? bu_us : td_us) += tr[i].us;
    if (trace)
      printf("level %d %-8s n_f=%lld m_f=%lld n_u=%lld %.1f us\n", tr[i].level,
             tr[i].strategy == XBFS_BU ? "bu" : (tr[i].strategy == XBFS_TD_SCAN ? "td_scan" : "td_queue"),
             (long long)tr[i].n_f, (long long)tr[i].m_f, (long long)tr[i].n_u, tr[i].us);
  }
  printf("\nCurrent level = %d reached = %lld padding=%d\n", s.depth, (long long)s.reached, padding);
  printf("Time consumption of top-down && bottom up BFS: %.9f seconds from the starting vertex %d\n",
         s.kernel_ms * 1e-3, src);
  printf("GTEPS = %.3f (m_c = %lld, kernel %.3f ms, device %.3f ms)\n",
         s.kernel_ms > 0 ? (double)s.edges_mc / (s.kernel_ms * 1e-3) / 1e9 : 0.0, (long long)s.edges_mc,
         s.kernel_ms, s.device_ms);
  printf("levels by strategy: td_queue %d, td_scan %d, bu %d; async level+2 vertices %d\n", s.n_td_queue,
         s.n_td_scan, s.n_bu, s.n_async);
  FILE* f = fopen(results, "a");
  if (f) {
    fprintf(f, "%s;%.9f;%.9f;%.9f\n", workload.c_str(), td_us * 1e-6, bu_us * 1e-6, (td_us + bu_us) * 1e-6);
    fclose(f);
  } else {
    fprintf(stderr, "bfs: cannot append to %s\n", results);
  }
  if (out_path) {
    FILE* fo = fopen(out_path, "wb");
    if (!fo || fwrite(levels.data(), 4, levels.size(), fo) != levels.size()) {
      fprintf(stderr, "bfs: cannot write %s\n", out_path);
      if (fo) fclose(fo);
      return 1;
    }
    fclose(fo);
  }
  if (par_path) {
    FILE* fp = fopen(par_path, "wb");
    if (!fp || fwrite(parents.data(), 4, parents.size(), fp) != parents.size()) {
      fprintf(stderr, "bfs: cannot write %s\n", par_path);
      if (fp) fclose(fp);
      return 1;
    }
    fclose(fp);
  }
  xbfs_graph_free(g);
  printf("Now we finish!\n");
  return 0;
}
