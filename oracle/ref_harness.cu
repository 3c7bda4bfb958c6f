// ref_harness.cu — runs the reference XBFS GPU path (BFS_ControlFlow,
// bfs_adaptiveFQ_wb_async.cuh:934-1258) on a CSR file pair and dumps its
// level array, so the CPU oracle and the new kernels can be pinned against
// the reference's own output. Test infrastructure only (oracle/).
//
// Built by oracle/Makefile from the reference headers where they lie (the
// include path points at the reference checkout; nothing is copied). The
// main() below is this project's: it mirrors what the reference's main does
// before and after the call (bfs_gpu_update.cu:105-127 CPU levels, which the
// reference needs for its termination test at cuh:1237-1253; device buffers
// as at bfs_gpu_update.cu:175-240; status copy-back at :255).
//
// Safety gate (the reference has latent out-of-bounds accesses): before any
// GPU work the harness replays the reference's direction switch from the CPU
// levels and refuses (exit 3, nothing launched) when
//   * the depth reaches 99 (count[100], cuh:1026, is indexed by level),
//   * the first level is bottom-up (the following scan-free top-down would
//     expand the whole unvisited queue, cuh:1078-1110),
//   * a "last phase" run could append past the end of small_FQ (the queue is
//     seeded with every unvisited vertex and grows in place, bfs_TD_scan_free.cuh:43).
//
// usage: xbfs_ref_harness beg csr src out_levels.bin [alpha] [BlockDim] [GridDim]
// prints one JSON line on stderr; the reference's own chatter goes to stdout.
#include "graph.h"  // reference include order (bfs_gpu_update.cu:2,14): wtime before the kernels
#include "bfs_adaptiveFQ_wb_async.cuh"

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s beg csr src out_levels.bin [alpha] [BlockDim] [GridDim]\n", argv[0]);
    return 2;
  }
  typedef int param_t;
  typedef long int index_t;
  const char* beg_file = argv[1];
  const char* csr_file = argv[2];
  const int src = atoi(argv[3]);
  const char* out = argv[4];
  const float alpha = argc > 5 ? (float)atof(argv[5]) : 0.1f;
  const int BlockDim = argc > 6 ? atoi(argv[6]) : 256;
  const int GridDim = argc > 7 ? atoi(argv[7]) : 256;
  if (BlockDim <= 0 || BlockDim > 512 || (BlockDim & (BlockDim - 1))) {
    fprintf(stderr, "{\"error\": \"BlockDim must be a power of two <= 512 (prefix_sum1.cuh)\"}\n");
    return 2;
  }
  graph<int, long, int, int, long, char>* g =
      new graph<int, long, int, int, long, char>(beg_file, csr_file, "/nonexistent-weight-file");
  const int V = (int)g->vert_count;
  if (src < 0 || src >= V) return 2;

  // CPU levels (same sweep as bfs_gpu_update.cu:105-127)
  param_t* status = new param_t[V];
  for (int i = 0; i < V; ++i) status[i] = -1;
  status[src] = 0;
  int k = 0;
  bool isdone = false;
  for (k = 0; !isdone; ++k) {
    isdone = true;
    for (int i = 0; i < V; ++i)
      if (status[i] == k)
        for (long j = g->beg_pos[i]; j < g->beg_pos[i + 1]; ++j)
          if (status[g->csr[j]] == -1) {
            isdone = false;
            status[g->csr[j]] = k + 1;
          }
  }
  // ---- safety gate: replay the reference's switch (cuh:1042-1078, 1114)
  int depth = 0;
  for (int i = 0; i < V; ++i)
    if (status[i] + 1 > depth) depth = status[i] + 1;
  if (depth >= 99) {
    fprintf(stderr, "{\"skipped\": \"depth %d >= 99: count[100] overflow\"}\n", depth);
    return 3;
  }
  std::vector<long long> cnt(depth + 2, 0), nsmall(depth + 2, 0), nlev(depth + 2, 0);
  for (int i = 0; i < V; ++i) {
    if (status[i] < 0) continue;
    const long d = g->beg_pos[i + 1] - g->beg_pos[i];
    cnt[status[i]] += d;
    nlev[status[i]] += 1;
    if (d > 0 && d <= 32) nsmall[status[i]] += 1;
  }
  {
    const long long E = g->beg_pos[V];
    int is_change = 0;
    long long td_adaptive = 10000, hub_before = 0, hub_after = 0;
    int tag_prev = 0;
    long long U = 0, appended = 0;
    long long reached_upto = 0;  // vertices with level <= L
    bool in_last = false;
    for (int L = 0; L < depth - 1; ++L) {
      const long long c = cnt[L];
      const long long cp = L > 0 ? cnt[L - 1] : 0;
      if (!is_change) {
        if (L == 0 && c >= 10000) { is_change = 1; td_adaptive = 1; }
        else if (L > 0 && cp >= 10000 && c >= 100000 && c / cp >= 8) { is_change = 1; td_adaptive = L; }
        else if ((L > 0 && c >= 1000000) || (L > 0 && cp < 10000 && cp > 0 && c >= 100000 && c / cp >= 1000)) {
          is_change = 1;
          td_adaptive = L;
        }
      }
      const float ratio = (float)c / (float)E;
      if (ratio >= alpha && tag_prev >= 0) hub_before = L;
      if (ratio < alpha && tag_prev == -1) hub_after = L;
      reached_upto += nlev[L];
      if (ratio < alpha) {
        if (hub_before == 0 && L < td_adaptive) tag_prev = 0;
        else if (hub_after > 0 && L > hub_after) {
          tag_prev = 0;
          if (!in_last) in_last = true;
          appended += nsmall[L + 1];
          if (U + appended > V) {
            fprintf(stderr, "{\"skipped\": \"last-phase queue could overflow at level %d\"}\n", L);
            return 3;
          }
        } else tag_prev = 1;
      } else {
        if (L == 0) {
          fprintf(stderr, "{\"skipped\": \"first level is bottom-up\"}\n");
          return 3;
        }
        tag_prev = -1;
        U = V - (reached_upto - nlev[L]);  // unvisited when this BU level starts
        appended = 0;
        in_last = false;
      }
    }
  }

  // ---- device buffers as in the reference's main (bfs_gpu_update.cu:175-240)
  index_t* beg_cu;
  H_ERR(cudaMalloc((void**)&beg_cu, sizeof(index_t) * (V + 1)));
  H_ERR(cudaMemcpy(beg_cu, g->beg_pos, sizeof(index_t) * (V + 1), cudaMemcpyHostToDevice));
  param_t* csr_cu;
  H_ERR(cudaMalloc((void**)&csr_cu, sizeof(param_t) * (g->beg_pos[V] > 0 ? g->beg_pos[V] : 1)));
  H_ERR(cudaMemcpy(csr_cu, g->csr, sizeof(param_t) * g->beg_pos[V], cudaMemcpyHostToDevice));
  param_t* status_cpp;
  H_ERR(cudaMalloc((void**)&status_cpp, sizeof(param_t) * V));
  H_ERR(cudaMemcpy(status_cpp, status, sizeof(param_t) * V, cudaMemcpyHostToDevice));
  param_t* small = new param_t[V];
  param_t* medium = new param_t[V];
  param_t* large = new param_t[V];
  memset(small, -1, sizeof(param_t) * V);
  memset(medium, -1, sizeof(param_t) * V);
  memset(large, -1, sizeof(param_t) * V);
  param_t *small_FQ, *medium_FQ, *large_FQ, *small_BU, *medium_BU, *large_BU;
  param_t** qs[6] = {&small_FQ, &medium_FQ, &large_FQ, &small_BU, &medium_BU, &large_BU};
  for (int i = 0; i < 6; ++i) {
    H_ERR(cudaMalloc((void**)qs[i], sizeof(param_t) * V));
    H_ERR(cudaMemcpy(*qs[i], small, sizeof(param_t) * V, cudaMemcpyHostToDevice));
  }
  param_t* Status = new param_t[V];
  memset(Status, -1, sizeof(param_t) * V);
  Status[src] = 0;
  param_t* Status_cu;
  H_ERR(cudaMalloc((void**)&Status_cu, sizeof(param_t) * V));
  H_ERR(cudaMemcpy(Status_cu, Status, sizeof(param_t) * V, cudaMemcpyHostToDevice));
  param_t* small_cnt = (param_t*)calloc(1, sizeof(param_t));
  param_t* medium_cnt = (param_t*)calloc(1, sizeof(param_t));
  param_t* large_cnt = (param_t*)calloc(1, sizeof(param_t));
  param_t *small_CNT, *medium_CNT, *large_CNT, *d_level;
  H_ERR(cudaMalloc((void**)&small_CNT, sizeof(param_t)));
  H_ERR(cudaMalloc((void**)&medium_CNT, sizeof(param_t)));
  H_ERR(cudaMalloc((void**)&large_CNT, sizeof(param_t)));
  H_ERR(cudaMemset(small_CNT, 0, sizeof(param_t)));
  H_ERR(cudaMemset(medium_CNT, 0, sizeof(param_t)));
  H_ERR(cudaMemset(large_CNT, 0, sizeof(param_t)));
  param_t* level = (param_t*)calloc(1, sizeof(param_t));
  H_ERR(cudaMalloc((void**)&d_level, sizeof(param_t)));
  H_ERR(cudaMemset(d_level, 0, sizeof(param_t)));
  // tag/iter/ratio with one slot of padding before index 0 (tag[-1] is read
  // at level 0, cuh:1069-1071)
  param_t* tag_base = new param_t[k + 2];
  for (int i = 0; i < k + 2; ++i) tag_base[i] = -1;
  tag_base[0] = 0;
  param_t* tag = tag_base + 1;
  double* iter = new double[k + 1]();
  float* ratio = new float[k + 1]();
  double T1 = 0, T2 = 0, T3 = 0, T4 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0;
  cudaDeviceSynchronize();
  const double w0 = wtime();
  BFS_ControlFlow<param_t, index_t>(1, std::string("harness"), src, 0, ratio, tag, iter, t1, t2, t3, t4, t5, t6, T1,
                                    T2, T3, T4, BlockDim, GridDim, status, status_cpp, Status, Status_cu, small,
                                    medium, large, small_FQ, medium_FQ, large_FQ, small_cnt, medium_cnt, large_cnt,
                                    small_CNT, medium_CNT, large_CNT, V, level, d_level, g->beg_pos, beg_cu, csr_cu,
                                    alpha, small_BU, medium_BU, large_BU);
  cudaDeviceSynchronize();
  const double wall = wtime() - w0;
  H_ERR(cudaMemcpy(Status, Status_cu, sizeof(param_t) * V, cudaMemcpyDeviceToHost));
  int mismatch = 0;
  for (int i = 0; i < V; ++i) mismatch += Status[i] != status[i];
  FILE* f = fopen(out, "wb");
  if (!f) return 4;
  fwrite(Status, sizeof(param_t), V, f);
  fclose(f);
  fprintf(stderr,
          "{\"V\": %d, \"E\": %ld, \"src\": %d, \"levels\": %d, \"mismatch\": %d, \"kernel_s\": %.9f, "
          "\"td_s\": %.9f, \"bu_s\": %.9f, \"wall_s\": %.9f, \"tags\": [",
          V, g->beg_pos[V], src, level[0], mismatch, T1 + T2 + T3 + T4, T1 + T2, T3 + T4, wall);
  for (int i = 0; i < level[0]; ++i) fprintf(stderr, "%s%d", i ? ", " : "", tag[i]);
  fprintf(stderr, "]}\n");
  return 0;
}
