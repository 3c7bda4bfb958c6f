// Internal host-side structures shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <vector>

#include "xbfs.h"

namespace xbfs {

xbfs_status set_error(xbfs_status st, const char* fmt, ...);

// A device allocation freed on destruction (the device must be current).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  xbfs_status ensure(size_t n);  // grow-only
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  xbfs_status ensure(size_t n);
};

struct LevelRecDev;  // device-side per-level record (bfs.cu)

// Scratch for single-source traversal, sized by V (allocated on first use).
struct SsWorkspace {
  bool ready = false;
  int64_t V = 0;
  size_t nwords = 0;       // bitmap words (32 vertices each), padded
  DevBuf levels_tmp;       // int32[V] when the caller passes host memory
  DevBuf parents_tmp;      // int32[V]
  DevBuf bits;             // vis + 4 frontier bitmaps, contiguous
  DevBuf qids[2][3];       // per parity, per bin: vertex ids
  DevBuf qeb[2][3];        // per parity, per bin: edge offsets (uint32)
  DevBuf qbg[2][3];        // per parity, per bin: CSR offsets (int64)
  size_t qcap[3] = {0, 0, 0};
  DevBuf heavy_ids, heavy_eb, heavy_bg;  // heavy vertices deferred by a fused sweep
  DevBuf ulist;            // bottom-up lists of unvisited vertices
  DevBuf ctl;              // control block
  DevBuf rs;               // loop state of a stepped traversal
  DevBuf snap;             // snapshot of the whole traversal state (stepped mode)
  DevBuf snap2;            // second snapshot: the state one strategy left after a level
  DevBuf hist;             // per-level records
  int hist_cap = 0;
  DevBuf forced;           // int8 per-level strategies
  int forced_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr;
  // pipelined traversals (xbfs_bfs_many): a second level buffer, the stream
  // that copies finished level arrays out, and the events between the two
  DevBuf levels_tmp2;
  DevBuf ctl_log;          // Ctl of every traversal of one call
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_done[2] = {nullptr, nullptr}, ev_copied[2] = {nullptr, nullptr};
  int grid = 0, block = 0;
  int last_levels = 0;
  std::vector<xbfs_level_trace> trace;
};

struct Graph {
  int device = 0;
  int64_t V = 0, E = 0;
  int64_t max_degree = 0;
  int64_t n_isolated = 0;
  bool symmetric = true;         // edge multiset symmetric: bottom-up steps allowed
  int adj_order = -1;            // XBFS_ADJ_* after xbfs_graph_sort_adjacency, -1 = as loaded
  int64_t cnt_deg_gt[16] = {0};  // vertices with degree > 2^k, k = 0..15
  DevBuf beg;                    // int64[V+1]
  DevBuf csr;                    // int32[E] (+16 bytes tail padding)
  DevBuf iso;                    // uint32 bitmap: isolated vertices + tail bits
  DevBuf head;                   // int4[V]: first three neighbours (-1 past the degree), degree
  cudaStream_t stream = nullptr;
  SsWorkspace ss;
  ~Graph();
};

// RAII device guard
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// graph.cpp
xbfs_status graph_finish_upload(Graph* g);  // degree stats, iso bitmap, stream, head records
// adjacency.cu: (re)writes g->head from the current neighbour order
xbfs_status graph_build_head(Graph* g);
// Degree field of a head record saturates here; the CSR offsets give the rest.
constexpr int kHeadDegSat = 0x7fffffff;
xbfs_status graph_from_host(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E,
                            int device, bool validate, Graph** out);
xbfs_status validate_csr(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E);
bool is_device_pointer(const void* p);

// gen.cu (device builders)
xbfs_status gen_rmat_device(int scale, int ef, uint64_t seed, double a, double b, double c,
                            int device, Graph** out);
xbfs_status gen_er_device(int64_t n, double mean_degree, uint64_t seed, int device, Graph** out);
xbfs_status gen_grid_device(int W, int H, int device, Graph** out);

// bfs.cu
xbfs_status bfs_single(Graph* g, int32_t src, int32_t* levels, int32_t* parents,
                       const xbfs_opts* opts, xbfs_stats* stats);

}  // namespace xbfs
