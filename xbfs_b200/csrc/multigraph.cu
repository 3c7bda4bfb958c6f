// Multi-graph BFS: many graphs of uneven size, one source each, in one
// persistent launch, replayed from a CUDA graph.
//
// No counterpart in the reference (one graph per process). B200 design:
//  * All graphs live in one arena (offsets per graph); a work list sorted by
//    edge count (largest first) is consumed by CTAs through an atomic ticket,
//    so the big graphs start first and the small ones fill the gaps
//    (longest-processing-time order).
//  * One CTA owns one graph for its whole traversal: visited / current /
//    next frontier bitmaps sit in shared memory when V fits (up to 2^18
//    vertices at 3 x 32 KB), so every status probe is a shared-memory access
//    and levels are separated by __syncthreads instead of grid barriers.
//    Larger graphs use a per-CTA slice of global scratch for the bitmaps.
//  * Each level picks top-down or bottom-up from CTA-local counts. Top-down
//    expands frontier vertices of degree <= `thread_max` one per lane and
//    heavier ones warp-cooperatively; bottom-up gives each lane one unvisited
//    vertex and stops at the first parent.
//  * The CTA shape (threads per CTA), the thread/warp degree threshold and the
//    direction threshold are picked by a small autotuner (xbfs_multi_tune).
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

namespace mg {

struct Desc {
  long long b_off;   // offset of the graph's V+1 local offsets in the beg arena
  long long e_off;   // offset of its neighbours in the csr arena
  long long v_off;   // offset of its levels in the output arena
  int V;
  int src;
  long long E;
};

struct Params {
  const long long* beg;   // local offsets, per graph
  const int* csr;         // local vertex ids
  const Desc* desc;
  const int* order;       // graph indices, largest first
  int n;
  int* levels;            // concatenated outputs
  unsigned* ticket;
  uint32_t* gscratch;     // per-CTA global bitmaps for graphs too large for shared memory
  long long gscratch_words;  // words per CTA (3 bitmaps)
  int smem_words;         // words per bitmap available in shared memory
  int thread_max;         // top-down: degree <= thread_max expanded by one lane
  float alpha;            // bottom-up when m_f * alpha > m_u
  unsigned long long* edges;  // per graph: sum of degrees of reached vertices
};

template <int BLOCK>
__device__ __forceinline__ long long block_sum_ll(long long v, long long* red) {
  return block_sum<BLOCK, long long>(v, red);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_multi(Params p) {
  extern __shared__ __align__(16) uint32_t sbits[];
  __shared__ long long red[BLOCK / 32 + 1];
  __shared__ int s_g;
  __shared__ unsigned long long s_nf, s_mf, s_mdone;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  for (;;) {
    if (threadIdx.x == 0) s_g = (int)atomicAdd(p.ticket, 1u);
    __syncthreads();
    const int gi = s_g;
    if (gi >= p.n) break;
    const Desc d = p.desc[p.order[gi]];
    const int V = d.V;
    const long long* beg = p.beg + d.b_off;
    const int* csr = p.csr + d.e_off;
    int* lv = p.levels + d.v_off;
    const int nw = (V + 31) / 32;
    // volatile: on the global-scratch path a plain load could hit an L1 line
    // made stale by another thread's atomic (atomics update L2 only)
    volatile uint32_t *vis, *cur, *nxt;
    if (nw <= p.smem_words) {
      vis = sbits;
      cur = sbits + p.smem_words;
      nxt = sbits + 2 * p.smem_words;
    } else {
      uint32_t* base = p.gscratch + (size_t)blockIdx.x * p.gscratch_words;
      vis = base;
      cur = base + nw;
      nxt = base + 2 * (size_t)nw;
    }
    for (int w = threadIdx.x; w < nw; w += BLOCK) {
      // bits past V count as visited so they are never searched
      const uint32_t tail = (w == nw - 1 && (V & 31)) ? ~((1u << (V & 31)) - 1u) : 0u;
      vis[w] = tail;
      cur[w] = 0u;
      nxt[w] = 0u;
    }
    __syncthreads();
    const int src = d.src;
    long long m_u = d.E;
    unsigned long long reached_deg = 0;
    if (threadIdx.x == 0) {
      vis[src >> 5] |= 1u << (src & 31);
      cur[src >> 5] |= 1u << (src & 31);
      lv[src] = 0;
      const long long dg = beg[src + 1] - beg[src];
      s_nf = 1;
      s_mf = (unsigned long long)dg;
    }
    __syncthreads();
    long long n_f = (long long)s_nf, m_f = (long long)s_mf;
    reached_deg = (unsigned long long)m_f;
    m_u -= m_f;
    int L = 0;
    while (n_f > 0) {
      const bool bu = (double)m_f * (double)p.alpha > (double)m_u;
      long long my_n = 0, my_m = 0;
      if (!bu) {
        // top-down: warps take frontier words; light vertices one per lane,
        // heavy ones warp-cooperatively
        for (int w = wid; w < nw; w += NW) {
          const uint32_t bits = cur[w];
          if (!bits) continue;
          const int u_l = w * 32 + lane;
          const bool mine = (bits >> lane) & 1u;
          long long e0 = 0, e1 = 0;
          if (mine) {
            e0 = __ldg(beg + u_l);
            e1 = __ldg(beg + u_l + 1);
          }
          const bool light = mine && (e1 - e0) <= p.thread_max;
          if (light) {
            for (long long e = e0; e < e1; ++e) {
              const int v = __ldg(csr + e);
              const uint32_t bit = 1u << (v & 31);
              if (vis[v >> 5] & bit) continue;
              if (atomicOr((uint32_t*)&vis[v >> 5], bit) & bit) continue;
              atomicOr((uint32_t*)&nxt[v >> 5], bit);
              lv[v] = L + 1;
              my_n += 1;
              my_m += __ldg(beg + v + 1) - __ldg(beg + v);
            }
          }
          unsigned heavy = __ballot_sync(0xffffffffu, mine && !light);
          while (heavy) {
            const int hl = __ffs(heavy) - 1;
            heavy &= heavy - 1;
            const long long h0 = __shfl_sync(0xffffffffu, e0, hl), h1 = __shfl_sync(0xffffffffu, e1, hl);
            for (long long e = h0 + lane; e < h1; e += 32) {
              const int v = __ldg(csr + e);
              const uint32_t bit = 1u << (v & 31);
              if (vis[v >> 5] & bit) continue;
              if (atomicOr((uint32_t*)&vis[v >> 5], bit) & bit) continue;
              atomicOr((uint32_t*)&nxt[v >> 5], bit);
              lv[v] = L + 1;
              my_n += 1;
              my_m += __ldg(beg + v + 1) - __ldg(beg + v);
            }
          }
        }
      } else {
        // bottom-up: lanes own unvisited vertices of a word
        for (int w = wid; w < nw; w += NW) {
          const uint32_t un = ~vis[w];
          if (!un) continue;
          const int v = w * 32 + lane;
          if ((un >> lane) & 1u) {
            const long long e0 = __ldg(beg + v), e1 = __ldg(beg + v + 1);
            for (long long e = e0; e < e1; ++e) {
              const int u = __ldg(csr + e);
              if ((cur[u >> 5] >> (u & 31)) & 1u) {
                lv[v] = L + 1;
                atomicOr((uint32_t*)&nxt[w], 1u << lane);
                my_n += 1;
                my_m += e1 - e0;
                break;
              }
            }
          }
        }
        __syncthreads();
        // newly found vertices become visited only after the sweep, so every
        // probe above saw the level-L frontier only
        for (int w = threadIdx.x; w < nw; w += BLOCK) vis[w] |= nxt[w];
      }
      const long long tn = block_sum_ll<BLOCK>(my_n, red);
      const long long tm = block_sum_ll<BLOCK>(my_m, red);
      // next frontier becomes current
      for (int w = threadIdx.x; w < nw; w += BLOCK) {
        cur[w] = nxt[w];
        nxt[w] = 0u;
      }
      __syncthreads();
      n_f = tn;
      m_f = tm;
      m_u -= tm;
      reached_deg += (unsigned long long)tm;
      ++L;
    }
    if (threadIdx.x == 0) p.edges[p.order[gi]] = reached_deg;
    __syncthreads();
  }
}

}  // namespace mg

struct MultiGraph {
  int device = 0;
  int n = 0;
  long long total_V = 0, total_E = 0;
  int maxV = 0;
  DevBuf beg, csr, desc, order, ticket, edges, gscratch, srcs_dev, levels_tmp;
  std::vector<mg::Desc> hdesc;
  std::vector<int> horder;
  PinnedBuf srcs_pin;
  cudaStream_t stream = nullptr;
  // tuned configuration
  int block = 512;
  int thread_max = 32;
  float alpha = 4.f;
  // captured replay
  cudaGraphExec_t exec = nullptr;
  int* exec_levels = nullptr;
  int exec_block = 0, exec_thread_max = 0;
  float exec_alpha = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~MultiGraph() {
    DeviceGuard dg(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) cudaStreamDestroy(stream);
  }
};

static int smem_words_for(int block) {
  (void)block;
  return 8192;  // 3 x 32 KB: graphs up to 262,144 vertices keep their bitmaps on chip
}

static xbfs_status enqueue_multi(MultiGraph* m, int* d_levels, int block, int thread_max, float alpha) {
  cudaStream_t s = m->stream;
  XBFS_CUDA_TRY(cudaMemsetAsync(d_levels, 0xff, (size_t)m->total_V * 4, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(m->ticket.p, 0, 16, s));
  // the per-graph sources are patched into the descriptors on the device
  mg::Params p;
  p.beg = m->beg.as<long long>();
  p.csr = m->csr.as<int>();
  p.desc = m->desc.as<mg::Desc>();
  p.order = m->order.as<int>();
  p.n = m->n;
  p.levels = d_levels;
  p.ticket = m->ticket.as<unsigned>();
  p.gscratch = m->gscratch.as<uint32_t>();
  p.gscratch_words = 3ll * ((m->maxV + 31) / 32);
  p.smem_words = smem_words_for(block);
  p.thread_max = thread_max;
  p.alpha = alpha;
  p.edges = m->edges.as<unsigned long long>();
  const size_t smem = (size_t)3 * p.smem_words * 4;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const void* kfn;
  switch (block) {
    case 256: kfn = (const void*)mg::k_multi<256>; break;
    case 1024: kfn = (const void*)mg::k_multi<1024>; break;
    default: kfn = (const void*)mg::k_multi<512>; block = 512; break;
  }
  XBFS_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  XBFS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, block, smem));
  if (per_sm < 1) return set_error(XBFS_ERR_INTERNAL, "multi-graph kernel cannot be resident");
  const int grid = std::min(nsm * per_sm, m->n);
  void* args[] = {&p};
  XBFS_CUDA_TRY(cudaLaunchKernel(kfn, dim3(grid), dim3(block), args, smem, s));
  return XBFS_OK;
}

__global__ void k_mg_set_sources(mg::Desc* desc, const int* srcs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) desc[i].src = srcs[i];
}

// One call: copy sources, patch descriptors, reset outputs, run. Captured into
// a CUDA graph on first use and replayed while the output pointer and the
// configuration stay the same.
static xbfs_status run_multi(MultiGraph* m, int* d_levels, int block, int thread_max, float alpha, float* ms_out) {
  cudaStream_t s = m->stream;
  const bool reuse = m->exec && m->exec_levels == d_levels && m->exec_block == block &&
                     m->exec_thread_max == thread_max && m->exec_alpha == alpha;
  if (!reuse) {
    if (m->exec) {
      cudaGraphExecDestroy(m->exec);
      m->exec = nullptr;
    }
    cudaGraph_t graph;
    XBFS_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    xbfs_status st = XBFS_OK;
    {
      cudaError_t e = cudaMemcpyAsync(m->srcs_dev.p, m->srcs_pin.p, sizeof(int) * m->n, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) {
        k_mg_set_sources<<<(m->n + 255) / 256, 256, 0, s>>>(m->desc.as<mg::Desc>(), m->srcs_dev.as<int>(), m->n);
        e = cudaGetLastError();
      }
      if (e != cudaSuccess) st = set_error(XBFS_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
      if (!st) st = enqueue_multi(m, d_levels, block, thread_max, alpha);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st) {
      if (ce == cudaSuccess) cudaGraphDestroy(graph);
      return st;
    }
    XBFS_CUDA_TRY(ce);
    cudaError_t ie = cudaGraphInstantiate(&m->exec, graph, 0);
    cudaGraphDestroy(graph);
    XBFS_CUDA_TRY(ie);
    m->exec_levels = d_levels;
    m->exec_block = block;
    m->exec_thread_max = thread_max;
    m->exec_alpha = alpha;
  }
  XBFS_CUDA_TRY(cudaEventRecord(m->e0, s));
  XBFS_CUDA_TRY(cudaGraphLaunch(m->exec, s));
  XBFS_CUDA_TRY(cudaEventRecord(m->e1, s));
  XBFS_CUDA_TRY(cudaEventSynchronize(m->e1));
  float ms = 0;
  XBFS_CUDA_TRY(cudaEventElapsedTime(&ms, m->e0, m->e1));
  if (ms_out) *ms_out = ms;
  return XBFS_OK;
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_multi_create(xbfs_graph* const* graphs, int32_t n, int32_t device, xbfs_multi** out) {
  if (!graphs || n <= 0 || !out) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  std::unique_ptr<MultiGraph> m(new MultiGraph());
  m->device = device;
  m->n = n;
  DeviceGuard dg(device);
  m->hdesc.resize(n);
  long long vb = 0, bb = 0, eb = 0;
  for (int i = 0; i < n; ++i) {
    const Graph* g = (const Graph*)graphs[i];
    if (!g) return set_error(XBFS_ERR_INVALID_ARG, "graph %d is NULL", i);
    if (g->device != device) return set_error(XBFS_ERR_INVALID_ARG, "graph %d lives on device %d", i, g->device);
    if (!g->symmetric) return set_error(XBFS_ERR_UNSUPPORTED, "graph %d is not symmetric", i);
    if (g->V > INT32_MAX - 64) return set_error(XBFS_ERR_UNSUPPORTED, "graph %d too large", i);
    m->hdesc[i] = mg::Desc{bb, eb, vb, (int)g->V, 0, g->E};
    vb += g->V;
    bb += g->V + 1;
    eb += g->E;
    m->maxV = std::max<int>(m->maxV, (int)g->V);
  }
  m->total_V = vb;
  m->total_E = eb;
  xbfs_status st;
  if ((st = m->beg.ensure((size_t)bb * 8)) || (st = m->csr.ensure((size_t)eb * 4 + 64)) ||
      (st = m->desc.ensure(sizeof(mg::Desc) * n)) || (st = m->order.ensure(sizeof(int) * n)) ||
      (st = m->ticket.ensure(16)) || (st = m->edges.ensure(8 * (size_t)n)) || (st = m->srcs_dev.ensure(4 * (size_t)n)) ||
      (st = m->srcs_pin.ensure(4 * (size_t)n)))
    return st;
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  XBFS_CUDA_TRY(cudaEventCreate(&m->e0));
  XBFS_CUDA_TRY(cudaEventCreate(&m->e1));
  for (int i = 0; i < n; ++i) {
    const Graph* g = (const Graph*)graphs[i];
    XBFS_CUDA_TRY(cudaMemcpyAsync(m->beg.as<long long>() + m->hdesc[i].b_off, g->beg.p, (size_t)(g->V + 1) * 8,
                                  cudaMemcpyDeviceToDevice, m->stream));
    if (g->E > 0)
      XBFS_CUDA_TRY(cudaMemcpyAsync(m->csr.as<int>() + m->hdesc[i].e_off, g->csr.p, (size_t)g->E * 4,
                                    cudaMemcpyDeviceToDevice, m->stream));
  }
  m->horder.resize(n);
  std::iota(m->horder.begin(), m->horder.end(), 0);
  std::stable_sort(m->horder.begin(), m->horder.end(), [&](int a, int b) {
    return m->hdesc[a].E + m->hdesc[a].V > m->hdesc[b].E + m->hdesc[b].V;
  });
  XBFS_CUDA_TRY(cudaMemcpyAsync(m->desc.p, m->hdesc.data(), sizeof(mg::Desc) * n, cudaMemcpyHostToDevice, m->stream));
  XBFS_CUDA_TRY(cudaMemcpyAsync(m->order.p, m->horder.data(), sizeof(int) * n, cudaMemcpyHostToDevice, m->stream));
  // global bitmap scratch only for graphs that do not fit the on-chip bitmaps
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const long long words = 3ll * ((m->maxV + 31) / 32);
  if ((m->maxV + 31) / 32 > smem_words_for(256)) {
    if ((st = m->gscratch.ensure((size_t)words * 4 * nsm * 8))) return st;
  } else {
    if ((st = m->gscratch.ensure(16))) return st;
  }
  XBFS_CUDA_TRY(cudaStreamSynchronize(m->stream));
  *out = (xbfs_multi*)m.release();
  return XBFS_OK;
}

xbfs_status xbfs_multi_info(const xbfs_multi* mh, int64_t* total_V, int64_t* total_E, int64_t* level_offsets) {
  const MultiGraph* m = (const MultiGraph*)mh;
  if (!m) return set_error(XBFS_ERR_INVALID_ARG, "NULL handle");
  if (total_V) *total_V = m->total_V;
  if (total_E) *total_E = m->total_E;
  if (level_offsets)
    for (int i = 0; i < m->n; ++i) level_offsets[i] = m->hdesc[i].v_off;
  return XBFS_OK;
}

xbfs_status xbfs_multi_bfs(xbfs_multi* mh, const int32_t* srcs, int32_t* levels, const xbfs_opts* opts,
                           xbfs_stats* stats) {
  MultiGraph* m = (MultiGraph*)mh;
  if (!m || !srcs || !levels) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  (void)opts;
  for (int i = 0; i < m->n; ++i)
    if (srcs[i] < 0 || srcs[i] >= m->hdesc[i].V) return set_error(XBFS_ERR_INVALID_ARG, "source of graph %d out of range", i);
  DeviceGuard dg(m->device);
  const auto t0 = std::chrono::steady_clock::now();
  memcpy(m->srcs_pin.p, srcs, sizeof(int) * m->n);
  const bool dev = is_device_pointer(levels);
  int* d_levels = levels;
  xbfs_status st;
  if (!dev) {
    if ((st = m->levels_tmp.ensure((size_t)m->total_V * 4))) return st;
    d_levels = m->levels_tmp.as<int>();
  }
  float ms = 0;
  if ((st = run_multi(m, d_levels, m->block, m->thread_max, m->alpha, &ms))) return st;
  if (!dev) XBFS_CUDA_TRY(cudaMemcpy(levels, d_levels, (size_t)m->total_V * 4, cudaMemcpyDeviceToHost));
  if (stats) {
    std::vector<unsigned long long> e(m->n);
    XBFS_CUDA_TRY(cudaMemcpy(e.data(), m->edges.p, 8 * (size_t)m->n, cudaMemcpyDeviceToHost));
    memset(stats, 0, sizeof(*stats));
    stats->struct_size = (int32_t)sizeof(xbfs_stats);
    unsigned long long tot = 0;
    for (auto x : e) tot += x / 2;
    stats->edges_mc = (int64_t)tot;
    stats->device_ms = ms;
    stats->kernel_ms = ms;
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return XBFS_OK;
}

// Autotuner: times every (threads per CTA, thread/warp degree threshold,
// direction threshold) candidate on the caller's sources and keeps the
// fastest. Returns the chosen configuration.
xbfs_status xbfs_multi_tune(xbfs_multi* mh, const int32_t* srcs, int32_t reps, int32_t* block_out,
                            int32_t* thread_max_out, float* alpha_out, float* best_ms_out) {
  MultiGraph* m = (MultiGraph*)mh;
  if (!m || !srcs) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(m->device);
  memcpy(m->srcs_pin.p, srcs, sizeof(int) * m->n);
  xbfs_status st;
  if ((st = m->levels_tmp.ensure((size_t)m->total_V * 4))) return st;
  const int blocks[] = {256, 512, 1024};
  const int tms[] = {8, 32, 128};
  const float alphas[] = {2.f, 4.f, 14.f};
  float best = 1e30f;
  int bb = m->block, bt = m->thread_max;
  float ba = m->alpha;
  if (reps < 1) reps = 1;
  for (int b : blocks)
    for (int t : tms)
      for (float a : alphas) {
        float tot = 0;
        for (int r = 0; r < reps + 1; ++r) {
          float ms = 0;
          if ((st = run_multi(m, m->levels_tmp.as<int>(), b, t, a, &ms))) return st;
          if (r > 0) tot += ms;  // first run builds the graph
        }
        tot /= reps;
        if (tot < best) {
          best = tot;
          bb = b;
          bt = t;
          ba = a;
        }
      }
  m->block = bb;
  m->thread_max = bt;
  m->alpha = ba;
  if (block_out) *block_out = bb;
  if (thread_max_out) *thread_max_out = bt;
  if (alpha_out) *alpha_out = ba;
  if (best_ms_out) *best_ms_out = best;
  return XBFS_OK;
}

xbfs_status xbfs_multi_set_config(xbfs_multi* mh, int32_t block, int32_t thread_max, float alpha) {
  MultiGraph* m = (MultiGraph*)mh;
  if (!m) return set_error(XBFS_ERR_INVALID_ARG, "NULL handle");
  if (block != 256 && block != 512 && block != 1024) return set_error(XBFS_ERR_INVALID_ARG, "block must be 256/512/1024");
  if (thread_max < 0 || !(alpha > 0)) return set_error(XBFS_ERR_INVALID_ARG, "bad threshold");
  m->block = block;
  m->thread_max = thread_max;
  m->alpha = alpha;
  return XBFS_OK;
}

void xbfs_multi_free(xbfs_multi* mh) { delete (MultiGraph*)mh; }

}  // extern "C"
