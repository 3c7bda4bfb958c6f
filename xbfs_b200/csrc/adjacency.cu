// Order of the neighbours within each vertex's CSR segment.
//
// Levels never depend on the order, but bottom-up steps do: an unvisited
// vertex scans its neighbours until one is in the frontier, and on power-law
// graphs the frontiers of the large bottom-up levels hold the hubs. With each
// segment sorted by descending neighbour degree, most unvisited vertices find
// a parent in their first probe. The reference keeps the file order; this is
// an optional preparation step on a loaded graph (off the traversal path).
//
// Method: one 64-bit key per CSR entry, (source vertex << 32 | rank of the
// neighbour), and a stable device radix sort of (key, neighbour) pairs. The
// rank is ~degree (descending degree, ties in the previous order) or the
// neighbour id itself (ascending ids, the order the generators write).
#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {
namespace {

// One warp per vertex (grid-stride), lanes over its segment.
__global__ void k_adj_keys(const long long* __restrict__ beg, const int* __restrict__ csr, long long V,
                           int order, unsigned long long* __restrict__ keys) {
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (long long u = warp; u < V; u += nwarps) {
    const long long b0 = beg[u], b1 = beg[u + 1];
    for (long long e = b0 + lane; e < b1; e += 32) {
      const int v = csr[e];
      uint32_t rank;
      if (order == XBFS_ADJ_DEGREE_DESC) {
        const long long d = beg[v + 1] - beg[v];
        rank = ~(uint32_t)(d > 0xffffffffll ? 0xffffffffll : d);
      } else {
        rank = (uint32_t)v;
      }
      keys[e] = ((unsigned long long)u << 32) | rank;
    }
  }
}

// Head record of every vertex (one thread each): its first three neighbours
// in CSR order, -1 past its degree, and its degree (saturated at
// kHeadDegSat). A bottom-up probe reads the 16-byte record, coalesced across
// the 32 vertices of a bitmap word, instead of the vertex's CSR offsets and
// then the first sector of its segment.
__global__ void k_head(const long long* __restrict__ beg, const int* __restrict__ csr, long long V,
                       int4* __restrict__ head) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    const long long b0 = beg[v], d = beg[v + 1] - b0;
    int4 h;
    h.x = d > 0 ? csr[b0] : -1;
    h.y = d > 1 ? csr[b0 + 1] : -1;
    h.z = d > 2 ? csr[b0 + 2] : -1;
    h.w = d < kHeadDegSat ? (int)d : kHeadDegSat;
    head[v] = h;
  }
}

}  // namespace

xbfs_status graph_build_head(Graph* g) {
  DeviceGuard dg(g->device);
  xbfs_status st = g->head.ensure((size_t)g->V * sizeof(int4));
  if (st) return st;
  int nsm = 0;
  XBFS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device));
  k_head<<<nsm * 8, 256, 0, g->stream>>>(g->beg.as<long long>(), g->csr.as<int>(), g->V, g->head.as<int4>());
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return XBFS_OK;
}

xbfs_status graph_sort_adjacency(Graph* g, int order) {
  if (!g) return set_error(XBFS_ERR_INVALID_ARG, "graph is NULL");
  if (order != XBFS_ADJ_ID_ASC && order != XBFS_ADJ_DEGREE_DESC)
    return set_error(XBFS_ERR_INVALID_ARG, "bad adjacency order %d", order);
  if (g->E == 0) return XBFS_OK;
  DeviceGuard dg(g->device);
  const size_t E = (size_t)g->E;
  cudaStream_t s = g->stream;
  DevBuf k0, k1, v1, tmp;
  xbfs_status st;
  if ((st = k0.ensure(E * 8)) || (st = k1.ensure(E * 8)) || (st = v1.ensure(E * 4))) return st;
  int nsm = 0;
  XBFS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device));
  k_adj_keys<<<nsm * 8, 256, 0, s>>>(g->beg.as<long long>(), g->csr.as<int>(), g->V, order,
                                     k0.as<unsigned long long>());
  XBFS_CUDA_TRY(cudaGetLastError());
  int vbits = 1;
  while (vbits < 31 && (1ll << vbits) < g->V) ++vbits;
  cub::DoubleBuffer<unsigned long long> keys(k0.as<unsigned long long>(), k1.as<unsigned long long>());
  cub::DoubleBuffer<int> vals(g->csr.as<int>(), v1.as<int>());
  size_t tmp_bytes = 0;
  XBFS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, vals, (int64_t)E, 0, 32 + vbits, s));
  if ((st = tmp.ensure(tmp_bytes))) return st;
  XBFS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys, vals, (int64_t)E, 0, 32 + vbits, s));
  if (vals.Current() != g->csr.as<int>())
    XBFS_CUDA_TRY(cudaMemcpyAsync(g->csr.p, vals.Current(), E * 4, cudaMemcpyDeviceToDevice, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  g->adj_order = order;
  return graph_build_head(g);
}

}  // namespace xbfs

using namespace xbfs;

extern "C" xbfs_status xbfs_graph_sort_adjacency(xbfs_graph* g, int32_t order) {
  return graph_sort_adjacency((Graph*)g, order);
}
