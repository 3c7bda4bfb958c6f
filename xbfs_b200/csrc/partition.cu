// 1D-partitioned single-source BFS: the per-rank device steps.
//
// No counterpart in the reference, which runs one source on one GPU
// (cudaSetDevice(gpu_id), bfs_gpu_update.cu:138). Here the vertex range is
// cut into P contiguous, 32-aligned slices, one per rank (one process per
// GPU); a rank holds the CSR rows of its slice (neighbour ids stay global)
// and the levels of its own vertices. A level is one of two exchanges,
// driven by the host (xbfs_b200/partition.py) between these kernels:
//  * top-down: every rank expands its own frontier vertices and marks their
//    neighbours in a byte-per-vertex candidate array over all V vertices
//    (xbfs_part_td_expand); the arrays are combined across ranks with a
//    MAX all-reduce (NCCL over NVLink); each rank then claims the unvisited
//    candidates of its slice (xbfs_part_claim);
//  * bottom-up: every rank packs its frontier into its word-aligned slice of
//    a V-bit bitmap (xbfs_part_frontier_bits), the slices are all-gathered,
//    and each rank's unvisited vertices probe their neighbours in the full
//    bitmap (xbfs_part_bottom_up); nothing else crosses ranks.
// Frontier statistics (n_f, m_f, n_u, m_u) are reduced per rank on the
// device and summed across ranks by the host, which takes the direction
// decision, so every rank takes the same steps in the same order.
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {
namespace part {

constexpr int kBlock = 256;

struct Part {
  int device = 0;
  long long V = 0, lo = 0, hi = 0, n = 0, E = 0;  // owned vertices [lo, hi), n = hi - lo, local edges
  int symmetric = 1;
  DevBuf beg;       // int64[n + 1], offsets into csr (rebased to 0)
  DevBuf csr;       // int32[E], global vertex ids
  DevBuf levels;    // int32[n]
  DevBuf vis;       // uint32[ceil(n/32)] owned visited bits
  DevBuf fq[2];     // int32[n] frontier lists (current / next)
  DevBuf ctr;       // unsigned long long[8]: next-frontier count, stats
  cudaStream_t stream = nullptr;
  int cur = 0;      // which fq holds the current frontier
  long long nf = 0; // its length
  ~Part() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }
};

// ctr layout
enum { kNext = 0, kNf = 1, kMf = 2, kNu = 3, kMu = 4 };

__global__ void k_reset(long long n, int* levels, uint32_t* vis, long long nwords) {
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock)
    levels[i] = -1;
  for (long long w = blockIdx.x * (long long)kBlock + threadIdx.x; w < nwords; w += (long long)gridDim.x * kBlock)
    vis[w] = 0u;
}

__global__ void k_seed(long long local, int* levels, uint32_t* vis, int* fq) {
  levels[local] = 0;
  vis[local >> 5] |= 1u << (local & 31);
  fq[0] = (int)local;
}

// Top-down: mark the neighbours of the owned frontier in the candidate
// bytes (one plain store each: every writer stores 1). One warp per
// frontier vertex, lanes over its neighbours (coalesced CSR reads).
__global__ void k_td_expand(const long long* __restrict__ beg, const int* __restrict__ csr,
                            const int* __restrict__ fq, long long nf, unsigned char* __restrict__ cand) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (kBlock / 32);
  for (long long i = blockIdx.x * (long long)(kBlock / 32) + (threadIdx.x >> 5); i < nf; i += warps) {
    const int u = fq[i];
    const long long e0 = beg[u], e1 = beg[u + 1];
    for (long long e = e0 + lane; e < e1; e += 32) cand[csr[e]] = 1;
  }
}

// Claim the unvisited candidates of the owned slice for level L+1 and queue
// them; the candidate bytes of the slice are cleared for the next exchange.
__global__ void k_claim(long long lo, long long n, const unsigned char* __restrict__ cand, int* levels,
                        uint32_t* vis, int* fq_next, unsigned long long* ctr, int next_level) {
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock) {
    if (!cand[lo + i]) continue;
    const uint32_t bit = 1u << (i & 31);
    if (vis[i >> 5] & bit) continue;
    atomicOr(&vis[i >> 5], bit);  // one thread per vertex: only it sets this bit
    levels[i] = next_level;
    const unsigned long long slot = atomicAdd(&ctr[kNext], 1ull);
    fq_next[slot] = (int)i;
  }
}

// Edges of the owned frontier (m_f).
__global__ void k_frontier_edges(const int* __restrict__ fq, long long nf, const long long* __restrict__ beg,
                                 unsigned long long* ctr) {
  unsigned long long m = 0;
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < nf; i += (long long)gridDim.x * kBlock) {
    const int v = fq[i];
    m += (unsigned long long)(beg[v + 1] - beg[v]);
  }
  m = warp_sum(m);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&ctr[kMf], m);
}

// Owned frontier -> its 32-aligned slice of the global frontier bitmap.
__global__ void k_frontier_bits(const int* __restrict__ fq, long long nf, uint32_t* slice) {
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < nf; i += (long long)gridDim.x * kBlock) {
    const int v = fq[i];
    atomicOr(&slice[v >> 5], 1u << (v & 31));
  }
}

// Bottom-up: every unvisited owned vertex looks for a neighbour in the
// global frontier bitmap (early exit); found -> level L+1, queued.
__global__ void k_bottom_up(long long n, const long long* __restrict__ beg, const int* __restrict__ csr,
                            const uint32_t* __restrict__ fbits, int* levels, uint32_t* vis, int* fq_next,
                            unsigned long long* ctr, int next_level) {
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock) {
    if (vis[i >> 5] & (1u << (i & 31))) continue;
    const long long e0 = beg[i], e1 = beg[i + 1];
    bool found = false;
    for (long long e = e0; e < e1 && !found; ++e) {
      const int u = csr[e];
      found = (fbits[u >> 5] >> (u & 31)) & 1u;
    }
    if (!found) continue;
    levels[i] = next_level;
    const unsigned long long slot = atomicAdd(&ctr[kNext], 1ull);
    fq_next[slot] = (int)i;
  }
}

// After a bottom-up step the new frontier's bits join the visited set (the
// step itself only reads the visited words, so its probes are not raced).
__global__ void k_mark_visited(const int* __restrict__ fq, long long nf, uint32_t* vis) {
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < nf; i += (long long)gridDim.x * kBlock) {
    const int v = fq[i];
    atomicOr(&vis[v >> 5], 1u << (v & 31));
  }
}

// Unvisited vertices of the slice and their edges (for the direction switch).
__global__ void k_unvisited(long long n, const long long* __restrict__ beg, const uint32_t* __restrict__ vis,
                            unsigned long long* ctr) {
  unsigned long long nu = 0, mu = 0;
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock) {
    if (vis[i >> 5] & (1u << (i & 31))) continue;
    const long long d = beg[i + 1] - beg[i];
    if (d == 0) continue;
    nu += 1;
    mu += (unsigned long long)d;
  }
  nu = warp_sum(nu);
  mu = warp_sum(mu);
  if ((threadIdx.x & 31) == 0) {
    if (nu) atomicAdd(&ctr[kNu], nu);
    if (mu) atomicAdd(&ctr[kMu], mu);
  }
}

static int grid_for(long long work) {
  return (int)std::max<long long>(1, std::min<long long>((work + kBlock - 1) / kBlock, 148 * 8));
}

}  // namespace part
}  // namespace xbfs

using namespace xbfs;
using xbfs::part::Part;

extern "C" {

xbfs_status xbfs_part_create(const int64_t* beg, const int32_t* csr, int64_t V, int64_t lo, int64_t hi,
                             int32_t symmetric, int32_t device, xbfs_part** out) {
  if (!beg || !out || V < 1 || lo < 0 || hi < lo || hi > V || ((lo % 32) != 0 && lo != hi))
    return set_error(XBFS_ERR_INVALID_ARG, "bad slice [%lld, %lld) of %lld vertices (lo must be 32-aligned)",
                     (long long)lo, (long long)hi, (long long)V);
  *out = nullptr;
  const int64_t n = hi - lo, E = beg[n] - beg[0];
  if (E < 0 || (E > 0 && !csr)) return set_error(XBFS_ERR_INVALID_ARG, "bad local CSR");
  if (V >= (1ll << 31)) return set_error(XBFS_ERR_UNSUPPORTED, "V must fit int32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(XBFS_ERR_NO_DEVICE, "no CUDA device available");
  }
  DeviceGuard dg(device);
  std::unique_ptr<Part> p(new Part());
  p->device = device;
  p->V = V;
  p->lo = lo;
  p->hi = hi;
  p->n = n;
  p->E = E;
  p->symmetric = symmetric ? 1 : 0;
  xbfs_status st;
  const size_t nwords = (size_t)(n + 31) / 32 + 1;
  if ((st = p->beg.ensure((size_t)(n + 1) * 8)) || (st = p->csr.ensure((size_t)E * 4 + 16)) ||
      (st = p->levels.ensure((size_t)n * 4 + 16)) || (st = p->vis.ensure(nwords * 4)) ||
      (st = p->fq[0].ensure((size_t)n * 4 + 16)) || (st = p->fq[1].ensure((size_t)n * 4 + 16)) ||
      (st = p->ctr.ensure(8 * 8)))
    return st;
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  // offsets rebased to the slice's first edge
  std::vector<long long> b((size_t)n + 1);
  for (int64_t i = 0; i <= n; ++i) b[(size_t)i] = beg[i] - beg[0];
  XBFS_CUDA_TRY(cudaMemcpy(p->beg.p, b.data(), (size_t)(n + 1) * 8, cudaMemcpyHostToDevice));
  if (E > 0) XBFS_CUDA_TRY(cudaMemcpy(p->csr.p, csr, (size_t)E * 4, cudaMemcpyHostToDevice));
  *out = (xbfs_part*)p.release();
  return XBFS_OK;
}

void xbfs_part_free(xbfs_part* h) { delete (Part*)h; }

xbfs_status xbfs_part_reset(xbfs_part* h, int32_t src) {
  Part* p = (Part*)h;
  if (!p || src < 0 || src >= p->V) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  const long long nwords = (p->n + 31) / 32 + 1;
  part::k_reset<<<part::grid_for(std::max<long long>(p->n, nwords)), part::kBlock, 0, p->stream>>>(
      p->n, p->levels.as<int>(), p->vis.as<uint32_t>(), nwords);
  p->cur = 0;
  p->nf = 0;
  if (src >= p->lo && src < p->hi) {
    part::k_seed<<<1, 1, 0, p->stream>>>(src - p->lo, p->levels.as<int>(), p->vis.as<uint32_t>(),
                                         p->fq[0].as<int>());
    p->nf = 1;
  }
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return XBFS_OK;
}

// Local statistics of the current frontier and the unvisited vertices:
// out[0] = n_f, out[1] = m_f, out[2] = n_u, out[3] = m_u (owned vertices).
xbfs_status xbfs_part_stats(xbfs_part* h, int64_t* out) {
  Part* p = (Part*)h;
  if (!p || !out) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  unsigned long long* ctr = p->ctr.as<unsigned long long>();
  XBFS_CUDA_TRY(cudaMemsetAsync(ctr + part::kMf, 0, 24, p->stream));
  part::k_unvisited<<<part::grid_for(p->n), part::kBlock, 0, p->stream>>>(p->n, p->beg.as<long long>(),
                                                                          p->vis.as<uint32_t>(), ctr);
  if (p->nf > 0)
    part::k_frontier_edges<<<part::grid_for(p->nf), part::kBlock, 0, p->stream>>>(p->fq[p->cur].as<int>(), p->nf,
                                                                                 p->beg.as<long long>(), ctr);
  XBFS_CUDA_TRY(cudaGetLastError());
  unsigned long long h_ctr[8];
  XBFS_CUDA_TRY(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, p->stream));
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  out[0] = p->nf;
  out[1] = (int64_t)h_ctr[part::kMf];
  out[2] = (int64_t)h_ctr[part::kNu];
  out[3] = (int64_t)h_ctr[part::kMu];
  return XBFS_OK;
}

// Top-down, first half: mark the neighbours of the owned frontier in
// cand (device, V bytes, zero outside what earlier claims cleared).
xbfs_status xbfs_part_td_expand(xbfs_part* h, uint8_t* cand) {
  Part* p = (Part*)h;
  if (!p || !cand) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  if (p->nf > 0) {
    const long long warps = p->nf;
    part::k_td_expand<<<part::grid_for(warps * 32), part::kBlock, 0, p->stream>>>(
        p->beg.as<long long>(), p->csr.as<int>(), p->fq[p->cur].as<int>(), p->nf, cand);
    XBFS_CUDA_TRY(cudaGetLastError());
  }
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return XBFS_OK;
}

static xbfs_status finish_step(Part* p) {
  unsigned long long h_ctr[8];
  XBFS_CUDA_TRY(cudaMemcpyAsync(h_ctr, p->ctr.p, sizeof(h_ctr), cudaMemcpyDeviceToHost, p->stream));
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  p->cur ^= 1;
  p->nf = (long long)h_ctr[part::kNext];
  return XBFS_OK;
}

// Top-down, second half: cand holds every rank's marks (after the MAX
// all-reduce); the unvisited marked vertices of the slice get next_level and
// form the next owned frontier. All V candidate bytes are cleared afterwards,
// ready for the next top-down level.
xbfs_status xbfs_part_claim(xbfs_part* h, uint8_t* cand, int32_t next_level) {
  Part* p = (Part*)h;
  if (!p || !cand) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  XBFS_CUDA_TRY(cudaMemsetAsync(p->ctr.p, 0, 8, p->stream));
  part::k_claim<<<part::grid_for(p->n), part::kBlock, 0, p->stream>>>(
      p->lo, p->n, cand, p->levels.as<int>(), p->vis.as<uint32_t>(), p->fq[p->cur ^ 1].as<int>(),
      p->ctr.as<unsigned long long>(), next_level);
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaMemsetAsync(cand, 0, (size_t)p->V, p->stream));
  return finish_step(p);
}

// Bottom-up, first half: the owned frontier into this rank's slice of the
// global bitmap (slice = words [lo/32, lo/32 + nwords_slice), zeroed here).
xbfs_status xbfs_part_frontier_bits(xbfs_part* h, uint32_t* slice, int64_t nwords_slice) {
  Part* p = (Part*)h;
  if (!p || !slice || nwords_slice * 32 < p->n) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  XBFS_CUDA_TRY(cudaMemsetAsync(slice, 0, (size_t)nwords_slice * 4, p->stream));
  if (p->nf > 0) {
    part::k_frontier_bits<<<part::grid_for(p->nf), part::kBlock, 0, p->stream>>>(p->fq[p->cur].as<int>(), p->nf,
                                                                                slice);
    XBFS_CUDA_TRY(cudaGetLastError());
  }
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return XBFS_OK;
}

// Bottom-up, second half: fbits is the whole V-bit frontier bitmap (after
// the all-gather). Needs a symmetric graph.
xbfs_status xbfs_part_bottom_up(xbfs_part* h, const uint32_t* fbits, int32_t next_level) {
  Part* p = (Part*)h;
  if (!p || !fbits) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  if (!p->symmetric) return set_error(XBFS_ERR_UNSUPPORTED, "bottom-up needs a symmetric graph");
  DeviceGuard dg(p->device);
  XBFS_CUDA_TRY(cudaMemsetAsync(p->ctr.p, 0, 8, p->stream));
  unsigned long long* ctr = p->ctr.as<unsigned long long>();
  part::k_bottom_up<<<part::grid_for(p->n), part::kBlock, 0, p->stream>>>(
      p->n, p->beg.as<long long>(), p->csr.as<int>(), fbits, p->levels.as<int>(), p->vis.as<uint32_t>(),
      p->fq[p->cur ^ 1].as<int>(), ctr, next_level);
  XBFS_CUDA_TRY(cudaGetLastError());
  unsigned long long h_ctr[8];
  XBFS_CUDA_TRY(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, p->stream));
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  const long long nn = (long long)h_ctr[part::kNext];
  if (nn > 0) {
    part::k_mark_visited<<<part::grid_for(nn), part::kBlock, 0, p->stream>>>(p->fq[p->cur ^ 1].as<int>(), nn,
                                                                            p->vis.as<uint32_t>());
    XBFS_CUDA_TRY(cudaGetLastError());
  }
  return finish_step(p);
}

// Levels of the owned vertices (n int32, host or device memory).
xbfs_status xbfs_part_levels(xbfs_part* h, int32_t* out) {
  Part* p = (Part*)h;
  if (!p || !out) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(p->device);
  XBFS_CUDA_TRY(cudaMemcpyAsync(out, p->levels.p, (size_t)p->n * 4, cudaMemcpyDefault, p->stream));
  XBFS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return XBFS_OK;
}

}  // extern "C"
