// Synthetic graph generators: R-MAT (Graph500 Kronecker parameters), 2D
// 4-neighbour grid, Erdos-Renyi G(n, m).
//
// There is no counterpart in the reference, which only reads pre-converted
// datasets (CSRGenerator/tuple_text_to_bin.cpp). Both the host build (used by
// CPU-only tests) and the device build (used for scale-23 inputs, where host
// sorting would dominate the run) draw every random number from a
// counter-based hash of (seed, tuple index, level), so they produce the same
// CSR bit for bit. Output: symmetric, self-loops removed, duplicates removed,
// adjacency sorted ascending, int64 offsets / int32 neighbours.
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <memory>
#include <parallel/algorithm>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct RmatParams {
  int scale;
  uint64_t base;   // per-graph hash base
  uint64_t t_ab;   // P(row bit = 0) = a + b, as a 32-bit threshold
  uint64_t t_a;    // P(col bit = 0 | row bit = 0) = a / (a + b)
  uint64_t t_c;    // P(col bit = 0 | row bit = 1) = c / (c + d)
  uint64_t pm[3];  // odd multipliers of the vertex scramble
  uint64_t pa[3];  // addends of the vertex scramble
};

static uint64_t prob_threshold(double p) {
  if (p <= 0) return 0;
  if (p >= 1) return 1ull << 32;
  return (uint64_t)(p * 4294967296.0);
}

static RmatParams make_rmat_params(int scale, uint64_t seed, double a, double b, double c) {
  RmatParams P;
  P.scale = scale;
  P.base = mix64(seed ^ 0x5851F42D4C957F2Dull);
  const double d = 1.0 - a - b - c;
  P.t_ab = prob_threshold(a + b);
  P.t_a = prob_threshold((a + b) > 0 ? a / (a + b) : 1.0);
  P.t_c = prob_threshold((c + d) > 0 ? c / (c + d) : 1.0);
  for (int r = 0; r < 3; ++r) {
    P.pm[r] = mix64(seed + 0x1000 + r) | 1ull;
    P.pa[r] = mix64(seed + 0x2000 + r);
  }
  return P;
}

// Seeded bijection on [0, 2^scale): the Graph500 convention of scrambling
// vertex labels so that high-degree vertices are not clustered at low ids.
__host__ __device__ __forceinline__ uint64_t scramble(uint64_t x, const RmatParams& P) {
  const uint64_t mask = (P.scale >= 64) ? ~0ull : ((1ull << P.scale) - 1);
  const int sh = (P.scale + 1) / 2;
  for (int r = 0; r < 3; ++r) {
    x = (x * P.pm[r] + P.pa[r]) & mask;
    if (sh > 0) x ^= x >> sh;
  }
  return x & mask;
}

__host__ __device__ __forceinline__ void rmat_edge(uint64_t k, const RmatParams& P, uint32_t* pu,
                                                   uint32_t* pv) {
  const uint64_t h = mix64(P.base + k);
  uint64_t u = 0, v = 0;
  for (int i = 0; i < P.scale; ++i) {
    const uint64_t r = mix64(h ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1)));
    const uint64_t r1 = r & 0xffffffffull, r2 = r >> 32;
    const uint64_t ii = (r1 >= P.t_ab) ? 1 : 0;
    const uint64_t jj = (r2 >= (ii ? P.t_c : P.t_a)) ? 1 : 0;
    u |= ii << i;
    v |= jj << i;
  }
  *pu = (uint32_t)scramble(u, P);
  *pv = (uint32_t)scramble(v, P);
}

__host__ __device__ __forceinline__ void er_edge(uint64_t k, uint64_t base, uint64_t n, uint32_t* pu,
                                                 uint32_t* pv) {
  const uint64_t h = mix64(base + k);
  *pu = (uint32_t)(((h & 0xffffffffull) * n) >> 32);
  *pv = (uint32_t)(((h >> 32) * n) >> 32);
}

static const uint64_t kSentinel = ~0ull;

// ---------------------------------------------------------------------------
// Host path
// ---------------------------------------------------------------------------
template <typename EdgeFn>
static xbfs_status host_build(uint64_t ntuples, int64_t V, EdgeFn fn, int64_t** pbeg, int32_t** pcsr,
                              int64_t* pV, int64_t* pE) {
  std::vector<uint64_t> keys;
  try {
    keys.resize(2 * ntuples);
  } catch (...) {
    return set_error(XBFS_ERR_OOM, "host allocation of %llu keys failed",
                     (unsigned long long)(2 * ntuples));
  }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)ntuples; ++k) {
    uint32_t u, v;
    fn((uint64_t)k, &u, &v);
    if (u == v) {
      keys[2 * k] = kSentinel;
      keys[2 * k + 1] = kSentinel;
    } else {
      keys[2 * k] = ((uint64_t)u << 32) | v;
      keys[2 * k + 1] = ((uint64_t)v << 32) | u;
    }
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if (!keys.empty() && keys.back() == kSentinel) keys.pop_back();
  const int64_t E = (int64_t)keys.size();
  int64_t* beg = (int64_t*)malloc(sizeof(int64_t) * (V + 1));
  int32_t* csr = (int32_t*)malloc(sizeof(int32_t) * (E > 0 ? E : 1));
  if (!beg || !csr) {
    free(beg);
    free(csr);
    return set_error(XBFS_ERR_OOM, "host allocation of the CSR failed");
  }
  std::vector<int64_t> deg(V + 1, 0);
  for (int64_t i = 0; i < E; ++i) {
    deg[keys[i] >> 32]++;
    csr[i] = (int32_t)(keys[i] & 0xffffffffull);
  }
  beg[0] = 0;
  for (int64_t v = 0; v < V; ++v) beg[v + 1] = beg[v] + deg[v];
  *pbeg = beg;
  *pcsr = csr;
  *pV = V;
  *pE = E;
  return XBFS_OK;
}

static void grid_host(int W, int H, int64_t* beg, int32_t* csr) {
  int64_t e = 0;
  for (int64_t r = 0; r < H; ++r)
    for (int64_t c = 0; c < W; ++c) {
      beg[r * W + c] = e;
      if (r > 0) csr[e++] = (int32_t)((r - 1) * W + c);
      if (c > 0) csr[e++] = (int32_t)(r * W + c - 1);
      if (c + 1 < W) csr[e++] = (int32_t)(r * W + c + 1);
      if (r + 1 < H) csr[e++] = (int32_t)((r + 1) * W + c);
    }
  beg[(int64_t)W * H] = e;
}

static int64_t grid_edges(int64_t W, int64_t H) { return 2 * (W - 1) * H + 2 * W * (H - 1); }

// ---------------------------------------------------------------------------
// Device path
// ---------------------------------------------------------------------------
__global__ void k_rmat_keys(uint64_t ntuples, RmatParams P, unsigned long long* keys) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ntuples;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    rmat_edge(k, P, &u, &v);
    unsigned long long a = kSentinel, b = kSentinel;
    if (u != v) {
      a = ((unsigned long long)u << 32) | v;
      b = ((unsigned long long)v << 32) | u;
    }
    keys[2 * k] = a;
    keys[2 * k + 1] = b;
  }
}

__global__ void k_er_keys(uint64_t ntuples, uint64_t base, uint64_t n, unsigned long long* keys) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ntuples;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    er_edge(k, base, n, &u, &v);
    unsigned long long a = kSentinel, b = kSentinel;
    if (u != v) {
      a = ((unsigned long long)u << 32) | v;
      b = ((unsigned long long)v << 32) | u;
    }
    keys[2 * k] = a;
    keys[2 * k + 1] = b;
  }
}

// keys sorted + unique (sentinel excluded, count E): fill beg[0..V] and csr.
__global__ void k_keys_to_csr(const unsigned long long* keys, long long E, long long V,
                              long long* beg, int* csr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= E;
       i += (long long)gridDim.x * blockDim.x) {
    long long u_prev = (i == 0) ? -1 : (long long)(keys[i - 1] >> 32);
    long long u_cur = (i == E) ? V : (long long)(keys[i] >> 32);
    for (long long w = u_prev + 1; w <= u_cur; ++w) beg[w] = i;
    if (i < E) csr[i] = (int)(keys[i] & 0xffffffffull);
  }
}

__global__ void k_grid(long long W, long long H, long long* beg, int* csr) {
  const long long V = W * H;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const long long r = v / W, c = v % W;
    long long rb = r * (4 * W - 2) - (r > 0 ? W : 0);
    long long off = 4 * c - (c > 0 ? 1 : 0) - (r == 0 ? c : 0) - (r == H - 1 ? c : 0);
    long long e = rb + off;
    beg[v] = e;
    if (r > 0) csr[e++] = (int)((r - 1) * W + c);
    if (c > 0) csr[e++] = (int)(r * W + c - 1);
    if (c + 1 < W) csr[e++] = (int)(r * W + c + 1);
    if (r + 1 < H) csr[e++] = (int)((r + 1) * W + c);
    if (v == V - 1) beg[V] = e;
  }
}

static xbfs_status device_build_from_keys(int device, int64_t V, DevBuf& keys, uint64_t nkeys,
                                          cudaStream_t s, Graph** out) {
  DevBuf keys2, tmp, dnum;
  xbfs_status st;
  if ((st = keys2.ensure(nkeys * 8))) return st;
  size_t tmp_bytes = 0, tmp2 = 0;
  XBFS_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys.as<unsigned long long>(),
                                               keys2.as<unsigned long long>(), (int64_t)nkeys, 0, 64, s));
  XBFS_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, tmp2, keys2.as<unsigned long long>(),
                                          keys.as<unsigned long long>(), dnum.as<long long>(),
                                          (int64_t)nkeys, s));
  if ((st = tmp.ensure(std::max(tmp_bytes, tmp2)))) return st;
  if ((st = dnum.ensure(16))) return st;
  XBFS_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp.p, tmp_bytes, keys.as<unsigned long long>(),
                                               keys2.as<unsigned long long>(), (int64_t)nkeys, 0, 64, s));
  tmp2 = tmp.bytes;
  XBFS_CUDA_TRY(cub::DeviceSelect::Unique(tmp.p, tmp2, keys2.as<unsigned long long>(),
                                          keys.as<unsigned long long>(), dnum.as<long long>(),
                                          (int64_t)nkeys, s));
  long long nuniq = 0;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&nuniq, dnum.p, 8, cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  unsigned long long last = 0;
  if (nuniq > 0) {
    XBFS_CUDA_TRY(cudaMemcpy(&last, keys.as<unsigned long long>() + nuniq - 1, 8, cudaMemcpyDeviceToHost));
    if (last == kSentinel) --nuniq;
  }
  keys2.release();
  tmp.release();
  std::unique_ptr<Graph> g(new Graph());
  g->device = device;
  g->V = V;
  g->E = nuniq;
  if ((st = g->beg.ensure((size_t)(V + 1) * 8))) return st;
  if ((st = g->csr.ensure((size_t)nuniq * 4 + 64))) return st;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  k_keys_to_csr<<<nsm * 8, 256, 0, s>>>(keys.as<unsigned long long>(), nuniq, V,
                                         g->beg.as<long long>(), g->csr.as<int>());
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  keys.release();
  if ((st = graph_finish_upload(g.get()))) return st;
  *out = g.release();
  return XBFS_OK;
}

static xbfs_status device_prologue(int device, cudaStream_t* s) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_error(XBFS_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (device < 0 || device >= n) return set_error(XBFS_ERR_INVALID_ARG, "bad device %d", device);
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  return XBFS_OK;
}

xbfs_status gen_rmat_device(int scale, int ef, uint64_t seed, double a, double b, double c,
                            int device, Graph** out) {
  DeviceGuard dg(device);
  cudaStream_t s = nullptr;
  xbfs_status st = device_prologue(device, &s);
  if (st) return st;
  const RmatParams P = make_rmat_params(scale, seed, a, b, c);
  const uint64_t ntuples = (uint64_t)ef << scale;
  DevBuf keys;
  if (!(st = keys.ensure(2 * ntuples * 8))) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    k_rmat_keys<<<nsm * 16, 256, 0, s>>>(ntuples, P, keys.as<unsigned long long>());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = set_error(XBFS_ERR_CUDA, "k_rmat_keys: %s", cudaGetErrorString(e));
    else st = device_build_from_keys(device, (int64_t)1 << scale, keys, 2 * ntuples, s, out);
  }
  cudaStreamDestroy(s);
  return st;
}

xbfs_status gen_er_device(int64_t n, double mean_degree, uint64_t seed, int device, Graph** out) {
  DeviceGuard dg(device);
  cudaStream_t s = nullptr;
  xbfs_status st = device_prologue(device, &s);
  if (st) return st;
  const uint64_t ntuples = (uint64_t)(mean_degree * (double)n / 2.0 + 0.5);
  const uint64_t base = mix64(seed ^ 0x6A09E667F3BCC909ull);
  DevBuf keys;
  if (!(st = keys.ensure(2 * std::max<uint64_t>(ntuples, 1) * 8))) {
    if (ntuples > 0) {
      k_er_keys<<<1184, 256, 0, s>>>(ntuples, base, (uint64_t)n, keys.as<unsigned long long>());
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = set_error(XBFS_ERR_CUDA, "k_er_keys: %s", cudaGetErrorString(e));
    else st = device_build_from_keys(device, n, keys, 2 * ntuples, s, out);
  }
  cudaStreamDestroy(s);
  return st;
}

xbfs_status gen_grid_device(int W, int H, int device, Graph** out) {
  DeviceGuard dg(device);
  cudaStream_t s = nullptr;
  xbfs_status st = device_prologue(device, &s);
  if (st) return st;
  std::unique_ptr<Graph> g(new Graph());
  g->device = device;
  g->V = (int64_t)W * H;
  g->E = grid_edges(W, H);
  if (!(st = g->beg.ensure((size_t)(g->V + 1) * 8)) && !(st = g->csr.ensure((size_t)g->E * 4 + 64))) {
    k_grid<<<1184, 256, 0, s>>>(W, H, g->beg.as<long long>(), g->csr.as<int>());
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_error(XBFS_ERR_CUDA, "k_grid: %s", cudaGetErrorString(e));
    else st = graph_finish_upload(g.get());
  }
  cudaStreamDestroy(s);
  if (st) return st;
  *out = g.release();
  return XBFS_OK;
}

static xbfs_status check_rmat_args(int scale, int ef, double a, double b, double c) {
  if (scale < 1 || scale > 30) return set_error(XBFS_ERR_INVALID_ARG, "scale %d not in [1, 30]", scale);
  if (ef < 1 || ef > 1024) return set_error(XBFS_ERR_INVALID_ARG, "edge factor %d not in [1, 1024]", ef);
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12)
    return set_error(XBFS_ERR_INVALID_ARG, "bad R-MAT probabilities a=%g b=%g c=%g", a, b, c);
  return XBFS_OK;
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_gen_rmat_host(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b,
                               double c, int64_t** beg, int32_t** csr, int64_t* V, int64_t* E) {
  if (!beg || !csr || !V || !E) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  xbfs_status st = check_rmat_args(scale, edge_factor, a, b, c);
  if (st) return st;
  const RmatParams P = make_rmat_params(scale, seed, a, b, c);
  const uint64_t ntuples = (uint64_t)edge_factor << scale;
  return host_build(ntuples, (int64_t)1 << scale,
                    [&](uint64_t k, uint32_t* u, uint32_t* v) { rmat_edge(k, P, u, v); }, beg, csr, V, E);
}

xbfs_status xbfs_gen_er_host(int64_t n, double mean_degree, uint64_t seed, int64_t** beg, int32_t** csr,
                             int64_t* V, int64_t* E) {
  if (!beg || !csr || !V || !E) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  if (n < 1 || n > (1ll << 31) - 64 || mean_degree < 0 || mean_degree > 1e6)
    return set_error(XBFS_ERR_INVALID_ARG, "bad ER arguments n=%lld mean_degree=%g", (long long)n,
                     mean_degree);
  const uint64_t ntuples = (uint64_t)(mean_degree * (double)n / 2.0 + 0.5);
  const uint64_t base = mix64(seed ^ 0x6A09E667F3BCC909ull);
  return host_build(ntuples, n, [&](uint64_t k, uint32_t* u, uint32_t* v) { er_edge(k, base, (uint64_t)n, u, v); },
                    beg, csr, V, E);
}

xbfs_status xbfs_gen_grid_host(int32_t width, int32_t height, int64_t** beg, int32_t** csr, int64_t* V,
                               int64_t* E) {
  if (!beg || !csr || !V || !E) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  if (width < 1 || height < 1 || (int64_t)width * height > (1ll << 31) - 64)
    return set_error(XBFS_ERR_INVALID_ARG, "bad grid %d x %d", width, height);
  const int64_t nv = (int64_t)width * height, ne = grid_edges(width, height);
  int64_t* b = (int64_t*)malloc(sizeof(int64_t) * (nv + 1));
  int32_t* c = (int32_t*)malloc(sizeof(int32_t) * (ne > 0 ? ne : 1));
  if (!b || !c) {
    free(b);
    free(c);
    return set_error(XBFS_ERR_OOM, "host allocation failed");
  }
  grid_host(width, height, b, c);
  *beg = b;
  *csr = c;
  *V = nv;
  *E = ne;
  return XBFS_OK;
}

xbfs_status xbfs_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b, double c,
                          int32_t device, xbfs_graph** out) {
  if (!out) return set_error(XBFS_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  xbfs_status st = check_rmat_args(scale, edge_factor, a, b, c);
  if (st) return st;
  Graph* g = nullptr;
  if ((st = gen_rmat_device(scale, edge_factor, seed, a, b, c, device, &g))) return st;
  *out = (xbfs_graph*)g;
  return XBFS_OK;
}

xbfs_status xbfs_gen_grid(int32_t width, int32_t height, int32_t device, xbfs_graph** out) {
  if (!out) return set_error(XBFS_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (width < 1 || height < 1 || (int64_t)width * height > (1ll << 31) - 64)
    return set_error(XBFS_ERR_INVALID_ARG, "bad grid %d x %d", width, height);
  Graph* g = nullptr;
  xbfs_status st = gen_grid_device(width, height, device, &g);
  if (st) return st;
  *out = (xbfs_graph*)g;
  return XBFS_OK;
}

xbfs_status xbfs_gen_er(int64_t n, double mean_degree, uint64_t seed, int32_t device, xbfs_graph** out) {
  if (!out) return set_error(XBFS_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (n < 1 || n > (1ll << 31) - 64 || mean_degree < 0 || mean_degree > 1e6)
    return set_error(XBFS_ERR_INVALID_ARG, "bad ER arguments");
  Graph* g = nullptr;
  xbfs_status st = gen_er_device(n, mean_degree, seed, device, &g);
  if (st) return st;
  *out = (xbfs_graph*)g;
  return XBFS_OK;
}

xbfs_status xbfs_pick_sources(const int64_t* beg, int64_t V, int32_t k, uint64_t seed, int32_t* out) {
  if (!beg || !out || V < 1 || k < 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  int64_t nonisolated = 0;
  for (int64_t v = 0; v < V; ++v) nonisolated += (beg[v + 1] > beg[v]);
  if (nonisolated == 0 && k > 0) return set_error(XBFS_ERR_INVALID_ARG, "graph has no edges");
  const bool distinct = k <= nonisolated;
  std::vector<int32_t> chosen;
  chosen.reserve(k);
  uint64_t ctr = 0;
  const uint64_t base = mix64(seed ^ 0x3C6EF372FE94F82Bull);
  while ((int32_t)chosen.size() < k) {
    const uint64_t h = mix64(base + ctr++);
    const int64_t v = (int64_t)(((h >> 11) % (uint64_t)V));
    if (beg[v + 1] == beg[v]) continue;
    if (distinct && std::find(chosen.begin(), chosen.end(), (int32_t)v) != chosen.end()) continue;
    chosen.push_back((int32_t)v);
  }
  memcpy(out, chosen.data(), sizeof(int32_t) * k);
  return XBFS_OK;
}

}  // extern "C"
