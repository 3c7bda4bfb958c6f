// Graph handles: CSR loading (file pair of the reference format), upload,
// validation, degree statistics and the isolated-vertex bitmap.
//
// Replaces graph<int,long,int,int,long,char>::graph (graph.hpp:4-104) and
// the beg_cu/csr_cu allocation in main (bfs_gpu_update.cu:175-180). The file
// format is identical (raw int64 offsets, raw int32 neighbours); unlike the
// reference, malformed input is reported as XBFS_ERR_FORMAT instead of an
// assert, and the file is streamed through a pinned double buffer so that
// reading, page-in and the host-to-device copy overlap.
#include <fcntl.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

static thread_local std::string g_last_error;

xbfs_status set_error(xbfs_status st, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

xbfs_status DevBuf::ensure(size_t n) {
  if (n <= bytes && p) return XBFS_OK;
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? XBFS_ERR_OOM : XBFS_ERR_CUDA,
                     "cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return XBFS_OK;
}

xbfs_status PinnedBuf::ensure(size_t n) {
  if (n <= bytes && p) return XBFS_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  bytes = 0;
  cudaError_t e = cudaMallocHost(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return set_error(XBFS_ERR_OOM, "cudaMallocHost(%zu): %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return XBFS_OK;
}

Graph::~Graph() {
  DeviceGuard dg(device);
  if (ss.ev0) cudaEventDestroy(ss.ev0);
  if (ss.ev1) cudaEventDestroy(ss.ev1);
  if (ss.evk0) cudaEventDestroy(ss.evk0);
  for (int i = 0; i < 2; ++i) {
    if (ss.ev_done[i]) cudaEventDestroy(ss.ev_done[i]);
    if (ss.ev_copied[i]) cudaEventDestroy(ss.ev_copied[i]);
  }
  if (ss.copy_stream) cudaStreamDestroy(ss.copy_stream);
  if (stream) cudaStreamDestroy(stream);
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// Device-side validation and statistics
// ---------------------------------------------------------------------------
struct GraphCheck {
  unsigned long long bad_beg;     // first index i with beg[i] > beg[i+1] (+1), 0 = ok
  unsigned long long bad_csr;     // first edge index with neighbour out of range (+1)
  unsigned long long fp_fwd;      // order-independent fingerprint of the (u, v) multiset
  unsigned long long fp_rev;      // ... and of the (v, u) multiset
  unsigned long long max_degree;
  unsigned long long n_isolated;
  unsigned long long cnt_deg_gt[16];
};

__global__ void k_check_beg(const long long* __restrict__ beg, long long V, GraphCheck* out,
                            uint32_t* __restrict__ iso, long long nwords) {
  __shared__ unsigned long long s_cnt[16];
  __shared__ unsigned long long s_iso, s_max;
  if (threadIdx.x < 16) s_cnt[threadIdx.x] = 0;
  if (threadIdx.x == 0) { s_iso = 0; s_max = 0; }
  __syncthreads();
  // One thread per 32-vertex bitmap word: vertices [32w, 32w+32).
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
       w += (long long)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    unsigned long long local_iso = 0, local_max = 0;
    unsigned c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = 0;
    for (int b = 0; b < 32; ++b) {
      long long v = w * 32 + b;
      if (v >= V) { bits |= 1u << b; continue; }
      long long d = beg[v + 1] - beg[v];
      if (d < 0) {
        atomicMin(&out->bad_beg, (unsigned long long)(v + 1));
        d = 0;
      }
      if (d == 0) { bits |= 1u << b; ++local_iso; }
      if ((unsigned long long)d > local_max) local_max = d;
#pragma unroll
      for (int k = 0; k < 16; ++k) c[k] += (d > (1ll << k)) ? 1u : 0u;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (c[k]) atomicAdd(&s_cnt[k], (unsigned long long)c[k]);
    iso[w] = bits;
    if (local_iso) atomicAdd(&s_iso, local_iso);
    atomicMax(&s_max, local_max);
  }
  __syncthreads();
  if (threadIdx.x < 16 && s_cnt[threadIdx.x]) atomicAdd(&out->cnt_deg_gt[threadIdx.x], s_cnt[threadIdx.x]);
  if (threadIdx.x == 0) {
    if (s_iso) atomicAdd(&out->n_isolated, s_iso);
    atomicMax(&out->max_degree, s_max);
  }
}

__device__ __forceinline__ unsigned long long fp_mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Range check of every neighbour id, plus two fingerprints (sums of a 64-bit
// hash over edges (u, v) and over reversed edges (v, u)). Equal fingerprints
// mean the edge multiset is symmetric (up to a 2^-64 collision), which is what
// makes bottom-up steps valid: they find parents through the out-adjacency.
// One warp per vertex. Requires beg to be monotone (checked by k_check_beg);
// runs only after that check passed.
__global__ void k_check_csr(const long long* __restrict__ beg, const int* __restrict__ csr, long long V,
                            GraphCheck* out) {
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  unsigned long long f1 = 0, f2 = 0;
  for (long long u = warp; u < V; u += nwarps) {
    const long long e0 = beg[u], e1 = beg[u + 1];
    for (long long e = e0 + lane; e < e1; e += 32) {
      const int v = csr[e];
      if (v < 0 || (long long)v >= V) {
        atomicMin(&out->bad_csr, (unsigned long long)(e + 1));
        continue;
      }
      f1 += fp_mix(((unsigned long long)u << 32) | (unsigned)v);
      f2 += fp_mix(((unsigned long long)(unsigned)v << 32) | (unsigned long long)u);
    }
  }
  f1 = warp_sum(f1);
  f2 = warp_sum(f2);
  if (lane == 0 && (f1 | f2)) {
    atomicAdd(&out->fp_fwd, f1);
    atomicAdd(&out->fp_rev, f2);
  }
}

xbfs_status graph_finish_upload(Graph* g) {
  DeviceGuard dg(g->device);
  if (!g->stream) XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  const long long nwords = (g->V + 31) / 32 + 64;  // padded: kernels may read a little past V
  xbfs_status st = g->iso.ensure(nwords * 4);
  if (st) return st;
  DevBuf dchk;
  if ((st = dchk.ensure(sizeof(GraphCheck)))) return st;
  GraphCheck init;
  memset(&init, 0, sizeof(init));
  init.bad_beg = ~0ull;
  init.bad_csr = ~0ull;
  XBFS_CUDA_TRY(cudaMemcpyAsync(dchk.p, &init, sizeof(init), cudaMemcpyHostToDevice, g->stream));
  // Check beg[0] == 0 and beg[V] == E on the host side with two tiny reads.
  long long b0 = -1, bV = -1;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&b0, g->beg.p, 8, cudaMemcpyDeviceToHost, g->stream));
  XBFS_CUDA_TRY(cudaMemcpyAsync(&bV, g->beg.as<long long>() + g->V, 8, cudaMemcpyDeviceToHost,
                                g->stream));
  XBFS_CUDA_TRY(cudaMemsetAsync(g->iso.p, 0xff, nwords * 4, g->stream));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device);
  const long long real_words = (g->V + 31) / 32;
  if (real_words > 0) {
    int grid = (int)std::min<long long>((real_words + 255) / 256, nsm * 8);
    k_check_beg<<<grid, 256, 0, g->stream>>>(g->beg.as<long long>(), g->V, dchk.as<GraphCheck>(),
                                             g->iso.as<uint32_t>(), real_words);
  }
  XBFS_CUDA_TRY(cudaGetLastError());
  GraphCheck res;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&res, dchk.p, sizeof(res), cudaMemcpyDeviceToHost, g->stream));
  XBFS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (b0 != 0) return set_error(XBFS_ERR_FORMAT, "beg_pos[0] = %lld, expected 0", b0);
  if (bV != g->E)
    return set_error(XBFS_ERR_FORMAT, "beg_pos[V] = %lld but the edge count is %lld", bV,
                     (long long)g->E);
  if (res.bad_beg != ~0ull)
    return set_error(XBFS_ERR_FORMAT, "beg_pos not monotone at vertex %llu", res.bad_beg - 1);
  // offsets are sane: now the per-vertex pass over the neighbours is in bounds
  if (g->E > 0) {
    int grid = (int)std::min<long long>((g->V * 32 + 255) / 256, nsm * 16);
    k_check_csr<<<grid, 256, 0, g->stream>>>(g->beg.as<long long>(), g->csr.as<int>(), g->V,
                                             dchk.as<GraphCheck>());
    XBFS_CUDA_TRY(cudaGetLastError());
    XBFS_CUDA_TRY(cudaMemcpyAsync(&res, dchk.p, sizeof(res), cudaMemcpyDeviceToHost, g->stream));
    XBFS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  g->symmetric = (res.fp_fwd == res.fp_rev);
  if (!g->symmetric && real_words > 0) {
    // In a directed CSR an out-degree-0 vertex can still be reached, so only
    // the padding bits past V may be pre-marked as visited.
    XBFS_CUDA_TRY(cudaMemsetAsync(g->iso.p, 0, real_words * 4, g->stream));
    if (g->V % 32) {
      const uint32_t tail = ~((1u << (g->V % 32)) - 1u);
      XBFS_CUDA_TRY(cudaMemcpyAsync(g->iso.as<uint32_t>() + real_words - 1, &tail, 4, cudaMemcpyHostToDevice,
                                    g->stream));
    }
    XBFS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  if (res.bad_csr != ~0ull)
    return set_error(XBFS_ERR_FORMAT, "csr[%llu] is not a vertex id in [0, %lld)",
                     res.bad_csr - 1, (long long)g->V);
  g->max_degree = (int64_t)res.max_degree;
  g->n_isolated = (int64_t)res.n_isolated;
  for (int k = 0; k < 16; ++k) g->cnt_deg_gt[k] = (int64_t)res.cnt_deg_gt[k];
  return graph_build_head(g);
}

xbfs_status validate_csr(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E) {
  if (V < 1) return set_error(XBFS_ERR_FORMAT, "graph has no vertices");
  if (beg[0] != 0) return set_error(XBFS_ERR_FORMAT, "beg_pos[0] = %lld", (long long)beg[0]);
  if (beg[V] != E)
    return set_error(XBFS_ERR_FORMAT, "beg_pos[V] = %lld != E = %lld", (long long)beg[V],
                     (long long)E);
  for (int64_t i = 0; i < V; ++i)
    if (beg[i] > beg[i + 1])
      return set_error(XBFS_ERR_FORMAT, "beg_pos not monotone at vertex %lld", (long long)i);
  for (int64_t e = 0; e < E; ++e)
    if (csr[e] < 0 || csr[e] >= V)
      return set_error(XBFS_ERR_FORMAT, "csr[%lld] = %d out of range", (long long)e, csr[e]);
  return XBFS_OK;
}

static xbfs_status check_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_error(XBFS_ERR_NO_DEVICE, "no CUDA device available (%s)",
                     e == cudaSuccess ? "count = 0" : cudaGetErrorString(e));
  }
  if (device < 0 || device >= n)
    return set_error(XBFS_ERR_INVALID_ARG, "device %d out of range [0, %d)", device, n);
  return XBFS_OK;
}

static xbfs_status alloc_graph(int device, int64_t V, int64_t E, Graph** out) {
  if (V < 1 || V > (int64_t)INT32_MAX - 64)
    return set_error(XBFS_ERR_UNSUPPORTED, "vertex count %lld outside [1, 2^31-64)", (long long)V);
  if (E < 0 || E >= (1ll << 33))
    return set_error(XBFS_ERR_UNSUPPORTED, "edge count %lld outside [0, 2^33)", (long long)E);
  xbfs_status st = check_device(device);
  if (st) return st;
  DeviceGuard dg(device);
  std::unique_ptr<Graph> g(new Graph());
  g->device = device;
  g->V = V;
  g->E = E;
  if ((st = g->beg.ensure((size_t)(V + 1) * 8))) return st;
  if ((st = g->csr.ensure((size_t)E * 4 + 64))) return st;
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  *out = g.release();
  return XBFS_OK;
}

// Copy `bytes` from host memory (pageable or mmap'd) to the device through a
// pinned double buffer so page-in and DMA overlap.
static xbfs_status staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return XBFS_OK;
  const size_t CH = 64u << 20;
  if (bytes <= CH) {
    XBFS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    XBFS_CUDA_TRY(cudaStreamSynchronize(s));
    return XBFS_OK;
  }
  PinnedBuf pin;
  xbfs_status st = pin.ensure(2 * CH);
  if (st) return st;
  cudaEvent_t ev[2];
  XBFS_CUDA_TRY(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  XBFS_CUDA_TRY(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  size_t off = 0;
  int k = 0;
  xbfs_status rc = XBFS_OK;
  while (off < bytes) {
    size_t n = std::min(CH, bytes - off);
    char* buf = (char*)pin.p + (size_t)k * CH;
    if (cudaEventSynchronize(ev[k]) != cudaSuccess) { cudaGetLastError(); }
    memcpy(buf, (const char*)src + off, n);
    cudaError_t e = cudaMemcpyAsync((char*)dst + off, buf, n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev[k], s);
    if (e != cudaSuccess) {
      rc = set_error(XBFS_ERR_CUDA, "staged copy: %s", cudaGetErrorString(e));
      break;
    }
    off += n;
    k ^= 1;
  }
  cudaError_t e = cudaStreamSynchronize(s);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (!rc && e != cudaSuccess) rc = set_error(XBFS_ERR_CUDA, "staged copy: %s", cudaGetErrorString(e));
  return rc;
}

xbfs_status graph_from_host(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E,
                            int device, bool /*validate*/, Graph** out) {
  Graph* g = nullptr;
  xbfs_status st = alloc_graph(device, V, E, &g);
  if (st) return st;
  std::unique_ptr<Graph> hold(g);
  DeviceGuard dg(device);
  if ((st = staged_h2d(g->beg.p, beg, (size_t)(V + 1) * 8, g->stream))) return st;
  if ((st = staged_h2d(g->csr.p, csr, (size_t)E * 4, g->stream))) return st;
  if ((st = graph_finish_upload(g))) return st;
  *out = hold.release();
  return XBFS_OK;
}

struct MappedFile {
  int fd = -1;
  void* p = nullptr;
  size_t size = 0;
  ~MappedFile() {
    if (p && p != MAP_FAILED) munmap(p, size);
    if (fd >= 0) close(fd);
  }
  xbfs_status open_ro(const char* path) {
    fd = ::open(path, O_RDONLY);
    if (fd < 0) return set_error(XBFS_ERR_IO, "cannot open %s: %s", path, strerror(errno));
    struct stat stt;
    if (fstat(fd, &stt) != 0) return set_error(XBFS_ERR_IO, "cannot stat %s", path);
    size = (size_t)stt.st_size;
    if (size == 0) return XBFS_OK;
    p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (p == MAP_FAILED) {
      p = nullptr;
      return set_error(XBFS_ERR_IO, "cannot mmap %s: %s", path, strerror(errno));
    }
    madvise(p, size, MADV_SEQUENTIAL);
    return XBFS_OK;
  }
};

}  // namespace xbfs

using namespace xbfs;

extern "C" {

const char* xbfs_strerror(xbfs_status st) {
  switch (st) {
    case XBFS_OK: return "ok";
    case XBFS_ERR_INVALID_ARG: return "invalid argument";
    case XBFS_ERR_IO: return "i/o error";
    case XBFS_ERR_FORMAT: return "malformed graph";
    case XBFS_ERR_CUDA: return "CUDA error";
    case XBFS_ERR_OOM: return "out of device memory";
    case XBFS_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case XBFS_ERR_UNSUPPORTED: return "unsupported input";
    case XBFS_ERR_INTERNAL: return "internal error";
    case XBFS_ERR_NO_DEVICE: return "no CUDA device";
    case XBFS_ERR_BUSY: return "busy";
    case XBFS_ERR_LEVEL_OVERFLOW: return "level overflow";
    default: return "unknown status";
  }
}

const char* xbfs_last_error(void) { return g_last_error.c_str(); }

int32_t xbfs_version(void) { return 10000; }

xbfs_status xbfs_device_count(int32_t* n) {
  if (!n) return set_error(XBFS_ERR_INVALID_ARG, "n is NULL");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *n = c;
  return XBFS_OK;
}

void xbfs_opts_init(xbfs_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(xbfs_opts);
  o->policy = XBFS_POLICY_HEURISTIC;
  o->alpha = 0.1f;
  o->async_bu = 1;
  o->small_max = 32;
  o->medium_max = 256;
  o->padding = 1;
  o->beamer_alpha = 14.f;
  o->beamer_beta = 24.f;
}

xbfs_status xbfs_graph_load(const char* beg_path, const char* csr_path, int32_t device,
                            xbfs_graph** out) {
  if (!beg_path || !csr_path || !out) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  MappedFile fb, fc;
  xbfs_status st = fb.open_ro(beg_path);
  if (st) return st;
  if (fb.size < 16 || fb.size % 8 != 0)
    return set_error(XBFS_ERR_FORMAT, "%s: size %zu is not 8*(V+1) with V >= 1", beg_path, fb.size);
  const int64_t V = (int64_t)(fb.size / 8) - 1;
  const int64_t E = ((const int64_t*)fb.p)[V];
  if (E < 0) return set_error(XBFS_ERR_FORMAT, "beg_pos[V] = %lld is negative", (long long)E);
  if ((st = fc.open_ro(csr_path))) return st;
  // The reference reads beg_pos[V] neighbours and asserts the read succeeded
  // (graph.hpp:97-100): a shorter file is an error, trailing bytes are unused.
  if (fc.size < (size_t)E * 4)
    return set_error(XBFS_ERR_FORMAT, "%s holds %zu bytes but beg_pos[V] = %lld needs %lld",
                     csr_path, fc.size, (long long)E, (long long)E * 4);
  Graph* g = nullptr;
  if ((st = alloc_graph(device, V, E, &g))) return st;
  std::unique_ptr<Graph> hold(g);
  DeviceGuard dg(device);
  if ((st = staged_h2d(g->beg.p, fb.p, (size_t)(V + 1) * 8, g->stream))) return st;
  if ((st = staged_h2d(g->csr.p, fc.p, (size_t)E * 4, g->stream))) return st;
  if ((st = graph_finish_upload(g))) return st;
  *out = (xbfs_graph*)hold.release();
  return XBFS_OK;
}

xbfs_status xbfs_graph_upload(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E,
                              int32_t device, xbfs_graph** out) {
  if (!beg || (!csr && E > 0) || !out) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  Graph* g = nullptr;
  xbfs_status st = graph_from_host(beg, csr, V, E, device, true, &g);
  if (st) return st;
  *out = (xbfs_graph*)g;
  return XBFS_OK;
}

xbfs_status xbfs_graph_info(const xbfs_graph* gh, int64_t* V, int64_t* E, int64_t* max_degree,
                            int64_t* n_isolated) {
  const Graph* g = (const Graph*)gh;
  if (!g) return set_error(XBFS_ERR_INVALID_ARG, "graph is NULL");
  if (V) *V = g->V;
  if (E) *E = g->E;
  if (max_degree) *max_degree = g->max_degree;
  if (n_isolated) *n_isolated = g->n_isolated;
  return XBFS_OK;
}

xbfs_status xbfs_graph_download(const xbfs_graph* gh, int64_t* beg, int32_t* csr) {
  const Graph* g = (const Graph*)gh;
  if (!g || !beg) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(g->device);
  XBFS_CUDA_TRY(cudaMemcpy(beg, g->beg.p, (size_t)(g->V + 1) * 8, cudaMemcpyDeviceToHost));
  if (csr && g->E > 0) XBFS_CUDA_TRY(cudaMemcpy(csr, g->csr.p, (size_t)g->E * 4, cudaMemcpyDeviceToHost));
  return XBFS_OK;
}

xbfs_status xbfs_graph_save(const xbfs_graph* gh, const char* beg_path, const char* csr_path) {
  const Graph* g = (const Graph*)gh;
  if (!g || !beg_path || !csr_path) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  std::vector<int64_t> beg(g->V + 1);
  std::vector<int32_t> csr(g->E);
  xbfs_status st = xbfs_graph_download(gh, beg.data(), csr.data());
  if (st) return st;
  FILE* f = fopen(beg_path, "wb");
  if (!f) return set_error(XBFS_ERR_IO, "cannot create %s", beg_path);
  size_t w = fwrite(beg.data(), 8, beg.size(), f);
  fclose(f);
  if (w != beg.size()) return set_error(XBFS_ERR_IO, "short write to %s", beg_path);
  f = fopen(csr_path, "wb");
  if (!f) return set_error(XBFS_ERR_IO, "cannot create %s", csr_path);
  w = csr.empty() ? 0 : fwrite(csr.data(), 4, csr.size(), f);
  fclose(f);
  if (w != csr.size()) return set_error(XBFS_ERR_IO, "short write to %s", csr_path);
  return XBFS_OK;
}

void xbfs_graph_free(xbfs_graph* gh) { delete (Graph*)gh; }

void xbfs_free_host(void* p) { free(p); }

}  // extern "C"
