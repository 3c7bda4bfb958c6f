// Shared device/host helpers for the xbfs_b200 kernels (sm_100a).
//
// Everything here is integer work: the BFS path has no dense contraction, so
// no tensor-core code appears anywhere in the library. What matters on B200
// is HBM/L2 traffic, latency hiding and the cost of grid-wide barriers in the
// persistent level loops, which is what these helpers serve.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "xbfs.h"

namespace xbfs {

// ---------------------------------------------------------------------------
// Small PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_acquire_i32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Relaxed (weak, L2-coherent) load: bypasses L1 so a value written by another
// SM earlier in the same persistent launch is observed once it reached L2.
__device__ __forceinline__ uint32_t ld_cg_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint64_t ld_cg_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
// Fire-and-forget atomic OR (no return value -> `red`, never stalls the issuer).
__device__ __forceinline__ void red_or_u32(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_or_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.or.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Streaming read of the (immutable during a launch) CSR: the adjacency is read
// once per traversal, so mark it first in line for L2 eviction and keep the
// status/bitmap working set resident instead.
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ int ld_stream_i32(const int* p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
      : "=r"(v)
      : "l"(p), "l"(l2_policy_evict_first()));
  return v;
}
// 16-byte read of data that is immutable during the launch, not kept in L1
// (read once per level: L1 stays for the bitmap words probed at random).
__device__ __forceinline__ int4 ld_nc_na_v4(const int4* p) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p));
  return v;
}
// 16-byte form of ld_stream_i32 (p 16-byte aligned).
__device__ __forceinline__ int4 ld_stream_v4(const int* p) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p), "l"(l2_policy_evict_first()));
  return v;
}
__device__ __forceinline__ long long ld_nc_i64(const long long* p) {
  long long v;
  asm volatile("ld.global.nc.b64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

// ---------------------------------------------------------------------------
// Bounded grid barrier for persistent cooperative launches.
//
// Every spin in the library is bounded in time (globaltimer); on expiry the
// waiting block records XBFS_ERR_DEVICE_TIMEOUT in the error word and returns
// false, so the launch ends and the host reads a status instead of the GPU
// hanging. Any block that sees a non-zero error word also leaves.
// ---------------------------------------------------------------------------
struct __align__(8) GridBarrier {
  uint32_t count;  // arrivals since launch (zeroed before the launch)
  int32_t err;     // launch status (xbfs_status), 0 = fine; shares count's 8 bytes
};

__device__ __forceinline__ void red_add_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Count-up barrier: the k-th barrier of a launch completes when `count`
// reaches k * nblocks. One release-add per CTA (the block barrier before it
// makes the whole CTA's writes part of the release), no reset and no
// generation flip on the critical path; `epoch` is the CTA's own count of
// barriers passed (identical in all CTAs). Each poll is one 8-byte acquire
// load that returns the arrival count and the error word together, so the
// barrier costs one release and the polls, with no separate fence or status
// read. 2^32 arrivals allow > 10^7 barriers at 296 CTAs.
__device__ __forceinline__ bool grid_sync(GridBarrier* bar, uint32_t nblocks, uint32_t& epoch,
                                          unsigned long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) {
    int ok = 1;
    const uint32_t target = epoch * nblocks;
    red_add_release_u32(&bar->count, 1u);
    uint32_t spins = 0;
    unsigned long long t0 = 0;
    for (;;) {
      const unsigned long long w = ld_acquire_u64(reinterpret_cast<const unsigned long long*>(bar));
      if ((int32_t)(w >> 32) != 0) {
        ok = 0;
        break;
      }
      if ((int32_t)((uint32_t)w - target) >= 0) break;
      ++spins;
      if (spins > 2048) __nanosleep(32);
      if ((spins & 1023u) == 0) {
        if (t0 == 0) t0 = globaltimer_ns();
        if (globaltimer_ns() - t0 > timeout_ns) {
          atomicCAS(&bar->err, 0, (int)XBFS_ERR_DEVICE_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// Warp / block reductions and scans (no library dependency on the hot path).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan. `s_warp` needs BLOCK/32 + 1 slots. Returns the
// exclusive prefix for the calling thread and the block total in *total.
template <int BLOCK, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T* total) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T w = (lane < NW) ? s_warp[lane] : T(0);
    T winc = warp_inclusive_scan(w);
    if (lane < NW) s_warp[lane] = winc - w;
    if (lane == NW - 1) s_warp[NW] = winc;
  }
  __syncthreads();
  T res = s_warp[wid] + inc - v;
  *total = s_warp[NW];
  __syncthreads();
  return res;
}

// Sums N values per thread over the block in one pass (two barriers).
// `s` needs N * (BLOCK/32) slots; every thread receives all N totals.
template <int BLOCK, int N, typename T>
__device__ __forceinline__ void block_sum_n(T (&v)[N], T* s) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const T t = warp_sum(v[k]);
    if (lane == 0) s[k * NW + wid] = t;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    T t = 0;
#pragma unroll
    for (int i = 0; i < NW; ++i) t += s[k * NW + i];
    v[k] = t;
  }
  __syncthreads();
}

template <int BLOCK, typename T>
__device__ __forceinline__ T block_sum(T v, T* s_warp) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) s_warp[wid] = v;
  __syncthreads();
  T r = 0;
  if (wid == 0) {
    T w = (lane < NW) ? s_warp[lane] : T(0);
    w = warp_sum(w);
    if (lane == 0) s_warp[NW] = w;
  }
  __syncthreads();
  r = s_warp[NW];
  __syncthreads();
  return r;
}

}  // namespace xbfs

// Host-side CUDA error plumbing: every CUDA failure becomes a status code with
// a thread-local detail string; nothing in the library exits the process.
#define XBFS_CUDA_TRY(expr)                                                   \
  do {                                                                        \
    cudaError_t e__ = (expr);                                                 \
    if (e__ != cudaSuccess) {                                                 \
      return ::xbfs::set_error(e__ == cudaErrorMemoryAllocation ? XBFS_ERR_OOM \
                                                               : XBFS_ERR_CUDA, \
                               "%s:%d %s: %s", __FILE__, __LINE__, #expr,     \
                               cudaGetErrorString(e__));                      \
    }                                                                         \
  } while (0)

namespace xbfs {
xbfs_status set_error(xbfs_status st, const char* fmt, ...);
}
