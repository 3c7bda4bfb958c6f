// Serving loop: BFS requests over device-resident graphs, continuously
// batched into 64-source bit slots.
//
// No counterpart in the reference. Design:
//  * Each graph owns a slot batch: one uint64 word per vertex for visited,
//    frontier (two, by tick parity) and an accumulator; bit s belongs to
//    slot s. A request joins a running batch at any tick t: its bit is set at
//    its source and its join tick recorded; from then on every tick advances
//    all slots by one level, and a vertex that gains bit s at tick t gets
//    level t + 1 - join[s] in that request's own int32[V] output.
//  * A slot finishes at the first tick that gives it no new vertex; its
//    visited bits are cleared and the slot is reused. Requests wait for a
//    free slot and for room in an HBM budget (their output array is
//    allocated from a stream-ordered pool when admitted).
//  * Ticks are top-down: the frontier queue (vertex ids with exclusive edge
//    offsets) is expanded edge-balanced across the GPU; each edge claims the
//    slots its target lacks with one 64-bit atomicOr, and the first claimant
//    of a vertex in a tick queues it for the next. On symmetric graphs a
//    slot whose own frontier holds more than E/8 edges advances bottom-up
//    instead (unvisited vertices probe their neighbours' masks); the other
//    slots of that tick stay top-down, so a request that joined late never
//    makes the bottom-up scan read whole adjacency lists. A round of ticks
//    runs in one cooperative launch with one grid barrier per tick. Graphs run
//    on their own streams so their ticks overlap on the device; the host
//    intervenes every K ticks (K grows with a graph's observed depth, so
//    long-diameter graphs are not host-bound).
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {
namespace sv {

constexpr int kBlock = 512;
constexpr int kSlots = 64;
constexpr int kRing = 64;  // ticks between host interventions, at most
constexpr unsigned long long kCountMask = (1ull << 31) - 1;

// Buffers by tick: frontier masks F[t % 3] (read at tick t, written for t+1,
// retired at t+1), frontier queues q[t % 4] (expanded at tick t, filled at
// t-1, their ids read again when retiring at t+1, counter reset at t-2).
struct Ctl {
  GridBarrier bar;                    // barrier of the round kernel (zeroed before each round)
  unsigned long long q[4];            // packed (edges << 31) | count, frontier queue ring
  unsigned long long active[kRing];   // OR of the bits gained at each tick of the window
  unsigned long long msum[kSlots];    // per slot: sum of degrees of reached vertices
  unsigned long long fe[4][kSlots];   // per slot: edges of its frontier, ring by tick like q
};

struct Params {
  const long long* beg;
  const int* csr;
  long long V, E;
  int allow_bu;        // symmetric CSR: bottom-up ticks are valid
  unsigned long long* vis;
  unsigned long long* F[3];
  int* qids[4];
  unsigned* qeb[4];
  long long* qbg[4];   // CSR offset of each queued vertex
  int** out;           // device table: output array of each slot (or null)
  long long* join;     // device table: join tick of each slot
  Ctl* ctl;
};

// Claim step of one edge (u, v) at tick t (see sv_tick), u offering the
// slot mask fu; returns whether this thread queues v for tick t+1, with v's
// degree and CSR offset.
__device__ __forceinline__ bool sv_claim_m(const Params& p, long long t, unsigned long long fu,
                                           unsigned long long* Fn, int v, long long& deg, long long& b0,
                                           unsigned long long& act, unsigned long long* s_msum) {
  const unsigned long long m = fu & ~ld_cg_u64(p.vis + v);
  if (!m) return false;
  const unsigned long long gained = m & ~atomicOr(p.vis + v, m);
  if (!gained) return false;
  b0 = ld_nc_i64(p.beg + v);
  deg = ld_nc_i64(p.beg + v + 1) - b0;
  // a vertex without edges is never expanded: it gets levels, no frontier bits
  const unsigned long long prev = deg > 0 ? atomicOr(Fn + v, gained) : ~0ull;
  act |= gained;
  for (unsigned long long bits = gained; bits; bits &= bits - 1) {
    const int sl = __ffsll((long long)bits) - 1;
    int* o = p.out[sl];
    if (o) o[v] = (int)(t + 1 - p.join[sl]);
    if (deg) atomicAdd(&s_msum[sl], (unsigned long long)deg);
  }
  return prev == 0 && deg > 0;
}

// The same with u's whole frontier mask.
__device__ __forceinline__ bool sv_claim(const Params& p, long long t, const unsigned long long* Fc,
                                         unsigned long long* Fn, int u, int v, long long& deg, long long& b0,
                                         unsigned long long& act, unsigned long long* s_msum) {
  return sv_claim_m(p, t, ld_cg_u64(Fc + u), Fn, v, deg, b0, act, s_msum);
}

// Warp-aggregated append of the lanes with `have` to queue qn (full warp).
__device__ __forceinline__ void sv_enqueue(const Params& p, int qn, bool have, int v, long long deg, long long b0) {
  const int lane = threadIdx.x & 31;
  const unsigned mask = __ballot_sync(0xffffffffu, have);
  if (!mask) return;
  const long long d = have ? deg : 0;
  const long long inc = warp_inclusive_scan(d);
  unsigned long long old = 0;
  if (lane == 31) old = atomicAdd(&p.ctl->q[qn], ((unsigned long long)inc << 31) | (unsigned long long)__popc(mask));
  old = __shfl_sync(0xffffffffu, old, 31);
  if (have) {
    const unsigned slot = (unsigned)(old & kCountMask) + __popc(mask & ((1u << lane) - 1));
    p.qids[qn][slot] = v;
    p.qeb[qn][slot] = (unsigned)((old >> 31) + (unsigned long long)(inc - d));
    p.qbg[qn][slot] = b0;
  }
}

// Tick t, one phase: every edge (u, v) of frontier queue t offers u's slot
// mask to v; the slots v did not have yet are claimed with one 64-bit
// atomicOr on vis[v] (each slot bit is won exactly once), recorded in v's
// output row for each won slot (level t + 1 - join), added to the next
// frontier mask, and the thread whose OR found v's next mask empty queues v
// for tick t+1 (so v is queued once). Edge-balanced: part takes an equal
// share of the queue's edges.
__device__ void sv_tick(const Params& p, long long t, unsigned nparts, unsigned part,
                        unsigned long long* s_msum, unsigned long long* s_act) {
  __shared__ long long wbeg[kBlock + 1];
  __shared__ unsigned web[kBlock + 1];
  __shared__ int wu[kBlock + 1];
  __shared__ int next_s;
  const int lane = threadIdx.x & 31;
  const int qs = (int)(t % 4), qn = (int)((t + 1) % 4);
  const unsigned long long pk = ld_cg_u64(&p.ctl->q[qs]);
  const unsigned cnt = (unsigned)(pk & kCountMask);
  const unsigned long long M = pk >> 31;
  const unsigned long long G = nparts;
  const unsigned long long lo = M * part / G, hi = M * (part + 1) / G;
  if (cnt == 0) return;
  const int* ids = p.qids[qs];
  const unsigned* eb = p.qeb[qs];
  const long long* bgs = p.qbg[qs];
  const unsigned long long* Fc = p.F[t % 3];
  unsigned long long* Fn = p.F[(t + 1) % 3];
  unsigned long long act = 0;
  if ((unsigned long long)cnt <= 32ull * G && M <= 32ull * cnt) {
    // small queue of low-degree vertices: each part takes an equal share of
    // the entries (at most 32), so no part searches the queue for its start
    const unsigned i0 = (unsigned)((unsigned long long)cnt * part / G);
    const unsigned i1 = (unsigned)((unsigned long long)cnt * (part + 1) / G);
    if (i0 >= i1) return;
    const int n = (int)(i1 - i0);
    const unsigned base = eb[i0];
    const unsigned long long T = ((i1 < cnt) ? (unsigned long long)eb[i1] : M) - base;
    if (threadIdx.x < n) {
      const unsigned slot = i0 + threadIdx.x;
      wu[threadIdx.x] = ids[slot];
      wbeg[threadIdx.x] = bgs[slot];
      web[threadIdx.x] = eb[slot] - base;
    }
    __syncthreads();
    for (unsigned long long e0 = 0; e0 < T; e0 += kBlock) {
      const unsigned long long e = e0 + threadIdx.x;
      bool first = false;
      int v = 0;
      long long deg = 0, b0 = 0;
      if (e < T) {
        int a = 0, c = n;
        while (c - a > 1) {
          const int mid = (a + c) >> 1;
          if ((unsigned long long)web[mid] <= e) a = mid; else c = mid;
        }
        v = ld_stream_i32(p.csr + wbeg[a] + (long long)(e - web[a]));
        first = sv_claim(p, t, Fc, Fn, wu[a], v, deg, b0, act, s_msum);
      }
      sv_enqueue(p, qn, first, v, deg, b0);
    }
  } else if (lo < hi) {
  if (threadIdx.x < 32) {
    unsigned a = 0, b = cnt;
    while (b - a > 32) {
      const unsigned span = b - a;
      const unsigned piv = a + (unsigned)(((unsigned long long)span * lane) / 32);
      const unsigned m = __ballot_sync(0xffffffffu, (unsigned long long)eb[piv] <= lo);
      const int last = 31 - __clz(m);
      const unsigned na = a + (unsigned)(((unsigned long long)span * last) / 32);
      const unsigned nb = (last == 31) ? b : a + (unsigned)(((unsigned long long)span * (last + 1)) / 32);
      a = na;
      b = nb;
    }
    const unsigned idx = a + lane;
    const unsigned m = __ballot_sync(0xffffffffu, idx < b && (unsigned long long)eb[idx] <= lo);
    if (lane == 0) next_s = (int)(a + 31 - __clz(m));
  }
  __syncthreads();
  unsigned s = (unsigned)next_s;
  for (unsigned long long r = lo; r < hi; r += kBlock) {
    const unsigned long long rhi = (r + kBlock < hi) ? r + kBlock : hi;
    for (int i = threadIdx.x; i <= kBlock; i += kBlock) {
      const unsigned slot = s + (unsigned)i;
      unsigned e0 = 0xffffffffu;
      if (slot < cnt) {
        const unsigned x = eb[slot];
        if ((unsigned long long)x < rhi) {
          e0 = x;
          wu[i] = ids[slot];
          wbeg[i] = bgs[slot];
        }
      }
      web[i] = e0;
    }
    __syncthreads();
    const unsigned long long e = r + threadIdx.x;
    bool first = false;
    int v = 0;
    long long deg = 0, b0 = 0;
    if (e < rhi) {
      int a = 0, c = kBlock + 1;
      while (c - a > 1) {
        const int mid = (a + c) >> 1;
        if ((unsigned long long)web[mid] <= e) a = mid; else c = mid;
      }
      v = ld_stream_i32(p.csr + wbeg[a] + (long long)(e - web[a]));
      first = sv_claim(p, t, Fc, Fn, wu[a], v, deg, b0, act, s_msum);
    }
    sv_enqueue(p, qn, first, v, deg, b0);
    if (threadIdx.x == 0 && rhi < hi) {
      int a = 0, c = kBlock + 1;
      while (c - a > 1) {
        const int mid = (a + c) >> 1;
        if ((unsigned long long)web[mid] <= rhi) a = mid; else c = mid;
      }
      next_s = (int)(s + a);
    }
    __syncthreads();
    s = (unsigned)next_s;
  }
  }
  act = __reduce_or_sync(0xffffffffu, (unsigned)act) |
        ((unsigned long long)__reduce_or_sync(0xffffffffu, (unsigned)(act >> 32)) << 32);
  if (lane == 0 && act) atomicOr(s_act, act);
}

// Top-down part of a mixed tick t: the queue entries whose frontier mask
// holds bits of `mask` (the slots not advanced bottom-up at this tick) are
// compacted per block (each block takes an equal share of the entries) and
// their edges expanded across the block for those bits only.
__device__ void sv_tick_td_part(const Params& p, long long t, unsigned long long mask, unsigned nparts,
                                unsigned part, unsigned long long* s_msum, unsigned long long& act) {
  __shared__ int cu[kBlock];
  __shared__ unsigned long long cm[kBlock];
  __shared__ long long cb[kBlock];
  __shared__ unsigned long long ce[kBlock];
  __shared__ unsigned long long s_scan[kBlock / 32 + 1];
  const int qs = (int)(t % 4), qn = (int)((t + 1) % 4);
  const unsigned cnt = (unsigned)(ld_cg_u64(&p.ctl->q[qs]) & kCountMask);
  const unsigned i0 = (unsigned)((unsigned long long)cnt * part / nparts);
  const unsigned i1 = (unsigned)((unsigned long long)cnt * (part + 1) / nparts);
  const unsigned long long* Fc = p.F[t % 3];
  unsigned long long* Fn = p.F[(t + 1) % 3];
  for (unsigned base = i0; base < i1; base += kBlock) {
    const unsigned i = base + threadIdx.x;
    int u = 0;
    unsigned long long fu = 0, d = 0;
    long long b0 = 0;
    if (i < i1) {
      u = p.qids[qs][i];
      fu = ld_cg_u64(Fc + u) & mask;
      if (fu) {
        b0 = p.qbg[qs][i];
        d = (unsigned long long)(ld_nc_i64(p.beg + u + 1) - b0);
      }
    }
    // (edges << 16) | entries: one scan gives both positions (d < 2^32)
    unsigned long long tot = 0;
    const unsigned long long x =
        block_exclusive_scan<kBlock, unsigned long long>(fu ? (d << 16) | 1ull : 0ull, s_scan, &tot);
    if (fu) {
      const int k = (int)(x & 0xffffull);
      cu[k] = u;
      cm[k] = fu;
      cb[k] = b0;
      ce[k] = x >> 16;
    }
    __syncthreads();
    const int n = (int)(tot & 0xffffull);
    const unsigned long long T = tot >> 16;
    for (unsigned long long e0 = 0; e0 < T; e0 += kBlock) {
      const unsigned long long e = e0 + threadIdx.x;
      bool first = false;
      int v = 0;
      long long deg = 0, vb0 = 0;
      if (e < T) {
        int a = 0, c = n;
        while (c - a > 1) {
          const int mid = (a + c) >> 1;
          if (ce[mid] <= e) a = mid; else c = mid;
        }
        v = ld_stream_i32(p.csr + cb[a] + (long long)(e - ce[a]));
        first = sv_claim_m(p, t, cm[a], Fn, v, deg, vb0, act, s_msum);
      }
      sv_enqueue(p, qn, first, v, deg, vb0);
    }
    __syncthreads();
  }
}

// Bottom-up tick t for the slots in `bu` (those whose own frontier is
// large): every vertex still lacking some of them probes its neighbours'
// frontier masks until it has found all of them or runs out of neighbours.
// The slots in `td` (running, with a frontier, but a small one) advance
// top-down in the same tick: a slot whose frontier is a handful of vertices
// would otherwise make every vertex scan its whole neighbour list. The two
// parts claim disjoint bits, so visited and next-frontier words take atomic
// ORs and the OR that finds v's next mask empty queues v. Blocks take
// contiguous vertex ranges.
__device__ void sv_tick_bu(const Params& p, long long t, unsigned long long bu, unsigned long long td,
                           unsigned nparts, unsigned part, unsigned long long* s_msum, unsigned long long* s_act) {
  const int lane = threadIdx.x & 31;
  const int qn = (int)((t + 1) % 4);
  const unsigned long long* Fc = p.F[t % 3];
  unsigned long long* Fn = p.F[(t + 1) % 3];
  unsigned long long act = 0;
  if (td) sv_tick_td_part(p, t, td, nparts, part, s_msum, act);
  const long long per = (p.V + nparts - 1) / nparts;
  const long long v0 = per * part, v1 = (v0 + per < p.V) ? v0 + per : p.V;
  for (long long base = v0; base < v1; base += blockDim.x) {
    const long long v = base + threadIdx.x;
    bool have = false;
    long long deg = 0, vb0 = 0;
    if (v < v1) {
      const unsigned long long vv = ld_cg_u64(p.vis + v);
      const unsigned long long needed = bu & ~vv;
      if (needed) {
        const long long b0 = ld_nc_i64(p.beg + v), b1 = ld_nc_i64(p.beg + v + 1);
        unsigned long long got = 0;
        // four neighbours per step: their CSR entries, then their masks, are
        // loaded together, so a lane has four probes in flight
        for (long long e = b0; e < b1 && got != needed; e += 4) {
          int u[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) u[k] = (e + k < b1) ? ld_stream_i32(p.csr + e + k) : -1;
          unsigned long long f[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) f[k] = (u[k] >= 0) ? ld_cg_u64(Fc + u[k]) : 0ull;
          got |= (f[0] | f[1] | f[2] | f[3]) & needed;
        }
        if (got) {
          deg = b1 - b0;
          vb0 = b0;
          atomicOr(p.vis + v, got);
          have = atomicOr(Fn + v, got) == 0ull;
          act |= got;
          for (unsigned long long bits = got; bits; bits &= bits - 1) {
            const int sl = __ffsll((long long)bits) - 1;
            int* o = p.out[sl];
            if (o) o[v] = (int)(t + 1 - p.join[sl]);
            atomicAdd(&s_msum[sl], (unsigned long long)deg);
          }
        }
      }
    }
    sv_enqueue(p, qn, have, (int)v, deg, vb0);
  }
  act = __reduce_or_sync(0xffffffffu, (unsigned)act) |
        ((unsigned long long)__reduce_or_sync(0xffffffffu, (unsigned)(act >> 32)) << 32);
  if (lane == 0 && act) atomicOr(s_act, act);
}

// Clears the frontier masks of tick t (the vertices of queue t).
__device__ void sv_retire(const Params& p, long long t, unsigned nparts, unsigned part) {
  const int qs = (int)(t % 4);
  const unsigned cnt = (unsigned)(ld_cg_u64(&p.ctl->q[qs]) & kCountMask);
  unsigned long long* Fc = p.F[t % 3];
  for (long long i = part * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)nparts * blockDim.x)
    Fc[p.qids[qs][i]] = 0ull;
}

// One round of k ticks from t0 in one cooperative launch, one grid barrier
// per tick. During tick t the blocks also retire frontier t-1 (its mask
// buffer is neither read nor written at tick t) and block 0 resets the
// queue counter and per-slot frontier edges of tick t+2 (last used at tick
// t-2) and, inside the round, the activity word of tick t+1. Every wait is
// bounded (XBFS_ERR_DEVICE_TIMEOUT).
// A slot advances bottom-up at tick t when its own frontier's edges exceed
// E / kBuRatio, the others top-down (sv_tick_bu); with no such slot the tick
// is top-down (sv_tick). The per-slot edge counts are final after the
// previous barrier, so every block takes the same decision. `running` = the
// slots in the batch.
constexpr long long kBuRatio = 8;

__global__ void __launch_bounds__(kBlock) k_sv_round(Params p, long long t0, int k, unsigned long long timeout_ns,
                                                     unsigned long long running) {
  __shared__ unsigned long long s_msum[kSlots];
  __shared__ unsigned long long s_act;
  __shared__ unsigned s_bu[2], s_live[2];
  const unsigned G = gridDim.x, b = blockIdx.x;
  uint32_t epoch = 0;
  for (int i = 0; i < k; ++i) {
    const long long t = t0 + i;
    if (threadIdx.x < kSlots) {
      s_msum[threadIdx.x] = 0;
      const unsigned long long f = ld_cg_u64(&p.ctl->fe[t % 4][threadIdx.x]);
      const bool big = p.allow_bu && ((running >> threadIdx.x) & 1ull) && (long long)f * kBuRatio > p.E;
      const unsigned bb = __ballot_sync(0xffffffffu, big), lb = __ballot_sync(0xffffffffu, f != 0);
      if ((threadIdx.x & 31) == 0) {
        s_bu[threadIdx.x >> 5] = bb;
        s_live[threadIdx.x >> 5] = lb;
      }
      if (b == 0) p.ctl->fe[(t + 2) % 4][threadIdx.x] = 0ull;
    }
    if (threadIdx.x == 0) s_act = 0;
    if (b == 0 && threadIdx.x == 0) {
      p.ctl->q[(t + 2) % 4] = 0ull;
      // the first tick's activity word is zeroed by the host before the round
      if (i + 1 < k) p.ctl->active[(t + 1) % kRing] = 0ull;
    }
    __syncthreads();
    if (t > 0) sv_retire(p, t - 1, G, b);
    const unsigned long long bu = s_bu[0] | ((unsigned long long)s_bu[1] << 32);
    const unsigned long long live = s_live[0] | ((unsigned long long)s_live[1] << 32);
    if (bu)
      sv_tick_bu(p, t, bu, running & live & ~bu, G, b, s_msum, &s_act);
    else
      sv_tick(p, t, G, b, s_msum, &s_act);
    __syncthreads();
    if (threadIdx.x < kSlots && s_msum[threadIdx.x]) {
      atomicAdd(&p.ctl->msum[threadIdx.x], s_msum[threadIdx.x]);
      atomicAdd(&p.ctl->fe[(t + 1) % 4][threadIdx.x], s_msum[threadIdx.x]);
    }
    if (threadIdx.x == 0 && s_act) atomicOr(&p.ctl->active[t % kRing], s_act);
    if (!grid_sync(&p.ctl->bar, G, epoch, timeout_ns)) return;
  }
}

// Seed slot s at src for tick t: its output array and join tick go into the
// slot tables (kernel arguments, so the host never copies from pageable
// memory onto a stream with a round in flight), then its visited and
// frontier bit, level 0 and a queue entry.
__global__ void k_sv_seed(Params p, long long t, int s, int src, int* out) {
  if (threadIdx.x != 0) return;
  const unsigned long long bit = 1ull << s;
  p.out[s] = out;
  p.join[s] = t;
  p.vis[src] |= bit;
  if (out) out[src] = 0;
  const long long b0 = p.beg[src], d = p.beg[src + 1] - b0;
  p.ctl->msum[s] = (unsigned long long)d;
  // no earlier tick gave slot s anything for tick t; the word was reset at t-2
  p.ctl->fe[t % 4][s] = (unsigned long long)d;
  if (d == 0) return;  // nothing to expand: the request completes at its first tick
  const unsigned long long prev = p.F[t % 3][src];
  p.F[t % 3][src] = prev | bit;
  if (prev == 0) {  // queued once per tick, whatever the number of slots seeded there
    const unsigned long long old = atomicAdd(&p.ctl->q[t % 4], ((unsigned long long)d << 31) | 1ull);
    p.qids[t % 4][old & kCountMask] = src;
    p.qeb[t % 4][old & kCountMask] = (unsigned)(old >> 31);
    p.qbg[t % 4][old & kCountMask] = b0;
  }
}

// Retire the slots in mask: no output array, visited bits cleared.
__global__ void k_sv_clear(Params p, unsigned long long mask) {
  if (blockIdx.x == 0 && threadIdx.x < kSlots && ((mask >> threadIdx.x) & 1ull)) p.out[threadIdx.x] = nullptr;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < p.V; v += (long long)gridDim.x * blockDim.x) {
    const unsigned long long x = p.vis[v];
    if (x & mask) p.vis[v] = x & ~mask;
  }
}

}  // namespace sv

// ---------------------------------------------------------------------------
// Host side: the serving engine. One step (engine_step) processes the rounds
// that have ended (finished slots leave, their outputs are freed, kept or
// copied out), admits waiting requests into free slots within the HBM
// budget, and issues the next round of every batch with work. Two drivers
// share it: xbfs_serve_run replays a request trace in the caller's thread,
// and the online mode runs it in the server's own host thread, fed by
// xbfs_serve_submit and read by xbfs_serve_poll.
// ---------------------------------------------------------------------------
struct ServeRequest {
  int graph = 0;
  int src = 0;
  double arrival_us = 0;
  double admit_us = -1, finish_us = -1;
  int slot = -1;
  int* out = nullptr;          // device output (int32[V])
  long long join = 0;
  int status = 0;              // 0 waiting, 1 running, 3 copying out, 2 done, 4 dropped at stop
  unsigned long long msum = 0;
  int mode = 0;                // output: 0 freed at completion, 1 kept on the device, 2 copied to host_out
  int32_t* host_out = nullptr;
};

// Finished requests whose levels are being copied to host arrays; done when
// the event (recorded after the copies) has passed.
struct Delivery {
  cudaEvent_t ev = nullptr;
  std::vector<int> reqs;
};

struct SlotBatch {
  Graph* g = nullptr;
  cudaStream_t stream = nullptr;
  DevBuf vis, F[3], q[4], qe[4], qb[4], ctl, out_tab, join_tab;
  sv::Params p;
  long long tick = 0;
  int req_of_slot[sv::kSlots];
  unsigned long long busy = 0;
  std::deque<int> waiting;
  int k_ticks = 1;
  int depth_est = 0;             // largest depth of a request finished on this graph (0: none yet)
  int grid = 0;
  int max_coop = 0;              // blocks of k_sv_round that can be resident at once
  bool inflight = false;         // a round of ticks is on the stream
  int round_k = 0;               // its length
  long long issued = 0;          // first tick not yet issued
  cudaEvent_t ev = nullptr;      // end of the round in flight
  std::deque<Delivery> deliveries;
  std::vector<cudaEvent_t> spare;  // delivery events for reuse
};

// Traversals at least this deep mark a long-diameter graph: its rounds are
// sized from the frontier (a few SMs), since its frontier grows slowly.
constexpr int kDeepGraph = 256;

struct Server {
  int device = 0;
  std::vector<std::unique_ptr<SlotBatch>> batches;
  size_t budget = 0, in_use = 0;
  cudaMemPool_t pool = nullptr;
  // requests of the current replay, or every request submitted online
  // (a deque: references stay valid while requests are appended)
  std::deque<ServeRequest> reqs;
  long long done = 0;
  std::chrono::steady_clock::time_point t0;
  PinnedBuf hctl_buf;            // control blocks read back after each round
  // online mode
  bool online = false;
  bool stop = false;
  std::thread worker;
  std::mutex mu;                 // guards everything above while online
  std::condition_variable cv;    // submissions, completions, releases, failure
  std::vector<int> inbox;        // submitted requests not yet queued to their batch
  cudaStream_t release_stream = nullptr;  // frees of kept level arrays (xbfs_serve_release)
  xbfs_status failed = XBFS_OK;  // the worker's error, if it stopped on one
  std::string fail_msg;
  ~Server();
};

static double now_us(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
}

static xbfs_status batch_init(SlotBatch& b, Graph* g, int nsm) {
  b.g = g;
  const long long V = g->V;
  xbfs_status st;
  if ((st = b.vis.ensure(V * 8)) || (st = b.ctl.ensure(sizeof(sv::Ctl))) ||
      (st = b.out_tab.ensure(sizeof(int*) * sv::kSlots)) || (st = b.join_tab.ensure(8 * sv::kSlots)))
    return st;
  for (int i = 0; i < 3; ++i)
    if ((st = b.F[i].ensure(V * 8))) return st;
  // a tick queues each vertex at most once, plus the seeds of one round
  for (int i = 0; i < 4; ++i)
    if ((st = b.q[i].ensure((V + sv::kSlots + 1) * 4)) || (st = b.qe[i].ensure((V + sv::kSlots + 1) * 4)) ||
        (st = b.qb[i].ensure((V + sv::kSlots + 1) * 8)))
      return st;
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  XBFS_CUDA_TRY(cudaMemsetAsync(b.vis.p, 0, V * 8, b.stream));
  for (int i = 0; i < 3; ++i) XBFS_CUDA_TRY(cudaMemsetAsync(b.F[i].p, 0, V * 8, b.stream));
  XBFS_CUDA_TRY(cudaMemsetAsync(b.ctl.p, 0, sizeof(sv::Ctl), b.stream));
  XBFS_CUDA_TRY(cudaMemsetAsync(b.out_tab.p, 0, sizeof(int*) * sv::kSlots, b.stream));
  XBFS_CUDA_TRY(cudaMemsetAsync(b.join_tab.p, 0, 8 * sv::kSlots, b.stream));
  sv::Params& p = b.p;
  p.beg = g->beg.as<long long>();
  p.csr = g->csr.as<int>();
  p.V = V;
  p.E = g->E;
  p.allow_bu = g->symmetric ? 1 : 0;
  p.vis = b.vis.as<unsigned long long>();
  for (int i = 0; i < 3; ++i) p.F[i] = b.F[i].as<unsigned long long>();
  for (int i = 0; i < 4; ++i) {
    p.qids[i] = b.q[i].as<int>();
    p.qeb[i] = b.qe[i].as<unsigned>();
    p.qbg[i] = b.qb[i].as<long long>();
  }
  p.out = b.out_tab.as<int*>();
  p.join = b.join_tab.as<long long>();
  p.ctl = b.ctl.as<sv::Ctl>();
  for (int s = 0; s < sv::kSlots; ++s) b.req_of_slot[s] = -1;
  int per_sm = 0;
  XBFS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)sv::k_sv_round, sv::kBlock, 0));
  if (per_sm < 1) return set_error(XBFS_ERR_INTERNAL, "serving round kernel cannot be resident");
  b.max_coop = nsm * per_sm;
  b.grid = b.max_coop;
  XBFS_CUDA_TRY(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
  return XBFS_OK;
}

Server::~Server() {
  if (worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    worker.join();
  }
  DeviceGuard dg(device);
  for (auto& b : batches) {
    if (b->stream) {
      cudaStreamSynchronize(b->stream);
      cudaStreamDestroy(b->stream);
    }
    if (b->ev) cudaEventDestroy(b->ev);
    for (auto& d : b->deliveries) cudaEventDestroy(d.ev);
    for (cudaEvent_t e : b->spare) cudaEventDestroy(e);
  }
  if (release_stream) {
    cudaStreamSynchronize(release_stream);
    cudaStreamDestroy(release_stream);
  }
}

// Issues k ticks on the batch's stream with `grid` blocks per tick kernel
// (sized by the caller from the frontier; the kernels are grid-stride, so a
// frontier that outgrows it is still covered).
static xbfs_status batch_ticks(SlotBatch& b, int k, int grid) {
  if (grid > b.max_coop) grid = b.max_coop;
  sv::Ctl* c = b.ctl.as<sv::Ctl>();
  XBFS_CUDA_TRY(cudaMemsetAsync(&c->bar, 0, sizeof(GridBarrier), b.stream));
  XBFS_CUDA_TRY(cudaMemsetAsync(&c->active[b.tick % sv::kRing], 0, 8, b.stream));
  long long t0 = b.tick;
  unsigned long long timeout_ns = 10ull * 1000 * 1000 * 1000;
  unsigned long long running = b.busy;
  void* args[] = {&b.p, &t0, &k, &timeout_ns, &running};
  XBFS_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)sv::k_sv_round, dim3(grid), dim3(sv::kBlock), args, 0,
                                            b.stream));
  return XBFS_OK;
}

// Marks a request done (the caller notifies waiters).
static void finish_request(Server* srv, ServeRequest& r, double t) {
  r.finish_us = t;
  r.status = 2;
  srv->done += 1;
}

// One step of the engine; *active is set when anything is waiting, running
// or being copied out (so the driver keeps stepping). `oom_is_error`: a
// waiting request that only kept outputs block, with nothing running, is an
// XBFS_ERR_OOM (replay) instead of a wait for xbfs_serve_release (online).
static xbfs_status engine_step(Server* srv, bool oom_is_error, bool* active, bool* progressed) {
  const int nb = (int)srv->batches.size();
  sv::Ctl* hctl = srv->hctl_buf.as<sv::Ctl>();
  *progressed = false;
  // ---- copies to host arrays that have completed
  for (int gi = 0; gi < nb; ++gi) {
    SlotBatch& b = *srv->batches[gi];
    while (!b.deliveries.empty()) {
      Delivery& d = b.deliveries.front();
      const cudaError_t q = cudaEventQuery(d.ev);
      if (q == cudaErrorNotReady) break;
      XBFS_CUDA_TRY(q);
      const double t = now_us(srv->t0);
      for (int ri : d.reqs) finish_request(srv, srv->reqs[ri], t);
      b.spare.push_back(d.ev);
      b.deliveries.pop_front();
      *progressed = true;
    }
  }
  // ---- rounds that have ended: the slots that gained nothing at some tick
  for (int gi = 0; gi < nb; ++gi) {
    SlotBatch& b = *srv->batches[gi];
    if (!b.inflight) continue;
    const cudaError_t q = cudaEventQuery(b.ev);
    if (q == cudaErrorNotReady) continue;
    XBFS_CUDA_TRY(q);
    b.inflight = false;
    *progressed = true;
    if (hctl[gi].bar.err != 0)
      return set_error((xbfs_status)hctl[gi].bar.err, "serving round on graph %d reported %s", gi,
                       xbfs_strerror(hctl[gi].bar.err));
    const int k = b.round_k;
    unsigned long long finished = 0;
    for (int i = 0; i < k; ++i) {
      const long long t = b.tick + i;
      const unsigned long long act = hctl[gi].active[t % sv::kRing];
      // slots joined at or before t that gained nothing at t are complete
      for (unsigned long long m = b.busy & ~finished; m; m &= m - 1) {
        const int sl = __builtin_ctzll(m);
        const ServeRequest& r = srv->reqs[b.req_of_slot[sl]];
        if (r.join <= t && !((act >> sl) & 1ull)) finished |= 1ull << sl;
      }
    }
    b.tick += k;
    // a request still running after t ticks is at least t levels deep: a
    // graph whose traversals are long is known as such before any finishes
    for (unsigned long long m = b.busy & ~finished; m; m &= m - 1) {
      const ServeRequest& r = srv->reqs[b.req_of_slot[__builtin_ctzll(m)]];
      b.depth_est = std::max(b.depth_est, (int)std::min<long long>(b.tick - r.join, 1 << 30));
    }
    if (!finished) {
      // longer rounds while nothing finishes, but never beyond an eighth of
      // the depth seen on this graph (a low-diameter graph keeps short rounds,
      // so the host notices its completions within a tick or two)
      if (b.depth_est == 0 || b.k_ticks * 8 < b.depth_est) b.k_ticks = std::min(sv::kRing, b.k_ticks * 2);
      continue;
    }
    const double tf = now_us(srv->t0);
    int max_depth = 0;
    // the slots leave the tables (k_sv_clear) before their arrays are freed
    sv::k_sv_clear<<<b.grid, 256, 0, b.stream>>>(b.p, finished);
    XBFS_CUDA_TRY(cudaGetLastError());
    Delivery dl;
    for (unsigned long long m = finished; m; m &= m - 1) {
      const int sl = __builtin_ctzll(m);
      const int ri = b.req_of_slot[sl];
      ServeRequest& r = srv->reqs[ri];
      r.msum = hctl[gi].msum[sl];
      max_depth = std::max<int>(max_depth, (int)(b.tick - r.join));
      if (r.mode == 2) {  // copy to the caller's host array, then give the memory back
        XBFS_CUDA_TRY(cudaMemcpyAsync(r.host_out, r.out, (size_t)b.g->V * 4, cudaMemcpyDeviceToHost, b.stream));
        dl.reqs.push_back(ri);
        r.status = 3;
      }
      if (r.mode != 1) {
        XBFS_CUDA_TRY(cudaFreeAsync(r.out, b.stream));
        srv->in_use -= (size_t)b.g->V * 4;
        r.out = nullptr;
      }
      if (r.mode != 2) finish_request(srv, r, tf);
      b.req_of_slot[sl] = -1;
    }
    if (!dl.reqs.empty()) {
      if (b.spare.empty()) {
        cudaEvent_t e;
        XBFS_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b.spare.push_back(e);
      }
      dl.ev = b.spare.back();
      b.spare.pop_back();
      XBFS_CUDA_TRY(cudaEventRecord(dl.ev, b.stream));
      b.deliveries.push_back(std::move(dl));
    }
    b.busy &= ~finished;
    b.depth_est = std::max(b.depth_est, max_depth);
    // host every ~1/8 of the depth seen so far, at least every tick
    b.k_ticks = std::max(1, std::min(sv::kRing, b.depth_est / 8));
  }
  // ---- admission: a free slot and room in the HBM budget; a request joins
  // at the batch's next unissued tick (its seed is stream-ordered after the
  // round in flight)
  for (int gi = 0; gi < nb; ++gi) {
    SlotBatch& b = *srv->batches[gi];
    while (!b.waiting.empty() && b.busy != ~0ull) {
      const size_t need = (size_t)b.g->V * 4;
      if (srv->in_use + need > srv->budget) break;
      const int ri = b.waiting.front();
      b.waiting.pop_front();
      ServeRequest& r = srv->reqs[ri];
      const int sl = __builtin_ctzll(~b.busy);
      b.busy |= 1ull << sl;
      b.req_of_slot[sl] = ri;
      void* mem = nullptr;
      XBFS_CUDA_TRY(cudaMallocFromPoolAsync(&mem, need, srv->pool, b.stream));
      srv->in_use += need;
      r.out = (int*)mem;
      r.slot = sl;
      r.join = b.issued;
      r.admit_us = now_us(srv->t0);
      r.status = 1;
      XBFS_CUDA_TRY(cudaMemsetAsync(r.out, 0xff, need, b.stream));
      // the seed goes into tick b.issued's frontier and records the slot's
      // output array and join tick
      sv::k_sv_seed<<<1, 32, 0, b.stream>>>(b.p, b.issued, sl, r.src, r.out);
      XBFS_CUDA_TRY(cudaGetLastError());
      *progressed = true;
    }
  }
  // ---- the next round of every idle batch with running slots; the
  // resident-block budget of the device is split between the batches that
  // have work, so that their cooperative rounds can be resident together
  // (a round needing the whole device would wait for every other to end)
  int with_work = 0;
  for (int gi = 0; gi < nb; ++gi) with_work += srv->batches[gi]->busy ? 1 : 0;
  bool any = false;
  for (int gi = 0; gi < nb; ++gi) {
    SlotBatch& b = *srv->batches[gi];
    if (!b.waiting.empty() || !b.deliveries.empty()) any = true;
    if (b.inflight) {
      any = true;
      continue;
    }
    if (!b.busy) continue;
    any = true;
    const int k = std::max(1, std::min(b.k_ticks, sv::kRing - (int)(b.tick % sv::kRing)));
    // Blocks of the round: on a long-diameter graph (deep traversals seen)
    // from the frontier the round starts with, with 4x headroom for growth
    // inside the round, so such batches use a few SMs and share the GPU
    // instead of taking turns. Low-diameter graphs, whose frontier can grow a
    // thousandfold in one tick, and graphs not yet seen to be deep get every
    // resident block of their share.
    int grid = b.grid;
    if (b.tick > 0 && b.depth_est >= kDeepGraph) {
      const unsigned long long pk = hctl[gi].q[b.tick % 4];
      const unsigned long long work = std::max<unsigned long long>(pk >> 31, pk & sv::kCountMask);
      const unsigned long long want = (work * 4 + sv::kBlock * 2 - 1) / (sv::kBlock * 2);
      grid = (int)std::min<unsigned long long>((unsigned long long)b.grid, std::max<unsigned long long>(8, want));
    }
    grid = std::min(grid, std::max(8, b.max_coop / std::max(1, with_work)));
    xbfs_status st = batch_ticks(b, k, grid);
    if (st) return st;
    XBFS_CUDA_TRY(cudaMemcpyAsync(&hctl[gi], b.ctl.p, sizeof(sv::Ctl), cudaMemcpyDeviceToHost, b.stream));
    XBFS_CUDA_TRY(cudaEventRecord(b.ev, b.stream));
    b.round_k = k;
    b.issued = b.tick + k;
    b.inflight = true;
    *progressed = true;
  }
  bool running = false;
  for (int gi = 0; gi < nb; ++gi) running |= srv->batches[gi]->inflight || !srv->batches[gi]->deliveries.empty();
  if (!running && oom_is_error) {
    // nothing runs, so nothing will give memory back: a request that waits
    // can only be blocked by kept outputs
    for (int gi = 0; gi < nb; ++gi)
      if (!srv->batches[gi]->waiting.empty())
        return set_error(XBFS_ERR_OOM,
                         "kept level arrays (%zu bytes) fill the HBM budget (%zu bytes): release them, or run "
                         "with keep_outputs = 0 or 2",
                         srv->in_use, srv->budget);
  }
  *active = any;
  return XBFS_OK;
}

// Prepares a server for a run of requests (replay or online): fresh clock,
// per-batch round state, the pinned read-back buffer.
static xbfs_status engine_reset(Server* srv) {
  const int nb = (int)srv->batches.size();
  if (xbfs_status st = srv->hctl_buf.ensure(sizeof(sv::Ctl) * (size_t)nb)) return st;
  for (auto& bp : srv->batches) {
    bp->inflight = false;
    bp->issued = bp->tick;
  }
  srv->reqs.clear();
  srv->done = 0;
  srv->t0 = std::chrono::steady_clock::now();
  return XBFS_OK;
}

// The online worker: hands submitted requests to their batches and steps
// the engine while there is work; sleeps on the condition variable when
// idle. Holds the mutex except while idle or yielding between steps.
static void worker_main(Server* srv) {
  cudaSetDevice(srv->device);
  std::unique_lock<std::mutex> lk(srv->mu);
  for (;;) {
    for (int ri : srv->inbox) srv->batches[srv->reqs[ri].graph]->waiting.push_back(ri);
    srv->inbox.clear();
    bool active = false, progressed = false;
    const long long done_before = srv->done;
    const xbfs_status st = engine_step(srv, false, &active, &progressed);
    if (st) {
      srv->failed = st;
      srv->fail_msg = xbfs_last_error();
      srv->cv.notify_all();
      return;
    }
    if (srv->done != done_before) srv->cv.notify_all();
    if (!active) {
      if (srv->stop) return;
      srv->cv.wait(lk, [&] { return !srv->inbox.empty() || srv->stop; });
      continue;
    }
    if (progressed) continue;
    bool running = false;
    for (auto& b : srv->batches) running |= b->inflight || !b->deliveries.empty();
    if (running) {
      // rounds in flight: let submitters and pollers in, then poll again
      lk.unlock();
      std::this_thread::yield();
      lk.lock();
    } else if (srv->stop) {
      // only requests that kept outputs block remain, and nothing will run
      // to free memory: they are dropped
      for (auto& b : srv->batches) {
        for (int ri : b->waiting) srv->reqs[ri].status = 4;
        b->waiting.clear();
      }
      srv->cv.notify_all();
      return;
    } else {
      // waiting requests that kept outputs block: a release wakes the worker
      srv->cv.wait_for(lk, std::chrono::milliseconds(1));
    }
  }
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_serve_create(xbfs_graph* const* graphs, int32_t n, int32_t device, int64_t hbm_budget_bytes,
                              xbfs_server** out) {
  if (!graphs || n <= 0 || !out) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  DeviceGuard dg(device);
  std::unique_ptr<Server> srv(new Server());
  srv->device = device;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  for (int i = 0; i < n; ++i) {
    Graph* g = (Graph*)graphs[i];
    if (!g || g->device != device) return set_error(XBFS_ERR_INVALID_ARG, "graph %d missing or on another device", i);
    if (g->E >= (1ll << 32)) return set_error(XBFS_ERR_UNSUPPORTED, "graph %d needs E < 2^32", i);
    std::unique_ptr<SlotBatch> b(new SlotBatch());
    xbfs_status st = batch_init(*b, g, nsm);
    if (st) return st;
    srv->batches.push_back(std::move(b));
  }
  size_t fr = 0, tot = 0;
  XBFS_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
  const size_t reserve = (size_t)2 << 30;
  srv->budget = hbm_budget_bytes > 0 ? (size_t)hbm_budget_bytes : (fr > reserve ? fr - reserve : fr / 2);
  XBFS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&srv->pool, device));
  uint64_t thr = UINT64_MAX;
  XBFS_CUDA_TRY(cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &thr));
  XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&srv->release_stream, cudaStreamNonBlocking));
  // grow the pool once to room for 16 level arrays of the largest graph (at
  // most half the budget), so the first requests of a run do not pay for
  // the pool's growth; the release threshold keeps the memory in the pool
  {
    size_t vmax = 0;
    for (auto& b : srv->batches) vmax = std::max(vmax, (size_t)b->g->V * 4);
    const size_t warm = std::min(vmax * 16, srv->budget / 2);
    if (warm > 0) {
      void* mem = nullptr;
      cudaStream_t s0 = srv->batches[0]->stream;
      if (cudaMallocFromPoolAsync(&mem, warm, srv->pool, s0) == cudaSuccess) {
        XBFS_CUDA_TRY(cudaFreeAsync(mem, s0));
      } else {
        cudaGetLastError();  // not enough memory for the warm-up: the pool grows on demand instead
      }
    }
  }
  XBFS_CUDA_TRY(cudaDeviceSynchronize());
  *out = (xbfs_server*)srv.release();
  return XBFS_OK;
}

// Runs a whole request trace in real time: request i (graph[i], src[i])
// arrives arrival_us[i] microseconds after the start. Outputs: admit / finish
// times (us since start) and the Graph500 edge count of each request. With
// keep_outputs = 1, levels[i] receives a device pointer to request i's
// int32[V] level array (release with xbfs_serve_release); with 2, levels[i]
// is the caller's host array that receives the levels when the request
// finishes; otherwise outputs are freed as requests finish. *wall_us = time from start to the last completion.
xbfs_status xbfs_serve_run(xbfs_server* sh, int32_t n, const int32_t* graph, const int32_t* src,
                           const double* arrival_us, int32_t keep_outputs, double* admit_us, double* finish_us,
                           int64_t* edges_mc, int32_t** levels, double* wall_us) {
  Server* srv = (Server*)sh;
  if (!srv || n < 0 || (n > 0 && (!graph || !src || !arrival_us || !admit_us || !finish_us))) {
    return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  }
  if (srv->online) return set_error(XBFS_ERR_BUSY, "the server runs online (xbfs_serve_start): stop it first");
  if (keep_outputs < 0 || keep_outputs > 2) return set_error(XBFS_ERR_INVALID_ARG, "keep_outputs must be 0, 1 or 2");
  if (keep_outputs && !levels) return set_error(XBFS_ERR_INVALID_ARG, "keep_outputs needs levels[]");
  if (keep_outputs == 2)
    for (int i = 0; i < n; ++i)
      if (!levels[i]) return set_error(XBFS_ERR_INVALID_ARG, "request %d: no host level array", i);
  DeviceGuard dg(srv->device);
  const int nb = (int)srv->batches.size();
  for (int i = 0; i < n; ++i) {
    if (graph[i] < 0 || graph[i] >= nb) return set_error(XBFS_ERR_INVALID_ARG, "request %d: bad graph", i);
    if (src[i] < 0 || src[i] >= srv->batches[graph[i]]->g->V)
      return set_error(XBFS_ERR_INVALID_ARG, "request %d: source out of range", i);
    if ((size_t)srv->batches[graph[i]]->g->V * 4 > srv->budget)
      return set_error(XBFS_ERR_OOM, "request %d: its level array does not fit the HBM budget", i);
  }
  if (xbfs_status st = engine_reset(srv)) return st;
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) {
    ServeRequest r;
    r.graph = graph[i];
    r.src = src[i];
    r.arrival_us = arrival_us[i];
    r.mode = keep_outputs;
    r.host_out = keep_outputs == 2 ? levels[i] : nullptr;
    srv->reqs.push_back(r);
    order[i] = i;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return arrival_us[a] < arrival_us[b]; });
  size_t next = 0;
  const double last_arrival = n ? srv->reqs[order.back()].arrival_us : 0.0;
  while (srv->done < n) {
    const double now = now_us(srv->t0);
    if (now > last_arrival + 1200e6)
      return set_error(XBFS_ERR_DEVICE_TIMEOUT, "serving loop made no progress for 20 minutes");
    while (next < order.size() && srv->reqs[order[next]].arrival_us <= now) {
      srv->batches[srv->reqs[order[next]].graph]->waiting.push_back(order[next]);
      ++next;
    }
    bool active = false, progressed = false;
    if (xbfs_status st = engine_step(srv, true, &active, &progressed)) return st;
    if (!active && next < order.size()) {
      const double wait = srv->reqs[order[next]].arrival_us - now_us(srv->t0);
      if (wait > 50) {
        // spin until the next arrival: a sleep would add its wake-up delay
        // to that request's latency
        const auto until = srv->t0 + std::chrono::microseconds((long long)srv->reqs[order[next]].arrival_us);
        while (std::chrono::steady_clock::now() < until) {
        }
      }
    }
  }
  for (auto& b : srv->batches) XBFS_CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (wall_us) *wall_us = now_us(srv->t0);
  for (int i = 0; i < n; ++i) {
    admit_us[i] = srv->reqs[i].admit_us;
    finish_us[i] = srv->reqs[i].finish_us;
    if (edges_mc) edges_mc[i] = (int64_t)(srv->reqs[i].msum / 2);
    if (keep_outputs == 1) levels[i] = srv->reqs[i].out;
  }
  return XBFS_OK;
}

xbfs_status xbfs_serve_start(xbfs_server* sh) {
  Server* srv = (Server*)sh;
  if (!srv) return set_error(XBFS_ERR_INVALID_ARG, "server is NULL");
  if (srv->online) return set_error(XBFS_ERR_BUSY, "the server is already running online");
  DeviceGuard dg(srv->device);
  if (xbfs_status st = engine_reset(srv)) return st;
  srv->stop = false;
  srv->failed = XBFS_OK;
  srv->fail_msg.clear();
  srv->inbox.clear();
  srv->online = true;
  try {
    srv->worker = std::thread(worker_main, srv);
  } catch (...) {
    srv->online = false;
    return set_error(XBFS_ERR_INTERNAL, "cannot start the serving thread");
  }
  return XBFS_OK;
}

xbfs_status xbfs_serve_submit(xbfs_server* sh, int32_t graph, int32_t src, int32_t output, int32_t* levels_host,
                              int64_t* ticket) {
  Server* srv = (Server*)sh;
  if (!srv || !ticket) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  if (output < 0 || output > 2) return set_error(XBFS_ERR_INVALID_ARG, "output must be 0, 1 or 2");
  if (output == 2 && !levels_host) return set_error(XBFS_ERR_INVALID_ARG, "output 2 needs a host level array");
  std::lock_guard<std::mutex> lk(srv->mu);
  if (!srv->online) return set_error(XBFS_ERR_INVALID_ARG, "the server is not running online (xbfs_serve_start)");
  if (srv->stop) return set_error(XBFS_ERR_BUSY, "the server is stopping");
  if (srv->failed) return set_error(srv->failed, "serving thread stopped: %s", srv->fail_msg.c_str());
  const int nb = (int)srv->batches.size();
  if (graph < 0 || graph >= nb) return set_error(XBFS_ERR_INVALID_ARG, "bad graph %d", graph);
  if (src < 0 || src >= srv->batches[graph]->g->V) return set_error(XBFS_ERR_INVALID_ARG, "source out of range");
  if ((size_t)srv->batches[graph]->g->V * 4 > srv->budget)
    return set_error(XBFS_ERR_OOM, "the level array does not fit the HBM budget");
  ServeRequest r;
  r.graph = graph;
  r.src = src;
  r.arrival_us = now_us(srv->t0);
  r.mode = output;
  r.host_out = output == 2 ? levels_host : nullptr;
  srv->reqs.push_back(r);
  const int id = (int)srv->reqs.size() - 1;
  srv->inbox.push_back(id);
  *ticket = id;
  srv->cv.notify_all();
  return XBFS_OK;
}

xbfs_status xbfs_serve_poll(xbfs_server* sh, int64_t ticket, int64_t wait_us, xbfs_serve_result* out) {
  Server* srv = (Server*)sh;
  if (!srv) return set_error(XBFS_ERR_INVALID_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(srv->mu);
  if (ticket < 0 || ticket >= (int64_t)srv->reqs.size()) return set_error(XBFS_ERR_INVALID_ARG, "unknown ticket");
  auto ready = [&] { return srv->reqs[ticket].status == 2 || srv->failed != XBFS_OK; };
  if (!ready() && wait_us != 0) {
    if (wait_us < 0) srv->cv.wait(lk, ready);
    else srv->cv.wait_for(lk, std::chrono::microseconds(wait_us), ready);
  }
  const ServeRequest& r = srv->reqs[ticket];
  if (out) {
    out->struct_size = (int32_t)sizeof(xbfs_serve_result);
    out->state = r.status == 3 ? 1 : (r.status == 4 ? 3 : r.status);
    out->submit_us = r.arrival_us;
    out->admit_us = r.admit_us;
    out->finish_us = r.finish_us;
    out->edges_mc = r.status == 2 ? (int64_t)(r.msum / 2) : 0;
    out->levels_dev = (r.status == 2 && r.mode == 1) ? r.out : nullptr;
  }
  if (r.status == 2) return XBFS_OK;
  if (srv->failed) return set_error(srv->failed, "serving thread stopped: %s", srv->fail_msg.c_str());
  if (r.status == 4)
    return set_error(XBFS_ERR_OOM, "request dropped when the server stopped: kept level arrays filled the HBM budget");
  return XBFS_ERR_BUSY;
}

xbfs_status xbfs_serve_stop(xbfs_server* sh) {
  Server* srv = (Server*)sh;
  if (!srv) return set_error(XBFS_ERR_INVALID_ARG, "server is NULL");
  if (!srv->online) return XBFS_OK;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  DeviceGuard dg(srv->device);
  for (auto& b : srv->batches) XBFS_CUDA_TRY(cudaStreamSynchronize(b->stream));
  srv->online = false;
  if (srv->failed) return set_error(srv->failed, "serving thread stopped: %s", srv->fail_msg.c_str());
  return XBFS_OK;
}

xbfs_status xbfs_serve_release(xbfs_server* sh, int32_t* levels_dev, int64_t V) {
  Server* srv = (Server*)sh;
  if (!srv || !levels_dev) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(srv->device);
  std::lock_guard<std::mutex> lk(srv->mu);
  // stream-ordered free on a stream of its own: no wait for rounds in flight
  XBFS_CUDA_TRY(cudaFreeAsync(levels_dev, srv->release_stream));
  srv->in_use -= std::min<size_t>(srv->in_use, (size_t)V * 4);
  for (auto& r : srv->reqs)
    if (r.out == levels_dev) r.out = nullptr;
  srv->cv.notify_all();  // room in the budget: the worker may admit again
  return XBFS_OK;
}

// Copies a kept level array to host memory, then releases it.
xbfs_status xbfs_serve_fetch(xbfs_server* sh, int32_t* levels_dev, int64_t V, int32_t* host_out) {
  Server* srv = (Server*)sh;
  if (!srv || !levels_dev || !host_out || V <= 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(srv->device);
  XBFS_CUDA_TRY(cudaMemcpy(host_out, levels_dev, (size_t)V * 4, cudaMemcpyDeviceToHost));
  return xbfs_serve_release(sh, levels_dev, V);
}

void xbfs_serve_free(xbfs_server* sh) { delete (Server*)sh; }

}  // extern "C"
