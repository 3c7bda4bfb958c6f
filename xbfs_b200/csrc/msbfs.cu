// Batched multi-source BFS: up to 64*W sources traversed together, 64
// sources packed per uint64 word, W words per vertex (W = 1, 2, 4, 8; 512
// sources = 8 groups of 64 in one pass at W = 8).
//
// No counterpart in the reference (it runs one source per process). The
// bit-parallel formulation is the standard multi-source BFS: per vertex a
// visited word set vis[v], a frontier word set F[v] (bits that arrived at the
// current level) and an accumulator N[v]. Top-down pushes F[u] & ~vis[v] into
// N[v] with atomicOr; bottom-up lets every not-yet-complete vertex OR in the
// frontier words of its neighbours until all missing bits are found (early
// exit). Both directions are exact for every source, whatever the schedule.
//
// B200 layout: a vertex's W words are contiguous (W = 4 fills one 32-byte
// sector, so a random neighbour probe costs one sector for 256 sources);
// frontier queues carry exclusive edge offsets so top-down expansion is
// edge-balanced across the whole GPU (same scheme as the single-source
// kernel); levels are recorded as one byte (or two, for deep graphs) per
// (vertex, source) in vertex-major rows and transposed at the end into the
// per-source int32 arrays of the API with coalesced 256-byte writes.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

namespace ms {

constexpr int kBlock = 512;
constexpr int kTE = kBlock;  // edges per gather round
constexpr int kMsLight = 64;  // bottom-up: larger degrees are pulled edge-balanced
constexpr unsigned long long kCountMask = (1ull << 31) - 1;

struct Ctl {
  GridBarrier bar;
  int depth;
  unsigned long long q[3];        // packed (edges << 31) | count, frontier queue ring
  unsigned int tcount[2];         // touched-list length by level parity
  unsigned long long m_done[3];   // degree sum of vertices completed, per level ring
  unsigned long long n_done[3];
  unsigned long long heavy[2];    // packed counter of the bottom-up heavy list, by level parity
  int strat_count[2];
};

template <int W, typename RowT>
struct Params {
  const long long* beg;
  const int* csr;
  long long V, E;
  unsigned long long* vis;  // [V][W]
  unsigned long long* F[2]; // [V][W], by level parity
  unsigned long long* N;    // [V][W]
  uint32_t* touched;        // bitmap
  uint32_t* done;           // bitmap: all active sources reached (isolated + tail pre-set)
  RowT* rows;               // [V][64W]
  int* qids[3];
  unsigned* qeb[3];
  int* tlist;
  int* ulist;
  int* hq_ids;              // bottom-up heavy list
  unsigned* hq_eb;
  Ctl* ctl;
  unsigned long long full[W];
  long long nwords;
  long long m_active;       // degree sum of non-isolated vertices
  float alpha;              // top-down while m_f <= m_u / alpha
  int allow_bu;
  int force;                // -1: heuristic, 0: always top-down, 1: bottom-up whenever allowed
  unsigned long long timeout_ns;
  long long max_levels;
  int row_max;              // largest level a row element can hold
};

struct __align__(16) Smem {
  long long wbeg[kTE + 1];
  unsigned web[kTE + 1];
  int wu[kTE + 1];
  int next_s;
  int bu_next, bu_n;
  int decision;
  long long red[kBlock / 32 + 1];
};

// Warp-aggregated append to a packed (edges | count) queue.
__device__ __forceinline__ void warp_enqueue(int* ids, unsigned* eb, unsigned long long* ctr, bool have, int v,
                                             long long deg) {
  const unsigned mask = __ballot_sync(0xffffffffu, have);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  long long d = have ? deg : 0;
  long long inc = warp_inclusive_scan(d);
  const int cnt = __popc(mask);
  unsigned long long old = 0;
  const int leader = __ffs(mask) - 1;
  if (lane == 31) {
    old = atomicAdd(ctr, ((unsigned long long)inc << 31) | (unsigned long long)cnt);
  }
  old = __shfl_sync(0xffffffffu, old, 31);
  (void)leader;
  if (have) {
    const unsigned slot = (unsigned)(old & kCountMask) + __popc(mask & ((1u << lane) - 1));
    ids[slot] = v;
    eb[slot] = (unsigned)((old >> 31) + (unsigned long long)(inc - d));
  }
}

// Record level L for the sources whose bits are set in `nw` (word w of v).
template <typename RowT>
__device__ __forceinline__ void record(RowT* row, int w, unsigned long long nw, int level) {
  while (nw) {
    const int b = __ffsll((long long)nw) - 1;
    nw &= nw - 1;
    row[w * 64 + b] = (RowT)level;
  }
}

template <int W, typename RowT>
__device__ __forceinline__ void complete_vertex(const Params<W, RowT>& p, int v, const unsigned long long* nw,
                                                const unsigned long long* vis_new, int level, unsigned long long* Fn,
                                                int* qids, unsigned* qeb, unsigned long long* qctr, long long deg,
                                                long long& m_done, long long& n_done, bool& have) {
  bool any = false;
  bool full = true;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    any |= nw[w] != 0;
    full &= vis_new[w] == p.full[w];
  }
  have = any;
  if (!any) return;
  RowT* row = p.rows + (size_t)v * 64 * W;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    p.vis[(size_t)v * W + w] = vis_new[w];
    Fn[(size_t)v * W + w] = nw[w];
    if (nw[w]) record(row, w, nw[w], level);
  }
  if (full) {
    red_or_u32(p.done + (v >> 5), 1u << (v & 31));
    m_done += deg;
    n_done += 1;
  }
}

// Edge-balanced pass over a queue (ids + exclusive edge offsets). PULL =
// false: top-down, the owner's frontier bits are pushed into each
// neighbour's accumulator. PULL = true: bottom-up for heavy vertices, each
// neighbour's frontier bits are pulled into the owner's accumulator. Every
// vertex whose accumulator gains bits is appended once to the touched list.
template <int W, typename RowT, bool PULL>
__device__ void ms_gather(const Params<W, RowT>& p, Smem& sm, const int* ids, const unsigned* eb, unsigned cnt,
                          unsigned long long M, const unsigned long long* Fc, unsigned* tctr) {
  const int lane = threadIdx.x & 31;
  const unsigned long long nb = gridDim.x;
  const unsigned long long lo = M * blockIdx.x / nb, hi = M * (blockIdx.x + 1) / nb;
  if (cnt == 0 || lo >= hi) return;
  if (threadIdx.x < 32) {
    unsigned a = 0, b = cnt;
    while (b - a > 32) {
      const unsigned span = b - a;
      const unsigned piv = a + (unsigned)(((unsigned long long)span * lane) / 32);
      const unsigned m = __ballot_sync(0xffffffffu, (unsigned long long)eb[piv] <= lo);
      const int last = 31 - __clz(m);
      const unsigned na = a + (unsigned)(((unsigned long long)span * last) / 32);
      const unsigned nbb = (last == 31) ? b : a + (unsigned)(((unsigned long long)span * (last + 1)) / 32);
      a = na;
      b = nbb;
    }
    const unsigned idx = a + lane;
    const unsigned m = __ballot_sync(0xffffffffu, idx < b && (unsigned long long)eb[idx] <= lo);
    if (lane == 0) sm.next_s = (int)(a + 31 - __clz(m));
  }
  __syncthreads();
  unsigned s = (unsigned)sm.next_s;
  for (unsigned long long r = lo; r < hi; r += kTE) {
    const unsigned long long rhi = (r + kTE < hi) ? r + kTE : hi;
    for (int i = threadIdx.x; i <= kTE; i += kBlock) {
      const unsigned slot = s + (unsigned)i;
      unsigned e0 = 0xffffffffu;
      if (slot < cnt) {
        const unsigned x = eb[slot];
        if ((unsigned long long)x < rhi) {
          e0 = x;
          const int u = ids[slot];
          sm.wu[i] = u;
          sm.wbeg[i] = ld_nc_i64(p.beg + u);
        }
      }
      sm.web[i] = e0;
    }
    __syncthreads();
    const unsigned long long e = r + threadIdx.x;
    bool first = false;
    int dst = 0;
    if (e < rhi) {
      int a = 0, c = kTE + 1;
      while (c - a > 1) {
        const int mid = (a + c) >> 1;
        if ((unsigned long long)sm.web[mid] <= e) a = mid; else c = mid;
      }
      const int owner = sm.wu[a];
      const int nbr = ld_stream_i32(p.csr + sm.wbeg[a] + (long long)(e - sm.web[a]));
      const int src = PULL ? nbr : owner;
      dst = PULL ? owner : nbr;
      bool any = false;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const unsigned long long f = Fc[(size_t)src * W + w];
        if (!f) continue;
        unsigned long long m = f & ~ld_cg_u64(p.vis + (size_t)dst * W + w);
        if (PULL) m &= p.full[w];
        if (m) {
          red_or_u64(p.N + (size_t)dst * W + w, m);
          any = true;
        }
      }
      if (any) {
        const uint32_t bit = 1u << (dst & 31);
        if (!(ld_cg_u32(p.touched + (dst >> 5)) & bit)) {
          const uint32_t old = atomicOr(p.touched + (dst >> 5), bit);
          first = !(old & bit);
        }
      }
    }
    const unsigned tm = __ballot_sync(0xffffffffu, first);
    if (tm) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(tctr, (unsigned)__popc(tm));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (first) p.tlist[base + __popc(tm & ((1u << lane) - 1))] = dst;
    }
    if (threadIdx.x == 0 && rhi < hi) {
      int a = 0, c = kTE + 1;
      while (c - a > 1) {
        const int mid = (a + c) >> 1;
        if ((unsigned long long)sm.web[mid] <= rhi) a = mid; else c = mid;
      }
      sm.next_s = (int)(s + a);
    }
    __syncthreads();
    s = (unsigned)sm.next_s;
  }
}

// Merge the accumulators of the touched vertices into visited / next frontier,
// record their levels and queue the ones that gained bits.
template <int W, typename RowT>
__device__ void ms_merge(const Params<W, RowT>& p, long long L, unsigned long long* Fn, int* qout, unsigned* qeb_out,
                         unsigned long long* qctr, long long& m_done, long long& n_done) {
  const unsigned tc = ld_cg_u32(&p.ctl->tcount[L & 1]);
  const long long nth = (long long)gridDim.x * kBlock;
  for (long long i0 = blockIdx.x * (long long)kBlock; i0 < tc; i0 += nth) {
    const long long i = i0 + threadIdx.x;
    bool have = false;
    int v = 0;
    long long deg = 0;
    if (i < tc) {
      v = p.tlist[i];
      p.touched[v >> 5] = 0u;  // every touched bit of this word is merged in this phase
      unsigned long long nw[W], vn[W];
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const size_t k = (size_t)v * W + w;
        const unsigned long long a = p.N[k];
        const unsigned long long vv = p.vis[k];
        if (a) p.N[k] = 0ull;
        nw[w] = a & ~vv;
        vn[w] = vv | nw[w];
      }
      deg = ld_nc_i64(p.beg + v + 1) - ld_nc_i64(p.beg + v);
      complete_vertex<W, RowT>(p, v, nw, vn, (int)(L + 1), Fn, qout, qeb_out, qctr, deg, m_done, n_done, have);
    }
    warp_enqueue(qout, qeb_out, qctr, have && deg > 0, v, deg);
  }
}

template <int W, typename RowT>
__global__ void __launch_bounds__(kBlock, (W >= 4 ? 1 : 2)) k_msbfs(Params<W, RowT> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  Ctl* ctl = p.ctl;
  const uint32_t nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const long long gtid = blockIdx.x * (long long)kBlock + threadIdx.x;
  const long long nth = (long long)gridDim.x * kBlock;
  long long m_done_total = 0;  // thread 0 only
  uint32_t epoch = 0;
  long long L = 0;
  for (;; ++L) {
    if (L >= p.max_levels) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&ctl->bar.err, 0, (int)XBFS_ERR_INTERNAL);
      break;
    }
    const int qs = (int)(L % 3), qn = (int)((L + 1) % 3), qo = (int)((L + 2) % 3);
    const unsigned long long pk = ld_cg_u64(&ctl->q[qs]);
    const unsigned cnt = (unsigned)(pk & kCountMask);
    const unsigned long long mf = pk >> 31;
    if (threadIdx.x == 0) {
      int d = -1;
      if (cnt > 0) {
        if (L > 0) m_done_total += (long long)ld_cg_u64(&ctl->m_done[(L - 1) % 3]);
        const long long m_u = p.m_active - m_done_total;
        if (L + 1 >= p.row_max) {
          atomicCAS(&ctl->bar.err, 0, (int)XBFS_ERR_LEVEL_OVERFLOW);
          d = -1;
        } else if (p.force == 0 || !p.allow_bu) {
          d = 0;
        } else if (p.force == 1) {
          d = 1;
        } else {
          d = ((double)mf * (double)p.alpha > (double)m_u) ? 1 : 0;
        }
        if (blockIdx.x == 0 && d >= 0) ctl->strat_count[d] += 1;
      }
      sm.decision = d;
    }
    __syncthreads();
    const int D = sm.decision;
    if (D < 0) break;
    const unsigned long long* Fc = p.F[L & 1];
    unsigned long long* Fn = p.F[(L + 1) & 1];
    int* qin = p.qids[qs];
    const unsigned* qeb_in = p.qeb[qs];
    int* qout = p.qids[qn];
    unsigned* qeb_out = p.qeb[qn];
    unsigned long long* qctr = &ctl->q[qn];
    // housekeeping: reset the retired queue counter (queue L-1, last read in
    // level L-1), the touched counter of level L-1, and the completion slot
    // that level L+1 will publish into (it was last read at the start of L-1)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl->q[qo] = 0;
      ctl->tcount[(L + 1) & 1] = 0;
      ctl->m_done[qn] = 0;
      ctl->n_done[qn] = 0;
      ctl->heavy[(L + 1) & 1] = 0ull;
    }
    long long m_done = 0, n_done = 0;
    if (D == 0) {
      // ---------------- top-down: push along the edges of the frontier queue
      ms_gather<W, RowT, false>(p, sm, qin, qeb_in, cnt, mf, Fc, &ctl->tcount[L & 1]);
      if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      ms_merge<W, RowT>(p, L, Fn, qout, qeb_out, qctr, m_done, n_done);
    } else {
      // ---------------- bottom-up: light vertices search their neighbours
      // (lane per vertex, early exit); heavy ones are queued and pulled
      // edge-balanced by the whole grid after the barrier
      unsigned long long* hctr = &ctl->heavy[L & 1];
      const long long nw_ = p.nwords;
      const long long w0 = nw_ * blockIdx.x / nb, w1 = nw_ * (blockIdx.x + 1) / nb;
      int* list = p.ulist + w0 * 32;
      long long pos = 0;
      for (long long wb = w0; wb < w1; wb += kBlock) {
        const long long w = wb + threadIdx.x;
        uint32_t bits = (w < w1) ? ~ld_cg_u32(p.done + w) : 0u;
        long long total;
        const long long ex = block_exclusive_scan<kBlock, long long>((long long)__popc(bits), sm.red, &total);
        long long o = pos + ex;
        while (bits) {
          const int bp = __ffs(bits) - 1;
          bits &= bits - 1;
          list[o++] = (int)(w * 32 + bp);
        }
        pos += total;
      }
      if (threadIdx.x == 0) {
        sm.bu_next = 0;
        sm.bu_n = (int)pos;
      }
      __syncthreads();
      const int n = sm.bu_n;
      for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&sm.bu_next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int i = base + lane;
        bool have = false, heavy = false;
        int v = 0;
        long long deg = 0, e0 = 0;
        if (i < n) {
          v = list[i];
          e0 = ld_nc_i64(p.beg + v);
          deg = ld_nc_i64(p.beg + v + 1) - e0;
          heavy = deg > kMsLight;
          if (!heavy) {
            unsigned long long need[W], acc[W], vv[W];
            bool open = false;
#pragma unroll
            for (int w = 0; w < W; ++w) {
              vv[w] = p.vis[(size_t)v * W + w];
              need[w] = p.full[w] & ~vv[w];
              acc[w] = 0;
              open |= need[w] != 0;
            }
            const long long e1 = e0 + deg;
            for (long long e = e0; e < e1 && open; e += 4) {
              int u[4];
#pragma unroll
              for (int k = 0; k < 4; ++k) u[k] = (e + k < e1) ? __ldg(p.csr + e + k) : -1;
#pragma unroll
              for (int k = 0; k < 4; ++k)
                if (u[k] >= 0) {
#pragma unroll
                  for (int w = 0; w < W; ++w) acc[w] |= Fc[(size_t)u[k] * W + w];
                }
              open = false;
#pragma unroll
              for (int w = 0; w < W; ++w) {
                acc[w] &= need[w];
                open |= need[w] != acc[w];
              }
            }
            unsigned long long vn[W];
#pragma unroll
            for (int w = 0; w < W; ++w) vn[w] = vv[w] | acc[w];
            complete_vertex<W, RowT>(p, v, acc, vn, (int)(L + 1), Fn, qout, qeb_out, qctr, deg, m_done, n_done,
                                     have);
          }
        }
        warp_enqueue(qout, qeb_out, qctr, have && deg > 0, v, deg);
        warp_enqueue(p.hq_ids, p.hq_eb, hctr, heavy, v, deg);
      }
      if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      const unsigned long long hk = ld_cg_u64(hctr);
      if ((hk & kCountMask) != 0) {
        ms_gather<W, RowT, true>(p, sm, p.hq_ids, p.hq_eb, (unsigned)(hk & kCountMask), hk >> 31, Fc,
                                 &ctl->tcount[L & 1]);
        if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
        ms_merge<W, RowT>(p, L, Fn, qout, qeb_out, qctr, m_done, n_done);
      }
    }
    // publish completion statistics of this level
    {
      long long md = block_sum<kBlock, long long>(m_done, sm.red);
      long long nd = block_sum<kBlock, long long>(n_done, sm.red);
      if (threadIdx.x == 0) {
        if (md) atomicAdd(&ctl->m_done[L % 3], (unsigned long long)md);
        if (nd) atomicAdd(&ctl->n_done[L % 3], (unsigned long long)nd);
      }
    }
    if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
    // retire frontier L: clear its F entries (nobody reads them any more)
    {
      unsigned long long* Fr = p.F[L & 1];
      for (long long i = gtid; i < cnt; i += nth) {
        const int u = qin[i];
#pragma unroll
        for (int w = 0; w < W; ++w) Fr[(size_t)u * W + w] = 0ull;
      }
    }
    // sources of degree 0 are never queued and keep their F bits; no vertex has
    // them as a neighbour (bottom-up runs on symmetric graphs only), so they are
    // never read again
    if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->depth = (int)L;
}

// Seeds source s (bit s) at vertex srcs[s]; duplicate vertices merge bits.
template <int W, typename RowT>
__global__ void k_ms_seed(Params<W, RowT> p, const int* srcs, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int v = srcs[s];
  const int w = s >> 6;
  const unsigned long long bit = 1ull << (s & 63);
  atomicOr(p.vis + (size_t)v * W + w, bit);
  atomicOr(p.F[0] + (size_t)v * W + w, bit);
  p.rows[(size_t)v * 64 * W + s] = (RowT)0;
}

// Queue the distinct source vertices (after seeding) and mark complete ones.
template <int W, typename RowT>
__global__ void k_ms_seed_queue(Params<W, RowT> p, const int* srcs, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  bool have = false;
  int v = 0;
  long long deg = 0;
  if (s < n) {
    v = srcs[s];
    // the lowest source index at this vertex owns the queue entry
    bool owner = true;
    for (int t = 0; t < s; ++t)
      if (srcs[t] == v) { owner = false; break; }
    if (owner) {
      deg = p.beg[v + 1] - p.beg[v];
      have = deg > 0;
    }
  }
  warp_enqueue(p.qids[0], p.qeb[0], &p.ctl->q[0], have, v, deg);
}

// Vertex-major level rows -> per-source int32 arrays (coalesced both ways)
// and per-source Graph500 edge counts m_c.
template <typename RowT>
__global__ void k_ms_transpose(const RowT* rows, int SW, long long V, const long long* beg, int s0, int ns,
                               int* out, long long out_stride, unsigned long long* msum, int row_max) {
  __shared__ RowT tile[64][65];
  __shared__ long long degs[64];
  __shared__ unsigned long long part[64];
  const long long v0 = (long long)blockIdx.x * 64;
  const int sb = blockIdx.y * 64;  // source block within the pass
  const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;  // 256 threads: 64 x 4
  for (int r = ty; r < 64; r += 4) {
    const long long v = v0 + r;
    tile[r][tx] = (v < V && sb + tx < SW) ? rows[(size_t)v * SW + sb + tx] : (RowT)row_max;
  }
  if (threadIdx.x < 64) {
    const long long v = v0 + threadIdx.x;
    degs[threadIdx.x] = (v < V) ? beg[v + 1] - beg[v] : 0;
    part[threadIdx.x] = 0;
  }
  __syncthreads();
  for (int c = ty; c < 64; c += 4) {  // c = source within block
    const int s = s0 + sb + c;
    if (sb + c >= SW || s >= ns) continue;
    const long long v = v0 + tx;
    const RowT x = tile[tx][c];
    const int lv = (x == (RowT)row_max) ? -1 : (int)x;
    if (v < V) out[(size_t)s * out_stride + v] = lv;
    unsigned long long dsum = (lv >= 0) ? (unsigned long long)degs[tx] : 0ull;
    dsum = warp_sum(dsum);
    if ((threadIdx.x & 31) == 0) atomicAdd(&part[c], dsum);
  }
  __syncthreads();
  if (threadIdx.x < 64 && sb + threadIdx.x < SW && s0 + sb + (int)threadIdx.x < ns && part[threadIdx.x])
    atomicAdd(&msum[s0 + sb + threadIdx.x], part[threadIdx.x]);
}

}  // namespace ms

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
struct MsWorkspace {
  DevBuf vis, F0, F1, N, touched, done, rows, q[3], qe[3], tlist, ulist, ctl, srcs, msum, hq, hqe;
  size_t bytes_rows = 0;
};

static MsWorkspace& ms_ws(Graph* g) {
  static thread_local std::vector<std::pair<Graph*, MsWorkspace*>> cache;
  for (auto& c : cache)
    if (c.first == g) return *c.second;
  // one workspace per graph handle, released with the process (handles are few)
  MsWorkspace* w = new MsWorkspace();
  cache.emplace_back(g, w);
  return *w;
}

template <int W, typename RowT>
static xbfs_status run_pass(Graph* g, const int32_t* srcs, int n, int* d_out, size_t out_stride, float alpha,
                            int force, cudaStream_t s, int* depth, int* strat, unsigned long long* d_msum,
                            int s_global0, MsWorkspace& w) {
  const long long V = g->V;
  const long long nwords = (V + 31) / 32;
  const int SW = 64 * W;
  xbfs_status st;
  if ((st = w.vis.ensure((size_t)V * W * 8)) || (st = w.F0.ensure((size_t)V * W * 8)) ||
      (st = w.F1.ensure((size_t)V * W * 8)) || (st = w.N.ensure((size_t)V * W * 8)) ||
      (st = w.touched.ensure((size_t)(nwords + 64) * 4)) || (st = w.done.ensure((size_t)(nwords + 64) * 4)) ||
      (st = w.rows.ensure((size_t)V * SW * sizeof(RowT))) || (st = w.tlist.ensure((size_t)V * 4 + 4)) ||
      (st = w.ulist.ensure((size_t)(nwords + 64) * 32 * 4)) || (st = w.ctl.ensure(sizeof(ms::Ctl))) ||
      (st = w.srcs.ensure((size_t)SW * 4)) || (st = w.hq.ensure((size_t)V * 4 + 4)) ||
      (st = w.hqe.ensure((size_t)V * 4 + 4)))
    return st;
  for (int i = 0; i < 3; ++i)
    if ((st = w.q[i].ensure((size_t)V * 4 + 4)) || (st = w.qe[i].ensure((size_t)V * 4 + 4))) return st;
  ms::Params<W, RowT> p;
  memset(&p, 0, sizeof(p));
  p.beg = g->beg.as<long long>();
  p.csr = g->csr.as<int>();
  p.V = V;
  p.E = g->E;
  p.vis = w.vis.as<unsigned long long>();
  p.F[0] = w.F0.as<unsigned long long>();
  p.F[1] = w.F1.as<unsigned long long>();
  p.N = w.N.as<unsigned long long>();
  p.touched = w.touched.as<uint32_t>();
  p.done = w.done.as<uint32_t>();
  p.rows = w.rows.as<RowT>();
  for (int i = 0; i < 3; ++i) {
    p.qids[i] = w.q[i].as<int>();
    p.qeb[i] = w.qe[i].as<unsigned>();
  }
  p.tlist = w.tlist.as<int>();
  p.ulist = w.ulist.as<int>();
  p.hq_ids = w.hq.as<int>();
  p.hq_eb = w.hqe.as<unsigned>();
  p.ctl = w.ctl.as<ms::Ctl>();
  for (int k = 0; k < W; ++k) {
    const int lo = k * 64, hi = std::min(n, lo + 64);
    p.full[k] = hi <= lo ? 0ull : (hi - lo == 64 ? ~0ull : ((1ull << (hi - lo)) - 1));
  }
  p.nwords = nwords;
  // edges of non-isolated vertices
  p.m_active = g->E;
  // the single-source default (0.1) means "use the batched default": 2, the
  // best of 1..32 for 512 sources on R-MAT scale 22 at 2 and 8 words per vertex
  p.alpha = alpha > 0.5f ? alpha : 2.0f;
  p.allow_bu = g->symmetric ? 1 : 0;
  p.force = force;
  p.timeout_ns = 20ull * 1000 * 1000 * 1000;
  p.max_levels = V + 2;
  p.row_max = (int)(RowT)(~(RowT)0);  // all-ones marks "unreached"
  XBFS_CUDA_TRY(cudaMemsetAsync(p.vis, 0, (size_t)V * W * 8, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.F[0], 0, (size_t)V * W * 8, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.F[1], 0, (size_t)V * W * 8, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.N, 0, (size_t)V * W * 8, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.touched, 0, (size_t)(nwords + 64) * 4, s));
  if (g->symmetric)
    XBFS_CUDA_TRY(cudaMemcpyAsync(p.done, g->iso.p, (size_t)(nwords + 64) * 4, cudaMemcpyDeviceToDevice, s));
  else
    XBFS_CUDA_TRY(cudaMemsetAsync(p.done, 0, (size_t)(nwords + 64) * 4, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.rows, 0xff, (size_t)V * SW * sizeof(RowT), s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(ms::Ctl), s));
  XBFS_CUDA_TRY(cudaMemcpyAsync(w.srcs.p, srcs, (size_t)n * 4, cudaMemcpyHostToDevice, s));
  ms::k_ms_seed<W, RowT><<<(n + 127) / 128, 128, 0, s>>>(p, w.srcs.as<int>(), n);
  ms::k_ms_seed_queue<W, RowT><<<(n + 127) / 128 * 1, 128, 0, s>>>(p, w.srcs.as<int>(), n);
  XBFS_CUDA_TRY(cudaGetLastError());
  const void* kfn = (const void*)ms::k_msbfs<W, RowT>;
  const size_t smem = sizeof(ms::Smem);
  XBFS_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nsm = 0, per_sm = 0;
  XBFS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device));
  XBFS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, ms::kBlock, smem));
  if (per_sm < 1) return set_error(XBFS_ERR_INTERNAL, "batched kernel cannot be resident");
  void* args[] = {&p};
  XBFS_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(nsm * per_sm), dim3(ms::kBlock), args, smem, s));
  ms::Ctl hc;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&hc, p.ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  if (hc.bar.err) return set_error((xbfs_status)hc.bar.err, "batched traversal kernel reported %s", xbfs_strerror(hc.bar.err));
  *depth = std::max(*depth, hc.depth);
  strat[0] += hc.strat_count[0];
  strat[1] += hc.strat_count[1];
  dim3 tg((unsigned)((V + 63) / 64), (unsigned)((SW + 63) / 64));
  ms::k_ms_transpose<RowT><<<tg, 256, 0, s>>>(p.rows, SW, V, p.beg, s_global0, s_global0 + n, d_out, out_stride, d_msum,
                                              p.row_max);
  XBFS_CUDA_TRY(cudaGetLastError());
  return XBFS_OK;
}

template <int W>
static xbfs_status run_pass_any(Graph* g, const int32_t* srcs, int n, int* d_out, size_t stride, float alpha,
                                int force, cudaStream_t s, int* depth, int* strat, unsigned long long* d_msum,
                                int s0, MsWorkspace& w) {
  xbfs_status st = run_pass<W, uint8_t>(g, srcs, n, d_out, stride, alpha, force, s, depth, strat, d_msum, s0, w);
  if (st == XBFS_ERR_LEVEL_OVERFLOW)
    st = run_pass<W, uint16_t>(g, srcs, n, d_out, stride, alpha, force, s, depth, strat, d_msum, s0, w);
  return st;
}

xbfs_status bfs_batch(Graph* g, const int32_t* srcs, int32_t n, int32_t* levels, const xbfs_opts* uo,
                      xbfs_stats* stats, int words_per_vertex) {
  const auto t_start = std::chrono::steady_clock::now();
  if (!g || !srcs || !levels || n <= 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  for (int i = 0; i < n; ++i)
    if (srcs[i] < 0 || srcs[i] >= g->V) return set_error(XBFS_ERR_INVALID_ARG, "source %d out of range", srcs[i]);
  if (g->E >= (1ll << 32)) return set_error(XBFS_ERR_UNSUPPORTED, "batched path needs E < 2^32");
  xbfs_opts o;
  xbfs_opts_init(&o);
  if (uo) {
    if (uo->struct_size != (int32_t)sizeof(xbfs_opts)) return set_error(XBFS_ERR_INVALID_ARG, "bad opts struct_size");
    o = *uo;
  }
  int force = -1;
  if (o.policy == XBFS_POLICY_FORCED && o.forced && o.n_forced > 0) force = (o.forced[0] == XBFS_BU) ? 1 : 0;
  int W = words_per_vertex;
  if (W <= 0) W = n > 256 ? 8 : (n > 128 ? 4 : (n > 64 ? 2 : 1));
  if (W != 1 && W != 2 && W != 4 && W != 8) return set_error(XBFS_ERR_INVALID_ARG, "words per vertex must be 1, 2, 4 or 8");
  DeviceGuard dg(g->device);
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;
  MsWorkspace& w = ms_ws(g);
  const bool dev_out = is_device_pointer(levels);
  const int per_pass = 64 * W;
  DevBuf tmp_out;
  xbfs_status st;
  int* d_out = levels;
  if (!dev_out) {
    if ((st = tmp_out.ensure((size_t)std::min(n, per_pass) * g->V * 4))) return st;
    d_out = tmp_out.as<int>();
  }
  if ((st = w.msum.ensure((size_t)n * 8))) return st;
  XBFS_CUDA_TRY(cudaMemsetAsync(w.msum.p, 0, (size_t)n * 8, s));
  cudaEvent_t e0, e1;
  XBFS_CUDA_TRY(cudaEventCreate(&e0));
  XBFS_CUDA_TRY(cudaEventCreate(&e1));
  float total_ms = 0;
  int depth = 0, strat[2] = {0, 0};
  for (int s0 = 0; s0 < n; s0 += per_pass) {
    const int cnt = std::min(per_pass, n - s0);
    // out_base + s * V is the level row of global source s
    int* out_base = dev_out ? levels : d_out - (ptrdiff_t)s0 * g->V;
    unsigned long long* msum_d = w.msum.as<unsigned long long>();
    XBFS_CUDA_TRY(cudaEventRecord(e0, s));
    switch (W) {
      case 1: st = run_pass_any<1>(g, srcs + s0, cnt, out_base, g->V, o.alpha, force, s, &depth, strat, msum_d, s0, w); break;
      case 2: st = run_pass_any<2>(g, srcs + s0, cnt, out_base, g->V, o.alpha, force, s, &depth, strat, msum_d, s0, w); break;
      case 4: st = run_pass_any<4>(g, srcs + s0, cnt, out_base, g->V, o.alpha, force, s, &depth, strat, msum_d, s0, w); break;
      default: st = run_pass_any<8>(g, srcs + s0, cnt, out_base, g->V, o.alpha, force, s, &depth, strat, msum_d, s0, w); break;
    }
    if (st) break;
    XBFS_CUDA_TRY(cudaEventRecord(e1, s));
    XBFS_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    total_ms += ms;
    if (!dev_out)
      XBFS_CUDA_TRY(cudaMemcpyAsync(levels + (size_t)s0 * g->V, d_out, (size_t)cnt * g->V * 4, cudaMemcpyDeviceToHost, s));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  std::vector<unsigned long long> msum(n);
  XBFS_CUDA_TRY(cudaMemcpyAsync(msum.data(), w.msum.p, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->struct_size = (int32_t)sizeof(xbfs_stats);
    stats->depth = depth;
    unsigned long long tot = 0;
    for (auto x : msum) tot += x;
    stats->edges_mc = (int64_t)(tot / 2);
    stats->device_ms = total_ms;
    stats->kernel_ms = total_ms;
    stats->n_td_queue = strat[0];
    stats->n_bu = strat[1];
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  }
  return XBFS_OK;
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_bfs_batch(xbfs_graph* g, const int32_t* srcs, int32_t n, int32_t* levels, const xbfs_opts* opts,
                           xbfs_stats* stats) {
  return bfs_batch((Graph*)g, srcs, n, levels, opts, stats, 0);
}

xbfs_status xbfs_bfs_batch_w(xbfs_graph* g, const int32_t* srcs, int32_t n, int32_t* levels, const xbfs_opts* opts,
                             xbfs_stats* stats, int32_t words_per_vertex) {
  return bfs_batch((Graph*)g, srcs, n, levels, opts, stats, words_per_vertex);
}

}  // extern "C"
