// Single-source direction-optimising BFS on B200: one persistent cooperative
// launch runs the whole level loop on the device.
//
// Reference path replaced (hpda-lab/XBFS):
//   BFS_ControlFlow            bfs_adaptiveFQ_wb_async.cuh:934-1258  (host level loop)
//   small/medium/large_SA_TD_update   bfs_adaptiveFQ_wb_async.cuh:50-162
//   small/medium/large_SA_TD_update1  bfs_TD_scan_free.cuh:23-135
//   atomic_FQ_Generator2 + *_SA_TD_update2   bfs_single_scan.cuh:26-126
//   ballot_counting, FQ_gen    bfs_adaptiveFQ_wb_async.cuh:189-284
//   my_prefixsum / IntraBlockSum / InterBlockSum   prefix_sum1.cuh:13-108
//   thread_centric_BU_update   bfs_adaptiveFQ_wb_async.cuh:738-777
//   swap (queue ping-pong)     swap.cuh:10-15
//   switch heuristic           bfs_adaptiveFQ_wb_async.cuh:946-958, 1042-1078, 1114
//
// Design (B200-first, not a translation):
//  * The reference returns to the host every level: it sums frontier edges
//    with an O(V) host loop, copies the whole status array back and checks
//    termination against the CPU answer. Here the level loop, the statistics
//    (n_f, m_f, n_u, m_u, reduced inside the kernels) and the strategy
//    decision live on the device; levels are separated by a bounded count-up
//    grid barrier instead of a host round trip.
//  * Status is kept twice: the int32 level array (the output contract) and
//    bitmaps - visited (pre-seeded with isolated vertices) and a ring of four
//    frontier bitmaps (level L, L+1, L+2 for the asynchronous bottom-up, and
//    one being cleared). At scale 23 a bitmap is 1 MB, so random status
//    probes hit L2 (126 MB) while the CSR streams with an evict-first hint.
//  * Frontier queues are degree-binned (small / medium / large, reference
//    thresholds 32 / 256). Every entry carries the vertex, its CSR offset and
//    an exclusive edge offset, reserved with one packed 64-bit atomic
//    (edges | count). Every bin is expanded edge-balanced: each CTA takes an
//    equal slice of the bin's edge space and walks its owners through a
//    shared-memory window, so a hub with 10^5 neighbours is spread over the
//    whole GPU and a lone degree-18 source costs one round, not 18 steps of one
//    thread (the reference maps bins to thread / warp / CTA per vertex; the
//    bins survive here as the processing order and the queue split).
//  * Top-down winners are staged per CTA in shared memory and flushed with
//    one global atomic per bin per flush.
//  * A top-down level whose frontier is only in bitmap form (after bottom-up
//    or single-scan) compacts and expands the bitmap in the same phase
//    ("single scan"), CTA by CTA, instead of building a queue first.
//  * Bottom-up: every CTA compacts the unvisited vertices of its slice with
//    block ballot/popcount scans (the reference's ballot_counting + prefix
//    sum + FQ_gen, without the host round trip of my_prefixsum); its warps
//    drain the list dynamically and lanes probe 2, 4, then 8 neighbours at a
//    time with early exit and the reference's asynchronous level+2 rule.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <limits.h>

#include <algorithm>
#include <chrono>
#include <mutex>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

constexpr int kBlock = 512;         // threads per CTA of the traversal kernel
constexpr int kK = 2;               // edges per thread per gather round
constexpr int kTE = kBlock * kK;    // edges per gather round
// Shared memory is kept near 54 KB per CTA on purpose: two CTAs per SM then
// leave about 140 KB of the SM's 256 KB unified L1/shared storage to L1,
// which caches the frontier-bitmap words and CSR offsets that bottom-up
// probes read at random (doubling the staging areas cost ~30% on the
// bottom-up level of R-MAT scale 23 through the smaller L1).
#ifndef XBFS_WIN_FACTOR
#define XBFS_WIN_FACTOR 1
#endif
constexpr int kWin = XBFS_WIN_FACTOR * kTE;  // shared window / tile list capacity (at least kTE)
constexpr int kRoundsNoStage = 4;   // edge-balanced rounds with bitmap output: up to this many kTE per round
// Asynchronous bottom-up winners of sparse (list-probing) bottom-up levels
// go into frontier L+2's queue (1) or only into its bitmap (0).
#ifndef XBFS_ASYNC_QUEUE
#define XBFS_ASYNC_QUEUE 1
#endif
// Top-down levels with bitmap output, many unvisited vertices and many
// frontier edges run in two phases, marks then finalize_marks (1), or claim
// their targets with returning atomics (0).
#ifndef XBFS_TD_MARK
#define XBFS_TD_MARK 1
#endif
// A mark first reads the target's word of frontier L+1's bitmap too and
// skips the reduction when the bit is already there (1), or reduces
// whenever the target is unvisited (0: one random read per edge fewer,
// measured slightly faster on the hub levels of R-MAT scale 23).
#ifndef XBFS_MARK_FBN_CHECK
#define XBFS_MARK_FBN_CHECK 0
#endif
// Levels-only two-phase levels mark blindly (no visited test per edge) when
// frontier L+1 holds no early entries (1), or always test (0).
#ifndef XBFS_TD_BLIND
#define XBFS_TD_BLIND 1
#endif
// The head neighbours of a frontier sweep are claimed through
// claim_filtered, six visited words read together (1), or as two batches of
// three through claim_batch (0).
#ifndef XBFS_TD_HEAD_FILTER
#define XBFS_TD_HEAD_FILTER 1
#endif
// The rest of the sweep's segments is claimed through claim_filtered (1) or
// claim_batch (0).
#ifndef XBFS_TD_REM_FILTER
#define XBFS_TD_REM_FILTER 0
#endif
// Bottom-up levels with at least V / XBFS_BU_DENSE_DIV unvisited vertices
// are word-parallel, sparser ones probe a compacted list.
#ifndef XBFS_BU_DENSE_DIV
#define XBFS_BU_DENSE_DIV 4
#endif
// Two-phase levels need at least V / XBFS_MARK_NU_DIV unvisited vertices
// (and V/2 frontier edges); marking the large levels with few unvisited
// vertices too (a divisor of 2^20) measured slower on R-MAT scale 23.
#ifndef XBFS_MARK_NU_DIV
#define XBFS_MARK_NU_DIV 16
#endif
// gather_bin_warp reads a chunk of edges that lies in one segment with
// 16-byte CSR loads (1) or one 4-byte load per edge (0). Measured equal on
// the hub levels of R-MAT scale 23 (188-192 us either way): a warp's CSR
// reads are one coalesced request per 32 edges against 32 random visited-
// word reads or reductions, so the CSR is not what bounds these levels.
#ifndef XBFS_TD_VEC
#define XBFS_TD_VEC 0
#endif
// Queue-output levels of symmetric graphs take the next frontier's counts
// from its bins (1) or publish them with atomics (0).
#ifndef XBFS_NM_FROM_BINS
#define XBFS_NM_FROM_BINS 1
#endif
// Bins with bitmap output are expanded by gather_bin_warp (1) or in
// gather_bin's block rounds (0).
#ifndef XBFS_TD_WARP_GATHER
#define XBFS_TD_WARP_GATHER 1
#endif
#ifndef XBFS_TD_ILP
#define XBFS_TD_ILP 4
#endif
// Sparse (list-probing) bottom-up levels apply the asynchronous level-(L+2)
// rule when async_bu is set (1) or never (0).
#ifndef XBFS_BU_ASYNC_LIST
#define XBFS_BU_ASYNC_LIST 1
#endif
constexpr int kTdIlp = XBFS_TD_ILP; // edges per thread in flight in the barrier-free top-down loops
constexpr int kCap = 1024;          // staging capacity, small and medium bins
constexpr int kCapL = 256;          // staging capacity, large bin
constexpr int kFlushAt = kCap - kTE;  // a round adds at most kTE winners: flush before each
constexpr int kFlushAtL = kCapL / 2;  // large-bin overflow goes straight to the global queue
static_assert(kFlushAt >= 0, "a gather round must fit the staging area");
constexpr int kHeavyDeg = 4096;     // fused sweep: larger degrees are deferred to the heavy list
constexpr long long kSpecEdges = 1 << 16;  // frontiers with at most this many edges claim speculatively

constexpr unsigned long long kCountMask = (1ull << 31) - 1;

struct FDesc {
  unsigned long long bin[3];  // packed: (edges << 31) | count
  unsigned long long n;       // vertices in the frontier (degree-0 included)
  unsigned long long m;       // sum of their degrees
  unsigned long long pend_n;  // part found early by asynchronous bottom-up
  unsigned long long pend_m;
  unsigned long long pad;     // 1: n and m are not published, the bins hold the frontier
};

struct LevelRecDev {
  int strategy;
  int flags;
  long long n_f, m_f, n_u, m_u;
  unsigned long long t0, t1;
};

struct Ctl {
  GridBarrier bar;
  int depth;
  unsigned long long n_async;   // vertices given level+2 by bottom-up
  unsigned long long reached;   // sum of frontier sizes
  unsigned long long msum;      // sum of frontier degrees
  unsigned long long heavy[2];  // packed counter of the heavy list, by level parity
  int strat_count[4];
  FDesc fd[4];
};

struct QBin {
  int* ids;
  unsigned* eb;    // exclusive edge offset within the bin
  long long* bg;   // CSR offset of the vertex
};

struct Params {
  const long long* beg;
  const int* csr;
  const int4* head;  // per-vertex head records (first three neighbours, degree); null: CSR offsets only
  long long V, E;
  int* levels;
  int* parents;
  uint32_t* vis;
  uint32_t* fb[4];
  QBin q[2][3];
  QBin heavy;
  int* ulist;        // bottom-up lists, one region per CTA slice
  Ctl* ctl;
  LevelRecDev* hist;
  int hist_cap;
  const signed char* forced;
  int n_forced;
  long long nwords;  // bitmap words covering V
  long long n_ni;    // non-isolated vertices
  int policy;
  float alpha;
  int async_bu;
  int small_max, medium_max;
  float beamer_alpha, beamer_beta;
  unsigned long long timeout_ns;
  long long max_levels;
  const float* mlp;  // packed MLP weights (may be null)
  int allow_bu;      // 0 when the CSR is not symmetric: bottom-up would miss parents
  struct ResumeState* rs;  // stepped mode: state saved at stop_level / loaded when resume
  long long stop_level;
  int resume;
  int bu_mode;       // bottom-up neighbour probe shape (see probe_range)
  int absent_block;  // failure-detection test hook: CTA absent_block-1 leaves at once
  int fresh;         // 1: the launch sets up the traversal from src itself (init_traversal)
  int src;
  const uint32_t* iso;  // isolated-vertex bitmap: the initial visited set
};

__device__ __forceinline__ int bin_of(long long d, int small_max, int medium_max) {
  return d <= small_max ? 0 : (d <= medium_max ? 1 : 2);
}

// ---------------------------------------------------------------------------
// Strategy policy (computed identically by thread 0 of every CTA).
// ---------------------------------------------------------------------------
struct PolicyState {
  // reference heuristic state (bfs_adaptiveFQ_wb_async.cuh:946-1078)
  long long count_prev;
  int is_change;
  long long td_adaptive;
  long long hub_before;
  long long hub_after;
  int tag_prev;  // 0: scan-free / last-phase TD, 1: second-phase TD, -1: BU
  // Beamer
  int bu_dir;
  // features
  long long n_prev;
  int prev_strategy;
};

// Per-CTA loop state owned by thread 0 (in shared memory).
struct LoopState {
  PolicyState ps;
  long long vis_n, vis_m;  // sums over frontiers <= L
  long long pend_q_for;    // frontier whose early (asynchronous bottom-up) entries are also queued
  // statistics of the whole traversal (used by block 0)
  unsigned long long st_reached, st_msum, st_async;
  int st_strat[3];
};

// ---------------------------------------------------------------------------
// Shared memory layout of the traversal kernel (dynamic).
// ---------------------------------------------------------------------------
struct __align__(16) Smem {
  long long wbeg[kWin + 1];   // window / tile: CSR offsets
  unsigned web[kWin + 1];     // window / tile: edge offsets
  int wu[kWin + 1];           // window / tile: vertices (also the bottom-up list)
  int st_id[2][kCap];
  int st_deg[2][kCap];
  long long st_bg[2][kCap];
  int stl_id[kCapL];
  int stl_deg[kCapL];
  long long stl_bg[kCapL];
  int cnt[3];
  int strategy;
  int spec;                     // this level's frontier is small: speculative claims
  int next_s;
  int bu_next;
  int bu_n;
  int bu_dense;                 // this level's unvisited vertices are at least a quarter of V
  int mark_ok;                  // many unvisited vertices and frontier edges: a bitmap-output level runs in two phases
  int qside_ok;                 // few unvisited vertices and every early next-frontier entry queued:
                                // a top-down level with bitmap output also fills the next queue
  int asyncq_ok;                // a sparse bottom-up level: its asynchronous winners are queued
  int chunk;
  unsigned long long bins[3];   // F_L bin counters, read once per level
  long long pend_next;          // F_{L+1} entries already found (async bottom-up)
  unsigned long long base_slot, base_edge;
  long long red[kBlock / 32 + 1];
  long long red4[4 * (kBlock / 32)];
  float mlp_raw[8];             // statistics the learned switch's features come from
  float mlp_cache_raw[8];       // statistics of its last evaluation
  int mlp_cache_dec;            // and its decision (-1: none yet)
  float mlp_cache_margin;       // and that decision's margin
  float mlp_q[8];               // sensitivity bound per feature over the feature's scale
  LoopState ls;
  float mlp_w[1472];            // the learned switch's weights and bound (XBFS_POLICY_MLP); must stay last
};

// Loop state carried across launches in stepped mode (xbfs_level_costs): a
// launch stops at the top of level `stop_level` and the next one resumes there.
struct ResumeState {
  long long L;
  int q_valid, b_valid;
  unsigned dirty;
  long long vis_n, vis_m;
  long long pend_q_for;
  PolicyState ps;
};

constexpr long long kInfinite = 10000;  // bfs_adaptiveFQ_wb_async.cuh:29

// The reference's switch restated on device statistics. The reference
// computes count[level] = sum of degrees of status==level vertices with a host
// sweep (cuh:1042-1046); here that number is m_f, reduced inside the kernels.
__device__ int decide_reference(PolicyState& ps, long long L, long long m_f, long long E, float alpha) {
  const long long cnt = m_f;
  if (!ps.is_change) {
    if (L == 0 && cnt >= kInfinite) {
      ps.is_change = 1;
      ps.td_adaptive = L + 1;
    } else if (L > 0 && ps.count_prev >= kInfinite && cnt >= kInfinite * 10 &&
               cnt / ps.count_prev >= 8) {
      ps.is_change = 1;
      ps.td_adaptive = L;
    } else if ((L > 0 && cnt >= kInfinite * 100) ||
               (L > 0 && ps.count_prev < kInfinite && cnt >= kInfinite * 10 && ps.count_prev > 0 &&
                cnt / ps.count_prev >= 1000)) {
      ps.is_change = 1;
      ps.td_adaptive = L;
    }
  }
  const float ratio = (float)cnt / (float)(E > 0 ? E : 1);
  if (ratio >= alpha && ps.tag_prev >= 0) ps.hub_before = L;
  if (ratio < alpha && ps.tag_prev == -1) ps.hub_after = L;
  int s;
  if (ratio < alpha) {
    if (ps.hub_before == 0 && L < ps.td_adaptive) {
      s = XBFS_TD_QUEUE;  // scan-free top-down (cuh:1078-1110)
      ps.tag_prev = 0;
    } else if (ps.hub_after > 0 && L > ps.hub_after) {
      s = XBFS_TD_QUEUE;  // "last phase" top-down (cuh:1114-1125)
      ps.tag_prev = 0;
    } else {
      s = XBFS_TD_SCAN;   // "second phase" single-scan top-down (cuh:1128-1153)
      ps.tag_prev = 1;
    }
  } else {
    s = XBFS_BU;
    ps.tag_prev = -1;
  }
  ps.count_prev = cnt;
  return s;
}

__device__ int decide_beamer(PolicyState& ps, long long n_f, long long m_f, long long m_u, long long V,
                             float a, float b) {
  if (!ps.bu_dir) {
    if ((double)m_f > (double)m_u / (double)a) ps.bu_dir = 1;
  } else {
    if ((double)n_f < (double)V / (double)b) ps.bu_dir = 0;
  }
  return ps.bu_dir ? XBFS_BU : XBFS_TD_QUEUE;
}

// MLP inference (8 -> 32 -> 32 -> 3), one warp, from a shared-memory copy of
// the weights made once per launch (mlp_stage). The packed global layout is
// [mean 8][std 8][W1 32x8][b1 32][W2 32x32][b2 32][W3 3x32][b3 3]; in shared
// memory W1 and W2 are stored transposed (input-major), so that lane j
// reading row j of either walks consecutive banks instead of one bank.
constexpr int kMlpParams = 16 + 256 + 32 + 1024 + 32 + 96 + 3;  // 1459
constexpr int kMlpStaged = kMlpParams + 8;  // + the per-feature sensitivity bound set at installation

static_assert(kMlpStaged <= 1472, "the staged weights must fit Smem::mlp_w");

__device__ void mlp_stage(const float* __restrict__ w, float* sw) {
  for (int t = threadIdx.x; t < kMlpStaged; t += blockDim.x) {
    int d = t;
    if (t >= 16 && t < 16 + 256) {  // W1[j][i] -> W1T[i][j]
      const int j = (t - 16) / 8, i = (t - 16) % 8;
      d = 16 + i * 32 + j;
    } else if (t >= 304 && t < 304 + 1024) {  // W2[j][i] -> W2T[i][j]
      const int j = (t - 304) / 32, i = (t - 304) % 32;
      d = 304 + i * 32 + j;
    }
    sw[d] = w[t];
  }
}

// Features (log1p of n_f, m_f, n_u, m_u and the level; the previous
// strategy; log growth of the frontier; log1p of its mean degree), one per
// lane, then the three layers with the hidden activations passed by shuffles.
// Called by one full warp.
// Certified reuse (mlp_reuse_bound, per CTA, in shared memory): the last
// evaluation's statistics, class and margin (its logit minus the best other,
// less a rounding allowance) are kept. With P the per-feature sensitivity
// bound installed with the weights, no logit difference can have moved by
// more than sum_i P[i] |x_i - x_last_i| over the normalised features x;
// while a bound of that sum computed from the raw statistics stays below the
// margin the network would pick the same class, and thread 0 reuses it
// without running the layers or a second block barrier. Long runs of similar
// levels (a grid's ring of a few thousand vertices growing by a few per
// level) then cost a few scalar operations, and decisions are those of
// evaluating the network at every level.
__device__ int mlp_decide(const float* sw, const float* raw, int lane, float* cache_raw, int* cache_dec,
                          float* cache_margin) {
  const float* mean = sw;
  const float* sd = sw + 8;
  const float* W1T = sw + 16;
  const float* B1 = W1T + 256;
  const float* W2T = B1 + 32;
  const float* B2 = W2T + 1024;
  const float* W3 = B2 + 32;
  const float* B3 = W3 + 96;
  float f = 0.f;
  if (lane < 8) {
    const float r = raw[lane];
    if (lane == 5) f = r;
    else if (lane == 6) f = logf(raw[0] + 1.f) - logf(raw[6] + 1.f);
    else f = log1pf(r > 0.f ? r : 0.f);
    f = (f - mean[lane]) / sd[lane];
  }
  float a = B1[lane];
#pragma unroll
  for (int i = 0; i < 8; ++i) a = fmaf(W1T[i * 32 + lane], __shfl_sync(0xffffffffu, f, i), a);
  a = fmaxf(a, 0.f);
  // four independent accumulators shorten the dependent FMA chain of layer 2
  float bq[4] = {B2[lane], 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 32; ++i) bq[i & 3] = fmaf(W2T[i * 32 + lane], __shfl_sync(0xffffffffu, a, i), bq[i & 3]);
  const float b = fmaxf((bq[0] + bq[1]) + (bq[2] + bq[3]), 0.f);
  float o[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = warp_sum(W3[k * 32 + lane] * b) + B3[k];
  int best = 0;
  if (o[1] > o[best]) best = 1;
  if (o[2] > o[best]) best = 2;
  const int o1 = best == 0 ? 1 : 0, o2 = best == 2 ? 1 : 2;
  const float second = fmaxf(o[o1], o[o2]);
  // rounding allowance: the logits are float sums of a few dozen terms
  const float slack = 1e-4f * (fabsf(o[best]) + fabsf(second) + 1.f);
  __syncwarp();
  if (lane < 8) cache_raw[lane] = raw[lane];
  if (lane == 0) {
    *cache_dec = best;
    *cache_margin = o[best] - second - slack;
  }
  __syncwarp();
  return best;
}


// Upper bound (with a rounding allowance) of sum_i P[i] |x_i - x_last_i| from
// the raw statistics a (now) and b (last evaluation), q[i] = P[i] / scale_i:
// |log1p(u) - log1p(v)| <= |u - v| / (1 + min(u, v)) for the log features;
// the growth feature log1p(n_f) - log1p(n_prev) moves by at most the sum of
// its two terms' moves; the previous strategy enters as it is.
__device__ __forceinline__ float mlp_dlog1p(float u, float v) {
  u = fmaxf(u, 0.f);
  v = fmaxf(v, 0.f);
  return __fdividef(fabsf(u - v), 1.f + fminf(u, v));  // approximate: the sum's allowance below covers it
}
__device__ float mlp_reuse_bound(const float* a, const float* b, const float* q) {
  const float d0 = mlp_dlog1p(a[0], b[0]);
  float t = q[0] * d0 + q[1] * mlp_dlog1p(a[1], b[1]) + q[2] * mlp_dlog1p(a[2], b[2]) +
            q[3] * mlp_dlog1p(a[3], b[3]) + q[4] * mlp_dlog1p(a[4], b[4]) + q[5] * fabsf(a[5] - b[5]) +
            q[6] * (d0 + mlp_dlog1p(a[6], b[6])) + q[7] * mlp_dlog1p(a[7], b[7]);
  return t * 1.01f + 1e-6f;
}

// ---------------------------------------------------------------------------
// Staging of top-down winners (per CTA) and flush to the global binned queue.
// ---------------------------------------------------------------------------
struct QOut {
  QBin b[3];
  unsigned long long* ctr;  // fd[..].bin
};

__device__ __forceinline__ void direct_enqueue(const QBin& q, unsigned long long* ctr, int v, long long d,
                                               long long bg) {
  const unsigned long long old = atomicAdd(ctr, ((unsigned long long)d << 31) | 1ull);
  const unsigned long long slot = old & kCountMask;
  q.ids[slot] = v;
  q.eb[slot] = (unsigned)(old >> 31);
  q.bg[slot] = bg;
}

// Vertices of the lanes with `have` (degree d > 0, CSR offset b0) into a
// binned queue: per bin one packed atomic for the warp (edges << 31 |
// count), entries at consecutive slots. Called by a full warp.
__device__ __forceinline__ void enqueue_warp(const Params& p, const QOut& q2, bool have, int v, long long d,
                                             long long b0) {
  const int lane = threadIdx.x & 31;
  have = have && d > 0;
  if (!__ballot_sync(0xffffffffu, have)) return;
  const int bin = have ? bin_of(d, p.small_max, p.medium_max) : -1;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const bool mine = bin == b;
    const unsigned mask = __ballot_sync(0xffffffffu, mine);
    if (!mask) continue;
    const long long dd = mine ? d : 0;
    const long long inc = warp_inclusive_scan(dd);
    unsigned long long old = 0;
    if (lane == 31) old = atomicAdd(&q2.ctr[b], ((unsigned long long)inc << 31) | (unsigned long long)__popc(mask));
    old = __shfl_sync(0xffffffffu, old, 31);
    if (mine) {
      const unsigned long long slot = (old & kCountMask) + __popc(mask & ((1u << lane) - 1));
      q2.b[b].ids[slot] = v;
      q2.b[b].eb[slot] = (unsigned)((old >> 31) + (unsigned long long)(inc - dd));
      q2.b[b].bg[slot] = b0;
    }
  }
}

__device__ __forceinline__ void stage(Smem& sm, const QOut& q, int bin, int v, long long d, long long bg) {
  const int slot = atomicAdd(&sm.cnt[bin], 1);
  if (bin < 2) {
    if (slot < kCap) {
      sm.st_id[bin][slot] = v;
      sm.st_deg[bin][slot] = (int)d;
      sm.st_bg[bin][slot] = bg;
      return;
    }
  } else if (slot < kCapL) {
    sm.stl_id[slot] = v;
    sm.stl_deg[slot] = (int)d;
    sm.stl_bg[slot] = bg;
    return;
  }
  direct_enqueue(q.b[bin], &q.ctr[bin], v, d, bg);
}

// Block-wide flush of all staged winners (call from all threads, uniform).
__device__ void flush(Smem& sm, const QOut& q) {
  __syncthreads();
  for (int bin = 0; bin < 3; ++bin) {
    const int cap = bin < 2 ? kCap : kCapL;
    int n = sm.cnt[bin];
    if (n > cap) n = cap;
    if (n == 0) continue;
    const int* ids = bin < 2 ? sm.st_id[bin] : sm.stl_id;
    const int* degs = bin < 2 ? sm.st_deg[bin] : sm.stl_deg;
    const long long* bgs = bin < 2 ? sm.st_bg[bin] : sm.stl_bg;
    constexpr int PER = (kCap + kBlock - 1) / kBlock;
    const int i0 = threadIdx.x * PER;
    long long loc = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k)
      if (i0 + k < n) loc += degs[i0 + k];
    long long total;
    const long long ex = block_exclusive_scan<kBlock, long long>(loc, sm.red, &total);
    if (threadIdx.x == 0) {
      const unsigned long long old =
          atomicAdd(&q.ctr[bin], ((unsigned long long)total << 31) | (unsigned long long)n);
      sm.base_slot = old & kCountMask;
      sm.base_edge = old >> 31;
    }
    __syncthreads();
    const unsigned long long bs = sm.base_slot, be = sm.base_edge;
    long long run = ex;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = i0 + k;
      if (i < n) {
        q.b[bin].ids[bs + i] = ids[i];
        q.b[bin].eb[bs + i] = (unsigned)(be + run);
        q.b[bin].bg[bs + i] = bgs[i];
        run += degs[i];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) sm.cnt[bin] = 0;
    __syncthreads();
  }
}

__device__ __forceinline__ bool need_flush(const Smem& sm) {
  return sm.cnt[0] >= kFlushAt || sm.cnt[1] >= kFlushAt || sm.cnt[2] >= kFlushAtL;
}

// ---------------------------------------------------------------------------
// Per-thread statistics for the frontier being produced.
// ---------------------------------------------------------------------------
struct Acc {
  long long n1, m1;  // level+1 winners
  long long n2, m2;  // level+2 (asynchronous bottom-up)
};

// Top-down claim of v (reached from u) for level L+1.
// On a large frontier most edges lead to visited vertices, so a plain read of
// the visited word filters them before the atomic; on a small one (spec) the
// latency of each level is what counts: the claim goes straight to the atomic
// and the vertex's CSR offsets are loaded alongside it, before it is known
// whether this thread wins.
template <bool PAR>
__device__ __forceinline__ void claim_td(const Params& p, Smem& sm, const QOut& q, Acc& acc, int v, int u,
                                         int L, bool enq, uint32_t* fbn, bool spec, bool qside = false) {
  const uint32_t word = (uint32_t)v >> 5, bit = 1u << (v & 31);
  long long b0 = 0, b1 = 0;
  if (spec) {
    b0 = ld_nc_i64(p.beg + v);
    b1 = ld_nc_i64(p.beg + v + 1);
  } else if (ld_cg_u32(p.vis + word) & bit) {
    return;
  }
  const uint32_t old = atomicOr(p.vis + word, bit);
  if (old & bit) return;
  p.levels[v] = L + 1;
  if (PAR) p.parents[v] = u;
  if (!spec) {
    b0 = ld_nc_i64(p.beg + v);
    b1 = ld_nc_i64(p.beg + v + 1);
  }
  const long long d = b1 - b0;
  acc.n1 += 1;
  acc.m1 += d;
  if (enq) {
    if (d > 0) stage(sm, q, bin_of(d, p.small_max, p.medium_max), v, d, b0);
  } else {
    red_or_u32(fbn + word, bit);
    if (qside && d > 0) {
      const int bin = bin_of(d, p.small_max, p.medium_max);
      direct_enqueue(q.b[bin], &q.ctr[bin], v, d, b0);
    }
  }
}

// Top-down claims of kTdIlp targets v[k] (reached from u[k]; v[k] < 0: none)
// for level L+1 with bitmap output, all in flight together: the visited
// words, then the atomics of the targets that looked unvisited, then the
// winners' writes and CSR offsets (for the frontier statistics). Same rules
// as claim_td; the independent loads and atomics of different targets
// overlap, and the offsets are read for winners only: on a level where many
// edges race for the same fresh targets, reading them for every candidate
// (claim_td's speculative order) costs a random DRAM sector per losing edge.
template <bool PAR, int N>
__device__ __forceinline__ void claim_batch(const Params& p, Acc& acc, const int (&v)[N], const int (&u)[N], int L,
                                            uint32_t* fbn, const QOut& q, bool qside) {
  uint32_t vw[N];
#pragma unroll
  for (int k = 0; k < N; ++k) vw[k] = (v[k] >= 0) ? ld_cg_u32(p.vis + (v[k] >> 5)) : ~0u;
  bool win[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    win[k] = false;
    if (v[k] >= 0 && !((vw[k] >> (v[k] & 31)) & 1u)) {
      const uint32_t bit = 1u << (v[k] & 31);
      win[k] = (atomicOr(p.vis + (v[k] >> 5), bit) & bit) == 0;
    }
  }
  long long b0[N], d[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    b0[k] = 0;
    d[k] = 0;
    if (!win[k]) continue;
    p.levels[v[k]] = L + 1;
    if (PAR) p.parents[v[k]] = u[k];
    red_or_u32(fbn + (v[k] >> 5), 1u << (v[k] & 31));
    b0[k] = ld_nc_i64(p.beg + v[k]);
    d[k] = ld_nc_i64(p.beg + v[k] + 1) - b0[k];
  }
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (win[k]) {
      acc.n1 += 1;
      acc.m1 += d[k];
      if (qside && d[k] > 0) {
        const int bin = bin_of(d[k], p.small_max, p.medium_max);
        direct_enqueue(q.b[bin], &q.ctr[bin], v[k], d[k], b0[k]);
      }
    }
}

// Top-down claims of N targets where few are expected to be unvisited (the
// head neighbours of a frontier sweep late in the traversal): the visited
// words of all N are read together, and the targets that look unvisited are
// then claimed one after another (the atomic, the winner's writes and CSR
// offsets), which keeps fewer registers live than claim_batch.
template <bool PAR, int N>
__device__ __forceinline__ void claim_filtered(const Params& p, Acc& acc, const int (&v)[N], const int (&u)[N], int L,
                                               uint32_t* fbn, const QOut& q, bool qside) {
  uint32_t vw[N];
#pragma unroll
  for (int k = 0; k < N; ++k) vw[k] = (v[k] >= 0) ? ld_cg_u32(p.vis + (v[k] >> 5)) : ~0u;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    if (v[k] < 0 || ((vw[k] >> (v[k] & 31)) & 1u)) continue;
    const uint32_t bit = 1u << (v[k] & 31);
    if (atomicOr(p.vis + (v[k] >> 5), bit) & bit) continue;
    p.levels[v[k]] = L + 1;
    if (PAR) p.parents[v[k]] = u[k];
    red_or_u32(fbn + (v[k] >> 5), bit);
    const long long b0 = ld_nc_i64(p.beg + v[k]);
    const long long d = ld_nc_i64(p.beg + v[k] + 1) - b0;
    acc.n1 += 1;
    acc.m1 += d;
    if (qside && d > 0) {
      const int bin = bin_of(d, p.small_max, p.medium_max);
      direct_enqueue(q.b[bin], &q.ctr[bin], v[k], d, b0);
    }
  }
}

// Marking form of claim_batch for a top-down level with many fresh targets
// (two-phase level): a target that is not visited (and, with
// XBFS_MARK_FBN_CHECK, not yet in frontier L+1's bitmap) gets its bit there
// by a reduction (no return value, so no thread waits on it), and with PAR
// its parent is stored: every edge that
// passes the test comes from frontier L, so whichever store lands last is a
// valid parent. Nothing else is written; finalize_marks then turns the new
// bits that no claim of the same level took (claims set the visited bit at
// once) into levels, visited bits and frontier statistics. A target may
// pass the test on several edges before the first reduction lands: its bit
// is just set more than once.
template <bool PAR, int N>
__device__ __forceinline__ void mark_batch(const Params& p, const int (&v)[N], const int (&u)[N], uint32_t* fbn,
                                           int mark) {
  if (!PAR && mark == 2) {
    // blind marks (see finalize_marks): no test at all
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (v[k] >= 0) red_or_u32(fbn + (v[k] >> 5), 1u << (v[k] & 31));
    return;
  }
  uint32_t vw[N], fw[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    vw[k] = (v[k] >= 0) ? ld_cg_u32(p.vis + (v[k] >> 5)) : ~0u;
    fw[k] = (XBFS_MARK_FBN_CHECK && v[k] >= 0) ? ld_cg_u32(fbn + (v[k] >> 5)) : 0u;
  }
#pragma unroll
  for (int k = 0; k < N; ++k) {
    if (v[k] < 0) continue;
    const uint32_t bit = 1u << (v[k] & 31);
    if ((vw[k] | fw[k]) & bit) continue;
    red_or_u32(fbn + (v[k] >> 5), bit);
    if (PAR) p.parents[v[k]] = u[k];
  }
}

// Warp-parallel search: last slot s in [0, cnt) with eb[s] <= key (eb strictly
// increasing from eb[0] = 0 <= key). Called by a full warp.
__device__ int find_owner(const unsigned* eb, unsigned cnt, unsigned long long key) {
  const int lane = threadIdx.x & 31;
  unsigned lo = 0, hi = cnt;  // answer in [lo, hi)
  while (hi - lo > 32) {
    const unsigned span = hi - lo;
    const unsigned piv = lo + (unsigned)(((unsigned long long)span * lane) / 32);
    const bool le = (unsigned long long)eb[piv] <= key;
    const unsigned mask = __ballot_sync(0xffffffffu, le);
    const int last = 31 - __clz(mask);  // lane 0 always true (eb[lo] <= key)
    const unsigned nlo = lo + (unsigned)(((unsigned long long)span * last) / 32);
    const unsigned nhi = (last == 31) ? hi : lo + (unsigned)(((unsigned long long)span * (last + 1)) / 32);
    lo = nlo;
    hi = nhi;
  }
  const unsigned idx = lo + lane;
  const bool le = idx < hi && (unsigned long long)eb[idx] <= key;
  const unsigned mask = __ballot_sync(0xffffffffu, le);
  return (int)(lo + 31 - __clz(mask));
}

// last index a in [0, n) with web[a] <= e (web non-decreasing, web[0] <= e)
__device__ __forceinline__ int smem_owner(const unsigned* web, int n, unsigned long long e) {
  int a = 0, c = n;
  while (c - a > 1) {
    const int mid = (a + c) >> 1;
    if ((unsigned long long)web[mid] <= e) a = mid; else c = mid;
  }
  return a;
}

// Edge-balanced expansion of a bin (or the heavy list) with bitmap output,
// barrier-free: the CTA's share of the bin's edges is split evenly between
// its warps, and each warp walks its range with the 32 bin entries that own
// the next edges held one per lane (vertex, CSR offset, first edge), kTdIlp
// edges per lane in flight; an edge's owner is found by a search over the
// lanes. The entries are reloaded only when the range passes the 32nd.
template <bool PAR>
__device__ void gather_bin_warp(const Params& p, Acc& acc, const QOut& q, const QBin& in, unsigned cnt,
                                unsigned long long M, int L, uint32_t* fbn, bool qside, int mark) {
  if (cnt == 0 || M == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kBlock / 32;
  const unsigned long long NW = (unsigned long long)gridDim.x * NWARP, gw = (unsigned long long)blockIdx.x * NWARP + warp;
  const unsigned long long lo = M * gw / NW, hi = M * (gw + 1) / NW;
  if (lo >= hi) return;
  unsigned s = (unsigned)find_owner(in.eb, cnt, lo);
  for (unsigned long long r = lo; r < hi;) {
    // entries s .. s + 31, one per lane, and the first edge past them
    const unsigned slot = s + (unsigned)lane;
    const unsigned eb = slot < cnt ? in.eb[slot] : 0xffffffffu;
    const int id = slot < cnt ? in.ids[slot] : 0;
    const long long bg = slot < cnt ? in.bg[slot] : 0;
    unsigned long long wend = M;
    if (lane == 31 && slot + 1 < cnt) wend = in.eb[slot + 1];
    wend = __shfl_sync(0xffffffffu, wend, 31);
    const unsigned long long rend = wend < hi ? wend : hi;
    for (; r < rend;) {
      int v[kTdIlp], u[kTdIlp];
      const unsigned long long cend = r + 32 * kTdIlp < rend ? r + 32 * kTdIlp : rend;
      int o0 = 0, o1 = 0;  // owners of the chunk's first and last edges
      if (XBFS_TD_VEC) {
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const unsigned x0 = __shfl_sync(0xffffffffu, eb, o0 + st);
          const unsigned x1 = __shfl_sync(0xffffffffu, eb, o1 + st);
          if ((unsigned long long)x0 <= r) o0 += st;
          if ((unsigned long long)x1 <= cend - 1) o1 += st;
        }
      }
      if (XBFS_TD_VEC && kTdIlp == 4 && o0 == o1) {
        // one segment: 16-byte loads from the aligned CSR index at or below
        // the chunk's first edge, lane l the four entries from 4l; the
        // chunk ends where the 32 vectors end
        const unsigned xo = __shfl_sync(0xffffffffu, eb, o0);
        const long long bo = __shfl_sync(0xffffffffu, bg, o0);
        const int uo = __shfl_sync(0xffffffffu, id, o0);
        const long long a0 = bo + (long long)(r - xo), aend = a0 + (long long)(cend - r);
        const long long al = a0 & ~3ll, my = al + 4 * lane;
        int4 x = make_int4(-1, -1, -1, -1);
        if (my < aend) x = ld_stream_v4(p.csr + my);
        const int xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int k = 0; k < kTdIlp; ++k) {
          v[k] = (my + k >= a0 && my + k < aend) ? xs[k] : -1;
          u[k] = uo;
        }
        const long long cov = (al + 32 * kTdIlp < aend ? al + 32 * kTdIlp : aend) - a0;
        r += (unsigned long long)cov;
      } else {
#pragma unroll
        for (int k = 0; k < kTdIlp; ++k) {
          const unsigned long long e = r + 32 * k + lane;
          int o = 0;  // last lane whose entry starts at or before e
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const unsigned x = __shfl_sync(0xffffffffu, eb, o + st);
            if ((unsigned long long)x <= e) o += st;
          }
          const unsigned xo = __shfl_sync(0xffffffffu, eb, o);
          const long long bo = __shfl_sync(0xffffffffu, bg, o);
          u[k] = __shfl_sync(0xffffffffu, id, o);
          v[k] = e < rend ? ld_stream_i32(p.csr + bo + (long long)(e - xo)) : -1;
        }
        r = cend;
      }
      if (mark)
        mark_batch<PAR>(p, v, u, fbn, mark);
      else
        claim_batch<PAR>(p, acc, v, u, L, fbn, q, qside);
    }
    if (rend < hi) {
      r = rend;
      s += 32;
    }
  }
}

// Edge-balanced expansion of one bin of the current frontier queue (medium
// and large bins, and the heavy list of a fused sweep).
template <bool PAR>
__device__ void gather_bin(const Params& p, Smem& sm, const QOut& q, Acc& acc, const QBin& in, unsigned cnt,
                           unsigned long long M, int L, bool enq, uint32_t* fbn, bool qside, int mark = 0) {
  if (cnt == 0 || M == 0) return;
  if (!enq && (XBFS_TD_WARP_GATHER || mark)) {
    gather_bin_warp<PAR>(p, acc, q, in, cnt, M, L, fbn, qside, mark);
    return;
  }
  const bool spec = sm.spec != 0;
  const unsigned long long G = gridDim.x, b = blockIdx.x;
  const unsigned long long lo = M * b / G, hi = M * (b + 1) / G;
  if (lo >= hi) return;
  if (threadIdx.x < 32) {
    const int s = find_owner(in.eb, cnt, lo);
    if (threadIdx.x == 0) sm.next_s = s;
  }
  __syncthreads();
  unsigned s = (unsigned)sm.next_s;
  if (!enq) {
    // bitmap output: nothing is staged, so a round may take up to
    // kRoundsNoStage x kTE edges (as far as the window's owners reach),
    // expanded kTdIlp edges per thread at a time with their visited words
    // loaded together: a quarter of the block barriers of the staged rounds
    constexpr unsigned long long kR = (unsigned long long)kRoundsNoStage * kTE;
    for (unsigned long long r = lo; r < hi;) {
      unsigned long long rhi = (r + kR < hi) ? r + kR : hi;
      if (s + kWin < cnt) {
        const unsigned long long w_end = in.eb[s + kWin];  // the window holds owners s .. s + kWin
        if (w_end < rhi) rhi = w_end;
      }
      for (int i = threadIdx.x; i <= kWin; i += kBlock) {
        const unsigned slot = s + (unsigned)i;
        unsigned e0 = 0xffffffffu;
        if (slot < cnt) {
          const unsigned x = in.eb[slot];
          if ((unsigned long long)x < rhi) {
            e0 = x;
            sm.wu[i] = in.ids[slot];
            sm.wbeg[i] = in.bg[slot];
          }
        }
        sm.web[i] = e0;
      }
      __syncthreads();
      for (unsigned long long e0 = r + threadIdx.x; e0 < rhi; e0 += (unsigned long long)kTdIlp * kBlock) {
        int v[kTdIlp], u[kTdIlp];
#pragma unroll
        for (int k = 0; k < kTdIlp; ++k) {
          const unsigned long long e = e0 + (unsigned long long)k * kBlock;
          v[k] = -1;
          u[k] = 0;
          if (e < rhi) {
            const int a = smem_owner(sm.web, kWin + 1, e);
            v[k] = ld_stream_i32(p.csr + sm.wbeg[a] + (long long)(e - sm.web[a]));
            u[k] = sm.wu[a];
          }
        }
        claim_batch<PAR>(p, acc, v, u, L, fbn, q, qside);
      }
      if (threadIdx.x == 0 && rhi < hi) sm.next_s = (int)(s + smem_owner(sm.web, kWin + 1, rhi));
      __syncthreads();
      s = (unsigned)sm.next_s;
      r = rhi;
    }
    return;
  }
  for (unsigned long long r = lo; r < hi; r += kTE) {
    const unsigned long long rhi = (r + kTE < hi) ? r + kTE : hi;
    for (int i = threadIdx.x; i <= kTE; i += kBlock) {
      const unsigned slot = s + (unsigned)i;
      unsigned e0 = 0xffffffffu;
      if (slot < cnt) {
        const unsigned x = in.eb[slot];
        if ((unsigned long long)x < rhi) {
          e0 = x;
          sm.wu[i] = in.ids[slot];
          sm.wbeg[i] = in.bg[slot];
        }
      }
      sm.web[i] = e0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kK; ++k) {
      const unsigned long long e = r + threadIdx.x + (unsigned long long)k * kBlock;
      if (e < rhi) {
        const int a = smem_owner(sm.web, kTE + 1, e);
        const int v = ld_stream_i32(p.csr + sm.wbeg[a] + (long long)(e - sm.web[a]));
        claim_td<PAR>(p, sm, q, acc, v, sm.wu[a], L, enq, fbn, spec);
      }
    }
    if (threadIdx.x == 0 && rhi < hi) sm.next_s = (int)(s + smem_owner(sm.web, kTE + 1, rhi));
    __syncthreads();
    s = (unsigned)sm.next_s;
    if (enq && need_flush(sm)) flush(sm, q);
  }
}

// Expansion of the small-degree bin (every entry has 1..small_max edges):
// each CTA takes an equal share of the ENTRIES, so no CTA has to search the
// queue for where its share starts. A tile of kBlock entries is loaded one
// per thread, a block scan of their degrees gives each edge its owner, and
// the tile's edges are expanded in rounds of kTE with the CSR loads issued
// before the claims. Degrees within the bin differ by at most
// small_max, so shares of many entries carry similar numbers of edges.
template <bool PAR>
__device__ void gather_entries(const Params& p, Smem& sm, const QOut& q, Acc& acc, const QBin& in, unsigned cnt,
                               unsigned long long M, int L, bool enq, uint32_t* fbn, bool qside, bool blind = false) {
  if (cnt == 0) return;
  const bool spec = sm.spec != 0;
  const unsigned long long G = gridDim.x, b = blockIdx.x;
  const unsigned i0 = (unsigned)((unsigned long long)cnt * b / G);
  const unsigned i1 = (unsigned)((unsigned long long)cnt * (b + 1) / G);
  for (unsigned t0 = i0; t0 < i1; t0 += kBlock) {
    const unsigned i = t0 + threadIdx.x;
    long long d = 0;
    if (i < i1) {
      const unsigned long long e0 = in.eb[i];
      const unsigned long long e1 = (i + 1 < cnt) ? (unsigned long long)in.eb[i + 1] : M;
      d = (long long)(e1 - e0);
      sm.wu[threadIdx.x] = in.ids[i];
      sm.wbeg[threadIdx.x] = in.bg[i];
    }
    long long total;
    const long long ex = block_exclusive_scan<kBlock, long long>(d, sm.red, &total);
    sm.web[threadIdx.x] = (unsigned)ex;
    __syncthreads();
    const int n = (int)min((unsigned)kBlock, i1 - t0);
    const long long T = total;
    // rounds of kTE edges (kK per thread, loads issued before the claims),
    // so one round's winners always fit the staging area
    for (long long r = 0; r < T; r += kTE) {
      int v[kK], u[kK];
#pragma unroll
      for (int k = 0; k < kK; ++k) {
        const long long e = r + threadIdx.x + (long long)k * kBlock;
        v[k] = -1;
        u[k] = 0;
        if (e < T) {
          const int a = smem_owner(sm.web, n, (unsigned long long)e);
          v[k] = ld_stream_i32(p.csr + sm.wbeg[a] + (e - (long long)sm.web[a]));
          u[k] = sm.wu[a];
        }
      }
#pragma unroll
      for (int k = 0; k < kK; ++k)
        if (v[k] >= 0) {
          if (blind)
            red_or_u32(fbn + (v[k] >> 5), 1u << (v[k] & 31));
          else
            claim_td<PAR>(p, sm, q, acc, v[k], u[k], L, enq, fbn, spec, qside);
        }
      __syncthreads();
      if (enq && need_flush(sm)) flush(sm, q);
    }
    __syncthreads();
  }
}

// Tiny share of the small bin (at most 32 entries for this CTA, the usual case
// on long-diameter graphs): warp 0 expands it alone with warp scans and
// shuffles, so the level costs this CTA no block barrier beyond the grid
// barrier's. Winners go to the next queue with one packed atomic per bin per
// warp (edges << 31 | count) and the warp's frontier counts straight to f1.
// Called by warp 0 only; returns nothing to stage or publish afterwards.
template <bool PAR>
__device__ void gather_entries_warp(const Params& p, const QOut& q, const QBin& in, unsigned cnt,
                                    unsigned long long M, unsigned i0, unsigned i1, int L, bool enq, uint32_t* fbn,
                                    bool spec, FDesc* f1, bool qside, bool blind = false) {
  const int lane = threadIdx.x & 31;
  const unsigned i = i0 + lane;
  const bool own = i < i1;
  long long d = 0, bg = 0;
  int u = 0;
  if (own) {
    const unsigned long long e0 = in.eb[i];
    const unsigned long long e1 = (i + 1 < cnt) ? (unsigned long long)in.eb[i + 1] : M;
    d = (long long)(e1 - e0);
    u = in.ids[i];
    bg = in.bg[i];
  }
  const long long incl = warp_inclusive_scan(d);
  const long long ex = incl - d;
  const long long T = __shfl_sync(0xffffffffu, incl, 31);
  const int n = (int)(i1 - i0);
  long long n1 = 0, m1 = 0;
  for (long long base = 0; base < T; base += 32) {
    const long long e = base + lane;
    // owner: the last of the n entries whose exclusive offset is <= e
    // (branch-free binary search, every lane takes part in every shuffle)
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int cand = lo + step;
      const long long exc = __shfl_sync(0xffffffffu, ex, cand < 32 ? cand : 31);
      if (cand < n && exc <= e) lo = cand;
    }
    const long long ex_a = __shfl_sync(0xffffffffu, ex, lo);
    const long long bg_a = __shfl_sync(0xffffffffu, bg, lo);
    const int par_u = __shfl_sync(0xffffffffu, u, lo);
    int v = -1;
    if (e < T) v = ld_stream_i32(p.csr + bg_a + (e - ex_a));
    if (blind && v >= 0) {  // a blind mark instead of a claim (see finalize_marks)
      red_or_u32(fbn + (v >> 5), 1u << (v & 31));
      v = -1;
    }
    // claim (same rules as claim_td)
    bool win = false;
    long long b0 = 0, b1 = 0;
    uint32_t word = 0, bit = 0;
    if (v >= 0) {
      word = (uint32_t)v >> 5;
      bit = 1u << (v & 31);
      bool skip = false;
      if (spec) {
        b0 = ld_nc_i64(p.beg + v);
        b1 = ld_nc_i64(p.beg + v + 1);
      } else {
        skip = (ld_cg_u32(p.vis + word) & bit) != 0;
      }
      if (!skip) win = (atomicOr(p.vis + word, bit) & bit) == 0;
      if (win) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = par_u;
        if (!spec) {
          b0 = ld_nc_i64(p.beg + v);
          b1 = ld_nc_i64(p.beg + v + 1);
        }
        n1 += 1;
        m1 += b1 - b0;
        if (!enq) {
          red_or_u32(fbn + word, bit);
          if (qside && b1 > b0) {
            const int qb = bin_of(b1 - b0, p.small_max, p.medium_max);
            direct_enqueue(q.b[qb], &q.ctr[qb], v, b1 - b0, b0);
          }
        }
      }
    }
    if (enq) {
      const long long dv = b1 - b0;
      const int bin = win ? bin_of(dv, p.small_max, p.medium_max) : -1;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const bool mine = win && dv > 0 && bin == b;
        const unsigned mask = __ballot_sync(0xffffffffu, mine);
        if (!mask) continue;
        const long long dd = mine ? dv : 0;
        const long long inc = warp_inclusive_scan(dd);
        unsigned long long old = 0;
        if (lane == 31) old = atomicAdd(&q.ctr[b], ((unsigned long long)inc << 31) | (unsigned long long)__popc(mask));
        old = __shfl_sync(0xffffffffu, old, 31);
        if (mine) {
          const unsigned long long slot = (old & kCountMask) + __popc(mask & ((1u << lane) - 1));
          q.b[b].ids[slot] = v;
          q.b[b].eb[slot] = (unsigned)((old >> 31) + (unsigned long long)(inc - dd));
          q.b[b].bg[slot] = b0;
        }
      }
    }
  }
  if (!f1) return;  // the next frontier's counts come from its bins
  n1 = warp_sum(n1);
  m1 = warp_sum(m1);
  if (lane == 0) {
    if (n1) atomicAdd(&f1->n, (unsigned long long)n1);
    if (m1) atomicAdd(&f1->m, (unsigned long long)m1);
  }
}

// Degree of v from its head record; a saturated field falls back to the CSR
// offsets.
__device__ __forceinline__ long long head_degree(const Params& p, const int4& h, int v) {
  return h.w != kHeadDegSat ? (long long)h.w : ld_nc_i64(p.beg + v + 1) - ld_nc_i64(p.beg + v);
}

// Position of the k-th (0-based) set bit of m; m has more than k set bits.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int k) {
  int pos = 0;  // largest pos with popc(m below pos) <= k
#pragma unroll
  for (int s = 16; s > 0; s >>= 1)
    if (__popc(m & ((1u << (pos + s)) - 1u)) <= k) pos += s;
  return pos;
}

// Last lane l of the warp with ex[l] <= t (ex non-decreasing over the lanes,
// ex[0] = 0 <= t): the lane whose range [ex[l], ex[l] + count[l]) holds t.
// Branch-free, every lane takes part in every shuffle.
__device__ __forceinline__ int lane_owner(int ex, int t) {
  int lo = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const int exc = __shfl_sync(0xffffffffu, ex, lo + s);
    if (exc <= t) lo += s;
  }
  return lo;
}

// Top-down from a frontier held only as a bitmap, with bitmap output, over
// head records, with no block barrier: each warp takes 32 words of its CTA's
// slice at a time (one per lane), numbers their set bits with a warp scan
// and takes the frontier vertices 64 at a time, two per lane. A lane reads
// its vertices' head records and claims (or, on a two-phase level, marks)
// the (up to) three neighbours in them; the rest of each segment (from the
// fourth neighbour) is expanded by the warp edge-balanced over its 32 lanes,
// kTdIlp edges per lane in flight, with the 64 vertices and their CSR
// offsets in the warp's part of the window arrays.
// Segments with more than kWarpSeg edges left go to the heavy list that is
// expanded grid-wide, edge-balanced, after the barrier (as expand_bitmap's
// vertices of degree above kHeavyDeg): warps do not wait for one another,
// and no warp is held up by a long segment.
#ifndef XBFS_TD_WARP_SEG
#define XBFS_TD_WARP_SEG 1024
#endif
constexpr int kWarpSeg = XBFS_TD_WARP_SEG;
template <bool PAR>
__device__ void expand_bitmap_heads(const Params& p, Smem& sm, Acc& acc, const QOut& q, const uint32_t* fbc, int L,
                                    uint32_t* fbn, int par, bool qside, int mark) {
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kBlock / 32;
  unsigned long long* hctr = &p.ctl->heavy[par];
  // the warp's 64 vertices and their segments' next CSR offsets, for the
  // edge-balanced expansion (the window arrays are free in this mode)
  int* wu = sm.wu + warp * 64;
  long long* wbg = sm.wbeg + warp * 64;
  for (long long c = w0 + (long long)warp * 32; c < w1; c += (long long)NWARP * 32) {
    const uint32_t bits = (c + lane < w1) ? ld_cg_u32(fbc + c + lane) : 0u;
    const int pc = __popc(bits);
    const int incl = warp_inclusive_scan(pc);
    const int ex = incl - pc;
    const int B = __shfl_sync(0xffffffffu, incl, 31);
    for (int base = 0; base < B; base += 64) {
      int uu[2];
      int4 h[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int t = base + 32 * j + lane;
        const int lo = lane_owner(ex, t);
        const uint32_t wbits = __shfl_sync(0xffffffffu, bits, lo);
        const int exl = __shfl_sync(0xffffffffu, ex, lo);
        uu[j] = t < B ? (int)((c + lo) * 32 + nth_set_bit(wbits, t - exl)) : -1;
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) h[j] = uu[j] >= 0 ? ld_nc_na_v4(p.head + uu[j]) : make_int4(-1, -1, -1, 0);
      // the segments' CSR offsets (where they go on past the head record)
      // are loaded alongside the claims of the head neighbours
      int r[2];
      long long bg[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const long long rem = uu[j] >= 0 ? head_degree(p, h[j], uu[j]) - 3 : 0;
        bg[j] = rem > 0 ? ld_nc_i64(p.beg + uu[j]) + 3 : 0;
        r[j] = rem > kWarpSeg ? -1 : (rem > 0 ? (int)rem : 0);
      }
      if (mark) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int v[3] = {h[j].x, h[j].y, h[j].z};
          const int u[3] = {uu[j], uu[j], uu[j]};
          mark_batch<PAR>(p, v, u, fbn, mark);
        }
      } else if (XBFS_TD_HEAD_FILTER) {
        const int v[6] = {h[0].x, h[0].y, h[0].z, h[1].x, h[1].y, h[1].z};
        const int u[6] = {uu[0], uu[0], uu[0], uu[1], uu[1], uu[1]};
        claim_filtered<PAR>(p, acc, v, u, L, fbn, q, qside);
      } else {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int v[3] = {h[j].x, h[j].y, h[j].z};
          const int u[3] = {uu[j], uu[j], uu[j]};
          claim_batch<PAR>(p, acc, v, u, L, fbn, q, qside);
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (r[j] < 0) {
          direct_enqueue(p.heavy, hctr, uu[j], head_degree(p, h[j], uu[j]) - 3, bg[j]);
          r[j] = 0;
        }
        wu[32 * j + lane] = uu[j];
        wbg[32 * j + lane] = bg[j];
      }
      __syncwarp();
      // the rest of the 64 segments, edge-balanced over the warp: lane l
      // owns edges [rex, rex + r[0] + r[1]) of the warp's total, its first
      // vertex's r[0] and then its second vertex's r[1]
      const int rr = r[0] + r[1];
      const int rincl = warp_inclusive_scan(rr);
      const int rex = rincl - rr;
      const int T = __shfl_sync(0xffffffffu, rincl, 31);
      for (int e0 = 0; e0 < T; e0 += 32 * kTdIlp) {
        int v[kTdIlp], u[kTdIlp];
#pragma unroll
        for (int k = 0; k < kTdIlp; ++k) {
          const int e = e0 + 32 * k + lane;
          const int o = lane_owner(rex, e);
          int off = e - __shfl_sync(0xffffffffu, rex, o);
          const int r0 = __shfl_sync(0xffffffffu, r[0], o);
          const int slot = off >= r0 ? 32 + o : o;
          off = off >= r0 ? off - r0 : off;
          u[k] = wu[slot];
          v[k] = e < T ? __ldg(p.csr + wbg[slot] + off) : -1;
        }
        if (mark)
          mark_batch<PAR>(p, v, u, fbn, mark);
        else if (XBFS_TD_REM_FILTER)
          claim_filtered<PAR>(p, acc, v, u, L, fbn, q, qside);
        else
          claim_batch<PAR>(p, acc, v, u, L, fbn, q, qside);
      }
      __syncwarp();  // the next round rewrites the warp's entries
    }
  }
}

// Second phase of a two-phase top-down level (after a grid barrier, when
// every mark has landed): the new vertices are the bits of frontier L+1's
// bitmap that are not visited. Each warp takes 32 words of its CTA's slice
// (one per lane), sets their visited bits (one thread per word; after blind
// marks it also clears the bits of visited targets from frontier L+1's
// word), and then takes the new vertices 64 at a time, two per lane: level
// L+1, and the frontier statistics with the degrees from their head records.
__device__ void finalize_marks(const Params& p, Acc& acc, int L, uint32_t* fbn, bool blind) {
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kBlock / 32;
  for (long long c = w0 + (long long)warp * 32; c < w1; c += (long long)NWARP * 32) {
    uint32_t nb = 0;
    if (c + lane < w1) {
      const uint32_t f = ld_cg_u32(fbn + c + lane);
      if (f) {
        const uint32_t vv = ld_cg_u32(p.vis + c + lane);
        nb = f & ~vv;
        if (nb) p.vis[c + lane] = vv | nb;
        if (blind && nb != f) fbn[c + lane] = nb;  // blind marks of visited targets
      }
    }
    const int pc = __popc(nb);
    const int incl = warp_inclusive_scan(pc);
    const int ex = incl - pc;
    const int B = __shfl_sync(0xffffffffu, incl, 31);
    for (int base = 0; base < B; base += 64) {
      int nv[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int t = base + 32 * j + lane;
        const int lo = lane_owner(ex, t);
        const uint32_t wbits = __shfl_sync(0xffffffffu, nb, lo);
        const int exl = __shfl_sync(0xffffffffu, ex, lo);
        nv[j] = t < B ? (int)((c + lo) * 32 + nth_set_bit(wbits, t - exl)) : -1;
      }
      int4 h[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) h[j] = nv[j] >= 0 ? ld_nc_na_v4(p.head + nv[j]) : make_int4(-1, -1, -1, 0);
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (nv[j] >= 0) {
          p.levels[nv[j]] = L + 1;
          acc.n1 += 1;
          acc.m1 += head_degree(p, h[j], nv[j]);
        }
    }
  }
}

// Top-down from a frontier held only as a bitmap ("single scan"): every CTA
// compacts the set bits of its slice tile by tile into shared memory, gives
// each vertex of degree <= kHeavyDeg its exclusive edge offset with a block
// scan and expands the tile edge-balanced; heavier vertices go to a global
// list expanded grid-wide after the barrier.
template <bool PAR>
__device__ void expand_bitmap(const Params& p, Smem& sm, const QOut& q, Acc& acc, const uint32_t* fbc, int L,
                              bool enq, uint32_t* fbn, int par, bool qside) {
  const bool spec = sm.spec != 0;
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  unsigned long long* hctr = &p.ctl->heavy[par];
  // A tile is kBlock words, one per thread. Its set bits are numbered by a
  // block scan of the words' popcounts and taken kWin at a time (one pass
  // for a sparse tile, ceil(bits / kWin) passes for a dense one).
  for (long long wt = w0; wt < w1; wt += kBlock) {
    uint32_t tbits = 0;
    const long long w = wt + threadIdx.x;
    if (w < w1) tbits = ld_cg_u32(fbc + w);
    const int tcount = __syncthreads_count(tbits != 0);
    if (tcount == 0) continue;
    long long tsum;
    const long long tex = block_exclusive_scan<kBlock, long long>((long long)__popc(tbits), sm.red, &tsum);
  for (long long c0 = 0; c0 < tsum; c0 += kWin) {
    // 1. list the tile's set bits numbered [c0, c0 + kWin)
    {
      const long long c1 = c0 + kWin;
      if (tbits && tex < c1 && tex + __popc(tbits) > c0) {
        uint32_t bits = tbits;
        long long o = tex;
        while (bits) {
          const int bp = __ffs(bits) - 1;
          bits &= bits - 1;
          if (o >= c0 && o < c1) sm.wu[o - c0] = (int)(w * 32 + bp);
          ++o;
        }
      }
    }
    __syncthreads();
    const int n = (int)((tsum - c0 < kWin) ? tsum - c0 : kWin);
    // 2. degrees and CSR offsets; heavy vertices are deferred
    constexpr int PER = (kWin + kBlock - 1) / kBlock;
    const int i0 = threadIdx.x * PER;
    long long loc = 0;
    int dd[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      dd[k] = 0;
      const int i = i0 + k;
      if (i < n) {
        const int u = sm.wu[i];
        const long long b0 = ld_nc_i64(p.beg + u);
        const long long d = ld_nc_i64(p.beg + u + 1) - b0;
        sm.wbeg[i] = b0;
        if (d > kHeavyDeg) {
          direct_enqueue(p.heavy, hctr, u, d, b0);
        } else {
          dd[k] = (int)d;
          loc += d;
        }
      }
    }
    long long T;
    long long run = block_exclusive_scan<kBlock, long long>(loc, sm.red, &T);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = i0 + k;
      if (i < n) {
        sm.web[i] = (unsigned)run;
        run += dd[k];
      }
    }
    __syncthreads();
    // 3. edge-balanced expansion of the tile
    if (!enq) {
      // bitmap output: nothing is staged, so the rounds need no block
      // barrier; each thread keeps kTdIlp edges in flight (their neighbour
      // ids, then the visited words of all of them) and claims only the
      // targets that looked unvisited
      for (long long e0 = threadIdx.x; e0 < T; e0 += (long long)kTdIlp * kBlock) {
        int v[kTdIlp], u[kTdIlp];
#pragma unroll
        for (int k = 0; k < kTdIlp; ++k) {
          const long long e = e0 + (long long)k * kBlock;
          v[k] = -1;
          u[k] = 0;
          if (e < T) {
            const int a = smem_owner(sm.web, n, (unsigned long long)e);
            v[k] = __ldg(p.csr + sm.wbeg[a] + (e - (long long)sm.web[a]));
            u[k] = sm.wu[a];
          }
        }
        claim_batch<PAR>(p, acc, v, u, L, fbn, q, qside);
      }
      __syncthreads();  // the next chunk rewrites the window
    } else {
      for (long long r = 0; r < T; r += kTE) {
#pragma unroll
        for (int k = 0; k < kK; ++k) {
          const long long e = r + threadIdx.x + (long long)k * kBlock;
          if (e < T) {
            const int a = smem_owner(sm.web, n, (unsigned long long)e);
            const int v = __ldg(p.csr + sm.wbeg[a] + (e - (long long)sm.web[a]));
            claim_td<PAR>(p, sm, q, acc, v, sm.wu[a], L, enq, fbn, spec);
          }
        }
        __syncthreads();
        if (need_flush(sm)) flush(sm, q);
      }
    }
  }
  }
}

// Queue of frontier L -> bitmap of frontier L.
__device__ void scatter_queue_to_bitmap(const Params& p, int par, const FDesc& fd, uint32_t* fbc) {
  const long long tid = blockIdx.x * (long long)kBlock + threadIdx.x;
  const long long nth = (long long)gridDim.x * kBlock;
  for (int bin = 0; bin < 3; ++bin) {
    const long long cnt = (long long)(ld_cg_u64(&fd.bin[bin]) & kCountMask);
    const int* ids = p.q[par][bin].ids;
    for (long long i = tid; i < cnt; i += nth) {
      const int v = ids[i];
      red_or_u32(fbc + (v >> 5), 1u << (v & 31));
    }
  }
}

// Bottom-up neighbour probe: scans [e, e_end) PW neighbours at a time (their
// CSR entries and frontier bits loaded together) until a level-L parent is
// found; with ASYNC, remembers the first level-(L+1) neighbour on the way.
template <int PW, bool LDG, bool ASYNC>
__device__ __forceinline__ void probe_range(const Params& p, const uint32_t* fbc, const uint32_t* fbn,
                                            long long& e, long long e_end, int& found, int& found2) {
  for (; e < e_end; e += PW) {
    int u[PW];
#pragma unroll
    for (int k = 0; k < PW; ++k)
      u[k] = (e + k < e_end) ? (LDG ? __ldg(p.csr + e + k) : ld_stream_i32(p.csr + e + k)) : -1;
    uint32_t wc[PW];
#pragma unroll
    for (int k = 0; k < PW; ++k) wc[k] = (u[k] >= 0) ? fbc[u[k] >> 5] : 0u;
#pragma unroll
    for (int k = 0; k < PW; ++k)
      if (found < 0 && u[k] >= 0 && ((wc[k] >> (u[k] & 31)) & 1u)) found = u[k];
    if (found >= 0) return;
    if (ASYNC && found2 < 0) {
      uint32_t wn[PW];
#pragma unroll
      for (int k = 0; k < PW; ++k) wn[k] = (u[k] >= 0) ? ld_cg_u32(fbn + (u[k] >> 5)) : 0u;
#pragma unroll
      for (int k = 0; k < PW; ++k)
        if (found2 < 0 && u[k] >= 0 && ((wn[k] >> (u[k] & 31)) & 1u)) found2 = u[k];
    }
  }
}

// Two vertices per lane: the same probe for vertex pairs, with the loads of
// both issued together, so a lane has two dependency chains in flight.
template <int PW, bool ASYNC>
__device__ __forceinline__ void probe_pair(const Params& p, const uint32_t* fbc, const uint32_t* fbn,
                                           long long (&e)[2], const long long (&lim)[2], int (&found)[2],
                                           int (&found2)[2]) {
  for (;;) {
    bool act[2];
    act[0] = found[0] < 0 && e[0] < lim[0];
    act[1] = found[1] < 0 && e[1] < lim[1];
    if (!act[0] && !act[1]) return;
    int u[2][PW];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < PW; ++k) u[j][k] = (act[j] && e[j] + k < lim[j]) ? __ldg(p.csr + e[j] + k) : -1;
    uint32_t wc[2][PW];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < PW; ++k) wc[j][k] = (u[j][k] >= 0) ? fbc[u[j][k] >> 5] : 0u;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < PW; ++k)
        if (found[j] < 0 && u[j][k] >= 0 && ((wc[j][k] >> (u[j][k] & 31)) & 1u)) found[j] = u[j][k];
    if (ASYNC) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (!act[j] || found[j] >= 0 || found2[j] >= 0) continue;
#pragma unroll
        for (int k = 0; k < PW; ++k)
          if (found2[j] < 0 && u[j][k] >= 0 && ((ld_cg_u32(fbn + (u[j][k] >> 5)) >> (u[j][k] & 31)) & 1u))
            found2[j] = u[j][k];
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (act[j]) e[j] += PW;
  }
}

// Publishes a warp's bottom-up results for 32 consecutive entries of a sorted
// list: vertices sharing a bitmap word sit in adjacent lanes, so their bits
// are ORed along each run of equal words and the run's first lane issues one
// atomic per word instead of one per vertex.
template <bool ASYNC>
__device__ __forceinline__ void bu_publish_words(const Params& p, uint32_t* fbn, uint32_t* fbn2, uint32_t word,
                                                 uint32_t m1, uint32_t m2, bool valid) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t ow = __shfl_down_sync(0xffffffffu, word, off);
    const uint32_t o1 = __shfl_down_sync(0xffffffffu, m1, off);
    const uint32_t o2 = __shfl_down_sync(0xffffffffu, m2, off);
    if (lane + off < 32 && ow == word) {
      m1 |= o1;
      m2 |= o2;
    }
  }
  const uint32_t pw = __shfl_up_sync(0xffffffffu, word, 1);
  if (valid && (lane == 0 || pw != word)) {
    if (m1 | m2) red_or_u32(p.vis + word, m1 | m2);
    if (m1) red_or_u32(fbn + word, m1);
    if (ASYNC && m2) red_or_u32(fbn2 + word, m2);
  }
}

// Bottom-up step for level L. Each CTA owns a contiguous slice of the vertex
// range (vertex ids are scrambled, so slices carry similar work): it compacts
// the slice's unvisited vertices into a sorted list with block ballot /
// popcount scans (the reference's ballot_counting + prefix sum + FQ_gen,
// without the host round trip of my_prefixsum), then its warps drain the list
// 32 vertices at a time from a shared counter, so a slow warp does not hold the
// others. Each lane probes its vertex's neighbours 2, then 4, then 8 at a time
// (most vertices find a parent among the first few).
// Frontier probe of the three neighbours in a head record (-1 entries are
// absent neighbours): a level-L parent, else with ASYNC the first of them
// already in frontier L+1.
template <bool ASYNC>
__device__ __forceinline__ void probe_head(const uint32_t* fbc, const uint32_t* fbn, const int4& h, int& found,
                                           int& found2) {
  const int u[3] = {h.x, h.y, h.z};
  uint32_t wc[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) wc[j] = u[j] >= 0 ? fbc[u[j] >> 5] : 0u;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (found < 0 && u[j] >= 0 && ((wc[j] >> (u[j] & 31)) & 1u)) found = u[j];
  if (ASYNC && found < 0 && found2 < 0) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
      if (found2 < 0 && u[j] >= 0 && ((ld_cg_u32(fbn + (u[j] >> 5)) >> (u[j] & 31)) & 1u)) found2 = u[j];
  }
}

template <bool PAR, bool ASYNC, bool HEAD>
__device__ void bottom_up(const Params& p, Smem& sm, Acc& acc, int L, const uint32_t* fbc, uint32_t* fbn,
                          uint32_t* fbn2, const QOut& q2, bool asyncq) {
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  int* list = p.ulist + w0 * 32;
  long long pos = 0;
  for (long long wb = w0; wb < w1; wb += kBlock) {
    const long long w = wb + threadIdx.x;
    uint32_t bits = (w < w1) ? ~ld_cg_u32(p.vis + w) : 0u;
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
  if (threadIdx.x == 0) sm.bu_next = 0;
  __syncthreads();
  const int n = (int)pos;
  const int lane = threadIdx.x & 31;
  if (p.bu_mode == 3) {
    // 64 list entries per warp grab, two per lane (entries base+lane and
    // base+32+lane), probed together: 2, then 4 neighbours at a time
    for (;;) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&sm.bu_next, 64);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) break;
      int v[2];
      long long eb[2], ee[2], e[2], lim[2];
      int found[2] = {-1, -1}, found2[2] = {-1, -1};
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int i = base + 32 * j + lane;
        v[j] = (i < n) ? list[i] : -1;
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        eb[j] = 0;
        ee[j] = 0;
        if (v[j] >= 0) {
          eb[j] = ld_nc_i64(p.beg + v[j]);
          ee[j] = ld_nc_i64(p.beg + v[j] + 1);
        }
        e[j] = eb[j];
        lim[j] = eb[j] + 2 < ee[j] ? eb[j] + 2 : ee[j];
      }
      probe_pair<2, ASYNC>(p, fbc, fbn, e, lim, found, found2);
      lim[0] = ee[0];
      lim[1] = ee[1];
      probe_pair<4, ASYNC>(p, fbc, fbn, e, lim, found, found2);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        uint32_t word = 0xffffffffu, m1 = 0, m2 = 0;
        if (v[j] >= 0) {
          word = (uint32_t)v[j] >> 5;
          const uint32_t bit = 1u << (v[j] & 31);
          if (found[j] >= 0) {
            p.levels[v[j]] = L + 1;
            if (PAR) p.parents[v[j]] = found[j];
            m1 = bit;
            acc.n1 += 1;
            acc.m1 += ee[j] - eb[j];
          } else if (ASYNC && found2[j] >= 0) {
            p.levels[v[j]] = L + 2;
            if (PAR) p.parents[v[j]] = found2[j];
            m2 = bit;
            acc.n2 += 1;
            acc.m2 += ee[j] - eb[j];
          }
        }
        if (ASYNC && asyncq) enqueue_warp(p, q2, m2 != 0, v[j], ee[j] - eb[j], eb[j]);
        bu_publish_words<ASYNC>(p, fbn, fbn2, word, m1, m2, v[j] >= 0);
      }
    }
    return;
  }
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&sm.bu_next, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int i = base + lane;
    uint32_t word = 0xffffffffu, m1 = 0, m2 = 0;  // bitmap word of this lane's vertex, bits to set
    int v = -1;
    long long e0 = 0, e1 = 0;
    if (i < n && HEAD) {
      // head record first: three neighbours and the degree in one read;
      // the CSR offsets only when the scan goes on (or a queue entry for
      // frontier L+2 needs the vertex's offset)
      v = list[i];
      const int4 h = ld_nc_na_v4(p.head + v);
      int found = -1, found2 = -1;
      probe_head<ASYNC>(fbc, fbn, h, found, found2);
      const long long d = head_degree(p, h, v);
      if (found < 0 && d > 3) {
        e0 = ld_nc_i64(p.beg + v);
        long long e = e0 + 3;
        probe_range<4, true, ASYNC>(p, fbc, fbn, e, e0 + 7 < e0 + d ? e0 + 7 : e0 + d, found, found2);
        if (found < 0) probe_range<8, true, ASYNC>(p, fbc, fbn, e, e0 + d, found, found2);
      } else if (ASYNC && asyncq && found < 0 && found2 >= 0) {
        e0 = ld_nc_i64(p.beg + v);
      }
      e1 = e0 + d;
      word = (uint32_t)v >> 5;
      const uint32_t bit = 1u << (v & 31);
      if (found >= 0) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = found;
        m1 = bit;
        acc.n1 += 1;
        acc.m1 += d;
      } else if (ASYNC && found2 >= 0) {
        p.levels[v] = L + 2;
        if (PAR) p.parents[v] = found2;
        m2 = bit;
        acc.n2 += 1;
        acc.m2 += d;
      }
    } else if (i < n) {
      v = list[i];
      e0 = ld_nc_i64(p.beg + v);
      e1 = ld_nc_i64(p.beg + v + 1);
      int found = -1, found2 = -1;
      long long e = e0;
      if (p.bu_mode == 2) {  // four at a time, streaming loads
        probe_range<4, false, ASYNC>(p, fbc, fbn, e, e1, found, found2);
      } else if (p.bu_mode == 1) {  // streaming (L1-bypassing) neighbour loads
        probe_range<2, false, ASYNC>(p, fbc, fbn, e, e0 + 2 < e1 ? e0 + 2 : e1, found, found2);
        if (found < 0) probe_range<4, false, ASYNC>(p, fbc, fbn, e, e0 + 6 < e1 ? e0 + 6 : e1, found, found2);
        if (found < 0) probe_range<8, false, ASYNC>(p, fbc, fbn, e, e1, found, found2);
      } else {  // L1-allocating neighbour loads: the next probes hit the same sector
        probe_range<2, true, ASYNC>(p, fbc, fbn, e, e0 + 2 < e1 ? e0 + 2 : e1, found, found2);
        if (found < 0) probe_range<4, true, ASYNC>(p, fbc, fbn, e, e0 + 6 < e1 ? e0 + 6 : e1, found, found2);
        if (found < 0) probe_range<8, true, ASYNC>(p, fbc, fbn, e, e1, found, found2);
      }
      word = (uint32_t)v >> 5;
      const uint32_t bit = 1u << (v & 31);
      if (found >= 0) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = found;
        m1 = bit;
        acc.n1 += 1;
        acc.m1 += e1 - e0;
      } else if (ASYNC && found2 >= 0) {
        p.levels[v] = L + 2;
        if (PAR) p.parents[v] = found2;
        m2 = bit;
        acc.n2 += 1;
        acc.m2 += e1 - e0;
      }
    }
    if (ASYNC && asyncq) enqueue_warp(p, q2, m2 != 0, v, e1 - e0, e0);
    // The warp's 32 vertices are consecutive entries of a sorted list, so
    // vertices sharing a bitmap word sit in adjacent lanes: OR their bits
    // along each run of equal words and let the run's first lane publish
    // them, one atomic per word instead of one per vertex.
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t ow = __shfl_down_sync(0xffffffffu, word, off);
      const uint32_t o1 = __shfl_down_sync(0xffffffffu, m1, off);
      const uint32_t o2 = __shfl_down_sync(0xffffffffu, m2, off);
      if (lane + off < 32 && ow == word) {
        m1 |= o1;
        m2 |= o2;
      }
    }
    const uint32_t pw = __shfl_up_sync(0xffffffffu, word, 1);
    if (i < n && (lane == 0 || pw != word)) {
      if (m1 | m2) red_or_u32(p.vis + word, m1 | m2);
      if (m1) red_or_u32(fbn + word, m1);
      if (ASYNC && m2) red_or_u32(fbn2 + word, m2);
    }
  }
}

// Shape of the word-parallel bottom-up step (below): bitmap words per warp
// step, neighbours probed before a vertex is deferred, neighbours per drain
// step, capacity of the per-CTA deferred queue.
#ifndef XBFS_BU_WORDS
#define XBFS_BU_WORDS 2
#endif
#ifndef XBFS_BU_FIRST
#define XBFS_BU_FIRST 2
#endif
constexpr int kBuWords = XBFS_BU_WORDS, kBuFirst = XBFS_BU_FIRST, kBuMore = 8;
constexpr int kBuQueue = 2 * kCap;
// Bottom-up probes read head records where the graph has them (1), or the
// CSR offsets only (0); the word-parallel step over head records loads the
// visited words of the warp's next step one step ahead (1) or not (0).
#ifndef XBFS_BU_HEADS
#define XBFS_BU_HEADS 1
#endif
// Top-down levels from a frontier bitmap with bitmap output read head
// records, barrier-free per warp (1), or take expand_bitmap's block tiles (0).
#ifndef XBFS_TD_HEADS
#define XBFS_TD_HEADS 1
#endif
#ifndef XBFS_BU_PREFETCH
#define XBFS_BU_PREFETCH 1
#endif
constexpr bool kBuPrefetch = XBFS_BU_PREFETCH;
// The word-parallel step over head records tests the vertices whose whole
// list is in the record for level L+2 (asynchronous rule) (1) or leaves
// them to the next level (0: one dependent read of frontier L+1's bitmap
// fewer per step; the first bottom-up level of R-MAT scale 23 measured
// 30-35% faster, the next level a little slower, the traversal 11%
// faster). The drain of deferred vertices applies the rule (1) or not (0:
// measured 1% faster; the list-probing levels keep the rule).
#ifndef XBFS_BU_FOUND2
#define XBFS_BU_FOUND2 0
#endif
#ifndef XBFS_BU_ASYNC_DRAIN
#define XBFS_BU_ASYNC_DRAIN 0
#endif

// Second phase of the word-parallel bottom-up step: the vertices deferred to
// the CTA's shared-memory queue (their first `first` neighbours probed
// without a hit) are scanned one per lane, kBuMore neighbours per step.
template <bool PAR, bool ASYNC>
__device__ void bu_drain(const Params& p, Smem& sm, Acc& acc, int L, const uint32_t* fbc, uint32_t* fbn,
                         uint32_t* fbn2, int first, const int* gq) {
  const int lane = threadIdx.x & 31;
  const int* q_v = &sm.st_id[0][0];
  const int nq = sm.bu_n;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&sm.bu_next, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= nq) break;
    const int i = base + lane;
    uint32_t word = 0xffffffffu, m1 = 0, m2 = 0;
    if (i < nq) {
      const int v = i < kBuQueue ? q_v[i] : gq[i - kBuQueue];
      const long long e0 = ld_nc_i64(p.beg + v), e1 = ld_nc_i64(p.beg + v + 1);
      long long e = e0 + first;
      int found = -1, found2 = -1;
      probe_range<kBuMore, true, ASYNC && XBFS_BU_ASYNC_DRAIN>(p, fbc, fbn, e, e1, found, found2);
      word = (uint32_t)v >> 5;
      const uint32_t bit = 1u << (v & 31);
      if (found >= 0) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = found;
        m1 = bit;
        acc.n1 += 1;
        acc.m1 += e1 - e0;
      } else if (ASYNC && found2 >= 0) {
        p.levels[v] = L + 2;
        if (PAR) p.parents[v] = found2;
        m2 = bit;
        acc.n2 += 1;
        acc.m2 += e1 - e0;
      }
    }
    bu_publish_words<ASYNC>(p, fbn, fbn2, word, m1, m2, i < nq);
  }
}

// Bottom-up step for level L, word-parallel (the default probe mode). Each
// warp takes kBuWords consecutive words of its CTA's slice of the visited
// bitmap at a time; lane i handles vertex 32w+i of each word when it is
// unvisited. A lane's vertices are probed together: their CSR offsets, then
// the first kBuFirst neighbours of each, then those neighbours' frontier
// bits, so every lane keeps kBuWords x kBuFirst loads in flight and a warp
// crosses its slice in few dependent steps. No list of unvisited vertices
// is built (the bitmap word is the lanes' work), and results go out with
// one atomic per word. On power-law graphs most unvisited vertices find a
// parent within the first few neighbours; one that still has neighbours
// left is deferred to a per-CTA queue (in shared memory, the top-down
// staging areas unused in a bottom-up level, and past kBuQueue entries in
// the CTA's part of the bottom-up list area) and drained afterwards one
// vertex per lane, kBuMore neighbours per step, so a long scan no longer
// holds the 31 other lanes of its warp.

template <bool PAR, bool ASYNC>
__device__ void bottom_up_words(const Params& p, Smem& sm, Acc& acc, int L, const uint32_t* fbc, uint32_t* fbn,
                                uint32_t* fbn2) {
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kBlock / 32;
  int* q_v = &sm.st_id[0][0];  // deferred vertices, then (past kBuQueue) the slice's part of p.ulist
  int* gq = p.ulist + w0 * 32;
  if (threadIdx.x == 0) {
    sm.bu_n = 0;
    sm.bu_next = 0;
  }
  __syncthreads();
  for (long long wb = w0 + (long long)warp * kBuWords; wb < w1; wb += (long long)NWARP * kBuWords) {
    uint32_t un[kBuWords];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) un[k] = (wb + k < w1) ? ~ld_cg_u32(p.vis + wb + k) : 0u;
    long long e[kBuWords], ee[kBuWords];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      e[k] = 0;
      ee[k] = 0;
      if ((un[k] >> lane) & 1u) {
        const int v = (int)((wb + k) * 32 + lane);
        e[k] = ld_nc_i64(p.beg + v);
        ee[k] = ld_nc_i64(p.beg + v + 1);
      }
    }
    int u[kBuWords][kBuFirst];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k)
#pragma unroll
      for (int j = 0; j < kBuFirst; ++j) u[k][j] = (e[k] + j < ee[k]) ? __ldg(p.csr + e[k] + j) : -1;
    uint32_t wc[kBuWords][kBuFirst];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k)
#pragma unroll
      for (int j = 0; j < kBuFirst; ++j) wc[k][j] = (u[k][j] >= 0) ? fbc[u[k][j] >> 5] : 0u;
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      const bool act = (un[k] >> lane) & 1u;
      int found = -1, found2 = -1;
#pragma unroll
      for (int j = 0; j < kBuFirst; ++j)
        if (found < 0 && u[k][j] >= 0 && ((wc[k][j] >> (u[k][j] & 31)) & 1u)) found = u[k][j];
      const long long d = ee[k] - e[k];
      bool defer = act && found < 0 && d > kBuFirst;
      // warp-aggregated slots in the deferred queue (shared memory first,
      // then the CTA's part of the list area, which holds its whole slice)
      const unsigned dm = __ballot_sync(0xffffffffu, defer);
      if (dm) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&sm.bu_n, __popc(dm));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (defer) {
          const int slot = base + __popc(dm & ((1u << lane) - 1u));
          if (slot < kBuQueue)
            q_v[slot] = (int)((wb + k) * 32 + lane);
          else
            gq[slot - kBuQueue] = (int)((wb + k) * 32 + lane);
        }
      }
      if (ASYNC && act && found < 0 && !defer && found2 < 0) {
        // whole neighbour list scanned without a level-L parent: a neighbour
        // already in frontier L+1 gives level L+2
#pragma unroll
        for (int j = 0; j < kBuFirst; ++j)
          if (found2 < 0 && u[k][j] >= 0 && ((ld_cg_u32(fbn + (u[k][j] >> 5)) >> (u[k][j] & 31)) & 1u))
            found2 = u[k][j];
      }
      const bool got1 = act && found >= 0;
      const bool got2 = ASYNC && act && !got1 && !defer && found2 >= 0;
      const int v = (int)((wb + k) * 32 + lane);
      if (got1) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = found;
        acc.n1 += 1;
        acc.m1 += d;
      } else if (got2) {
        p.levels[v] = L + 2;
        if (PAR) p.parents[v] = found2;
        acc.n2 += 1;
        acc.m2 += d;
      }
      const uint32_t m1 = __ballot_sync(0xffffffffu, got1);
      const uint32_t m2 = __ballot_sync(0xffffffffu, got2);
      if (lane == 0 && (m1 | m2)) {
        const long long w = wb + k;
        red_or_u32(p.vis + w, m1 | m2);
        if (m1) red_or_u32(fbn + w, m1);
        if (ASYNC && m2) red_or_u32(fbn2 + w, m2);
      }
    }
  }
  __syncthreads();
  bu_drain<PAR, ASYNC>(p, sm, acc, L, fbc, fbn, fbn2, kBuFirst, gq);
}

// Word-parallel bottom-up step over head records: the same work split and
// deferred queue as bottom_up_words, but a lane reads its vertex's 16-byte
// head record (first three neighbours and degree; the 32 records of a word
// are one coalesced 512-byte read) in place of its CSR offsets followed by
// the first CSR sector, and the visited words of the warp's next step are
// loaded one step ahead. A probe is then two dependent reads (record, then
// frontier bits) instead of four.
template <bool PAR, bool ASYNC>
__device__ void bottom_up_heads(const Params& p, Smem& sm, Acc& acc, int L, const uint32_t* fbc, uint32_t* fbn,
                                uint32_t* fbn2) {
  constexpr int F = 3;  // neighbours in a head record
  const long long nw = p.nwords;
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kBlock / 32;
  constexpr long long kStride = (long long)NWARP * kBuWords;
  int* q_v = &sm.st_id[0][0];  // deferred vertices, then (past kBuQueue) the slice's part of p.ulist
  int* gq = p.ulist + w0 * 32;
  if (threadIdx.x == 0) {
    sm.bu_n = 0;
    sm.bu_next = 0;
  }
  __syncthreads();
  uint32_t un_nx[kBuWords];
  if (kBuPrefetch) {
    const long long wb = w0 + (long long)warp * kBuWords;
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) un_nx[k] = (wb + k < w1) ? ~ld_cg_u32(p.vis + wb + k) : 0u;
  }
  for (long long wb = w0 + (long long)warp * kBuWords; wb < w1; wb += kStride) {
    uint32_t un[kBuWords];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      if (kBuPrefetch) {
        un[k] = un_nx[k];
        un_nx[k] = (wb + kStride + k < w1) ? ~ld_cg_u32(p.vis + wb + kStride + k) : 0u;
      } else {
        un[k] = (wb + k < w1) ? ~ld_cg_u32(p.vis + wb + k) : 0u;
      }
    }
    int4 h[kBuWords];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k)
      h[k] = ((un[k] >> lane) & 1u) ? ld_nc_na_v4(p.head + (wb + k) * 32 + lane) : make_int4(-1, -1, -1, 0);
    uint32_t wc[kBuWords][F];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      wc[k][0] = h[k].x >= 0 ? fbc[h[k].x >> 5] : 0u;
      wc[k][1] = h[k].y >= 0 ? fbc[h[k].y >> 5] : 0u;
      wc[k][2] = h[k].z >= 0 ? fbc[h[k].z >> 5] : 0u;
    }
    int found[kBuWords], found2[kBuWords];
    long long d[kBuWords];
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      const bool act = (un[k] >> lane) & 1u;
      const int u[F] = {h[k].x, h[k].y, h[k].z};
      found[k] = -1;
      found2[k] = -1;
#pragma unroll
      for (int j = 0; j < F; ++j)
        if (found[k] < 0 && u[j] >= 0 && ((wc[k][j] >> (u[j] & 31)) & 1u)) found[k] = u[j];
      d[k] = act ? head_degree(p, h[k], (int)((wb + k) * 32 + lane)) : 0;
    }
    if (ASYNC && XBFS_BU_FOUND2) {
      // a vertex whose whole list is in its head record and has no level-L
      // parent: a neighbour already in frontier L+1 gives level L+2 (the
      // words of both vertices read together)
      uint32_t wn[kBuWords][F];
#pragma unroll
      for (int k = 0; k < kBuWords; ++k) {
        const bool need = ((un[k] >> lane) & 1u) && found[k] < 0 && d[k] <= F;
        const int u[F] = {h[k].x, h[k].y, h[k].z};
#pragma unroll
        for (int j = 0; j < F; ++j) wn[k][j] = (need && u[j] >= 0) ? ld_cg_u32(fbn + (u[j] >> 5)) : 0u;
      }
#pragma unroll
      for (int k = 0; k < kBuWords; ++k) {
        const int u[F] = {h[k].x, h[k].y, h[k].z};
#pragma unroll
        for (int j = 0; j < F; ++j)
          if (found2[k] < 0 && u[j] >= 0 && ((wn[k][j] >> (u[j] & 31)) & 1u)) found2[k] = u[j];
      }
    }
#pragma unroll
    for (int k = 0; k < kBuWords; ++k) {
      const bool act = (un[k] >> lane) & 1u;
      const int v = (int)((wb + k) * 32 + lane);
      const bool defer = act && found[k] < 0 && d[k] > F;
      const unsigned dm = __ballot_sync(0xffffffffu, defer);
      if (dm) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&sm.bu_n, __popc(dm));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (defer) {
          const int slot = base + __popc(dm & ((1u << lane) - 1u));
          if (slot < kBuQueue)
            q_v[slot] = v;
          else
            gq[slot - kBuQueue] = v;
        }
      }
      const bool got1 = act && found[k] >= 0;
      const bool got2 = ASYNC && act && !got1 && !defer && found2[k] >= 0;
      if (got1) {
        p.levels[v] = L + 1;
        if (PAR) p.parents[v] = found[k];
        acc.n1 += 1;
        acc.m1 += d[k];
      } else if (got2) {
        p.levels[v] = L + 2;
        if (PAR) p.parents[v] = found2[k];
        acc.n2 += 1;
        acc.m2 += d[k];
      }
      const uint32_t m1 = __ballot_sync(0xffffffffu, got1);
      const uint32_t m2 = __ballot_sync(0xffffffffu, got2);
      if (lane == 0 && (m1 | m2)) {
        const long long w = wb + k;
        red_or_u32(p.vis + w, m1 | m2);
        if (m1) red_or_u32(fbn + w, m1);
        if (ASYNC && m2) red_or_u32(fbn2 + w, m2);
      }
    }
  }
  __syncthreads();
  bu_drain<PAR, ASYNC>(p, sm, acc, L, fbc, fbn, fbn2, F, gq);
}

// Block-reduce the accumulators and publish them to the frontier descriptors
// (f1 and f2 null: nothing to publish, the accumulators are reset).
__device__ void publish_acc(Smem& sm, Acc& acc, FDesc* f1, FDesc* f2) {
  if (!f1 && !f2) {
    acc = Acc{0, 0, 0, 0};
    return;
  }
  long long v[4] = {acc.n1, acc.m1, acc.n2, acc.m2};
  block_sum_n<kBlock, 4, long long>(v, sm.red4);
  const long long n1 = v[0], m1 = v[1], n2 = v[2], m2 = v[3];
  if (threadIdx.x == 0) {
    if (f1 && n1) atomicAdd(&f1->n, (unsigned long long)n1);
    if (f1 && m1) atomicAdd(&f1->m, (unsigned long long)m1);
    if (f2 && n2) {
      atomicAdd(&f2->n, (unsigned long long)n2);
      atomicAdd(&f2->m, (unsigned long long)m2);
      atomicAdd(&f2->pend_n, (unsigned long long)n2);
      atomicAdd(&f2->pend_m, (unsigned long long)m2);
    }
  }
  acc = Acc{0, 0, 0, 0};
}

// Distributed clear of a bitmap (each CTA its slice).
__device__ void clear_bitmap(uint32_t* bm, long long nw) {
  const long long G = gridDim.x, b = blockIdx.x;
  const long long w0 = nw * b / G, w1 = nw * (b + 1) / G;
  for (long long w = w0 + threadIdx.x; w < w1; w += kBlock) bm[w] = 0u;
}

// Fills n int32 with val; the 16-byte aligned body is split evenly between
// the CTAs and written with vector stores, CTA 0 also writes the unaligned
// head and tail (the array is 4-byte aligned).
__device__ void fill_i32(int* a, long long n, int val) {
  const long long G = gridDim.x, b = blockIdx.x;
  long long head = (long long)(((16u - ((unsigned)(uintptr_t)a & 15u)) & 15u) >> 2);
  if (head > n) head = n;
  const long long body = (n - head) >> 2;
  const long long tail = head + body * 4;
  int4* b4 = reinterpret_cast<int4*>(a + head);
  const int4 v4 = make_int4(val, val, val, val);
  for (long long i = body * b / G + threadIdx.x, i1 = body * (b + 1) / G; i < i1; i += kBlock) b4[i] = v4;
  if (b == 0) {
    if (threadIdx.x < head) a[threadIdx.x] = val;
    if (tail + threadIdx.x < n) a[tail + threadIdx.x] = val;
  }
}

// Set-up of a traversal from p.src inside the traversal launch (the host
// only zeroes the control block): levels (and parents) -1, visited = the
// isolated vertices plus the source, frontier bitmaps empty but for the
// source's bit in level 0's, and, by CTA 0, the source's queue entry and
// level 0's frontier descriptor. Every word is written by one thread only,
// so the source's bits are part of the copy, not a second write; the
// source's own level and parent are written after the grid barrier that
// follows (the traversal never reads the level array).
template <bool PAR>
__device__ void init_traversal(const Params& p) {
  fill_i32(p.levels, p.V, -1);
  if (PAR) fill_i32(p.parents, p.V, -1);
  const long long G = gridDim.x, b = blockIdx.x;
  const long long nw = p.nwords;
  const long long sw = p.src >> 5;
  const uint32_t sbit = 1u << (p.src & 31);
  // the bitmaps' 64 padding words past V (all-visited in iso) go to the last CTA
  const long long w0 = nw * b / G, w1 = (b == G - 1) ? nw + 64 : nw * (b + 1) / G;
  for (long long w = w0 + threadIdx.x; w < w1; w += kBlock) {
    const uint32_t own = (w == sw) ? sbit : 0u;
    p.vis[w] = p.iso[w] | own;
    p.fb[0][w] = own;
    p.fb[1][w] = 0u;
    p.fb[2][w] = 0u;
    p.fb[3][w] = 0u;
  }
  if (b == 0 && threadIdx.x == 0) {
    const long long b0 = p.beg[p.src];
    const long long d = p.beg[p.src + 1] - b0;
    FDesc& f = p.ctl->fd[0];
    f.n = 1;
    f.m = (unsigned long long)d;
    if (d > 0) {
      const int bin = bin_of(d, p.small_max, p.medium_max);
      p.q[0][bin].ids[0] = p.src;
      p.q[0][bin].eb[0] = 0;
      p.q[0][bin].bg[0] = b0;
      f.bin[bin] = ((unsigned long long)d << 31) | 1ull;
    }
  }
}

// ---------------------------------------------------------------------------
// The persistent traversal kernel.
// ---------------------------------------------------------------------------
template <bool PAR>
__global__ void __launch_bounds__(kBlock, 2) k_bfs(Params p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  Ctl* ctl = p.ctl;
  if (p.absent_block > 0 && (int)blockIdx.x == p.absent_block - 1) return;  // test hook: never arrives
  if (threadIdx.x < 3) sm.cnt[threadIdx.x] = 0;
  if (p.policy == XBFS_POLICY_MLP && p.mlp) mlp_stage(p.mlp, sm.mlp_w);
  if (threadIdx.x == 0) sm.mlp_cache_dec = -1;
  __syncthreads();

  // Policy state and running sums live in shared memory, owned by thread 0:
  // kept in registers they would be carried by every thread through every
  // inner loop of the level.
  LoopState& ls = sm.ls;
  if (threadIdx.x == 0) {
    if (p.policy == XBFS_POLICY_MLP && p.mlp) {
      // the installed bound after the weights, over each feature's scale
      const float* sd = sm.mlp_w + 8;
      const float* P = sm.mlp_w + kMlpParams;
      for (int k = 0; k < 8; ++k) sm.mlp_q[k] = P[k] / sd[k];
    }
    ls.ps.count_prev = 0;
    ls.ps.is_change = 0;
    ls.ps.td_adaptive = kInfinite;
    ls.ps.hub_before = 0;
    ls.ps.hub_after = 0;
    ls.ps.tag_prev = 0;
    ls.ps.bu_dir = 0;
    ls.ps.n_prev = 1;
    ls.ps.prev_strategy = XBFS_TD_QUEUE;
    ls.vis_n = 0;
    ls.vis_m = 0;
    ls.pend_q_for = -1;
    ls.st_reached = 0;
    ls.st_msum = 0;
    ls.st_async = 0;
    for (int k = 0; k < 3; ++k) ls.st_strat[k] = 0;
    if (p.resume) {
      const ResumeState r = *p.rs;
      ls.vis_n = r.vis_n;
      ls.vis_m = r.vis_m;
      ls.pend_q_for = r.pend_q_for;
      ls.ps = r.ps;
    }
  }

  bool q_valid = true, b_valid = true;
  unsigned dirty = 1u;  // fb[i] may contain set bits
  Acc acc{0, 0, 0, 0};
  const uint32_t nb = gridDim.x;
  uint32_t epoch = 0;
  long long L = 0;
  if (p.fresh) {
    init_traversal<PAR>(p);
    if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.levels[p.src] = 0;
      if (PAR) p.parents[p.src] = p.src;
    }
  }
  if (p.resume) {
    const ResumeState r = *p.rs;
    L = r.L;
    q_valid = r.q_valid != 0;
    b_valid = r.b_valid != 0;
    dirty = r.dirty;
  }
  __syncthreads();
  for (;; ++L) {
    if (L >= p.stop_level) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        ResumeState r;
        r.L = L;
        r.q_valid = q_valid;
        r.b_valid = b_valid;
        r.dirty = dirty;
        r.vis_n = ls.vis_n;
        r.vis_m = ls.vis_m;
        r.pend_q_for = ls.pend_q_for;
        r.ps = ls.ps;
        *p.rs = r;
      }
      break;
    }
    if (L >= p.max_levels) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&ctl->bar.err, 0, (int)XBFS_ERR_INTERNAL);
      break;
    }
    FDesc* F0 = &ctl->fd[L & 3];
    FDesc* F1 = &ctl->fd[(L + 1) & 3];
    FDesc* F2 = &ctl->fd[(L + 2) & 3];
    FDesc* F3 = &ctl->fd[(L + 3) & 3];
    if (threadIdx.x == 0) {
      // every descriptor word this level needs, loaded together
      long long n_f = (long long)ld_cg_u64(&F0->n);
      long long m_f = (long long)ld_cg_u64(&F0->m);
      const long long pn = (long long)ld_cg_u64(&F1->pend_n);
      const long long pm = (long long)ld_cg_u64(&F1->pend_m);
      const long long own_pend = (long long)ld_cg_u64(&F0->pend_n);
      const bool from_bins = ld_cg_u64(&F0->pad) != 0;
#pragma unroll
      for (int b2 = 0; b2 < 3; ++b2) sm.bins[b2] = ld_cg_u64(&F0->bin[b2]);
      if (from_bins) {
        // a queue-output level of a symmetric graph: every vertex it found
        // has a neighbour, so its bins hold the whole frontier
        n_f = 0;
        m_f = 0;
#pragma unroll
        for (int b2 = 0; b2 < 3; ++b2) {
          n_f += (long long)(sm.bins[b2] & kCountMask);
          m_f += (long long)(sm.bins[b2] >> 31);
        }
      }
      sm.pend_next = pn;
      sm.spec = m_f <= kSpecEdges ? 1 : 0;
      int s = -1;
      if (n_f > 0) {
        ls.vis_n += n_f;
        ls.vis_m += m_f;
        if (blockIdx.x == 0) {
          ls.st_reached += n_f;
          ls.st_msum += m_f;
          ls.st_async += own_pend;
        }
        long long n_u = p.n_ni - ls.vis_n - pn;
        long long m_u = p.E - ls.vis_m - pm;
        if (n_u < 0) n_u = 0;
        if (m_u < 0) m_u = 0;
        sm.bu_dense = (n_u * XBFS_BU_DENSE_DIV >= p.V) ? 1 : 0;
        sm.asyncq_ok = (n_u * 4 < p.V) ? 1 : 0;
        sm.mark_ok = (n_u * XBFS_MARK_NU_DIV >= p.V && m_f * 2 >= p.V) ? 1 : 0;
        sm.qside_ok = (n_u * 64 <= p.V && (pn == 0 || ls.pend_q_for == L + 1)) ? 1 : 0;
        switch (p.policy) {
          case XBFS_POLICY_FORCED: {
            const long long i = L < p.n_forced ? L : p.n_forced - 1;
            s = (i >= 0) ? (int)p.forced[i] : XBFS_TD_QUEUE;
            if (s < 0 || s > 2) s = XBFS_TD_QUEUE;
            break;
          }
          case XBFS_POLICY_BEAMER:
            s = decide_beamer(ls.ps, n_f, m_f, m_u, p.V, p.beamer_alpha, p.beamer_beta);
            break;
          case XBFS_POLICY_MLP: {
            const float raw[8] = {(float)n_f, (float)m_f, (float)n_u, (float)m_u, (float)L,
                                  (float)ls.ps.prev_strategy, (float)ls.ps.n_prev, (float)m_f / (float)n_f};
            if (sm.mlp_cache_dec >= 0 && mlp_reuse_bound(raw, sm.mlp_cache_raw, sm.mlp_q) < sm.mlp_cache_margin) {
              s = sm.mlp_cache_dec;  // certified: the network would choose the same
            } else {
              s = -2;  // decided by warp 0 below
#pragma unroll
              for (int k = 0; k < 8; ++k) sm.mlp_raw[k] = raw[k];
            }
            break;
          }
          default:
            s = decide_reference(ls.ps, L, m_f, p.E, p.alpha);
        }
        if (s == XBFS_BU && !p.allow_bu) s = XBFS_TD_QUEUE;
        if (blockIdx.x == 0 && L < p.hist_cap) {
          LevelRecDev& r = p.hist[L];
          r.n_f = n_f;
          r.m_f = m_f;
          r.n_u = n_u;
          r.m_u = m_u;
          r.t0 = globaltimer_ns();
          r.t1 = 0;
          if (L > 0 && L - 1 < p.hist_cap) p.hist[L - 1].t1 = r.t0;
        }
        ls.ps.n_prev = n_f;
      }
      sm.strategy = s;
    }
    __syncthreads();
    if (sm.strategy == -2) {
      // the learned switch: warp 0 evaluates it while the block waits (one
      // warp keeps the shared-memory and shuffle traffic of the network small)
      if (threadIdx.x < 32) {
        int s2 = p.mlp ? mlp_decide(sm.mlp_w, sm.mlp_raw, threadIdx.x, sm.mlp_cache_raw, &sm.mlp_cache_dec,
                                    &sm.mlp_cache_margin)
                       : XBFS_TD_QUEUE;
        if (s2 == XBFS_BU && !p.allow_bu) s2 = XBFS_TD_QUEUE;
        if (threadIdx.x == 0) sm.strategy = s2;
      }
      __syncthreads();
    }
    const int S = sm.strategy;
    if (S < 0) break;  // empty frontier: done
    if (threadIdx.x == 0) {
      ls.ps.prev_strategy = S;
      if (blockIdx.x == 0) {
        if (L < p.hist_cap) p.hist[L].strategy = S;
        ls.st_strat[S] += 1;
        // counter used at level L+1 (last used at level L-1)
        ctl->heavy[(L + 1) & 1] = 0ull;
      }
    }
    // ---- housekeeping for slots no longer in use (first phase of the level)
    if (blockIdx.x == 0 && threadIdx.x < 8) reinterpret_cast<unsigned long long*>(F3)[threadIdx.x] = 0ull;
    const int c3 = (int)((L + 3) & 3);
    if (dirty & (1u << c3)) {
      clear_bitmap(p.fb[c3], p.nwords);
      dirty &= ~(1u << c3);
    }
    uint32_t* fbc = p.fb[L & 3];
    uint32_t* fbn = p.fb[(L + 1) & 3];
    uint32_t* fbn2 = p.fb[(L + 2) & 3];
    const int par = (int)(L & 1);

    if (S == XBFS_TD_QUEUE || S == XBFS_TD_SCAN) {
      const bool enq = (S == XBFS_TD_QUEUE) && (sm.pend_next == 0);
      // A top-down level with bitmap output (single scan, or a queue level
      // after an asynchronous bottom-up) can only have as many winners as
      // there are unvisited vertices; when those are few, the winners also
      // go straight into the next level's binned queue (one atomic each),
      // so a small next level expands the queue instead of sweeping the
      // bitmap (the bitmap stays valid too)
      const bool qside = !enq && sm.qside_ok;
      // A queue-output level of a symmetric graph publishes no frontier
      // counts: every vertex it finds has degree > 0 and lands in a bin, so
      // the next decision sums the bins (flagged in the descriptor's last
      // word) and the level saves the count atomics before its barrier.
      // Stepped launches keep the counts (the host reads them).
      const bool nm_bins = XBFS_NM_FROM_BINS && enq && p.allow_bu && p.fresh;
      FDesc* P1 = nm_bins ? nullptr : F1;
      if (nm_bins && blockIdx.x == 0 && threadIdx.x == 0) F1->pad = 1ull;
      // A level with bitmap output and many unvisited vertices runs in two
      // phases: marks of fresh targets into frontier L+1's bitmap without
      // atomics that return (the bitmap sweep, the medium and large bins
      // and the heavy list; the small bin still claims), then, after a
      // barrier, finalize_marks: levels, visited bits and statistics of the
      // marked vertices that no claim took
      // Without parents and with no early (asynchronous) entries in frontier
      // L+1's bitmap, the marks are blind: every edge sets its target's bit
      // with no read of the visited bitmap (on these levels nearly every
      // target is unvisited), and finalize_marks also clears the bits of
      // visited targets; claims then make way for marks in every expansion
      // path of the level, so no visited bit is set before the finalize.
      const int mark = !(XBFS_TD_MARK && !enq && p.head && sm.mark_ok && !qside)
                           ? 0
                           : ((!PAR && XBFS_TD_BLIND && sm.pend_next == 0) ? 2 : 1);
      QOut qo;
      for (int b2 = 0; b2 < 3; ++b2) qo.b[b2] = p.q[par ^ 1][b2];
      qo.ctr = F1->bin;
      // a CTA whose whole share is at most 32 small-bin entries takes the
      // warp-only path (no staging, no block reductions)
      const unsigned long long pk0 = sm.bins[0];
      const unsigned cnt0 = (unsigned)(pk0 & kCountMask);
      const unsigned i0 = (unsigned)((unsigned long long)cnt0 * blockIdx.x / nb);
      const unsigned i1 = (unsigned)((unsigned long long)cnt0 * (blockIdx.x + 1) / nb);
      const bool tiny = q_valid && (sm.bins[1] & kCountMask) == 0 && (sm.bins[2] & kCountMask) == 0 && i1 - i0 <= 32;
      if (tiny) {
        if (threadIdx.x < 32 && i1 > i0)
          gather_entries_warp<PAR>(p, qo, p.q[par][0], cnt0, pk0 >> 31, i0, i1, (int)L, enq, fbn, sm.spec != 0, P1,
                                   qside, mark == 2);
      } else {
        if (q_valid) {
          for (int bin = 2; bin >= 1; --bin) {
            const unsigned long long pk = sm.bins[bin];
            gather_bin<PAR>(p, sm, qo, acc, p.q[par][bin], (unsigned)(pk & kCountMask), pk >> 31, (int)L, enq, fbn,
                            qside, mark);
          }
          gather_entries<PAR>(p, sm, qo, acc, p.q[par][0], cnt0, pk0 >> 31, (int)L, enq, fbn, qside, mark == 2);
        } else if ((XBFS_TD_HEADS || mark) && !enq && p.head) {
          expand_bitmap_heads<PAR>(p, sm, acc, qo, fbc, (int)L, fbn, par, qside, mark);
        } else {
          expand_bitmap<PAR>(p, sm, qo, acc, fbc, (int)L, enq, fbn, par, qside);
        }
        if (enq) flush(sm, qo);
        publish_acc(sm, acc, P1, nullptr);
      }
      if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      if (!q_valid) {
        // heavy vertices deferred by the fused sweep: expand them grid-wide
        // (the list is complete only after the barrier; usually it is empty)
        const unsigned long long hk = ld_cg_u64(&ctl->heavy[par]);
        if ((hk & kCountMask) != 0) {
          gather_bin<PAR>(p, sm, qo, acc, p.heavy, (unsigned)(hk & kCountMask), hk >> 31, (int)L, enq, fbn, qside,
                          mark);
          if (enq) flush(sm, qo);
          publish_acc(sm, acc, P1, nullptr);
          if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
        }
      }
      if (mark) {
        finalize_marks(p, acc, (int)L, fbn, mark == 2);
        publish_acc(sm, acc, F1, nullptr);
        if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      }
      q_valid = enq || qside;
      b_valid = !enq;
      if (!enq) dirty |= 1u << ((L + 1) & 3);
    } else {
      if (!b_valid) {
        scatter_queue_to_bitmap(p, par, *F0, fbc);
        dirty |= 1u << (L & 3);
        if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      }
      // word-parallel while unvisited vertices are dense (the first
      // bottom-up level of a power-law graph), else over the compacted list
      // of unvisited vertices (few per bitmap word: most lanes of a word
      // would idle)
      const bool words = p.bu_mode >= 5 || (p.bu_mode == 0 && sm.bu_dense);
      // head records, where the graph has them, in the default mode (and
      // mode 6, word-parallel over head records only)
      const bool heads = XBFS_BU_HEADS && p.head != nullptr && (p.bu_mode == 0 || p.bu_mode == 6);
      // on a sparse bottom-up level (list probing, few unvisited vertices)
      // the level-(L+2) winners of the asynchronous rule also go into
      // frontier L+2's queue, warp-aggregated (its counters are not used by
      // anything else before level L+1), so a top-down level L+1 can
      // complete that queue beside its bitmap
      QOut qo2;
      for (int b2 = 0; b2 < 3; ++b2) qo2.b[b2] = p.q[par][b2];
      qo2.ctr = F2->bin;
      const bool asyncq = XBFS_ASYNC_QUEUE && XBFS_BU_ASYNC_LIST && p.async_bu && !words && sm.asyncq_ok;
      if (threadIdx.x == 0 && asyncq) ls.pend_q_for = L + 2;
      if (words && heads) {
        if (p.async_bu)
          bottom_up_heads<PAR, true>(p, sm, acc, (int)L, fbc, fbn, fbn2);
        else
          bottom_up_heads<PAR, false>(p, sm, acc, (int)L, fbc, fbn, fbn2);
      } else if (words) {
        if (p.async_bu)
          bottom_up_words<PAR, true>(p, sm, acc, (int)L, fbc, fbn, fbn2);
        else
          bottom_up_words<PAR, false>(p, sm, acc, (int)L, fbc, fbn, fbn2);
      } else if (p.async_bu && XBFS_BU_ASYNC_LIST) {
        if (heads)
          bottom_up<PAR, true, true>(p, sm, acc, (int)L, fbc, fbn, fbn2, qo2, asyncq);
        else
          bottom_up<PAR, true, false>(p, sm, acc, (int)L, fbc, fbn, fbn2, qo2, asyncq);
      } else if (heads) {
        bottom_up<PAR, false, true>(p, sm, acc, (int)L, fbc, fbn, fbn2, qo2, false);
      } else {
        bottom_up<PAR, false, false>(p, sm, acc, (int)L, fbc, fbn, fbn2, qo2, false);
      }
      publish_acc(sm, acc, F1, F2);
      if (!grid_sync(&ctl->bar, nb, epoch, p.timeout_ns)) break;
      q_valid = false;
      b_valid = true;
      dirty |= 1u << ((L + 1) & 3);
      if (p.async_bu) dirty |= 1u << ((L + 2) & 3);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->depth = (int)L;
    // a stepped launch adds its levels to what earlier launches counted
    ctl->reached += ls.st_reached;
    ctl->msum += ls.st_msum;
    ctl->n_async += ls.st_async;
    for (int k = 0; k < 3; ++k) ctl->strat_count[k] += ls.st_strat[k];
    if (L > 0 && L - 1 < p.hist_cap) p.hist[L - 1].t1 = globaltimer_ns();
  }
}

// Seeds the traversal: level/parent of the source, its bits, queue entry and
// frontier descriptor for level 0.
__global__ void k_seed(Params p, int src, int par_enabled) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  p.levels[src] = 0;
  if (par_enabled) p.parents[src] = src;
  const uint32_t word = (uint32_t)src >> 5, bit = 1u << (src & 31);
  p.vis[word] |= bit;
  p.fb[0][word] |= bit;
  const long long b0 = p.beg[src];
  const long long d = p.beg[src + 1] - b0;
  FDesc& f = p.ctl->fd[0];
  f.n = 1;
  f.m = (unsigned long long)d;
  if (d > 0) {
    const int bin = bin_of(d, p.small_max, p.medium_max);
    p.q[0][bin].ids[0] = src;
    p.q[0][bin].eb[0] = 0;
    p.q[0][bin].bg[0] = b0;
    f.bin[bin] = ((unsigned long long)d << 31) | 1ull;
  }
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
static xbfs_status ensure_workspace(Graph* g, int small_max, int medium_max) {
  SsWorkspace& w = g->ss;
  xbfs_status st;
  const long long nwords = (g->V + 31) / 32 + 64;
  if (!w.ready) {
    w.V = g->V;
    w.nwords = (size_t)nwords;
    if ((st = w.bits.ensure((size_t)nwords * 4 * 5))) return st;
    if ((st = w.ctl.ensure(sizeof(Ctl)))) return st;
    if ((st = w.rs.ensure(sizeof(ResumeState)))) return st;
    if ((st = w.ulist.ensure((size_t)nwords * 32 * 4))) return st;
    w.hist_cap = 1 << 16;
    if ((st = w.hist.ensure(sizeof(LevelRecDev) * (size_t)w.hist_cap))) return st;
    // heavy list of the fused sweep: vertices with degree > kHeavyDeg (<= degree > 16)
    const size_t hcap = (size_t)g->cnt_deg_gt[4] + 1;
    if ((st = w.heavy_ids.ensure(hcap * 4)) || (st = w.heavy_eb.ensure(hcap * 4)) ||
        (st = w.heavy_bg.ensure(hcap * 8)))
      return st;
    XBFS_CUDA_TRY(cudaEventCreate(&w.ev0));
    XBFS_CUDA_TRY(cudaEventCreate(&w.ev1));
    XBFS_CUDA_TRY(cudaEventCreate(&w.evk0));
    w.ready = true;
  }
  // queue capacities per bin: vertices with degree in the bin's range
  auto count_gt = [&](long long t) -> size_t {
    if (t < 1) return (size_t)g->V;
    int k = 0;
    while (k < 15 && (1ll << (k + 1)) <= t) ++k;
    return (size_t)g->cnt_deg_gt[k];
  };
  size_t cap[3];
  cap[0] = (size_t)g->V;
  cap[1] = std::min<size_t>((size_t)g->V, count_gt(small_max));
  cap[2] = std::min<size_t>((size_t)g->V, count_gt(medium_max));
  for (int b = 0; b < 3; ++b) {
    if (cap[b] + 1 > w.qcap[b] || !w.qids[0][b].p) {
      for (int par = 0; par < 2; ++par) {
        if ((st = w.qids[par][b].ensure((cap[b] + 1) * 4))) return st;
        if ((st = w.qeb[par][b].ensure((cap[b] + 1) * 4))) return st;
        if ((st = w.qbg[par][b].ensure((cap[b] + 1) * 8))) return st;
      }
      w.qcap[b] = cap[b] + 1;
    }
  }
  return XBFS_OK;
}

// Fills the kernel parameters for one traversal of g with options o.
static xbfs_status setup_params(Graph* g, const xbfs_opts& o, int* d_levels, int* d_parents, Params& p,
                                const void** kfn_out, size_t* smem_out, int* grid_out) {
  SsWorkspace& w = g->ss;
  memset(&p, 0, sizeof(p));
  p.beg = g->beg.as<long long>();
  p.head = g->head.as<int4>();
  p.csr = g->csr.as<int>();
  p.V = g->V;
  p.E = g->E;
  p.levels = d_levels;
  p.parents = d_parents;
  uint32_t* bits = w.bits.as<uint32_t>();
  p.vis = bits;
  for (int i = 0; i < 4; ++i) p.fb[i] = bits + (size_t)(i + 1) * w.nwords;
  for (int par = 0; par < 2; ++par)
    for (int b = 0; b < 3; ++b) {
      p.q[par][b].ids = w.qids[par][b].as<int>();
      p.q[par][b].eb = w.qeb[par][b].as<unsigned>();
      p.q[par][b].bg = w.qbg[par][b].as<long long>();
    }
  p.heavy.ids = w.heavy_ids.as<int>();
  p.heavy.eb = w.heavy_eb.as<unsigned>();
  p.heavy.bg = w.heavy_bg.as<long long>();
  p.ulist = w.ulist.as<int>();
  p.ctl = w.ctl.as<Ctl>();
  p.hist = w.hist.as<LevelRecDev>();
  p.hist_cap = w.hist_cap;
  p.forced = w.forced.as<signed char>();
  p.n_forced = o.n_forced;
  p.nwords = (g->V + 31) / 32;
  p.n_ni = g->symmetric ? g->V - g->n_isolated : g->V;
  p.policy = o.policy;
  p.alpha = o.alpha;
  p.async_bu = o.async_bu ? 1 : 0;
  p.small_max = o.small_max;
  p.medium_max = o.medium_max;
  p.beamer_alpha = o.beamer_alpha > 0 ? o.beamer_alpha : 14.f;
  p.beamer_beta = o.beamer_beta > 0 ? o.beamer_beta : 24.f;
  p.timeout_ns = o.wait_timeout_us > 0 ? (unsigned long long)o.wait_timeout_us * 1000ull
                                        : 10ull * 1000 * 1000 * 1000;
  p.absent_block = o.test_absent_block;
  p.max_levels = g->V + 2;
  extern const float* mlp_device_weights(int device);
  p.mlp = mlp_device_weights(g->device);
  if (o.policy == XBFS_POLICY_MLP && !p.mlp) p.policy = XBFS_POLICY_HEURISTIC;
  p.allow_bu = g->symmetric ? 1 : 0;

  const bool par_on = d_parents != nullptr;
  const void* kfn = par_on ? (const void*)k_bfs<true> : (const void*)k_bfs<false>;
  // the weight copy of the learned switch sits at the end of Smem and is only
  // allocated for launches that use it (shared memory taken from L1)
  const size_t smem = sizeof(Smem) - (p.policy == XBFS_POLICY_MLP ? 0 : sizeof(((Smem*)0)->mlp_w));
  XBFS_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)));
  int nsm = 0, per_sm = 0;
  XBFS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device));
  XBFS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kBlock, smem));
  if (per_sm < 1) return set_error(XBFS_ERR_INTERNAL, "traversal kernel cannot be resident");
  int grid = nsm * per_sm;
  if (o.grid_dim > 0 && o.grid_dim < grid) grid = o.grid_dim;
  w.grid = grid;
  w.block = kBlock;
  p.rs = w.rs.as<ResumeState>();
  p.bu_mode = o.bu_probe;
  p.stop_level = LLONG_MAX;
  p.resume = 0;
  p.fresh = 0;
  p.iso = g->iso.as<uint32_t>();
  *kfn_out = kfn;
  *smem_out = smem;
  *grid_out = grid;
  return XBFS_OK;

}

// Initial state of a traversal from src: levels/parents -1, visited = isolated
// vertices, frontier bitmaps and control block cleared, source seeded.
static xbfs_status init_state(Graph* g, const Params& p, int src, bool par_on, cudaStream_t s) {
  SsWorkspace& w = g->ss;
  XBFS_CUDA_TRY(cudaMemsetAsync(p.levels, 0xff, (size_t)g->V * 4, s));
  if (par_on) XBFS_CUDA_TRY(cudaMemsetAsync(p.parents, 0xff, (size_t)g->V * 4, s));
  XBFS_CUDA_TRY(cudaMemcpyAsync(p.vis, g->iso.p, w.nwords * 4, cudaMemcpyDeviceToDevice, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.fb[0], 0, w.nwords * 4 * 4, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(Ctl), s));
  k_seed<<<1, 32, 0, s>>>(p, src, par_on ? 1 : 0);
  XBFS_CUDA_TRY(cudaGetLastError());
  return XBFS_OK;
}

xbfs_status bfs_single(Graph* g, int32_t src, int32_t* levels, int32_t* parents, const xbfs_opts* uopts,
                       xbfs_stats* stats) {
  const auto t_start = std::chrono::steady_clock::now();
  xbfs_opts o;
  xbfs_opts_init(&o);
  if (uopts) {
    if (uopts->struct_size != (int32_t)sizeof(xbfs_opts))
      return set_error(XBFS_ERR_INVALID_ARG, "xbfs_opts.struct_size = %d, expected %zu (call xbfs_opts_init)",
                       uopts->struct_size, sizeof(xbfs_opts));
    o = *uopts;
  }
  if (!g) return set_error(XBFS_ERR_INVALID_ARG, "graph is NULL");
  if (!levels) return set_error(XBFS_ERR_INVALID_ARG, "levels is NULL");
  if (src < 0 || (int64_t)src >= g->V)
    return set_error(XBFS_ERR_INVALID_ARG, "source %d out of range [0, %lld)", src, (long long)g->V);
  if (g->E >= (1ll << 32))
    return set_error(XBFS_ERR_UNSUPPORTED, "single-source path needs E < 2^32 (E = %lld)", (long long)g->E);
  if (o.padding != 1)
    return set_error(XBFS_ERR_INVALID_ARG,
                     "padding = %d: only 1 is supported (the reference's bottom-up is incorrect for "
                     "padding > 1)", o.padding);
  if (o.small_max <= 0) o.small_max = 32;
  if (o.medium_max < o.small_max) o.medium_max = o.small_max;
  if (o.policy == XBFS_POLICY_FORCED && (!o.forced || o.n_forced <= 0))
    return set_error(XBFS_ERR_INVALID_ARG, "forced policy needs a non-empty forced[] array");
  if (o.policy < 0 || o.policy > 3) return set_error(XBFS_ERR_INVALID_ARG, "bad policy %d", o.policy);
  if (o.bu_probe < 0 || o.bu_probe > 6) return set_error(XBFS_ERR_INVALID_ARG, "bad bu_probe %d", o.bu_probe);
  if (!(o.alpha > 0)) o.alpha = 0.1f;

  DeviceGuard dg(g->device);
  xbfs_status st = ensure_workspace(g, o.small_max, o.medium_max);
  if (st) return st;
  SsWorkspace& w = g->ss;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;

  const bool lv_dev = is_device_pointer(levels);
  const bool par_dev = parents && is_device_pointer(parents);
  int* d_levels = lv_dev ? levels : nullptr;
  int* d_parents = par_dev ? parents : nullptr;
  if (!lv_dev) {
    if ((st = w.levels_tmp.ensure((size_t)g->V * 4))) return st;
    d_levels = w.levels_tmp.as<int>();
  }
  if (parents && !par_dev) {
    if ((st = w.parents_tmp.ensure((size_t)g->V * 4))) return st;
    d_parents = w.parents_tmp.as<int>();
  }
  if (o.policy == XBFS_POLICY_FORCED) {
    if (o.n_forced > w.forced_cap) {
      if ((st = w.forced.ensure((size_t)o.n_forced))) return st;
      w.forced_cap = o.n_forced;
    }
    XBFS_CUDA_TRY(cudaMemcpyAsync(w.forced.p, o.forced, (size_t)o.n_forced, cudaMemcpyHostToDevice, s));
  }

  Params p;
  const void* kfn = nullptr;
  size_t smem = 0;
  int grid = 0;
  if ((st = setup_params(g, o, d_levels, d_parents, p, &kfn, &smem, &grid))) return st;

  // ---- one launch: it sets up the traversal state itself (init_traversal);
  // only the control block, which holds the launch's grid barrier, is
  // zeroed beforehand
  XBFS_CUDA_TRY(cudaEventRecord(w.ev0, s));
  XBFS_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(Ctl), s));
  p.fresh = 1;
  p.src = src;
  void* args[] = {&p};
  XBFS_CUDA_TRY(cudaEventRecord(w.evk0, s));
  XBFS_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kBlock), args, smem, s));
  XBFS_CUDA_TRY(cudaEventRecord(w.ev1, s));
  Ctl hctl;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&hctl, p.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  if (!lv_dev) XBFS_CUDA_TRY(cudaMemcpyAsync(levels, d_levels, (size_t)g->V * 4, cudaMemcpyDeviceToHost, s));
  if (parents && !par_dev)
    XBFS_CUDA_TRY(cudaMemcpyAsync(parents, d_parents, (size_t)g->V * 4, cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  if (hctl.bar.err != 0)
    return set_error((xbfs_status)hctl.bar.err, "traversal kernel reported %s", xbfs_strerror(hctl.bar.err));
  w.last_levels = hctl.depth;
  float ms = 0, kms = 0;
  XBFS_CUDA_TRY(cudaEventElapsedTime(&ms, w.ev0, w.ev1));
  XBFS_CUDA_TRY(cudaEventElapsedTime(&kms, w.evk0, w.ev1));

  if (o.trace || stats) {
    const int nl = std::min(hctl.depth, w.hist_cap);
    std::vector<LevelRecDev> h(nl);
    if (nl > 0) XBFS_CUDA_TRY(cudaMemcpy(h.data(), p.hist, sizeof(LevelRecDev) * nl, cudaMemcpyDeviceToHost));
    w.trace.resize(nl);
    for (int i = 0; i < nl; ++i) {
      w.trace[i].level = i;
      w.trace[i].strategy = h[i].strategy;
      w.trace[i].n_f = h[i].n_f;
      w.trace[i].m_f = h[i].m_f;
      w.trace[i].n_u = h[i].n_u;
      w.trace[i].m_u = h[i].m_u;
      w.trace[i].us = (h[i].t1 > h[i].t0) ? (double)(h[i].t1 - h[i].t0) * 1e-3 : 0.0;
    }
  }
  if (stats) {
    stats->struct_size = (int32_t)sizeof(xbfs_stats);
    stats->depth = hctl.depth;
    stats->reached = (int64_t)hctl.reached;
    stats->edges_mc = (int64_t)(hctl.msum / 2);
    stats->device_ms = ms;
    stats->kernel_ms = kms;
    stats->n_td_queue = hctl.strat_count[0];
    stats->n_td_scan = hctl.strat_count[1];
    stats->n_bu = hctl.strat_count[2];
    stats->n_async = (int32_t)hctl.n_async;
    stats->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  }
  return XBFS_OK;
}

// n single-source traversals in one call, pipelined: while traversal i runs
// on the graph's stream, the level array of traversal i-1 is copied out on a
// second stream, so a host output costs max(kernel, copy) per source instead
// of their sum. Two device level buffers alternate; traversal i+2 waits for
// the copy that frees its buffer. With device outputs the kernels write the
// rows directly and nothing is copied.
xbfs_status bfs_many(Graph* g, const int32_t* srcs, int32_t n, int32_t* levels, const xbfs_opts* uopts,
                     xbfs_stats* stats) {
  const auto t_start = std::chrono::steady_clock::now();
  xbfs_opts o;
  xbfs_opts_init(&o);
  if (uopts) {
    if (uopts->struct_size != (int32_t)sizeof(xbfs_opts))
      return set_error(XBFS_ERR_INVALID_ARG, "xbfs_opts.struct_size = %d, expected %zu (call xbfs_opts_init)",
                       uopts->struct_size, sizeof(xbfs_opts));
    o = *uopts;
  }
  if (!g || !srcs || !levels || n <= 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  for (int i = 0; i < n; ++i)
    if (srcs[i] < 0 || (int64_t)srcs[i] >= g->V)
      return set_error(XBFS_ERR_INVALID_ARG, "source %d (%d) out of range [0, %lld)", i, srcs[i], (long long)g->V);
  if (g->E >= (1ll << 32))
    return set_error(XBFS_ERR_UNSUPPORTED, "single-source path needs E < 2^32 (E = %lld)", (long long)g->E);
  if (o.padding != 1) return set_error(XBFS_ERR_INVALID_ARG, "padding = %d: only 1 is supported", o.padding);
  if (o.policy == XBFS_POLICY_FORCED && (!o.forced || o.n_forced <= 0))
    return set_error(XBFS_ERR_INVALID_ARG, "forced policy needs a non-empty forced[] array");
  if (o.policy < 0 || o.policy > 3) return set_error(XBFS_ERR_INVALID_ARG, "bad policy %d", o.policy);
  if (o.bu_probe < 0 || o.bu_probe > 6) return set_error(XBFS_ERR_INVALID_ARG, "bad bu_probe %d", o.bu_probe);
  if (o.small_max <= 0) o.small_max = 32;
  if (o.medium_max < o.small_max) o.medium_max = o.small_max;
  if (!(o.alpha > 0)) o.alpha = 0.1f;

  DeviceGuard dg(g->device);
  xbfs_status st = ensure_workspace(g, o.small_max, o.medium_max);
  if (st) return st;
  SsWorkspace& w = g->ss;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;
  const bool dev_out = is_device_pointer(levels);
  const size_t row = (size_t)g->V;
  if (!dev_out) {
    if ((st = w.levels_tmp.ensure(row * 4)) || (st = w.levels_tmp2.ensure(row * 4))) return st;
    if (!w.copy_stream) XBFS_CUDA_TRY(cudaStreamCreateWithFlags(&w.copy_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      if (!w.ev_done[b]) XBFS_CUDA_TRY(cudaEventCreateWithFlags(&w.ev_done[b], cudaEventDisableTiming));
      if (!w.ev_copied[b]) XBFS_CUDA_TRY(cudaEventCreateWithFlags(&w.ev_copied[b], cudaEventDisableTiming));
    }
  }
  if ((st = w.ctl_log.ensure(sizeof(Ctl) * (size_t)n))) return st;
  if (o.policy == XBFS_POLICY_FORCED) {
    if (o.n_forced > w.forced_cap) {
      if ((st = w.forced.ensure((size_t)o.n_forced))) return st;
      w.forced_cap = o.n_forced;
    }
    XBFS_CUDA_TRY(cudaMemcpyAsync(w.forced.p, o.forced, (size_t)o.n_forced, cudaMemcpyHostToDevice, s));
  }
  int* dbuf[2] = {w.levels_tmp.as<int>(), w.levels_tmp2.as<int>()};
  Params p;
  const void* kfn = nullptr;
  size_t smem = 0;
  int grid = 0;
  if ((st = setup_params(g, o, dev_out ? levels : dbuf[0], nullptr, p, &kfn, &smem, &grid))) return st;

  XBFS_CUDA_TRY(cudaEventRecord(w.ev0, s));
  // every traversal has its own control block (grid barrier, descriptors,
  // results), all zeroed here at once, so a traversal is a single launch
  Ctl* ctls = w.ctl_log.as<Ctl>();
  XBFS_CUDA_TRY(cudaMemsetAsync(ctls, 0, sizeof(Ctl) * (size_t)n, s));
  p.fresh = 1;
  auto copy_out = [&](int i) -> xbfs_status {
    const int b = i & 1;
    XBFS_CUDA_TRY(cudaStreamWaitEvent(w.copy_stream, w.ev_done[b], 0));
    XBFS_CUDA_TRY(cudaMemcpyAsync(levels + (size_t)i * row, dbuf[b], row * 4, cudaMemcpyDeviceToHost,
                                  w.copy_stream));
    XBFS_CUDA_TRY(cudaEventRecord(w.ev_copied[b], w.copy_stream));
    return XBFS_OK;
  };
  for (int i = 0; i < n; ++i) {
    const int b = i & 1;
    if (dev_out) {
      p.levels = levels + (size_t)i * row;
    } else {
      p.levels = dbuf[b];
      if (i >= 2) XBFS_CUDA_TRY(cudaStreamWaitEvent(s, w.ev_copied[b], 0));  // buffer copied out
    }
    p.src = srcs[i];
    p.ctl = ctls + i;
    void* args[] = {&p};
    XBFS_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kBlock), args, smem, s));
    if (!dev_out) {
      XBFS_CUDA_TRY(cudaEventRecord(w.ev_done[b], s));
      // the copy of the previous traversal is issued after this launch, so
      // a pageable destination (whose copy blocks the host) still overlaps
      if (i > 0 && (st = copy_out(i - 1))) return st;
    }
  }
  if (!dev_out && (st = copy_out(n - 1))) return st;
  XBFS_CUDA_TRY(cudaEventRecord(w.ev1, s));
  std::vector<Ctl> hctl((size_t)n);
  XBFS_CUDA_TRY(cudaMemcpyAsync(hctl.data(), w.ctl_log.p, sizeof(Ctl) * (size_t)n, cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  if (!dev_out) XBFS_CUDA_TRY(cudaStreamSynchronize(w.copy_stream));
  long long reached = 0, msum = 0, n_async = 0;
  int depth = 0, sc[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    if (hctl[i].bar.err != 0)
      return set_error((xbfs_status)hctl[i].bar.err, "traversal %d reported %s", i, xbfs_strerror(hctl[i].bar.err));
    reached += (long long)hctl[i].reached;
    msum += (long long)hctl[i].msum;
    n_async += (long long)hctl[i].n_async;
    depth = std::max(depth, hctl[i].depth);
    for (int k = 0; k < 3; ++k) sc[k] += hctl[i].strat_count[k];
  }
  if (stats) {
    float ms = 0;
    XBFS_CUDA_TRY(cudaEventElapsedTime(&ms, w.ev0, w.ev1));
    stats->struct_size = (int32_t)sizeof(xbfs_stats);
    stats->depth = depth;
    stats->reached = reached;
    stats->edges_mc = msum / 2;
    stats->device_ms = ms;
    stats->kernel_ms = 0.0;
    stats->n_td_queue = sc[0];
    stats->n_td_scan = sc[1];
    stats->n_bu = sc[2];
    stats->n_async = (int32_t)n_async;
    stats->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  }
  return XBFS_OK;
}

// Per-level strategy costs for training the learned switch: at every level
// the whole traversal state is snapshotted, the level is run once with each
// strategy from that snapshot (one stepped launch each, timed with the
// device's globaltimer between the level's start and its closing barrier),
// and the traversal continues along the cheapest strategy (follow = 0) or
// the reference heuristic's choice (follow = 1).
xbfs_status level_costs(Graph* g, int32_t src, int32_t follow, int32_t cap, float* costs, xbfs_level_trace* trace,
                        int32_t* n_out) {
  if (!g || !costs || !trace || !n_out || cap <= 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  if (src < 0 || (int64_t)src >= g->V) return set_error(XBFS_ERR_INVALID_ARG, "source out of range");
  if (g->E >= (1ll << 32)) return set_error(XBFS_ERR_UNSUPPORTED, "needs E < 2^32");
  xbfs_opts o;
  xbfs_opts_init(&o);
  DeviceGuard dg(g->device);
  xbfs_status st = ensure_workspace(g, o.small_max, o.medium_max);
  if (st) return st;
  SsWorkspace& w = g->ss;
  cudaStream_t s = g->stream;
  if ((st = w.levels_tmp.ensure((size_t)g->V * 4))) return st;
  if (cap + 1 > w.forced_cap) {
    if ((st = w.forced.ensure((size_t)cap + 1))) return st;
    w.forced_cap = cap + 1;
  }
  std::vector<signed char> forced((size_t)cap + 1, 0);
  o.policy = XBFS_POLICY_FORCED;
  o.forced = (const int8_t*)forced.data();
  o.n_forced = cap + 1;
  Params p;
  const void* kfn = nullptr;
  size_t smem = 0;
  int grid = 0;
  if ((st = setup_params(g, o, w.levels_tmp.as<int>(), nullptr, p, &kfn, &smem, &grid))) return st;
  // A snapshot holds the state a level starts from: levels, the five
  // bitmaps, the live part of the frontier queue (parity of the level, the
  // entries its descriptor counts), the control block and the resume state.
  struct Piece { void* p; size_t n; };
  struct Snap { DevBuf* buf; std::vector<Piece> pieces; };
  auto live_pieces = [&](long long level, const FDesc& f) {
    std::vector<Piece> v;
    v.push_back({w.levels_tmp.p, (size_t)g->V * 4});
    v.push_back({w.bits.p, w.nwords * 4 * 5});
    const int par = (int)(level & 1);
    for (int b = 0; b < 3; ++b) {
      const size_t cnt = (size_t)(f.bin[b] & kCountMask);
      if (!cnt) continue;
      v.push_back({w.qids[par][b].p, cnt * 4});
      v.push_back({w.qeb[par][b].p, cnt * 4});
      v.push_back({w.qbg[par][b].p, cnt * 8});
    }
    v.push_back({w.ctl.p, sizeof(Ctl)});
    v.push_back({w.rs.p, sizeof(ResumeState)});
    return v;
  };
  size_t total = 0;
  {
    FDesc full;
    memset(&full, 0, sizeof(full));
    for (int b = 0; b < 3; ++b) full.bin[b] = (unsigned long long)w.qcap[b];
    for (auto& pc : live_pieces(0, full)) total += (pc.n + 255) & ~(size_t)255;
  }
  if ((st = w.snap.ensure(total))) return st;
  if ((st = w.snap2.ensure(total))) return st;
  Snap s1{&w.snap, {}}, s2{&w.snap2, {}};
  auto copy_snap = [&](Snap& sn, bool save) -> xbfs_status {
    size_t off = 0;
    for (auto& pc : sn.pieces) {
      char* sp = sn.buf->as<char>() + off;
      XBFS_CUDA_TRY(cudaMemcpyAsync(save ? sp : pc.p, save ? pc.p : sp, pc.n, cudaMemcpyDeviceToDevice, s));
      off += (pc.n + 255) & ~(size_t)255;
    }
    return XBFS_OK;
  };
  auto save_snap = [&](Snap& sn, long long level, const FDesc& f) -> xbfs_status {
    sn.pieces = live_pieces(level, f);
    return copy_snap(sn, true);
  };
  auto copy_all = [&](bool save) -> xbfs_status { return copy_snap(s1, save); };
  auto run_level = [&](int L, int strategy, int policy, LevelRecDev* rec) -> xbfs_status {
    forced[L] = (signed char)strategy;
    XBFS_CUDA_TRY(cudaMemcpyAsync(w.forced.p, forced.data(), (size_t)L + 1, cudaMemcpyHostToDevice, s));
    XBFS_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(GridBarrier), s));  // fresh barrier epoch
    Params q = p;
    q.policy = policy;
    q.resume = L > 0 ? 1 : 0;
    q.stop_level = L + 1;
    void* args[] = {&q};
    XBFS_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kBlock), args, smem, s));
    XBFS_CUDA_TRY(cudaMemcpyAsync(rec, p.hist + L, sizeof(LevelRecDev), cudaMemcpyDeviceToHost, s));
    int err = 0;
    XBFS_CUDA_TRY(cudaMemcpyAsync(&err, &p.ctl->bar.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    XBFS_CUDA_TRY(cudaStreamSynchronize(s));
    if (err) return set_error((xbfs_status)err, "stepped traversal reported %s", xbfs_strerror(err));
    return XBFS_OK;
  };
  if ((st = init_state(g, p, src, false, s))) return st;
  int n = 0;
  for (int L = 0; L < cap; ++L) {
    // is there a level-L frontier?
    FDesc f;
    XBFS_CUDA_TRY(cudaMemcpyAsync(&f, &p.ctl->fd[L & 3], sizeof(FDesc), cudaMemcpyDeviceToHost, s));
    XBFS_CUDA_TRY(cudaStreamSynchronize(s));
    if (f.n == 0) break;
    if ((st = save_snap(s1, L, f))) return st;
    LevelRecDev rec[3];
    for (int k = 0; k < 3; ++k) {
      if (k > 0 && (st = copy_all(false))) return st;
      if ((st = run_level(L, k, XBFS_POLICY_FORCED, &rec[k]))) return st;
      costs[L * 3 + k] = (rec[k].t1 > rec[k].t0) ? (float)((rec[k].t1 - rec[k].t0) * 1e-3) : 0.f;
      // one level of lookahead: a strategy also fixes the form of the next
      // frontier (queue or bitmap) and with it the next level's input cost,
      // so the cost of k is this level plus the cheapest next level (each
      // strategy tried from the state k left behind)
      if (L + 1 < cap) {
        FDesc nf;
        XBFS_CUDA_TRY(cudaMemcpyAsync(&nf, &p.ctl->fd[(L + 1) & 3], sizeof(FDesc), cudaMemcpyDeviceToHost, s));
        XBFS_CUDA_TRY(cudaStreamSynchronize(s));
        if (nf.n != 0) {
          if ((st = save_snap(s2, L + 1, nf))) return st;
          float best = 0.f;
          for (int j = 0; j < 3; ++j) {
            if (j > 0 && (st = copy_snap(s2, false))) return st;
            LevelRecDev r2;
            if ((st = run_level(L + 1, j, XBFS_POLICY_FORCED, &r2))) return st;
            const float t2 = (r2.t1 > r2.t0) ? (float)((r2.t1 - r2.t0) * 1e-3) : 0.f;
            if (j == 0 || t2 < best) best = t2;
          }
          costs[L * 3 + k] += best;
        }
      }
    }
    int choice = 0;
    if (follow == 1) {
      LevelRecDev hr;
      if ((st = copy_all(false))) return st;
      if ((st = run_level(L, 0, XBFS_POLICY_HEURISTIC, &hr))) return st;
      choice = hr.strategy;
    } else {
      for (int k = 1; k < 3; ++k)
        if (costs[L * 3 + k] < costs[L * 3 + choice]) choice = k;
    }
    if ((st = copy_all(false))) return st;
    LevelRecDev cr;
    if ((st = run_level(L, choice, XBFS_POLICY_FORCED, &cr))) return st;
    trace[L].level = L;
    trace[L].strategy = cr.strategy;
    trace[L].n_f = cr.n_f;
    trace[L].m_f = cr.m_f;
    trace[L].n_u = cr.n_u;
    trace[L].m_u = cr.m_u;
    trace[L].us = (cr.t1 > cr.t0) ? (double)(cr.t1 - cr.t0) * 1e-3 : 0.0;
    n = L + 1;
  }
  *n_out = n;
  return XBFS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free traversal. Callers that must not allocate device memory at
// traversal time: processes whose device memory is pre-divided by an arena or
// pool that owns nearly all of HBM (a cudaMalloc beside it fails or fragments
// the pool), and latency-bound service loops in which cudaMalloc/cudaFree
// would stall the device (cudaFree synchronises it). They load the graph once
// at start-up and then traverse with this path, which takes the k_bfs
// workspace from the fixed array of static_scratch.cu instead of the per-graph
// workspace that bfs_single grows with cudaMalloc. The launch is the same
// kernel with the same parameters; only where the workspace lives differs.
//
// Layout of the scratch (each region 256-byte aligned), for a graph of V
// vertices, nw = ceil(V/32) + 64 bitmap words:
//   bits    5 * nw * 4      visited + 4 frontier bitmaps   cleared every call
//   ctl     sizeof(Ctl)     barrier, descriptors, counters cleared every call
//   rs      sizeof(ResumeState)                            unused (no stepping)
//   ulist   nw * 32 * 4     bottom-up vertex lists         written before read
//   heavy   3 arrays, (vertices of degree > 16) + 1 each   written before read
//   queues  2 parities x 3 bins x (cap + 1) x (4 + 4 + 8)  written before read
//   forced  n_forced bytes (forced policy only)            copied every call
// No per-level history is kept (hist_cap = 0), so trace is not available.
// ---------------------------------------------------------------------------
extern cudaError_t noalloc_scratch_address(void** ptr);

namespace {

// Shared memory of a traversal launch: the learned switch's weight copy at
// the end of Smem is only allocated for launches that use it (the rest of
// the SM's unified storage stays L1).
constexpr size_t kSmemNoMlp = sizeof(Smem) - sizeof(((Smem*)0)->mlp_w);

struct NoallocDevice {
  bool ready = false;
  int grid[2][2] = {{0, 0}, {0, 0}};  // resident CTAs: [parents on][learned switch on]
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc[64];

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Per-device set-up, run once with `device` current: the launch shapes of
// both kernel instantiations, with and without the learned switch's shared
// memory. The scratch address itself is resolved again on every call
// (noalloc_scratch), so a context that was reset and re-created gets the
// address of the array in its own module image.
xbfs_status noalloc_setup(int device, NoallocDevice** out) {
  if (device < 0 || device >= 64) return set_error(XBFS_ERR_INVALID_ARG, "device %d out of range", device);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocDevice& d = g_noalloc[device];
  if (!d.ready) {
    int nsm = 0;
    XBFS_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const void* fns[2] = {(const void*)k_bfs<false>, (const void*)k_bfs<true>};
    for (int i = 0; i < 2; ++i) {
      XBFS_CUDA_TRY(cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)));
      for (int m = 0; m < 2; ++m) {
        int per_sm = 0;
        XBFS_CUDA_TRY(
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fns[i], kBlock, m ? sizeof(Smem) : kSmemNoMlp));
        if (per_sm < 1) return set_error(XBFS_ERR_INTERNAL, "traversal kernel cannot be resident");
        d.grid[i][m] = nsm * per_sm;
      }
    }
    d.ready = true;
  }
  *out = &d;
  return XBFS_OK;
}

// Device address of the static scratch in the current context; checked.
xbfs_status noalloc_scratch(int device, unsigned char** out) {
  void* ptr = nullptr;
  const cudaError_t e = noalloc_scratch_address(&ptr);
  if (e != cudaSuccess || !ptr) {
    cudaGetLastError();
    return set_error(XBFS_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed on device %d: %s", device,
                     cudaGetErrorString(e));
  }
  *out = (unsigned char*)ptr;
  return XBFS_OK;
}

// Device memory of `device` (plain or managed): the traversal kernel writes
// the outputs directly.
bool on_device(const void* ptr, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

}  // namespace

xbfs_status bfs_noalloc(Graph* g, int32_t src, int32_t* levels, int32_t* parents, const xbfs_opts* uopts,
                        xbfs_stats* stats) {
  const auto t_start = std::chrono::steady_clock::now();
  xbfs_opts o;
  xbfs_opts_init(&o);
  if (uopts) {
    if (uopts->struct_size != (int32_t)sizeof(xbfs_opts))
      return set_error(XBFS_ERR_INVALID_ARG, "xbfs_opts.struct_size = %d, expected %zu (call xbfs_opts_init)",
                       uopts->struct_size, sizeof(xbfs_opts));
    o = *uopts;
  }
  if (!g) return set_error(XBFS_ERR_INVALID_ARG, "graph is NULL");
  if (!levels) return set_error(XBFS_ERR_INVALID_ARG, "levels is NULL");
  if (src < 0 || (int64_t)src >= g->V)
    return set_error(XBFS_ERR_INVALID_ARG, "source %d out of range [0, %lld)", src, (long long)g->V);
  if (g->E >= (1ll << 32))
    return set_error(XBFS_ERR_UNSUPPORTED, "single-source path needs E < 2^32 (E = %lld)", (long long)g->E);
  if (o.padding != 1) return set_error(XBFS_ERR_INVALID_ARG, "padding = %d: only 1 is supported", o.padding);
  if (o.trace) return set_error(XBFS_ERR_UNSUPPORTED, "xbfs_bfs_noalloc keeps no per-level trace (trace = 1)");
  if (o.small_max <= 0) o.small_max = 32;
  if (o.medium_max < o.small_max) o.medium_max = o.small_max;
  if (o.policy == XBFS_POLICY_FORCED && (!o.forced || o.n_forced <= 0))
    return set_error(XBFS_ERR_INVALID_ARG, "forced policy needs a non-empty forced[] array");
  if (o.policy < 0 || o.policy > 3) return set_error(XBFS_ERR_INVALID_ARG, "bad policy %d", o.policy);
  if (o.bu_probe < 0 || o.bu_probe > 6) return set_error(XBFS_ERR_INVALID_ARG, "bad bu_probe %d", o.bu_probe);
  if (!(o.alpha > 0)) o.alpha = 0.1f;

  DeviceGuard dg(g->device);
  if (!on_device(levels, g->device))
    return set_error(XBFS_ERR_INVALID_ARG, "xbfs_bfs_noalloc needs levels in device memory of the graph's device %d",
                     g->device);
  if (parents && !on_device(parents, g->device))
    return set_error(XBFS_ERR_INVALID_ARG, "xbfs_bfs_noalloc needs parents in device memory of the graph's device %d",
                     g->device);
  NoallocDevice* dev = nullptr;
  xbfs_status st = noalloc_setup(g->device, &dev);
  if (st) return st;
  unsigned char* base = nullptr;
  if ((st = noalloc_scratch(g->device, &base))) return st;

  // ---- carve the scratch; refuse graphs whose workspace does not fit
  const size_t nw = (size_t)((g->V + 31) / 32 + 64);
  auto count_gt = [&](long long t) -> size_t {
    if (t < 1) return (size_t)g->V;
    int k = 0;
    while (k < 15 && (1ll << (k + 1)) <= t) ++k;
    return (size_t)g->cnt_deg_gt[k];
  };
  size_t cap[3];
  cap[0] = (size_t)g->V;
  cap[1] = std::min<size_t>((size_t)g->V, count_gt(o.small_max));
  cap[2] = std::min<size_t>((size_t)g->V, count_gt(o.medium_max));
  const size_t hcap = (size_t)g->cnt_deg_gt[4] + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align256(off + bytes);
    return at;
  };
  const size_t o_bits = take(nw * 4 * 5);
  const size_t o_ctl = take(sizeof(Ctl));
  const size_t o_rs = take(sizeof(ResumeState));
  const size_t o_ulist = take(nw * 32 * 4);
  const size_t o_hid = take(hcap * 4), o_heb = take(hcap * 4), o_hbg = take(hcap * 8);
  size_t o_q[2][3][3];
  for (int par = 0; par < 2; ++par)
    for (int b = 0; b < 3; ++b) {
      o_q[par][b][0] = take((cap[b] + 1) * 4);
      o_q[par][b][1] = take((cap[b] + 1) * 4);
      o_q[par][b][2] = take((cap[b] + 1) * 8);
    }
  const size_t o_forced = take(o.policy == XBFS_POLICY_FORCED ? (size_t)o.n_forced : 0);
  if (off > (size_t)XBFS_NOALLOC_SCRATCH_BYTES)
    return set_error(XBFS_ERR_UNSUPPORTED,
                     "graph needs %zu bytes of traversal scratch (V = %lld); the static scratch of "
                     "xbfs_bfs_noalloc holds %llu bytes (XBFS_NOALLOC_SCRATCH_BYTES): use xbfs_bfs",
                     off, (long long)g->V, (unsigned long long)XBFS_NOALLOC_SCRATCH_BYTES);

  // ---- kernel parameters: as setup_params, with the workspace in the scratch
  Params p;
  memset(&p, 0, sizeof(p));
  p.beg = g->beg.as<long long>();
  p.head = g->head.as<int4>();
  p.csr = g->csr.as<int>();
  p.V = g->V;
  p.E = g->E;
  p.levels = levels;
  p.parents = parents;
  uint32_t* bits = (uint32_t*)(base + o_bits);
  p.vis = bits;
  for (int i = 0; i < 4; ++i) p.fb[i] = bits + (size_t)(i + 1) * nw;
  for (int par = 0; par < 2; ++par)
    for (int b = 0; b < 3; ++b) {
      p.q[par][b].ids = (int*)(base + o_q[par][b][0]);
      p.q[par][b].eb = (unsigned*)(base + o_q[par][b][1]);
      p.q[par][b].bg = (long long*)(base + o_q[par][b][2]);
    }
  p.heavy.ids = (int*)(base + o_hid);
  p.heavy.eb = (unsigned*)(base + o_heb);
  p.heavy.bg = (long long*)(base + o_hbg);
  p.ulist = (int*)(base + o_ulist);
  p.ctl = (Ctl*)(base + o_ctl);
  p.hist = nullptr;
  p.hist_cap = 0;
  p.forced = (signed char*)(base + o_forced);
  p.n_forced = o.n_forced;
  p.nwords = (g->V + 31) / 32;
  p.n_ni = g->symmetric ? g->V - g->n_isolated : g->V;
  p.policy = o.policy;
  p.alpha = o.alpha;
  p.async_bu = o.async_bu ? 1 : 0;
  p.small_max = o.small_max;
  p.medium_max = o.medium_max;
  p.beamer_alpha = o.beamer_alpha > 0 ? o.beamer_alpha : 14.f;
  p.beamer_beta = o.beamer_beta > 0 ? o.beamer_beta : 24.f;
  p.timeout_ns = o.wait_timeout_us > 0 ? (unsigned long long)o.wait_timeout_us * 1000ull
                                        : 10ull * 1000 * 1000 * 1000;
  p.absent_block = o.test_absent_block;
  p.max_levels = g->V + 2;
  extern const float* mlp_device_weights(int device);
  p.mlp = mlp_device_weights(g->device);
  if (o.policy == XBFS_POLICY_MLP && !p.mlp) p.policy = XBFS_POLICY_HEURISTIC;
  p.allow_bu = g->symmetric ? 1 : 0;
  p.rs = (ResumeState*)(base + o_rs);
  p.bu_mode = o.bu_probe;
  p.stop_level = LLONG_MAX;
  p.resume = 0;
  const bool par_on = parents != nullptr;
  const bool mlp_on = p.policy == XBFS_POLICY_MLP;
  const void* kfn = par_on ? (const void*)k_bfs<true> : (const void*)k_bfs<false>;
  const size_t smem = mlp_on ? sizeof(Smem) : kSmemNoMlp;
  int grid = dev->grid[par_on ? 1 : 0][mlp_on ? 1 : 0];
  if (o.grid_dim > 0 && o.grid_dim < grid) grid = o.grid_dim;

  // ---- the launch sets up the traversal state itself (init_traversal);
  // the control block, which holds its grid barrier, is zeroed first
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;
  XBFS_CUDA_TRY(cudaMemsetAsync(p.ctl, 0, sizeof(Ctl), s));
  if (o.policy == XBFS_POLICY_FORCED)
    XBFS_CUDA_TRY(cudaMemcpyAsync((void*)p.forced, o.forced, (size_t)o.n_forced, cudaMemcpyHostToDevice, s));
  p.fresh = 1;
  p.src = src;
  p.iso = g->iso.as<uint32_t>();
  void* args[] = {&p};
  XBFS_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kBlock), args, smem, s));
  Ctl hctl;
  XBFS_CUDA_TRY(cudaMemcpyAsync(&hctl, p.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  XBFS_CUDA_TRY(cudaStreamSynchronize(s));
  if (hctl.bar.err != 0)
    return set_error((xbfs_status)hctl.bar.err, "traversal kernel reported %s", xbfs_strerror(hctl.bar.err));
  if (stats) {
    stats->struct_size = (int32_t)sizeof(xbfs_stats);
    stats->depth = hctl.depth;
    stats->reached = (int64_t)hctl.reached;
    stats->edges_mc = (int64_t)(hctl.msum / 2);
    stats->device_ms = 0.0;  // not timed: this path creates no CUDA events
    stats->kernel_ms = 0.0;
    stats->n_td_queue = hctl.strat_count[0];
    stats->n_td_scan = hctl.strat_count[1];
    stats->n_bu = hctl.strat_count[2];
    stats->n_async = (int32_t)hctl.n_async;
    stats->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  }
  return XBFS_OK;
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_bfs(xbfs_graph* gh, int32_t src, int32_t* levels, int32_t* parents, const xbfs_opts* opts,
                     xbfs_stats* stats) {
  return bfs_single((Graph*)gh, src, levels, parents, opts, stats);
}

xbfs_status xbfs_bfs_many(xbfs_graph* gh, const int32_t* srcs, int32_t n, int32_t* levels, const xbfs_opts* opts,
                          xbfs_stats* stats) {
  return bfs_many((Graph*)gh, srcs, n, levels, opts, stats);
}

xbfs_status xbfs_bfs_noalloc(xbfs_graph* gh, int32_t src, int32_t* levels, int32_t* parents,
                             const xbfs_opts* opts, xbfs_stats* stats) {
  return bfs_noalloc((Graph*)gh, src, levels, parents, opts, stats);
}

xbfs_status xbfs_level_costs(xbfs_graph* gh, int32_t src, int32_t follow, int32_t cap, float* costs,
                             xbfs_level_trace* trace, int32_t* n) {
  return level_costs((Graph*)gh, src, follow, cap, costs, trace, n);
}

xbfs_status xbfs_last_trace(xbfs_graph* gh, xbfs_level_trace* out, int32_t cap, int32_t* n) {
  Graph* g = (Graph*)gh;
  if (!g || !n) return set_error(XBFS_ERR_INVALID_ARG, "NULL argument");
  const int total = (int)g->ss.trace.size();
  *n = total;
  if (out && cap > 0) memcpy(out, g->ss.trace.data(), sizeof(xbfs_level_trace) * std::min(cap, total));
  return XBFS_OK;
}

}  // extern "C"
