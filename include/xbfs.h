/*
 * xbfs.h — C ABI of the B200-native XBFS library (libxbfs.so).
 *
 * The reference (hpda-lab/XBFS) exposes no library: its interface is the
 * `bfs` command line (bfs_gpu_update.cu:33-48), the CSR file pair read by
 * graph.hpp:4-104, and the internal call BFS_ControlFlow<int,long>(...)
 * (bfs_adaptiveFQ_wb_async.cuh:934-935) that main() makes after allocating
 * every device buffer itself (bfs_gpu_update.cu:175-251). Each entry point
 * below names the piece of that interface it replaces.
 *
 * Conventions
 *  - Every call returns an xbfs_status (0 = OK). The library never exits the
 *    process (the reference's H_ERR calls exit(1), bfs_single_scan.cuh:11-19).
 *    xbfs_last_error() gives a thread-local detail string for the last failure.
 *  - Level arrays are int32[V]: source -> 0, BFS depth for reached vertices,
 *    -1 for unreached (the reference's SA/status contract,
 *    bfs_gpu_update.cu:105-127, 213-218).
 *  - Output pointers may be host or device memory; the library detects which.
 *  - A graph handle owns its device copy of the CSR and the traversal scratch.
 *    One handle must not be used from two host threads at once.
 */
#ifndef XBFS_H_
#define XBFS_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t xbfs_status;
enum {
  XBFS_OK = 0,
  XBFS_ERR_INVALID_ARG = 1,
  XBFS_ERR_IO = 2,
  XBFS_ERR_FORMAT = 3,
  XBFS_ERR_CUDA = 4,
  XBFS_ERR_OOM = 5,
  XBFS_ERR_DEVICE_TIMEOUT = 6, /* a bounded device-side wait expired */
  XBFS_ERR_UNSUPPORTED = 7,
  XBFS_ERR_INTERNAL = 8,
  XBFS_ERR_NO_DEVICE = 9,
  XBFS_ERR_BUSY = 10,
  XBFS_ERR_LEVEL_OVERFLOW = 11 /* depth exceeded the packed level width */
};

/* Per-level strategies (the three classes the direction switch chooses among). */
enum {
  XBFS_TD_QUEUE = 0, /* top-down, binned frontier queue built during expansion
                        (replaces small/medium/large_SA_TD_update,
                        bfs_adaptiveFQ_wb_async.cuh:50-162, and the in-place
                        variants bfs_TD_scan_free.cuh:23-135) */
  XBFS_TD_SCAN = 1,  /* top-down, frontier found by a status sweep
                        (replaces atomic_FQ_Generator2 + *_SA_TD_update2,
                        bfs_single_scan.cuh:26-126) */
  XBFS_BU = 2        /* bottom-up over a ballot-scan queue of unvisited vertices
                        (replaces ballot_counting/FQ_gen/my_prefixsum/
                        thread_centric_BU_update, bfs_adaptiveFQ_wb_async.cuh:
                        189-284, 738-777, prefix_sum1.cuh:13-108) */
};

/* Direction/strategy policies. */
enum {
  XBFS_POLICY_HEURISTIC = 0, /* the reference's switch: ratio = m_f/E < alpha
                                -> top-down, TD_adaptive / hub_before /
                                hub_after pick the TD variant
                                (bfs_adaptiveFQ_wb_async.cuh:946-1078, 1114) */
  XBFS_POLICY_MLP = 1,       /* learned predictor (xbfs_mlp_set_weights) */
  XBFS_POLICY_FORCED = 2,    /* xbfs_opts.forced[level] (last entry repeats) */
  XBFS_POLICY_BEAMER = 3     /* classic alpha/beta direction optimisation */
};

typedef struct xbfs_opts {
  int32_t struct_size;  /* = sizeof(xbfs_opts); set by xbfs_opts_init */
  int32_t policy;       /* XBFS_POLICY_* */
  float alpha;          /* reference threshold, argv[8] (default 0.1) */
  int32_t block_dim;    /* reference BlockDim argv[4]; 0 = tuned default */
  int32_t grid_dim;     /* reference GridDim argv[5]; 0 = all resident CTAs */
  int32_t async_bu;     /* 1 = bottom-up may write level+2 (reference "async",
                           bfs_adaptiveFQ_wb_async.cuh:764-770); 0 = off */
  int32_t small_max;    /* degree bin edges: small <= small_max < medium <=  */
  int32_t medium_max;   /*   medium_max < large (reference: 32 / 256)        */
  const int8_t* forced; /* XBFS_POLICY_FORCED: host array of XBFS_TD_* / XBFS_BU */
  int32_t n_forced;
  int32_t trace;        /* 1 = record a per-level trace (xbfs_last_trace) */
  void* stream;         /* cudaStream_t to run on; NULL = the handle's stream */
  int32_t padding;      /* reference argv[11]; only 1 is meaningful (the
                           reference is wrong for padding > 1) */
  float beamer_alpha;   /* XBFS_POLICY_BEAMER: TD->BU when m_f > m_u/alpha (14) */
  float beamer_beta;    /*                     BU->TD when n_f < V/beta (24)   */
  int32_t bu_probe;     /* bottom-up probe shape: 0 = by density (default):
                           while unvisited vertices are at least V/4,
                           word-parallel over head records (6), else over a
                           compacted list of them, head record first and then
                           the CSR segment (4 after the first three
                           neighbours); 5 = word-parallel over CSR offsets,
                           each lane probing the first 2 neighbours of two
                           vertices at once, longer scans deferred to a
                           per-CTA queue; 6 = the same over the graph's head
                           records (first three neighbours and degree of each
                           vertex, 16 bytes, written at upload and after
                           xbfs_graph_sort_adjacency); over the list, CSR
                           offsets only: 1 = 2, 4, then 8 neighbours at a
                           time, streaming (L1 bypass); 2 = 4 at a time,
                           streaming; 3 = two vertices per lane; 4 = 2, 4,
                           then 8 at a time through L1. Other values:
                           XBFS_ERR_INVALID_ARG */
  int32_t wait_timeout_us; /* bound of every device-side wait of a traversal
                              (grid barriers); 0 = 10 s. On expiry the call
                              returns XBFS_ERR_DEVICE_TIMEOUT */
  int32_t test_absent_block; /* failure-detection test hook: k > 0 makes CTA
                                k-1 leave the traversal kernel before its first
                                grid barrier, so the others' bounded wait runs
                                out; 0 = off */
  int32_t reserved;
} xbfs_opts;

typedef struct xbfs_stats {
  int32_t struct_size;
  int32_t depth;      /* number of levels: max level + 1 */
  int64_t reached;    /* vertices with level >= 0 */
  int64_t edges_mc;   /* Graph500 m_c: (sum of degrees of reached vertices)/2 */
  double device_ms;   /* traversal time on the device (CUDA events) */
  double total_ms;    /* wall time of the whole call, copies included */
  int32_t n_td_queue; /* levels run with each strategy */
  int32_t n_td_scan;
  int32_t n_bu;
  int32_t n_async;    /* vertices given level+2 by bottom-up */
  double kernel_ms;   /* the persistent traversal launch alone (CUDA events) */
} xbfs_stats;

typedef struct xbfs_level_trace {
  int32_t level;
  int32_t strategy;
  int64_t n_f; /* frontier vertices at this level */
  int64_t m_f; /* frontier edges (sum of degrees) */
  int64_t n_u; /* unvisited non-isolated vertices */
  int64_t m_u; /* their edges */
  double us;   /* device time of this level (globaltimer) */
} xbfs_level_trace;

typedef struct xbfs_graph xbfs_graph;

const char* xbfs_strerror(xbfs_status st);
const char* xbfs_last_error(void);
int32_t xbfs_version(void);
xbfs_status xbfs_device_count(int32_t* n);
void xbfs_opts_init(xbfs_opts* o);

/* Load the reference's CSR pair: <beg> = raw little-endian int64[V+1],
 * <csr> = raw int32[beg[V]]; V = size(beg)/8 - 1. Replaces
 * graph<int,long,int,int,long,char>::graph (graph.hpp:4-104) — but validates
 * (monotone offsets, beg[0]=0, in-range neighbours, sizes agree) and returns
 * XBFS_ERR_FORMAT instead of asserting. */
xbfs_status xbfs_graph_load(const char* beg_path, const char* csr_path, int32_t device,
                            xbfs_graph** out);
/* Upload a host CSR (same layout). Replaces the cudaMalloc/cudaMemcpy of
 * beg_cu/csr_cu in main (bfs_gpu_update.cu:175-180). Every graph handle
 * (loaded, uploaded or generated) also keeps one 16-byte head record per
 * vertex on the device (its first three neighbours in CSR order and its
 * degree), which the traversal's bottom-up probes and bitmap sweeps read
 * instead of the CSR offsets and the segment's first sector: device memory
 * is 8(V+1) + 4E + 16V bytes plus the traversal workspace. */
xbfs_status xbfs_graph_upload(const int64_t* beg, const int32_t* csr, int64_t V, int64_t E,
                              int32_t device, xbfs_graph** out);
xbfs_status xbfs_graph_info(const xbfs_graph* g, int64_t* V, int64_t* E, int64_t* max_degree,
                            int64_t* n_isolated);
/* Copy the device CSR back to host buffers (beg: V+1, csr: E entries; csr
 * may be NULL to fetch the offsets only). */
xbfs_status xbfs_graph_download(const xbfs_graph* g, int64_t* beg, int32_t* csr);
/* Reorders the neighbours inside every vertex's CSR segment (the offsets and
 * the edge multiset stay the same). XBFS_ADJ_DEGREE_DESC puts high-degree
 * neighbours first, so bottom-up steps on power-law graphs find a frontier
 * parent in fewer probes; XBFS_ADJ_ID_ASC restores ascending ids. Levels
 * never depend on the order (parents may). No reference counterpart: the
 * reference traverses the file order. Needs about 20 bytes per edge of
 * temporary device memory; xbfs_graph_download returns the new order, and
 * the head records are rewritten to match it. */
enum { XBFS_ADJ_ID_ASC = 0, XBFS_ADJ_DEGREE_DESC = 1 };
xbfs_status xbfs_graph_sort_adjacency(xbfs_graph* g, int32_t order);
/* Write the handle's CSR in the reference's file format. */
xbfs_status xbfs_graph_save(const xbfs_graph* g, const char* beg_path, const char* csr_path);
void xbfs_graph_free(xbfs_graph* g);

/* Single-source BFS. Replaces BFS_ControlFlow<int,long>(...)
 * (bfs_adaptiveFQ_wb_async.cuh:934-1258) plus the status copy-back in main
 * (bfs_gpu_update.cu:255). levels: V entries (host or device). parents:
 * nullable, V entries; parents[src] = src, -1 when unreached. opts, stats:
 * nullable. The whole level loop runs on the device (one persistent
 * cooperative launch); no per-level host round trip. */
xbfs_status xbfs_bfs(xbfs_graph* g, int32_t src, int32_t* levels, int32_t* parents,
                     const xbfs_opts* opts, xbfs_stats* stats);

/* n single-source traversals in one call (row i of levels, n x V int32, host
 * or device, belongs to srcs[i]). Same kernel and results as n xbfs_bfs
 * calls, pipelined: traversal i runs while the level array of traversal i-1
 * is copied to host memory on a second stream. No reference counterpart
 * (the reference runs one source per process); stats are summed over the
 * traversals (depth = the largest), device_ms spans the whole pipeline. */
xbfs_status xbfs_bfs_many(xbfs_graph* g, const int32_t* srcs, int32_t n, int32_t* levels,
                          const xbfs_opts* opts, xbfs_stats* stats);

/* Allocation-free single-source BFS. No counterpart in the reference (its
 * main cudaMallocs the status arrays and queues itself); added for callers
 * that may not allocate device memory while they traverse: a process whose
 * HBM is pre-divided by its own pool or arena, or a latency-bound loop in
 * which cudaMalloc/cudaFree would stall the device. Same kernel, options and
 * results as xbfs_bfs, but the traversal workspace comes from one fixed
 * static device array of XBFS_NOALLOC_SCRATCH_BYTES per device, not from
 * cudaMalloc. Requirements and limits:
 *  - levels (and parents, if not NULL) must be device memory on g's device
 *    (XBFS_ERR_INVALID_ARG otherwise, host memory and other devices' memory
 *    included);
 *  - graphs whose workspace exceeds the array are refused with
 *    XBFS_ERR_UNSUPPORTED and a message giving the bytes needed (R-MAT with
 *    edge factor 16 fits up to about 2^20 vertices; xbfs_bfs has no limit);
 *  - every call resolves the array's address in the current context
 *    (cudaGetSymbolAddress; the first one also makes the runtime load the
 *    module holding the array); the first call on a device also sets the
 *    kernel's launch attributes: make that first call before any stream
 *    capture begins;
 *  - wait_timeout_us and test_absent_block bound and test the device-side
 *    waits exactly as in xbfs_bfs;
 *  - nothing in the array has to start at zero: each call clears the
 *    visited/frontier bitmaps and the control block it reads first;
 *  - calls on the same device share the one array: calls that overlap in time
 *    (other threads, other streams) race and corrupt each other's traversal.
 *    Serialise them;
 *  - the call waits for its stream to read back the status; opts->trace is
 *    refused and stats->device_ms / kernel_ms are 0 (no events are created). */
#define XBFS_NOALLOC_SCRATCH_BYTES (64ull << 20)
xbfs_status xbfs_bfs_noalloc(xbfs_graph* g, int32_t src, int32_t* levels, int32_t* parents,
                             const xbfs_opts* opts, xbfs_stats* stats);

/* Batched multi-source BFS: n sources, levels = n x V int32 (source-major,
 * host or device). Sources are traversed 64 per uint64 word, up to 8 words
 * (512 sources) per pass. No counterpart in the reference (one source per
 * process). opts.policy FORCED with forced[0] = XBFS_TD_QUEUE / XBFS_BU pins
 * the direction; otherwise opts.alpha (default 2 when <= 0.5) sets the
 * top-down/bottom-up switch on frontier vs unfinished edges. */
xbfs_status xbfs_bfs_batch(xbfs_graph* g, const int32_t* srcs, int32_t n, int32_t* levels,
                           const xbfs_opts* opts, xbfs_stats* stats);
/* Same with an explicit number of uint64 words per vertex (1, 2, 4 or 8). */
xbfs_status xbfs_bfs_batch_w(xbfs_graph* g, const int32_t* srcs, int32_t n, int32_t* levels,
                             const xbfs_opts* opts, xbfs_stats* stats, int32_t words_per_vertex);

/* Multi-graph traversal: many graphs (symmetric CSRs on one device) packed
 * into one arena, one source each, traversed by one persistent launch that is
 * captured into a CUDA graph and replayed. No counterpart in the reference.
 * Levels are concatenated: graph i's array starts at level_offsets[i]
 * (xbfs_multi_info). */
typedef struct xbfs_multi xbfs_multi;
xbfs_status xbfs_multi_create(xbfs_graph* const* graphs, int32_t n, int32_t device, xbfs_multi** out);
xbfs_status xbfs_multi_info(const xbfs_multi* m, int64_t* total_V, int64_t* total_E, int64_t* level_offsets);
xbfs_status xbfs_multi_bfs(xbfs_multi* m, const int32_t* srcs, int32_t* levels, const xbfs_opts* opts,
                           xbfs_stats* stats);
/* Autotuner: times every candidate (threads per CTA 256/512/1024, thread/warp
 * degree threshold, direction threshold) on these sources and keeps the
 * fastest for later xbfs_multi_bfs calls. */
xbfs_status xbfs_multi_tune(xbfs_multi* m, const int32_t* srcs, int32_t reps, int32_t* block,
                            int32_t* thread_max, float* alpha, float* best_ms);
xbfs_status xbfs_multi_set_config(xbfs_multi* m, int32_t block, int32_t thread_max, float alpha);
void xbfs_multi_free(xbfs_multi* m);

/* Serving loop (no reference counterpart): BFS requests over device-resident
 * graphs, continuously batched 64 per graph into uint64 bit slots; a request
 * joins a running batch at any level step, is admitted when a slot is free
 * and its int32[V] output fits the HBM budget (hbm_budget_bytes <= 0: free
 * memory minus 2 GiB), and leaves when its traversal is complete. */
typedef struct xbfs_server xbfs_server;
xbfs_status xbfs_serve_create(xbfs_graph* const* graphs, int32_t n, int32_t device, int64_t hbm_budget_bytes,
                              xbfs_server** out);
/* Replays a request trace in real time (request i targets graph[i] from
 * src[i] and arrives arrival_us[i] after the start). Returns per request the
 * admission and completion times (us since start) and its Graph500 edge
 * count. keep_outputs = 0: level arrays are freed as requests finish;
 * 1: levels[i] receives a device pointer to request i's level array (free
 * with xbfs_serve_release; kept arrays count against the HBM budget, and a
 * request they block is an XBFS_ERR_OOM); 2: levels[i] is the caller's host
 * array of V int32 that receives the levels when request i finishes (its
 * device array is freed at once). */
xbfs_status xbfs_serve_run(xbfs_server* s, int32_t n, const int32_t* graph, const int32_t* src,
                           const double* arrival_us, int32_t keep_outputs, double* admit_us, double* finish_us,
                           int64_t* edges_mc, int32_t** levels, double* wall_us);
/* Online mode: the same engine in the server's own host thread, fed as
 * requests arrive. xbfs_serve_start starts it (the server must not be in a
 * xbfs_serve_run call; a running server refuses xbfs_serve_run with
 * XBFS_ERR_BUSY). xbfs_serve_submit queues one request and returns at once
 * with its ticket; it is admitted when a slot of its graph and room in the
 * HBM budget are free, joins the running batch at its next level step, and
 * leaves when complete. output: 0 = only the edge count and times are kept;
 * 1 = the level array stays on the device (xbfs_serve_poll returns it; free
 * with xbfs_serve_release); 2 = it is copied into levels_host (V int32,
 * page-locked memory lets the copy overlap) before the request counts as
 * done. Kept device arrays count against the budget: requests they block
 * wait for a release. Any host thread may submit and poll. */
typedef struct xbfs_serve_result {
  int32_t struct_size;
  int32_t state;       /* 0 waiting, 1 running (or copying out), 2 done, 3 dropped at stop */
  double submit_us;    /* times since xbfs_serve_start */
  double admit_us;     /* -1 until admitted */
  double finish_us;    /* -1 until done */
  int64_t edges_mc;    /* Graph500 m_c of the traversal (when done) */
  int32_t* levels_dev; /* output 1: the device level array (when done) */
} xbfs_serve_result;
xbfs_status xbfs_serve_start(xbfs_server* s);
xbfs_status xbfs_serve_submit(xbfs_server* s, int32_t graph, int32_t src, int32_t output, int32_t* levels_host,
                              int64_t* ticket);
/* State of a request. wait_us: 0 = look only, > 0 = wait up to that long,
 * < 0 = wait until done. Returns XBFS_OK when done (result filled),
 * XBFS_ERR_BUSY while waiting or running, or the engine's error. */
xbfs_status xbfs_serve_poll(xbfs_server* s, int64_t ticket, int64_t wait_us, xbfs_serve_result* out);
/* Lets every submitted request complete, then stops the thread. Requests
 * that only kept device arrays block at that point are dropped (state 3). */
xbfs_status xbfs_serve_stop(xbfs_server* s);
xbfs_status xbfs_serve_release(xbfs_server* s, int32_t* levels_dev, int64_t V);
/* Copies a kept level array (V entries) to host memory, then releases it. */
xbfs_status xbfs_serve_fetch(xbfs_server* s, int32_t* levels_dev, int64_t V, int32_t* host_out);
void xbfs_serve_free(xbfs_server* s);

/* 1D-partitioned single-source BFS, the per-rank device steps (no reference
 * counterpart: the reference runs one source on one GPU, cudaSetDevice at
 * bfs_gpu_update.cu:138). Rank r owns the vertices [lo, hi) (lo a multiple
 * of 32) and the CSR rows of those vertices (beg: hi - lo + 1 offsets into
 * csr, which holds global neighbour ids). The host driver
 * (xbfs_b200/partition.py) runs the level loop across ranks: a top-down
 * level is xbfs_part_td_expand into a V-byte candidate array, a MAX
 * all-reduce of that array, xbfs_part_claim; a bottom-up level (symmetric
 * graphs) is xbfs_part_frontier_bits into this rank's words of a V-bit
 * bitmap, an all-gather of the bitmap, xbfs_part_bottom_up. Candidate and
 * bitmap buffers are device memory owned by the caller. Each call returns
 * when its kernels have completed. */
typedef struct xbfs_part xbfs_part;
xbfs_status xbfs_part_create(const int64_t* beg, const int32_t* csr, int64_t V, int64_t lo, int64_t hi,
                             int32_t symmetric, int32_t device, xbfs_part** out);
void xbfs_part_free(xbfs_part* p);
/* Levels -1, the source (if owned) level 0 and the only frontier vertex. */
xbfs_status xbfs_part_reset(xbfs_part* p, int32_t src);
/* out[4] = owned n_f, m_f (frontier vertices, their edges) and n_u, m_u
 * (unvisited vertices with edges, their edges). */
xbfs_status xbfs_part_stats(xbfs_part* p, int64_t* out);
xbfs_status xbfs_part_td_expand(xbfs_part* p, uint8_t* cand);
/* cand: after the all-reduce; cleared (all V bytes) on return. */
xbfs_status xbfs_part_claim(xbfs_part* p, uint8_t* cand, int32_t next_level);
/* slice: this rank's words of the global bitmap (nwords_slice >= ceil((hi-lo)/32)). */
xbfs_status xbfs_part_frontier_bits(xbfs_part* p, uint32_t* slice, int64_t nwords_slice);
/* fbits: the whole V-bit frontier bitmap after the all-gather. */
xbfs_status xbfs_part_bottom_up(xbfs_part* p, const uint32_t* fbits, int32_t next_level);
/* Levels of the owned vertices (hi - lo int32, host or device memory). */
xbfs_status xbfs_part_levels(xbfs_part* p, int32_t* out);

/* Per-level trace of the last xbfs_bfs call made with opts.trace = 1
 * (replaces the reference's tag[]/ratio[]/iter[] arrays, written to
 * Hybrid_iteration.csv at bfs_gpu_update.cu:270-272). */
xbfs_status xbfs_last_trace(xbfs_graph* g, xbfs_level_trace* out, int32_t cap, int32_t* n);

/* Learned direction/strategy switch (no reference counterpart; the
 * reference's fixed heuristic stays the fallback).
 * xbfs_level_costs: for every level of a traversal from src, snapshot the
 * state, run the level once with each strategy (XBFS_TD_QUEUE, XBFS_TD_SCAN,
 * XBFS_BU), then, from the state each one leaves, the next level once with
 * each strategy (a strategy also decides whether the next frontier is a
 * queue or a bitmap), and record the level's device time plus the cheapest
 * next level's in costs[level*3 + strategy] (us);
 * continue along the cheapest (follow = 0) or the heuristic's choice
 * (follow = 1). trace[level] gets the level's statistics and the strategy
 * taken. *n = number of levels. Levels never depend on the strategies. */
xbfs_status xbfs_level_costs(xbfs_graph* g, int32_t src, int32_t follow, int32_t cap, float* costs,
                             xbfs_level_trace* trace, int32_t* n);
/* MLP 8 -> 32 -> 32 -> 3 (ReLU, softmax), packed as [feature mean 8][feature
 * std 8][W1 32x8][b1 32][W2 32x32][b2 32][W3 3x32][b3 3] = 1,459 floats of
 * which 1,443 are trained. */
int32_t xbfs_mlp_num_params(void);
/* Install weights for XBFS_POLICY_MLP on a device (n = 0 or NULL removes). */
xbfs_status xbfs_mlp_set_weights(int32_t device, const float* packed, int32_t n);
/* Forward pass on the device: logits (n x 3) of features (n x 8). */
xbfs_status xbfs_mlp_logits(int32_t device, const float* packed, const float* feats, int32_t n, float* logits);
/* Mean softmax cross-entropy loss and its gradient (1,443 floats, trainable
 * part only) over n labelled samples, computed by the device kernels. */
xbfs_status xbfs_mlp_grad(int32_t device, const float* packed, const float* feats, const int32_t* labels,
                          int32_t n, float* grad, float* loss);
/* Full-batch SGD with momentum on the device; weights updated in place. */
xbfs_status xbfs_mlp_train(int32_t device, float* packed, const float* feats, const int32_t* labels, int32_t n,
                           int32_t epochs, float lr, float momentum, float* losses);

/* Synthetic inputs (no reference counterpart: the reference reads datasets
 * converted by CSRGenerator/tuple_text_to_bin.cpp). All generators are
 * deterministic functions of their arguments; the host and device builds
 * produce identical CSRs. Graphs are symmetric, self-loop free, deduplicated,
 * adjacency sorted ascending. */
xbfs_status xbfs_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, double a, double b,
                          double c, int32_t device, xbfs_graph** out);
xbfs_status xbfs_gen_grid(int32_t width, int32_t height, int32_t device, xbfs_graph** out);
xbfs_status xbfs_gen_er(int64_t n, double mean_degree, uint64_t seed, int32_t device,
                        xbfs_graph** out);
/* Host-only generation (no GPU needed): returns malloc'd arrays that the
 * caller releases with xbfs_free_host. */
xbfs_status xbfs_gen_rmat_host(int32_t scale, int32_t edge_factor, uint64_t seed, double a,
                               double b, double c, int64_t** beg, int32_t** csr, int64_t* V,
                               int64_t* E);
xbfs_status xbfs_gen_grid_host(int32_t width, int32_t height, int64_t** beg, int32_t** csr,
                               int64_t* V, int64_t* E);
xbfs_status xbfs_gen_er_host(int64_t n, double mean_degree, uint64_t seed, int64_t** beg,
                             int32_t** csr, int64_t* V, int64_t* E);
void xbfs_free_host(void* p);
/* Edge-list text (one "u v" pair per line, '#'/'%' comments, skip_lines
 * header lines) -> <out_prefix>_beg_pos.bin + <out_prefix>_csr.bin (int32
 * neighbours). Replaces CSRGenerator/tuple_text_to_bin.cpp (:59-426), which
 * writes int64 neighbours its own reader cannot load. reverse = 1 adds every
 * tuple's reversed edge; dedupe / drop_self_loops as named; write_weights
 * adds <out_prefix>_weight.bin (int32, 1..63, seeded), which the BFS ignores. */
xbfs_status xbfs_convert_edge_list(const char* text_path, int32_t reverse, int32_t skip_lines, int32_t dedupe,
                                   int32_t drop_self_loops, int32_t write_weights, const char* out_prefix,
                                   int64_t* V, int64_t* E);
/* Deterministic source sampling: k sources uniform over vertices with
 * degree > 0 (host CSR offsets). */
xbfs_status xbfs_pick_sources(const int64_t* beg, int64_t V, int32_t k, uint64_t seed,
                              int32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* XBFS_H_ */
