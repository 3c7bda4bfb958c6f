/*
 * oracle.c — CPU restatement of the reference's BFS, used ONLY as test
 * infrastructure: by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline / reference legs. The product (libxbfs.so) never links or
 * calls this code.
 *
 * Parity pins: the restatement is checked against (a) golden level arrays
 * produced by the reference's own GPU code (BFS_ControlFlow, compiled from
 * the reference sources by oracle/Makefile into oracle/_ref/ and run on a
 * B200; fixtures in tests/golden/ with the generating script beside them),
 * and (b) networkx on tiny graphs. The reference ships no fixtures of its own.
 *
 * Functions
 *  oracle_bfs_sweep  - the reference's serial CPU BFS, bfs_gpu_update.cu:105-127:
 *                      level-synchronous sweep over all vertices, status -1 for
 *                      unreached; optionally parallel over vertices (OpenMP).
 *  oracle_bfs_queue  - serial FIFO BFS (ground truth at every scale).
 *  oracle_bfs_do     - OpenMP direction-optimising BFS (top-down / bottom-up,
 *                      Beamer alpha/beta), a multi-core CPU baseline.
 *  oracle_check_tree - parent-tree check: parent[src] = src, every reached v
 *                      has level[parent[v]] = level[v] - 1 and the edge
 *                      (parent[v], v) exists; unreached v has parent -1.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Serial FIFO BFS. Returns the number of levels (max level + 1). */
int32_t oracle_bfs_queue(const int64_t* beg, const int32_t* csr, int64_t V, int32_t src, int32_t* levels) {
  for (int64_t i = 0; i < V; ++i) levels[i] = -1;
  if (src < 0 || src >= V) return 0;
  int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  if (!q) return -1;
  int64_t head = 0, tail = 0;
  q[tail++] = src;
  levels[src] = 0;
  int32_t depth = 1;
  while (head < tail) {
    const int32_t u = q[head++];
    const int32_t lu = levels[u];
    for (int64_t e = beg[u]; e < beg[u + 1]; ++e) {
      const int32_t v = csr[e];
      if (levels[v] < 0) {
        levels[v] = lu + 1;
        if (lu + 2 > depth) depth = lu + 2;
        q[tail++] = v;
      }
    }
  }
  free(q);
  return depth;
}

/* The reference's sweep BFS (bfs_gpu_update.cu:105-127): for k = 0, 1, ...
 * every vertex with status k marks its unreached neighbours k+1; stop after
 * a sweep that marked nothing. Returns the number of sweeps (the reference's
 * k, = depth + 1 for a non-empty graph). With nthreads > 1 the sweep over
 * vertices runs in parallel; concurrent writes store the same value k+1 and
 * use relaxed atomics, so the result is identical to the serial sweep. */
int32_t oracle_bfs_sweep(const int64_t* beg, const int32_t* csr, int64_t V, int32_t src, int32_t* status,
                         int32_t nthreads) {
  for (int64_t i = 0; i < V; ++i) status[i] = -1;
  status[src] = 0;
  int32_t k = 0;
  int done = 0;
  if (nthreads < 1) nthreads = 1;
  for (k = 0; !done; ++k) {
    int isdone = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4096) reduction(&& : isdone)
    for (int64_t i = 0; i < V; ++i) {
      if (__atomic_load_n(&status[i], __ATOMIC_RELAXED) == k) {
        for (int64_t j = beg[i]; j < beg[i + 1]; ++j) {
          const int32_t v = csr[j];
          if (__atomic_load_n(&status[v], __ATOMIC_RELAXED) == -1) {
            isdone = 0;
            __atomic_store_n(&status[v], k + 1, __ATOMIC_RELAXED);
          }
        }
      }
    }
    done = isdone;
  }
  return k;
}

/* OpenMP direction-optimising BFS (top-down with CAS claims into per-thread
 * queues; bottom-up over unvisited vertices with early exit). Returns depth. */
int32_t oracle_bfs_do(const int64_t* beg, const int32_t* csr, int64_t V, int32_t src, int32_t* levels,
                      int32_t nthreads, double alpha, double beta) {
  if (nthreads < 1) nthreads = omp_get_max_threads();
  for (int64_t i = 0; i < V; ++i) levels[i] = -1;
  int32_t* front = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  int32_t* next = (int32_t*)malloc(sizeof(int32_t) * (size_t)V);
  if (!front || !next) {
    free(front);
    free(next);
    return -1;
  }
  int64_t nf = 1, m_u = beg[V];
  front[0] = src;
  levels[src] = 0;
  m_u -= beg[src + 1] - beg[src];
  int32_t L = 0;
  int bottom_up = 0;
  while (nf > 0) {
    int64_t m_f = 0;
    if (!bottom_up) {
#pragma omp parallel for num_threads(nthreads) reduction(+ : m_f)
      for (int64_t i = 0; i < nf; ++i) m_f += beg[front[i] + 1] - beg[front[i]];
      if ((double)m_f > (double)m_u / alpha) bottom_up = 1;
    } else if ((double)nf < (double)V / beta) {
      bottom_up = 0;
    }
    int64_t nn = 0;
    int64_t m_new = 0;
    if (!bottom_up) {
#pragma omp parallel num_threads(nthreads) reduction(+ : m_new)
      {
        int32_t buf[256];
        int nb = 0;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < nf; ++i) {
          const int32_t u = front[i];
          for (int64_t e = beg[u]; e < beg[u + 1]; ++e) {
            const int32_t v = csr[e];
            int32_t expect = -1;
            if (__atomic_load_n(&levels[v], __ATOMIC_RELAXED) == -1 &&
                __atomic_compare_exchange_n(&levels[v], &expect, L + 1, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
              m_new += beg[v + 1] - beg[v];
              buf[nb++] = v;
              if (nb == 256) {
                int64_t at = __atomic_fetch_add(&nn, 256, __ATOMIC_RELAXED);
                memcpy(next + at, buf, sizeof(buf));
                nb = 0;
              }
            }
          }
        }
        if (nb) {
          int64_t at = __atomic_fetch_add(&nn, nb, __ATOMIC_RELAXED);
          memcpy(next + at, buf, sizeof(int32_t) * (size_t)nb);
        }
      }
    } else {
#pragma omp parallel num_threads(nthreads) reduction(+ : m_new)
      {
        int32_t buf[256];
        int nb = 0;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t v = 0; v < V; ++v) {
          if (levels[v] != -1) continue;
          for (int64_t e = beg[v]; e < beg[v + 1]; ++e) {
            if (__atomic_load_n(&levels[csr[e]], __ATOMIC_RELAXED) == L) {
              __atomic_store_n(&levels[v], L + 1, __ATOMIC_RELAXED);
              m_new += beg[v + 1] - beg[v];
              buf[nb++] = (int32_t)v;
              if (nb == 256) {
                int64_t at = __atomic_fetch_add(&nn, 256, __ATOMIC_RELAXED);
                memcpy(next + at, buf, sizeof(buf));
                nb = 0;
              }
              break;
            }
          }
        }
        if (nb) {
          int64_t at = __atomic_fetch_add(&nn, nb, __ATOMIC_RELAXED);
          memcpy(next + at, buf, sizeof(int32_t) * (size_t)nb);
        }
      }
    }
    m_u -= m_new;
    int32_t* t = front;
    front = next;
    next = t;
    nf = nn;
    ++L;
  }
  free(front);
  free(next);
  return L;
}

static int has_edge(const int64_t* beg, const int32_t* csr, int32_t u, int32_t v) {
  /* adjacency may be unsorted in user graphs: linear scan */
  for (int64_t e = beg[u]; e < beg[u + 1]; ++e)
    if (csr[e] == v) return 1;
  return 0;
}

/* Returns 0 when the parent array is a valid BFS tree for the level array,
 * else 1 + the first offending vertex. */
int64_t oracle_check_tree(const int64_t* beg, const int32_t* csr, int64_t V, int32_t src, const int32_t* levels,
                          const int32_t* parents) {
  int64_t first = INT64_MAX;
  if (parents[src] != src || levels[src] != 0) return 1 + src;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < V; ++v) {
    if (v == src) continue;
    int ok;
    if (levels[v] < 0) {
      ok = parents[v] == -1;
    } else {
      const int32_t p = parents[v];
      ok = p >= 0 && p < V && levels[p] == levels[v] - 1 && has_edge(beg, csr, p, (int32_t)v);
    }
    if (!ok) {
      int64_t cur = __atomic_load_n(&first, __ATOMIC_RELAXED);
      while (v < cur && !__atomic_compare_exchange_n(&first, &cur, v, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      }
    }
  }
  return first == INT64_MAX ? 0 : first + 1;
}

/* Graph500 m_c: half the sum of degrees of reached vertices. */
int64_t oracle_edges_mc(const int64_t* beg, int64_t V, const int32_t* levels) {
  int64_t s = 0;
#pragma omp parallel for reduction(+ : s)
  for (int64_t v = 0; v < V; ++v)
    if (levels[v] >= 0) s += beg[v + 1] - beg[v];
  return s / 2;
}
