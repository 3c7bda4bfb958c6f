/*
 * gen.c — input preparation for the oracle side, TEST INFRASTRUCTURE ONLY
 * (bench.py's reference and cpu_baseline legs, tests/). It lets the
 * reference arm build its graph and pick its sources without loading the
 * product library (libxbfs.so), and gives the tests a second, independent
 * build of the seeded inputs to compare the library's generators against.
 *
 * The graphs are the ones the library's generators define (the same seeded
 * counter-based hash per tuple, so the two builds agree bit for bit; a CPU
 * test checks this):
 *  - R-MAT (Graph500 Kronecker, probabilities a, b, c, d = 1-a-b-c): tuple k
 *    of ef * 2^scale draws, for each of the `scale` bit levels, one 64-bit
 *    hash; its low half picks the row bit (1 when >= (a+b) * 2^32), its high
 *    half the column bit (threshold a/(a+b) for row bit 0, c/(c+d) for row
 *    bit 1); both endpoints then pass a seeded bijection of [0, 2^scale)
 *    (three rounds of multiply-add by an odd constant and xorshift), the
 *    Graph500 label scramble. The hash is the splitmix64 finalizer.
 *  - 2D grid W x H, vertex r*W + c, 4-neighbourhood, neighbours ascending.
 *  - Every tuple (u, v), u != v, gives edges u->v and v->u; duplicates and
 *    self-loops are dropped; each adjacency list is sorted ascending.
 *
 * The construction here is a different one from the library's (which sorts
 * 64-bit (u, v) keys): degrees are counted, tuples are scattered into
 * per-vertex buckets, and each bucket is sorted and deduplicated on its own
 * (OpenMP over vertices).
 *
 *  oracle_gen_rmat / oracle_gen_grid return malloc'd arrays that the caller
 *  frees with oracle_free; oracle_pick_sources draws k distinct sources
 *  uniformly over vertices with degree > 0 (seeded hash, rejection).
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t ogen_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

typedef struct {
  int scale;
  uint64_t base, t_ab, t_a, t_c;
  uint64_t pm[3], pa[3];
} ogen_rmat;

static uint64_t ogen_threshold(double p) {
  if (p <= 0) return 0;
  if (p >= 1) return 1ull << 32;
  return (uint64_t)(p * 4294967296.0);
}

static void ogen_rmat_init(ogen_rmat* P, int scale, uint64_t seed, double a, double b, double c) {
  const double d = 1.0 - a - b - c;
  P->scale = scale;
  P->base = ogen_mix64(seed ^ 0x5851F42D4C957F2Dull);
  P->t_ab = ogen_threshold(a + b);
  P->t_a = ogen_threshold((a + b) > 0 ? a / (a + b) : 1.0);
  P->t_c = ogen_threshold((c + d) > 0 ? c / (c + d) : 1.0);
  for (int r = 0; r < 3; ++r) {
    P->pm[r] = ogen_mix64(seed + 0x1000 + (uint64_t)r) | 1ull;
    P->pa[r] = ogen_mix64(seed + 0x2000 + (uint64_t)r);
  }
}

static inline uint64_t ogen_scramble(uint64_t x, const ogen_rmat* P) {
  const uint64_t mask = (1ull << P->scale) - 1;
  const int sh = (P->scale + 1) / 2;
  for (int r = 0; r < 3; ++r) {
    x = (x * P->pm[r] + P->pa[r]) & mask;
    x ^= x >> sh;
  }
  return x & mask;
}

static inline void ogen_rmat_tuple(uint64_t k, const ogen_rmat* P, uint32_t* pu, uint32_t* pv) {
  const uint64_t h = ogen_mix64(P->base + k);
  uint64_t u = 0, v = 0;
  for (int i = 0; i < P->scale; ++i) {
    const uint64_t r = ogen_mix64(h ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1)));
    const uint64_t row = ((r & 0xffffffffull) >= P->t_ab) ? 1 : 0;
    const uint64_t col = ((r >> 32) >= (row ? P->t_c : P->t_a)) ? 1 : 0;
    u |= row << i;
    v |= col << i;
  }
  *pu = (uint32_t)ogen_scramble(u, P);
  *pv = (uint32_t)ogen_scramble(v, P);
}

static int ogen_cmp_i32(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static void ogen_sort_i32(int32_t* a, int64_t n) {
  if (n < 2) return;
  if (n <= 32) {  // insertion sort for the many short lists
    for (int64_t i = 1; i < n; ++i) {
      const int32_t x = a[i];
      int64_t j = i - 1;
      while (j >= 0 && a[j] > x) {
        a[j + 1] = a[j];
        --j;
      }
      a[j + 1] = x;
    }
    return;
  }
  qsort(a, (size_t)n, sizeof(int32_t), ogen_cmp_i32);
}

void oracle_free(void* p) { free(p); }

/* Returns 0 on success, -1 on bad arguments, -2 when out of memory. */
int32_t oracle_gen_rmat(int32_t scale, int32_t ef, uint64_t seed, double a, double b, double c,
                        int64_t** pbeg, int32_t** pcsr, int64_t* pV, int64_t* pE) {
  if (scale < 1 || scale > 30 || ef < 1 || !pbeg || !pcsr || !pV || !pE) return -1;
  ogen_rmat P;
  ogen_rmat_init(&P, scale, seed, a, b, c);
  const int64_t V = (int64_t)1 << scale;
  const int64_t nt = (int64_t)ef << scale;
  int64_t* cnt = (int64_t*)calloc((size_t)V + 1, sizeof(int64_t));
  if (!cnt) return -2;
  /* pass 1: degrees before deduplication */
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nt; ++k) {
    uint32_t u, v;
    ogen_rmat_tuple((uint64_t)k, &P, &u, &v);
    if (u == v) continue;
#pragma omp atomic
    cnt[u + 1] += 1;
#pragma omp atomic
    cnt[v + 1] += 1;
  }
  for (int64_t i = 0; i < V; ++i) cnt[i + 1] += cnt[i];
  const int64_t total = cnt[V];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)V);
  if (!adj || !pos) {
    free(cnt);
    free(adj);
    free(pos);
    return -2;
  }
  memcpy(pos, cnt, sizeof(int64_t) * (size_t)V);
  /* pass 2: the same tuples again, scattered into per-vertex buckets */
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nt; ++k) {
    uint32_t u, v;
    ogen_rmat_tuple((uint64_t)k, &P, &u, &v);
    if (u == v) continue;
    int64_t iu, iv;
#pragma omp atomic capture
    iu = pos[u]++;
#pragma omp atomic capture
    iv = pos[v]++;
    adj[iu] = (int32_t)v;
    adj[iv] = (int32_t)u;
  }
  free(pos);
  /* sort and deduplicate every bucket in place; cnt[] keeps the bucket starts */
  int64_t* deg = (int64_t*)malloc(sizeof(int64_t) * (size_t)V);
  if (!deg) {
    free(cnt);
    free(adj);
    return -2;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t x = 0; x < V; ++x) {
    int32_t* s = adj + cnt[x];
    const int64_t n = cnt[x + 1] - cnt[x];
    ogen_sort_i32(s, n);
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i)
      if (m == 0 || s[i] != s[m - 1]) s[m++] = s[i];
    deg[x] = m;
  }
  int64_t* beg = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V + 1));
  if (!beg) {
    free(cnt);
    free(adj);
    free(deg);
    return -2;
  }
  beg[0] = 0;
  for (int64_t x = 0; x < V; ++x) beg[x + 1] = beg[x] + deg[x];
  const int64_t E = beg[V];
  int32_t* csr = (int32_t*)malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
  if (!csr) {
    free(cnt);
    free(adj);
    free(deg);
    free(beg);
    return -2;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t x = 0; x < V; ++x) memcpy(csr + beg[x], adj + cnt[x], sizeof(int32_t) * (size_t)deg[x]);
  free(cnt);
  free(adj);
  free(deg);
  *pbeg = beg;
  *pcsr = csr;
  *pV = V;
  *pE = E;
  return 0;
}

int32_t oracle_gen_grid(int32_t W, int32_t H, int64_t** pbeg, int32_t** pcsr, int64_t* pV, int64_t* pE) {
  if (W < 1 || H < 1 || !pbeg || !pcsr || !pV || !pE) return -1;
  const int64_t V = (int64_t)W * H;
  const int64_t E = 2 * (int64_t)(W - 1) * H + 2 * (int64_t)W * (H - 1);
  int64_t* beg = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V + 1));
  int32_t* csr = (int32_t*)malloc(sizeof(int32_t) * (size_t)(E > 0 ? E : 1));
  if (!beg || !csr) {
    free(beg);
    free(csr);
    return -2;
  }
  /* degrees first (2..4 by position), then neighbours in ascending id order:
   * up (r-1), left (c-1), right (c+1), down (r+1) */
  beg[0] = 0;
  for (int64_t x = 0; x < V; ++x) {
    const int64_t r = x / W, c = x % W;
    beg[x + 1] = beg[x] + (r > 0) + (c > 0) + (c + 1 < W) + (r + 1 < H);
  }
#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < V; ++x) {
    const int64_t r = x / W, c = x % W;
    int64_t e = beg[x];
    if (r > 0) csr[e++] = (int32_t)(x - W);
    if (c > 0) csr[e++] = (int32_t)(x - 1);
    if (c + 1 < W) csr[e++] = (int32_t)(x + 1);
    if (r + 1 < H) csr[e++] = (int32_t)(x + W);
  }
  *pbeg = beg;
  *pcsr = csr;
  *pV = V;
  *pE = E;
  return 0;
}

/* k sources uniform over vertices with degree > 0, distinct when k does not
 * exceed their number. Returns 0, or -1 when the graph has no edges. */
int32_t oracle_pick_sources(const int64_t* beg, int64_t V, int32_t k, uint64_t seed, int32_t* out) {
  if (!beg || !out || V < 1 || k < 0) return -1;
  int64_t nonisolated = 0;
  for (int64_t v = 0; v < V; ++v) nonisolated += (beg[v + 1] > beg[v]);
  if (nonisolated == 0) return k > 0 ? -1 : 0;
  const int distinct = k <= nonisolated;
  const uint64_t base = ogen_mix64(seed ^ 0x3C6EF372FE94F82Bull);
  uint64_t ctr = 0;
  int32_t n = 0;
  while (n < k) {
    const uint64_t h = ogen_mix64(base + ctr++);
    const int64_t v = (int64_t)((h >> 11) % (uint64_t)V);
    if (beg[v + 1] == beg[v]) continue;
    int dup = 0;
    if (distinct)
      for (int32_t i = 0; i < n && !dup; ++i) dup = out[i] == (int32_t)v;
    if (dup) continue;
    out[n++] = (int32_t)v;
  }
  return 0;
}

static int ogen_cmp_u64(const void* a, const void* b) {
  const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return (x > y) - (x < y);
}

/* Reorders each vertex's neighbours by descending neighbour degree, ties by
 * ascending id (the order the library's xbfs_graph_sort_adjacency gives an
 * id-sorted CSR). In place; returns 0, or -2 when out of memory. */
int32_t oracle_sort_adjacency_degree(const int64_t* beg, int32_t* csr, int64_t V) {
  int64_t maxd = 0;
  for (int64_t v = 0; v < V; ++v) maxd = beg[v + 1] - beg[v] > maxd ? beg[v + 1] - beg[v] : maxd;
  int failed = 0;
#pragma omp parallel
  {
    uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(maxd > 0 ? maxd : 1));
    if (!key) {
#pragma omp atomic write
      failed = 1;
    }
#pragma omp for schedule(dynamic, 1024)
    for (int64_t v = 0; v < V; ++v) {
      if (!key) continue;
      const int64_t b = beg[v], n = beg[v + 1] - b;
      if (n < 2) continue;
      for (int64_t i = 0; i < n; ++i) {
        const int32_t u = csr[b + i];
        const uint64_t d = (uint64_t)(beg[u + 1] - beg[u]);
        key[i] = ((uint64_t)(uint32_t)~(uint32_t)(d > 0xffffffffull ? 0xffffffffull : d) << 32) | (uint32_t)u;
      }
      qsort(key, (size_t)n, sizeof(uint64_t), ogen_cmp_u64);
      for (int64_t i = 0; i < n; ++i) csr[b + i] = (int32_t)(key[i] & 0xffffffffull);
    }
    free(key);
  }
  return failed ? -2 : 0;
}
