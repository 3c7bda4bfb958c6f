// Edge-list text -> CSR file pair, replacing CSRGenerator/tuple_text_to_bin.cpp.
//
// Same inputs as the reference converter (tuple_text_to_bin.cpp:59-72): a text
// file of whitespace-separated vertex pairs, one per line, `skip_lines` header
// lines, `reverse` = 1 to add the reversed edge of every tuple. Differences,
// all deliberate:
//  * neighbours are written as int32 - the format the BFS reader loads
//    (graph.hpp:55-59); the reference converter writes int64 neighbours
//    (tuple_text_to_bin.cpp:48, 359), which its own reader cannot use;
//  * duplicates and self-loops are removed unless asked to keep them;
//  * the input is opened read-only (the reference opens it O_CREAT|O_RDWR,
//    tuple_text_to_bin.cpp:74), parsed in parallel chunks split at line
//    boundaries, and lines starting with '#' or '%' are comments;
//  * the weight file (random 1..63 in the reference, :325-328, and never used
//    by the BFS) is written only on request, from a seeded hash.
#include <fcntl.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "internal.hpp"

namespace xbfs {

static bool parse_u64(const char*& p, const char* end, unsigned long long* out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == ',' || *p == '\r')) ++p;
  if (p >= end || *p < '0' || *p > '9') return false;
  unsigned long long v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    v = v * 10 + (unsigned long long)(*p - '0');
    ++p;
  }
  *out = v;
  return true;
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

xbfs_status xbfs_convert_edge_list(const char* text_path, int32_t reverse, int32_t skip_lines, int32_t dedupe,
                                   int32_t drop_self_loops, int32_t write_weights, const char* out_prefix,
                                   int64_t* V_out, int64_t* E_out) {
  if (!text_path || !out_prefix) return set_error(XBFS_ERR_INVALID_ARG, "NULL path");
  const int fd = open(text_path, O_RDONLY);
  if (fd < 0) return set_error(XBFS_ERR_IO, "cannot open %s", text_path);
  struct stat st;
  if (fstat(fd, &st) != 0) {
    close(fd);
    return set_error(XBFS_ERR_IO, "cannot stat %s", text_path);
  }
  const size_t size = (size_t)st.st_size;
  const char* base = nullptr;
  if (size > 0) {
    base = (const char*)mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (base == (const char*)MAP_FAILED) {
      close(fd);
      return set_error(XBFS_ERR_IO, "cannot mmap %s", text_path);
    }
  }
  close(fd);
  const char* end = base + size;
  // skip header lines
  const char* body = base;
  for (int i = 0; i < skip_lines && body < end; ++i) {
    const char* nl = (const char*)memchr(body, '\n', end - body);
    body = nl ? nl + 1 : end;
  }
  // chunk boundaries at line starts
  const int nt = std::max(1, omp_get_max_threads());
  std::vector<const char*> cut(nt + 1);
  cut[0] = body;
  cut[nt] = end;
  for (int t = 1; t < nt; ++t) {
    const char* c = body + (size_t)(end - body) * t / nt;
    if (c < cut[t - 1]) c = cut[t - 1];
    const char* nl = (const char*)memchr(c, '\n', end - c);
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<std::vector<unsigned long long>> parts(nt);
  std::vector<long long> bad_line(nt, -1);
  std::vector<unsigned long long> maxid(nt, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const char* p = cut[t];
    const char* e = cut[t + 1];
    auto& out = parts[t];
    unsigned long long mx = 0;
    while (p < e) {
      const char* nl = (const char*)memchr(p, '\n', e - p);
      const char* le = nl ? nl : e;
      const char* q = p;
      while (q < le && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
      if (q < le && *q != '#' && *q != '%') {
        unsigned long long u, v;
        if (!parse_u64(q, le, &u) || !parse_u64(q, le, &v) || u > 0x7fffffbfull || v > 0x7fffffbfull) {
          if (bad_line[t] < 0) bad_line[t] = (long long)(p - base);
        } else {
          if (!(drop_self_loops && u == v)) {
            out.push_back((u << 32) | v);
            if (reverse && u != v) out.push_back((v << 32) | u);
          }
          mx = std::max(mx, std::max(u, v));
        }
      }
      p = le + 1;
    }
    maxid[t] = mx;
  }
  if (base) munmap((void*)base, size);
  for (int t = 0; t < nt; ++t)
    if (bad_line[t] >= 0)
      return set_error(XBFS_ERR_FORMAT, "%s: malformed edge line at byte %lld", text_path, bad_line[t]);
  size_t total = 0;
  unsigned long long mx = 0;
  for (int t = 0; t < nt; ++t) {
    total += parts[t].size();
    mx = std::max(mx, maxid[t]);
  }
  std::vector<unsigned long long> keys;
  keys.reserve(total);
  for (auto& pt : parts) {
    keys.insert(keys.end(), pt.begin(), pt.end());
    std::vector<unsigned long long>().swap(pt);
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  if (dedupe) keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  const long long V = total == 0 && mx == 0 ? (size > 0 ? 1 : 0) : (long long)mx + 1;
  if (V < 1) return set_error(XBFS_ERR_FORMAT, "%s holds no edges", text_path);
  const long long E = (long long)keys.size();
  std::vector<long long> beg(V + 1, 0);
  std::vector<int> csr(E);
  for (long long i = 0; i < E; ++i) {
    beg[(keys[i] >> 32) + 1]++;
    csr[i] = (int)(keys[i] & 0xffffffffull);
  }
  for (long long v = 0; v < V; ++v) beg[v + 1] += beg[v];
  const std::string pre(out_prefix);
  auto write = [&](const std::string& path, const void* data, size_t bytes) -> xbfs_status {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return set_error(XBFS_ERR_IO, "cannot create %s", path.c_str());
    const size_t w = bytes ? fwrite(data, 1, bytes, f) : 0;
    fclose(f);
    if (w != bytes) return set_error(XBFS_ERR_IO, "short write to %s", path.c_str());
    return XBFS_OK;
  };
  xbfs_status rc;
  if ((rc = write(pre + "_beg_pos.bin", beg.data(), beg.size() * 8))) return rc;
  if ((rc = write(pre + "_csr.bin", csr.data(), csr.size() * 4))) return rc;
  if (write_weights) {
    std::vector<int> wts(E);
    for (long long i = 0; i < E; ++i) {
      unsigned long long z = (unsigned long long)i + 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      wts[i] = (int)((z ^ (z >> 31)) % 63) + 1;
    }
    if ((rc = write(pre + "_weight.bin", wts.data(), wts.size() * 4))) return rc;
  }
  if (V_out) *V_out = V;
  if (E_out) *E_out = E;
  return XBFS_OK;
}

}  // extern "C"
