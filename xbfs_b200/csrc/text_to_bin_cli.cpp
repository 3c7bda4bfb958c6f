// text_to_bin — edge-list text to the CSR file pair, with the reference
// converter's argument contract (CSRGenerator/tuple_text_to_bin.cpp:64-72):
//
//   text_to_bin edge_list reverse skip_lines thread_count
//               [--keep-duplicates] [--keep-self-loops] [--weights] [--out prefix]
//
// Writes <prefix>_beg_pos.bin (int64[V+1]) and <prefix>_csr.bin (int32[E]);
// prefix defaults to the input path, as in the reference. thread_count is
// accepted and ignored (the reference parses it but never uses it, :72).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "xbfs.h"

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s edge_list reverse skip_lines thread_count [--keep-duplicates] "
                    "[--keep-self-loops] [--weights] [--out prefix]\n", argv[0]);
    return 2;
  }
  const char* in = argv[1];
  const int reverse = atoi(argv[2]);
  const int skip = atoi(argv[3]);
  int dedupe = 1, drop_loops = 1, weights = 0;
  std::string prefix = in;
  for (int i = 5; i < argc; ++i) {
    if (!strcmp(argv[i], "--keep-duplicates")) dedupe = 0;
    else if (!strcmp(argv[i], "--keep-self-loops")) drop_loops = 0;
    else if (!strcmp(argv[i], "--weights")) weights = 1;
    else if (!strcmp(argv[i], "--out") && i + 1 < argc) prefix = argv[++i];
    else {
      fprintf(stderr, "text_to_bin: unknown option %s\n", argv[i]);
      return 2;
    }
  }
  int64_t V = 0, E = 0;
  const xbfs_status st = xbfs_convert_edge_list(in, reverse, skip, dedupe, drop_loops, weights, prefix.c_str(), &V, &E);
  if (st) {
    fprintf(stderr, "text_to_bin: %s (%s)\n", xbfs_strerror(st), xbfs_last_error());
    return 1;
  }
  printf("%s_beg_pos.bin / %s_csr.bin: %lld vertices, %lld edges\n", prefix.c_str(), prefix.c_str(), (long long)V,
         (long long)E);
  return 0;
}
