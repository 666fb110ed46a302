// cli.cpp -- the ulb / lb command-line drivers.
//
//   ulb <graph prefix> <pattern.g>     (unlabeled; built with TDFS_LABELED=0)
//   lb  <graph prefix> <pattern.g>     (labeled;   built with TDFS_LABELED=1)
//
// Same arguments and the same final line as the reference driver
// (cu_test.cu:10-110, README.md:30-36): "<pattern path>\t<kernel ms>\t<count>".
// Errors go to stderr with exit status 1 instead of asserts.
#include <cstdio>

#include "../../include/tdfs.h"

#ifndef TDFS_LABELED
#define TDFS_LABELED 0
#endif

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <graph prefix> <pattern.g>\n", argv[0]);
    return 2;
  }
  tdfs_graph *g = nullptr;
  tdfs_plan *p = nullptr;
  if (tdfs_graph_open(argv[1], TDFS_LABELED, 0, &g) || tdfs_plan_compile(argv[2], TDFS_LABELED, &p)) {
    std::fprintf(stderr, "%s\n", tdfs_last_error());
    return 1;
  }
  uint64_t count = 0;
  float ms = 0.f;
  if (tdfs_count(g, p, nullptr, &count, &ms)) {
    std::fprintf(stderr, "%s\n", tdfs_last_error());
    return 1;
  }
  std::printf("%s\t%f\t%llu\n", argv[2], ms, (unsigned long long)count);
  tdfs_plan_free(p);
  tdfs_graph_free(g);
  return 0;
}
