// convert.cpp -- tdfs_convert: writes graphs in the reference's binary CSR
// format (the output format of graph_converter/, src/graph.h:136-193) from
// the seeded generators, and applies the reference converter's relabel and
// halve steps to a graph on disk.  Host-only: no CUDA runtime, no GPU.
//
//   tdfs_convert er    <n> <avg_degree> <seed> <out prefix>
//   tdfs_convert cl    <n> <undirected edges> <gamma> <degree cap> <seed> <out prefix>
//   tdfs_convert rmat  <scale> <edge factor> <a> <b> <c> <seed> <out prefix>
//   tdfs_convert labels  <prefix> <nlabels> <seed>   (writes <prefix>.label.bin)
//   tdfs_convert relabel <in prefix> <out prefix>    (graph_converter/relabel.cpp)
//   tdfs_convert halve   <in prefix> <out prefix>    (graph_converter/halve.cpp)
//   tdfs_convert pattern <k> <density> <nlabels> <seed>   (prints a .g pattern)
//
// Prints "n E max_degree" of the written graph (the pattern text for
// `pattern`).  Errors go to stderr with exit status 1.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/tdfs.h"

namespace {

int usage(const char *argv0) {
  std::fprintf(stderr,
               "usage: %s er <n> <avg_degree> <seed> <out>\n"
               "       %s cl <n> <edges> <gamma> <cap> <seed> <out>\n"
               "       %s rmat <scale> <edge_factor> <a> <b> <c> <seed> <out>\n"
               "       %s labels <prefix> <nlabels> <seed>\n"
               "       %s relabel <in> <out>\n"
               "       %s halve <in> <out>\n"
               "       %s pattern <k> <density> <nlabels> <seed>\n",
               argv0, argv0, argv0, argv0, argv0, argv0, argv0);
  return 2;
}

int report(tdfs_csr *c, const char *prefix) {
  int rc = tdfs_csr_write(c, prefix);
  if (rc) return rc;
  int64_t n = 0, e = 0;
  int32_t md = 0;
  tdfs_csr_view(c, &n, &e, nullptr, nullptr, nullptr, &md);
  std::printf("%lld %lld %d\n", (long long)n, (long long)e, md);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) return usage(argv[0]);
  const std::string cmd = argv[1];
  tdfs_csr *c = nullptr, *d = nullptr;
  int rc = 0;
  const char *out = nullptr;
  if (cmd == "pattern" && argc == 6) {
    char buf[1024];
    rc = tdfs_gen_pattern(std::atoi(argv[2]), std::atof(argv[3]), std::atoi(argv[4]),
                          std::strtoull(argv[5], nullptr, 10), buf, sizeof buf);
    if (rc) {
      std::fprintf(stderr, "%s\n", tdfs_last_error());
      return 1;
    }
    std::fputs(buf, stdout);
    return 0;
  }
  if (cmd == "er" && argc == 6) {
    rc = tdfs_gen_er(std::atoll(argv[2]), std::atof(argv[3]), std::strtoull(argv[4], nullptr, 10), &c);
    out = argv[5];
  } else if (cmd == "cl" && argc == 8) {
    rc = tdfs_gen_chung_lu(std::atoll(argv[2]), std::atoll(argv[3]), std::atof(argv[4]), std::atoi(argv[5]),
                           std::strtoull(argv[6], nullptr, 10), &c);
    out = argv[7];
  } else if (cmd == "rmat" && argc == 9) {
    rc = tdfs_gen_rmat(std::atoi(argv[2]), std::atoi(argv[3]), std::atof(argv[4]), std::atof(argv[5]),
                       std::atof(argv[6]), std::strtoull(argv[7], nullptr, 10), &c);
    out = argv[8];
  } else if (cmd == "labels" && argc == 5) {
    rc = tdfs_csr_read(argv[2], 0, &c);
    if (!rc) rc = tdfs_csr_set_labels(c, std::atoi(argv[3]), std::strtoull(argv[4], nullptr, 10));
    out = argv[2];
  } else if ((cmd == "relabel" || cmd == "halve") && argc == 4) {
    // labels travel with the graph when the input has a .label.bin
    const std::string lab = std::string(argv[2]) + ".label.bin";
    FILE *f = std::fopen(lab.c_str(), "rb");
    const int labeled = f != nullptr;
    if (f) std::fclose(f);
    rc = tdfs_csr_read(argv[2], labeled, &c);
    if (!rc) rc = cmd == "relabel" ? tdfs_csr_relabel(c, &d) : tdfs_csr_halve(c, &d);
    out = argv[3];
  } else {
    return usage(argv[0]);
  }
  if (!rc) rc = report(d ? d : c, out);
  if (rc) std::fprintf(stderr, "%s\n", tdfs_last_error());
  tdfs_csr_free(c);
  tdfs_csr_free(d);
  return rc ? 1 : 0;
}
