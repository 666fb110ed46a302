// csr.h -- host CSR graph: reference binary format I/O and generators.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "common.h"

struct tdfs_csr {
  int64_t n = 0;
  int64_t nedges = 0;                // directed (each undirected edge twice)
  std::vector<int64_t> rowptr;       // n + 1
  std::vector<int32_t> colidx;       // nedges, rows strictly increasing
  std::vector<int32_t> labels;       // n or empty
  int32_t max_degree = 0;
  // sampling tables of tdfs_estimate (estimate.cpp), built on first use
  mutable std::shared_ptr<void> estimate_tables;
};

namespace tdfs {

// splitmix64: the one seeded generator used by every synthetic input.
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * 0x1.0p-53; }  // [0, 1)
  uint64_t below(uint64_t m) { return next() % m; }
};

// Counter-based value for element i of stream `seed` (order independent).
inline uint64_t hash64(uint64_t seed, uint64_t i) {
  Rng r(seed * 0xD1B54A32D192ED03ull + i);
  return r.next();
}

// Check a CSR for the reference's invariants; returns TDFS_OK or error code.
int validate_csr(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                 int32_t *max_degree);

// Build a symmetric, deduplicated, loop-free CSR from undirected pairs.
void csr_from_pairs(int64_t n, std::vector<std::pair<uint32_t, uint32_t>> &pairs, tdfs_csr *out);

}  // namespace tdfs
