// common.h -- types shared by the host plan compiler, the C ABI and the
// sm_100a kernels of the tdfs B200 engine.
#pragma once

#include <cstdint>
#include <string>

#include "../../include/tdfs.h"

namespace tdfs {

constexpr int kMaxK = TDFS_MAX_PATTERN;  // pattern vertices (src/config.h:11)
constexpr int kWarp = 32;

// Condition operators, numbered as the reference's CondOperator
// (src/pattern.h:21).
enum CondOp : int { kLess = 0, kLarger = 1, kNonEqual = 2 };

// Device plan table: everything the DFS kernel reads about one pattern.  It
// is passed by value as a __grid_constant__ kernel parameter (or sits in a
// device array for batched launches), so it lives in the constant bank.
struct DevPlan {
  int32_t k;          // pattern vertices, 3..7
  int32_t labeled;    // lb (1) or ulb (0) semantics
  int32_t orient;     // level-0 edges kept only when r < c (unlabeled)
  int32_t deg[3];     // pattern degrees of vertices 0, 1, 2 (job filter)
  int32_t label[kMaxK];       // pattern vertex labels (255 = matches nothing)
  int32_t nbn[kMaxK];         // backward neighbours of vertex i
  int8_t bn[kMaxK][kMaxK];
  int32_t dep[kMaxK];         // reuse: candidates of vertex dep[i] (or -1)
  int32_t nsh[kMaxK];         // extra backward neighbours under reuse
  int8_t bnsh[kMaxK][kMaxK];
  uint8_t larger[kMaxK];      // bit j: x > phi(j)
  uint8_t less[kMaxK];        // bit j: x < phi(j)
  uint8_t neq[kMaxK];         // bit j: x != phi(j)
  uint8_t pad_;
  uint64_t multiplicity;      // |Aut| multiplier (unlabeled)
};

// Device view of a resident data graph.
struct DevGraph {
  const int64_t *rowptr;   // n + 1
  const int32_t *colidx;   // nedges (+ padding)
  const int32_t *src;      // edge -> source vertex, nedges
  const uint8_t *label;    // n, or nullptr
  const int32_t *maxnd;    // max degree over each vertex's neighbours
  const int32_t *lperm;    // level-0 label index (labeled graphs), or nullptr
  const int32_t *colidx_l; // labeled graphs with few labels: every row re-sorted by (label, id), or nullptr
  const int32_t *loff;     // its segment starts: loff[v * (nlab + 1) + l], relative to rowptr[v]
  int32_t nlab;            // labels 0..nlab-1 have segments
  int64_t nedges;
  int32_t n;
  int32_t max_degree;
};

// Per-launch control block in device memory.  Counters that many warps touch
// sit on their own 128-byte lines so ticket atomics, idle polling and the
// final count do not serialise on one L2 line.
struct alignas(128) RunCtl {
  int32_t hungry;                // warps idle and looking for work
  char pad0_[124];
  unsigned long long steals;     // diagnostics: intra-block steals
  unsigned long long splits;     // diagnostics: units through the global queue
  int32_t error;                 // TDFS_ERR_* raised by the kernel
  int32_t pad_;
  unsigned long long idle_ns;    // diagnostics: summed time warps spent without work
  unsigned long long warp_ns;    // diagnostics: summed time warps ran
  char pad1_[88];
};

// Error reporting shared by the C ABI implementation files.
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

}  // namespace tdfs
