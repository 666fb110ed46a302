// graph.h -- device-resident data graph handle and launch workspace.
#pragma once

#include <cstddef>
#include <cstdint>

#include "common.h"

namespace tdfs {

constexpr int kColPad = 256;         // int32 padding after colidx (>= merge window)
constexpr int kUnitItems = 24;       // candidate vertices carried by one split unit
constexpr int kQueueCap = 1 << 16;   // split units in the global queue

// A heavy subtree split off by a busy warp: the prefix phi(0..level-1) and up
// to kUnitItems candidates of pattern vertex `level`.
struct SplitUnit {
  int32_t level;
  int32_t nitems;
  int32_t phi[kMaxK];
  int32_t items[kUnitItems];
  int32_t pad_[7];
};
static_assert(sizeof(SplitUnit) % 16 == 0, "unit alignment");

// Bounded MPMC ring (per-slot sequence numbers) header, followed in memory
// by kQueueCap sequence words and kQueueCap units.
struct alignas(128) QueueHdr {
  unsigned long long head;
  char pad0_[120];
  unsigned long long tail;
  char pad1_[120];
  unsigned long long seq[kQueueCap];
};

}  // namespace tdfs

struct tdfs_graph {
  int device;
  int64_t n;
  int64_t nedges;
  int32_t max_degree;
  bool labeled;
  int64_t *rowptr;
  int32_t *colidx;
  int32_t *src;
  int32_t *maxnd;
  uint8_t *label;
  tdfs::RunCtl *ctl;     // launch control block (one launch at a time per handle)
  tdfs::SplitUnit *queue; // split-unit ring: kQueueCap units then a QueueHdr
  size_t bytes;
};

namespace tdfs {

int graph_upload(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const int32_t *labels,
                 int device, int32_t max_degree, tdfs_graph **out);
void graph_release(tdfs_graph *g);
DevGraph graph_view(const tdfs_graph *g);
inline QueueHdr *queue_hdr(tdfs_graph *g) { return reinterpret_cast<QueueHdr *>(g->queue + kQueueCap); }

}  // namespace tdfs
