// graph.h -- device-resident data graph handle and launch workspace.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "common.h"

namespace tdfs {

constexpr int kColPad = 256;         // int32 padding after colidx (>= merge window)
constexpr int kSegLabels = 16;       // label-partitioned rows for graphs with at most this many labels
constexpr int kUnitItems = 24;       // candidate vertices carried by one split unit
constexpr int kQueueCap = 1 << 16;   // split units in the global queue

// A heavy subtree split off by a busy warp: the prefix phi(0..level-1) and up
// to kUnitItems candidates of pattern vertex `level`.
struct SplitUnit {
  int32_t level;
  int32_t nitems;
  int32_t phi[kMaxK];
  int32_t items[kUnitItems];
  int32_t slot;     // query the subtree belongs to
  int32_t pad_[6];
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

// ---- query slots ----------------------------------------------------------
// Every launch works through a table of query slots: one slot per pattern of
// a batched launch, or one per admitted query of the serving loop.  Slots are
// filled by the host before the kernel may see them (`admitted`) and are never
// reused within one launch, so a warp holding a stale slot index can only
// touch a finished slot, never a recycled one.
constexpr int kMaxSlots = 16384;

enum : int32_t { kSlotEmpty = 0, kSlotActive = 1, kSlotDone = 2 };

// Counters that warps update: the ticket counter, the hottest (one atomic
// per level-0 ticket), on a 128-byte line of its own; the rest on a second.
struct alignas(128) SlotHot {
  unsigned long long ticket;  // next level-0 chunk ticket
  char pad_ticket_[120];
  unsigned long long count;   // raw count (before the |Aut| multiplier)
  int32_t holders;            // warps holding this query's work + its queued units
  int32_t state;              // kSlotActive -> kSlotDone (by the completing warp)
  unsigned long long t_first; // globaltimer when the first ticket was taken
  unsigned long long t_done;  // globaltimer at completion
  unsigned long long work;    // work units spent so far (flushed by warps; budgeted launches)
  int32_t aborted;            // 1: the work budget ran out; the count is not valid
};

// Written by the host at admission, read-only for the kernel.
struct SlotInfo {
  int64_t e_begin;   // level-0 edge range and round-robin dealing (positions in the
  int64_t e_end;     //   label index when `perm` is set, else edge ids)
  int64_t ntickets;  // tickets of this slot
  int32_t stride, phase;
  int32_t chunk;     // directed edges per ticket (1, 2, 4, ..., 32)
  int32_t perm;      // 1: level-0 positions index DevGraph::lperm (labeled plans)
  int64_t budget;    // work units this query may spend (0 = unlimited)
};

struct alignas(128) SlotCtl {
  unsigned long long admitted;   // host: slots [0, admitted) are filled in
  char pad0_[120];
  unsigned long long completed;  // device: slots completed
  char pad1_[120];
  int32_t shutdown;              // host: 1 = no further admissions this launch
  int32_t idle_exit_ms;          // serving: retire after this long with no work
  char pad2_[120];
  unsigned long long first_open; // device hint: slots below this have no tickets left
  char pad3_[120];
};

struct SlotTable {
  SlotCtl ctl;
  SlotHot hot[kMaxSlots];
  SlotInfo info[kMaxSlots];
  DevPlan plan[kMaxSlots];
};

}  // namespace tdfs

namespace tdfs {

// Launch workspace: what one persistent launch needs besides the graph --
// the control block, the split ring, the slot table and its pinned host
// staging copy.  About 12 MB of device memory and 1.7 MB of pinned host
// memory, so it is pooled per device (graph.cu) instead of being allocated
// with every graph: a graph takes one at its first launch and hands it back
// when it is freed.
struct Workspace {
  int device;
  RunCtl *ctl;
  SplitUnit *queue;    // split-unit ring: kQueueCap units then a QueueHdr
  SlotTable *tab;
  SlotTable *htab;     // pinned
  RunCtl *hctl;        // pinned
  void *gstream;       // cudaStream_t for captured launches (created on first use)
};

}  // namespace tdfs

namespace tdfs {

// Level-0 label index of a labeled graph: every directed edge id, grouped by
// the label pair (label(src), label(dst)) and in ascending id within a group.
// A labeled plan's level-0 tickets run over its group only, so none of them is
// spent on edges the label test would drop.
struct LabelIndex {
  std::vector<int64_t> off;       // group of key = nl * l0 + l1 is perm[off[key], off[key + 1])
  int nl = 0;                     // labels of the graph lie in [0, nl)
  int64_t nedges = 0;
  // host copy of the sorted edge ids: written by the host build (in the
  // graph's pinned staging block), or fetched from the device array at the
  // first launch over part of the edge ids (a whole-range launch needs only off)
  const int32_t *perm = nullptr;
  const int32_t *dev_perm = nullptr;
  std::vector<int32_t> fetched;
  std::once_flag fetch_once;
};

// Group range of plan labels (l0, l1) restricted to edge ids [eb, ee).
// False when the host copy of the index could not be fetched (the caller
// then walks every edge id of the range instead).  The graph's device must be
// current.
bool label_range(LabelIndex &x, int l0, int l1, int64_t eb, int64_t ee, int64_t *b, int64_t *e);

}  // namespace tdfs

struct tdfs_graph {
  int device;
  int64_t n;
  int64_t nedges;
  int32_t max_degree;
  bool labeled;
  void *arrays;           // the one device allocation holding the arrays below
  int64_t *rowptr;
  int32_t *colidx;
  int32_t *src;
  int32_t *maxnd;
  uint8_t *label;
  int32_t *lperm;         // device label index (labeled graphs), see LabelIndex
  int32_t *colidx_l;      // label-partitioned rows (labeled graphs with <= kSegLabels labels)
  int32_t *loff;          //   and their segment starts per vertex and label
  int32_t nlab;
  tdfs::LabelIndex *lindex;  // its host copy and group offsets
  size_t array_bytes;     // size of the `arrays` block (cached for reuse when the graph is freed)
  void *staging;          // pinned host block: the derived arrays as uploaded (labeled graphs)
  size_t staging_bytes;
  tdfs::Workspace *ws;    // launch workspace (pooled; taken at the first launch)
  tdfs::RunCtl *ctl;      // = ws->ctl etc. while a workspace is held
  tdfs::SplitUnit *queue;
  tdfs::SlotTable *tab;
  tdfs::SlotTable *htab;
  tdfs::RunCtl *hctl;
  void *graphs;           // cache of instantiated launch graphs (capi.cpp)
  size_t bytes;
  int64_t last_warps;     // warps in the grid of the last count launch (diagnostics)
};

namespace tdfs {

int graph_upload(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const int32_t *labels,
                 int device, int32_t max_degree, tdfs_graph **out);
void graph_release(tdfs_graph *g);
// Give g a launch workspace from its device's pool (allocating one when none
// is idle); the device must be current.  Idempotent.
int acquire_workspace(tdfs_graph *g);
void release_graphs(tdfs_graph *g);  // capi.cpp: destroys cached launch graphs
DevGraph graph_view(const tdfs_graph *g);
int prepare_graph_arrays(const int64_t *rowptr, const int32_t *colidx, int32_t n, const int32_t *labels,
                         int32_t *src, int32_t *maxnd, uint8_t *label8, int32_t *bad, cudaStream_t st);
inline QueueHdr *queue_hdr(tdfs_graph *g) { return reinterpret_cast<QueueHdr *>(g->queue + kQueueCap); }

}  // namespace tdfs
