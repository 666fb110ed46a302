// match.cuh -- the sm_100a DFS subgraph-counting kernel.
//
// Replaces the reference kernel _parallel_match (src/gpu_match.cu:951-1080)
// with the same count semantics and a different execution design:
//
//  * Persistent grid, one warp per DFS.  The plan is a __grid_constant__
//    parameter (constant bank); per-warp state and the candidate buffers of
//    every stored level live in shared memory, not in a 240 KB/warp global
//    stack (src/callstack.h, cu_test.cu:36-49).
//  * Candidate sets are produced in bounded chunks of `cap` vertices from a
//    resumable source cursor, so a hub's candidate set never overflows a
//    buffer (the reference writes past GRAPH_DEGREE=4096, src/config.h:12).
//  * One scan produces the set directly as filter(source) ∩ other lists:
//    the symmetry conditions become a lower bound (the source is sorted, so
//    the prefix below it is skipped by a 32-ary warp search) plus at most six
//    inequality tests; labels and injectivity are fused into the same pass
//    (src/gpu_match.cu:260-494 does this as separate passes through global
//    memory).
//  * Membership is tested with per-lane searches from a monotone cursor, or by
//    staging the matching window of the other list in shared memory with
//    16-byte loads (merge), picked per 32-element step by how wide the window
//    is, i.e. by the local degree ratio.
//  * The last pattern vertex is only counted (ballot + popc); a last vertex
//    with a single backward neighbour and no label test is counted in closed
//    form from the bound and the excluded vertices.
//  * Load balance: level-0 edge chunks from an atomic ticket (as get_job,
//    src/gpu_match.cu:496-569, but one edge per lane and the neighbour-degree
//    test precomputed); idle warps steal half of another warp's buffered
//    candidates at its shallowest level through 64-bit shared-memory words
//    (gen | next | end) and CAS; busy warps donate candidates to a bounded
//    lock-free ring in HBM when warps anywhere are hungry (the reference's
//    timeout queue, src/queue.h, src/gpu_match.cu:875-909).  Every wait is
//    bounded and reports TDFS_ERR_TIMEOUT through RunCtl::error.
#pragma once

#include <cstdint>

#include "common.h"
#include "graph.h"

namespace tdfs {

struct KernelCfg {
  int64_t e_begin;      // level-0 edge range
  int64_t e_end;
  int32_t stride;       // chunks dealt round-robin over `stride` shards
  int32_t phase;        // this launch's shard
  int32_t cap;          // candidates per stored level (multiple of 32)
  int32_t warp_bytes;   // shared memory per warp
  int32_t steal;        // 1: stealing + donation on
  int32_t window;       // merge window in ints (multiple of 128) or 0 = off
  int32_t idle_ms;      // bounded idle wait before a warp reports a timeout
  int32_t steal_min;    // a thief takes half of a level only when >= steal_min items remain
  int32_t merge_ratio;  // merge a list when its length <= merge_ratio x the source span
  int32_t fixed;        // 1: stage the last vertex's fixed lists once per parent
  int32_t split_after_ns;  // work becomes stealable after this long on one base subtree
                           // (donation to the HBM ring after 4x as long)
  int32_t wide_regs;    // 1: the 80-register build (at most 3 CTAs of 256 threads per SM)
  int32_t steal_first;  // first look for levels with >= steal_first items, then the ring, then steal_min
  int32_t lane_list;    // last level: siblings' lists up to max(lane_list, 4 |F|) long go to the
                        // flattened batch pass (0 = off: one warp pass per sibling)
  int32_t budgeted;     // 1: some slot has a work budget (SlotInfo::budget); warps account their work
  int32_t rush_hungry;  // with at least this many warps idle (0 = never) ...
  int32_t rush_ns;      // ... subtrees may be split after this long instead of split_after_ns
  int32_t leaf_min;     // the last stored level (its items only count leaves) is split only
                        // with at least this many items left
  int32_t hoist;        // 1: levels whose candidates hang on an ancestor reuse a core set
  int32_t segments;     // 1: labeled plans read the label segments of rows (DevGraph::colidx_l)
  int32_t tail;         // 1: nodes above an independent tail count it in closed form (count_tail)
  int32_t prune;        // 1: nodes whose subtree must be empty are not descended (subtree_dead)
};

constexpr int kEdgeChunk = 32;  // largest level-0 ticket (one edge per lane)

// Edges per level-0 ticket: a requested power of two up to 32; else 32 when
// the range is dealt over several shards (the documented round-robin split),
// else the largest power of two that still gives every warp of the grid two
// tickets to start with -- down to single edges for the short ranges of a
// power-law slice, whose heavy edges then start on different warps instead
// of waiting in one warp's ticket to be stolen.
inline int auto_chunk(int64_t edges, int stride, int total_warps, int requested) {
  if (requested > 0 && requested <= kEdgeChunk && (requested & (requested - 1)) == 0) return requested;
  if (stride > 1) return kEdgeChunk;
  int c = kEdgeChunk;
  while (c > 1 && edges / c < 2ll * total_warps) c >>= 1;
  return c;
}

size_t warp_smem_bytes(int k, int cap, int window, bool fixed);

// CTAs of the match kernel that fit on one SM at once (registers, shared
// memory, threads) for its 64-register (wide = false) or 80-register build;
// -1 on a CUDA error.  The persistent grid must not exceed this times the SM
// count: idle warps wait for busy ones.
int resident_blocks_per_sm(bool labeled, int warps_per_block, size_t smem, bool wide);

// Reset the control block and the split ring (stream-ordered).
void init_launch(RunCtl *ctl, QueueHdr *qh, cudaStream_t stream);

// Launch the match kernel over the slot table `tab` (filled by the host).
int launch_match(bool labeled, const DevGraph &g, RunCtl *ctl, SlotTable *tab, SplitUnit *units, QueueHdr *qh,
                 const KernelCfg &cfg, int blocks, int warps_per_block, cudaStream_t stream);

}  // namespace tdfs
